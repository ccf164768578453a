// Device-side state of the reference-semantics path and the launch
// interfaces of its kernels.  Layout in HBM (all arrays 256-byte aligned,
// float3 quantities widened to float4 so every particle is one 16-byte load):
//   compound particle (c, l) -> slot c*64 + l   (the reference's own indexing,
//                               Box::compound_state_array / Compound::*[64])
//   solvent s                -> slot s
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lima_abi.h"

namespace lima {

constexpr int kMaxCP = LIMA_MAX_COMPOUND_PARTICLES;   // 64
constexpr int kCsChunk = 256;                         // solvent neighbours per compound<-solvent block

// device error bits (read by lima_synchronize)
enum : int {
    ERR_BIT_SS_OVERFLOW = 1,
    ERR_BIT_CS_OVERFLOW = 2,
    ERR_BIT_CC_OVERFLOW = 4,
    ERR_BIT_NAN = 8,
    ERR_BIT_CRITICAL_FORCE = 16,
    ERR_BIT_PHYS_LIST_OVERFLOW = 32,
    ERR_BIT_LIST_STALE = 64,      // a particle moved more than skin/2 since the last list build
    ERR_BIT_TILE_TIMEOUT = 128,   // a shared-memory staging wait ran out (bounded mbarrier wait)
    ERR_BIT_REBUILD_LAUNCH = 256, // the device could not launch a due list rebuild
};

struct RefDev {
    int n_c, n_s, n_b;
    float L, Lh, C;          // box, half box, reference CUTOFF
    double dt;
    const lima_compound* comps;                 // topology, the reference struct verbatim
    const lima_compound_bridge_compact* bridges;
    const lima_particle_parameters* pp;         // [LIMA_MAX_ATOM_TYPES]
    float4* cpos[2];         // CompoundState::positions, double-buffered [n_c*64]
    float4* cprev;           // Compound::prev_positions [n_c*64]
    float4* cbridge;         // Compound::forces (bridge -> compound hand-off) [n_c*64]
    float4* spos[2];         // Solvent::pos, double-buffered [n_s]
    float4* sprev[2];        // Solvent::pos_tsub1, double-buffered [n_s]
    // neighbour lists: fixed capacity rows, ids ascending
    uint32_t* ss_ids; uint32_t* ss_cnt; int ss_cap;
    uint32_t* cs_ids; uint32_t* cs_cnt; int cs_cap;
    uint32_t* cc_ids; uint32_t* cc_cnt;         // row capacity 64 (NEIGHBORLIST_MAX_COMPOUNDS)
    uint8_t* cc_prev;        // [n_c*n_c] previous compound-compound membership
    // cell grid for the solvent-solvent search
    int m;                   // cells per dimension (1 = no grid)
    float cell;
    uint32_t* cell_count; uint32_t* cell_start; uint32_t* cell_fill; uint32_t* cell_items; uint32_t* sol_cell;
    // compound <- solvent partial sums [n_c][n_chunks][64]
    float4* cs_partial; int n_chunks;
    // compound LJ partial sums [n_c][1 + 64][64]: slot 0 the intramolecular
    // sum, slot 1 + k the sum over compound-list entry k
    float4* cc_partial;
    // lanes per solvent (1, 2, 4, 8 or 16) in the solvent kernels' loop over
    // the compounds and over the solvent list
    int sol_lanes, sol_list_lanes;
    int sol_list_block;      // threads per block of the list loop's kernel (32, 64 or 128)
    // per solvent [n_s]: the force summed over the compounds, the list
    // loop's sum, and the image the list loop ends on
    float4* sol_force; float4* sol_acc; float4* sol_image;
    // outputs of the last step
    float4* force_c;         // [n_c*64]
    float4* force_s;         // [n_s]
    double* potE;            // [n_c*64] (solvent entries are always 0 in the reference)
    float4* force_ljsol;     // [n_c*64] the LJ force from solvents (data_GAN value 1, Engine.cu:1034)
    float* lambda;           // thermostat scalar applied in the next step
    int* err;
    // reference thermostat (Engine::getBoxTemperature) scratch
    float4* csnap; float4* ssnap;   // positions two steps back
    double* ke_accum;               // [1]
    // per compound particle, the bonded-term results it receives, in the
    // order the reference accumulates them (bonds, then angles, then
    // dihedrals, each by term index): CSR rows c*65+t, codes
    // (kind << 14) | (term << 2) | slot, kind 0 bond, 1 angle, 2 dihedral
    uint32_t* bt_off; uint16_t* bt_code;
};

// nlist_reference.cu
void ref_build_nlists(const RefDev& d, int cur, cudaStream_t s);
// kernels_reference.cu
// Two more streams and three events: the solvent kernels run beside the
// compound kernels (they read the same current buffers and write disjoint
// next ones), the solvents' loop over the compounds beside their list loop.
struct StepFork {
    cudaStream_t side = nullptr, side2 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, join2 = nullptr;
};
int ref_step_kernels(const RefDev& d, int cur, cudaStream_t s, cudaEvent_t* ev = nullptr, const StepFork* fk = nullptr);
void ref_thermostat_snapshot(const RefDev& d, int cur, cudaStream_t s);
void ref_thermostat_update(const RefDev& d, int cur, int n_particles, float t_target, bool apply, cudaStream_t s);
void set_device_float(float* p, float v, cudaStream_t s);

}  // namespace lima
