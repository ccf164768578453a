// Physics-semantics path: conservative forces of the LIMA_MD model on one
// unified particle array, laid out for throughput.
//
// Particle ids: "orig" = compound particles compound by compound (c, l) ->
// base[c] + l, then solvents (n_cp + s).  "slot" = position in the cell-sorted
// order used by every per-step array; re-sorted at each list rebuild.
//
// Cells: a uniform grid of m^3 cells of side >= r_list/2, so every particle
// within r_list of a cell lies in the 5x5x5 block of cells around it (all
// m^3 cells when m < 5).  A cell's particles occupy a contiguous slot range
// [cstart[c], cstart[c+1]), and cells (x, y, z..z+4) are consecutive, so a
// neighbourhood is 25 contiguous ranges (columns along z).
//
// HBM layout (float3 quantities widened to float4, one 16-byte access each):
//   pos[2][n_pad]   x, y, z in [0, L), w = type index (bit-cast)   (double-buffered)
//   vel[n_pad]      half-step velocity, w = 1/m
//   posc/velc       low parts of pos/vel (mixed precision)
//   xref[n_pad]     positions at the last rebuild (list validity check)
//   force[n_pad]    total force of the last evaluation, w = per-particle potential energy
//   nl[cap][n_pad]  Verlet list of sorted slots (uint16 ids when n_pad <= 65536,
//                   else uint32), entry k of particle i at word
//                   ((k / 32) * n_pad + i) * 32 + (k % 8) * 4 + (k / 8) % 4
//                   (nl_word): lane g of a particle's 8 reads entries
//                   g, g + 8, g + 16, g + 24 as one vector, and consecutive
//                   particles follow each other
//   term_force      one float4 per (term, atom) of every bonded term; gathered
//                   per particle through bterm_off/bterm_slot (CSR over orig)
//   part[blocks][4] per-block FP64 partial sums of the last step kernel; the
//                   block that finishes last adds them in block order
// A list rebuild permutes every per-slot array (both position buffers,
// velocities, forces, low parts, orig ids), so readbacks after it stay
// consistent with the forces of the step before it.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "lima_abi.h"

namespace lima {

// FP64 sums of a step kernel: kinetic energy, LJ energy, LJ virial (the
// bonded kernel sums bond, angle, dihedral energy and bonded virial)
constexpr int kRed = 3;
constexpr int kRedStride = 4;   // doubles per block partial
// step-kernel slots: 0/1 = the step of that parity (sets lambda[parity ^ 1]),
// 2 = an energy evaluation without integration
constexpr int kSlotEval = 2;

struct PhysDev {
    int n;              // particles
    int n_pad;          // n rounded up to 32
    int n_cp;           // compound particles
    int n_c, n_s;
    float L, invL, rc, rc2, rlist, rlist2, ron2, inv_sw_d, half_skin2;   // inv_sw_d = 1/(rc^2 - r_on^2)
    float sw_c0, sw_k10;        // rc^2 inv_sw_d and 10 inv_sw_d (the step kernel's switch)
    float inv_rc2;              // 1 / rc^2
    int use_switch;
    double dt;
    int precision;      // lima_precision
    int thermostat;     // lima_thermostat
    double t_target, tau_t;
    int n_types;
    float4* pos[2];
    float4* vel;
    float4* posc;
    float4* velc;
    float4* xref;
    float4* force;
    float4* pos_orig[2];        // [n_cp] compound-particle positions in orig order (the bonded terms' input)
    float4* posc_orig[2];       // [n_cp] their low parts (mixed precision)
    uint32_t* orig_of_sorted;   // [n]
    uint32_t* sorted_of_orig;   // [n]
    uint32_t* cp_base;          // [n_c + 1] orig id of each compound's particle 0 (n_cp at the end)
    float2* lj_table;           // [n_types^2] (sigma^2, 4 eps), Lorentz-Berthelot
    // cell grid and the counting sort by cell (stable: ascending slot inside a cell)
    int m;                      // cells per dimension
    int n_cells;                // m^3
    uint32_t* cell_key;         // [n] cell of each slot
    uint32_t* cell_rank;        // [n] arrival order of the slot in its cell
    uint32_t* ccount;           // [n_cells] occupancy during a sort; zero between sorts
    uint32_t* order;            // [n] slots in cell order
    uint32_t* cstart;           // [n_cells + 1]: cell c holds sorted slots [cstart[c], cstart[c+1])
    float4* pos_tmp[2]; float4* vel_tmp; float4* posc_tmp; float4* velc_tmp; float4* force_tmp; uint32_t* orig_tmp;
    // Verlet list (tile-local indices)
    uint32_t* nl; uint32_t* nl_cnt; int nl_cap;
    int nl16;                   // 1: nl holds uint16 slot ids (half the bytes per step), 0: uint32
    int* nl_need;               // largest row length a build found beyond nl_cap (0: none)
    // dynamic lists (nlist_period <= 0): the step kernel's last block sees
    // that a particle moved more than skin/2 since the last build and
    // tail-launches the device-launchable rebuild graph of the next parity,
    // which runs before anything that follows the step in its stream; fixed
    // period: the same test is an error (ERR_BIT_LIST_STALE)
    int dynamic_list;
    int* need_rebuild;
    unsigned long long* rebuild_count;   // rebuilds launched from the device
    cudaGraphExec_t rebuild_exec[2];     // device-launchable rebuild of pos[parity] (null: host decides)
    // exclusions (CSR over orig ids)
    uint32_t* excl_off; uint32_t* excl_ids;
    // bonded terms (orig ids); a term slot numbers (term, role): bond b role r
    // -> 2b + r, angle a -> 2 n_bonds + 3a + r, dihedral q -> 2 n_bonds +
    // 3 n_angles + 4q + r
    int n_bonds, n_angles, n_dih;
    int4* bond_idx; float2* bond_par;          // (r0, k)
    int4* angle_idx; float2* angle_par;        // (theta0, k)
    int4* dih_idx; float4* dih_par;            // (phi0, k, n)
    uint32_t* bterm_off; uint32_t* bterm_slot;
    float4* term_force;         // [n_term_slots] the bonded kernel's force per (term, role), w = energy share
    int n_term_slots;
    // FP64 reductions: block partials, the count of blocks that wrote theirs,
    // the latest totals (LIMA_E_*) and the Berendsen scalar per parity
    double* part;
    double* bpart;      // [bonded blocks][4] the bonded kernel's block partials
    unsigned int* done;
    double* e_last;
    float* lambda;      // [2]
    int* err;
};

struct PhysHost {
    const lima_params* params;
    const lima_forcefield* ff;
    const lima_compound* comps;
    const lima_compound_state* states;
    int n_c;
    const lima_compound_bridge_compact* bridges;
    int n_b;
    const lima_solvent* sols;
    int n_s;
};

// Stream-ordered device allocations from a pool of the current device shared
// by every context of the process; freed blocks stay cached in it, so a new
// context reuses the memory of destroyed ones instead of mapping new memory.
void* pool_alloc(size_t bytes, cudaStream_t s);   // nullptr on failure
void pool_free(void* p, cudaStream_t s);
// Pinned host blocks from a process-wide cache: a freed block is kept and
// handed to a later request of up to its size (cudaMallocHost costs about a
// millisecond per call).
void* pinned_alloc(size_t bytes);   // nullptr on failure
void pinned_free(void* p);

// returns 0 or a lima_status; device buffers (from the pool) are appended to `allocs`
int phys_setup(const PhysHost& h, PhysDev& d, cudaStream_t s, std::vector<void*>& allocs, std::string& msg);
void phys_upload_state(const PhysHost& h, PhysDev& d, int cur, cudaStream_t s);
void phys_rebuild(const PhysDev& d, int cur, cudaStream_t s);
// list of `pos` (particle order unchanged; reference positions reset)
void phys_rebuild_inplace(const PhysDev& d, const float4* pos, cudaStream_t s);
void phys_prime(PhysDev& d, int cur, cudaStream_t s);
// after a build: if a row overflowed the list capacity, grow the list to 1.25x
// the longest row (the capacity starts from the box's mean density, which a
// dense solute exceeds) and return true so the caller rebuilds; waits for s.
// allocs: the pool allocations of phys_setup (the list is one of them)
bool phys_fit_list(PhysDev& d, cudaStream_t s, std::vector<void*>& allocs);
// dynamic lists: the step graph of parity `cur` (the step kernel, which tail-launches
// the rebuild when one is due); returns its kernel count, or -1 if the graph cannot be built.
// extra (nullable): more kernels for the same graph, launched into the
// capturing stream after the step (the frame log of a logged step), returning
// how many it launched
int phys_capture_dynamic(const PhysDev& d, int cur, bool energy, cudaStream_t s, cudaGraphExec_t* out,
                         int (*extra)(void*, cudaStream_t) = nullptr, void* extra_ctx = nullptr);
bool phys_rebuild_pending(const PhysDev& d, cudaStream_t s);
unsigned long long phys_device_rebuilds(const PhysDev& d, cudaStream_t s);
// the device-launchable rebuild graphs of both parities (after the list capacity is final)
int phys_capture_rebuild(PhysDev& d, cudaStream_t s, std::string& msg);
void phys_free_rebuild(PhysDev& d);
// k_sort_count, k_sort_scan, k_sort_fill, k_sort_order, k_permute, k_build_list
constexpr int kRebuildKernels = 6;
// One step: the bonded kernel, then the step kernel (pair terms,
// integration, FP64 sums) launched programmatically so that it overlaps the
// bonded kernel.  tail: launch the due rebuild from the device (the launch
// must be captured in a graph).  ev (nullable): events before the bonded
// kernel, after it, after the step kernel.  Returns kernels launched.
int phys_step_kernels(const PhysDev& d, int cur, cudaStream_t s, bool energy = false, cudaEvent_t* ev = nullptr,
                      bool tail = false);
void phys_energy_now(PhysDev& d, int cur, cudaStream_t s);
// Host copy of the state in orig order (position and previous position, in
// double), kept while the state it was read from is unchanged: `key` names
// that state (the caller changes it whenever the state may have changed).
// The state in the reference's layout, straight into device copies of its
// structs: every compound slot (particle 0 in the box, the others in the image
// nearest to it, Engine.cu:993-996; previous position x - v dt in the same
// image; empty slots zero) and every solvent (position, previous position).
// Either compound output may be null.
void launch_read_compounds(const PhysDev& d, int cur, lima_compound_state* states, lima_float3* prev, cudaStream_t s);
void launch_read_solvents(const PhysDev& d, int cur, lima_solvent* out, cudaStream_t s);
void phys_read_forces(const PhysDev& d, const lima_compound* comps, float4* fc, float4* fs);
// the Verlet list as CSR over orig ids (offsets[n + 1]; ids, nullable, sorted
// ascending in each row); returns the total entry count
uint32_t phys_read_list(const PhysDev& d, uint32_t* offsets, uint32_t* ids);
void phys_read_energies(const PhysDev& d, double* totals, double* per_particle, const lima_compound* comps, int n_c,
                        int n_s);

}  // namespace lima
