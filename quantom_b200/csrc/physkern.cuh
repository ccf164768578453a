// Launchers of the physics-semantics kernels (kernels_physics.cu), called by
// the host side in physics_host.cu.
#pragma once
#include <algorithm>

#include "physdev.cuh"

namespace lima {

constexpr int kTB = 256;         // threads per block of the per-particle kernels and the step kernel
constexpr int kGroup = 8;        // lanes per particle in the list and step kernels
constexpr int kBuildWarps = 4;   // warps per block of the list build (8 particles per warp)
constexpr int kMaxTypes = 32;    // LIMA_MAX_ATOM_TYPES
constexpr int kScanThreads = 1024;

// lanes per particle in the step kernel: one list column each
constexpr int kStepLanes = 8;
static_assert(kStepLanes == kGroup, "the step kernel gives each lane one list column");
// the step kernel reads its list rows from shared memory, staged by bulk
// copies in groups of kStageRows rows (false: per-lane loads from the list).
// Built into liblima_b200_staged.so (LIMA_STAGED_LIST=1) beside the default
// library; it measured no faster on the 32k box.
#ifndef LIMA_STAGED_LIST
#define LIMA_STAGED_LIST 0
#endif
constexpr bool kStagedList = LIMA_STAGED_LIST != 0;
constexpr int kStageRows = 8;
// Verlet-list layout: entry k of particle slot i is column k % 8 of row k / 8,
// and a particle's rows come in chunks of kListChunk / 8 = 4: column g of
// chunk q holds rows 4q .. 4q + 3 in consecutive words, so the lane that owns
// column g reads its next four entries with one 8-byte (16-bit ids) or
// 16-byte (32-bit ids) load, and the 32 words of one chunk of consecutive
// particles follow each other.  The capacity per particle is a multiple of
// kListChunk.
constexpr int kListChunk = 32;
static_assert(kGroup == 8 && kListChunk == 4 * kGroup, "chunks of four 8-entry rows");
__host__ __device__ inline uint32_t nl_word(uint32_t n_pad, uint32_t i, uint32_t k) {
    return ((k >> 5) * n_pad + i) * 32u + (k & 7u) * 4u + ((k >> 3) & 3u);
}
// list capacity per particle: `want` entries rounded up to whole chunks
__host__ __device__ inline int nl_round_cap(int want) { return (want + kListChunk - 1) / kListChunk * kListChunk; }
// list entry `idx` (a word index of the layout above) in either id width
__device__ __forceinline__ uint32_t nl_load(const PhysDev& d, size_t idx) {
    return d.nl16 ? (uint32_t)reinterpret_cast<const uint16_t*>(d.nl)[idx] : d.nl[idx];
}
__device__ __forceinline__ void nl_store(const PhysDev& d, size_t idx, uint32_t j) {
    if (d.nl16)
        reinterpret_cast<uint16_t*>(d.nl)[idx] = (uint16_t)j;
    else
        d.nl[idx] = j;
}
// whether the step kernels of this library take 16-bit list ids for n_pad
// slots: whenever they fit, except in the staged variant (32-bit rows)
bool list_ids_16bit(int n_pad);
// bytes of one list entry
__host__ __device__ inline size_t nl_entry_bytes(const PhysDev& d) { return d.nl16 ? 2 : 4; }

// blocks of the step kernel (kStepLanes lanes per particle slot, n_pad a multiple of 32)
__host__ __device__ inline int step_blocks(const PhysDev& d) {
    return (int)(((size_t)d.n_pad * kStepLanes + kTB - 1) / kTB);
}
// blocks of the bonded kernel (one thread per term)
__host__ __device__ inline int bonded_blocks(const PhysDev& d) {
    const int nt = d.n_bonds + d.n_angles + d.n_dih;
    return nt > 0 ? (nt + kTB - 1) / kTB : 1;
}

// the counting sort of the slots by the cell of `pos`: cell_key, cstart, order
void launch_sort(const PhysDev& d, const float4* pos, cudaStream_t s);
// every per-slot array into cell order in the tmp arrays, reference positions
void launch_permute(const PhysDev& d, int cur, bool mixed, cudaStream_t s);
// reference positions of an in-place build (particles not moved)
void launch_set_xref(const PhysDev& d, const float4* pos, cudaStream_t s);
// The Verlet list of positions pos (orig: orig ids by slot).  items
// (nullable): slots in cell order when the particles were not re-sorted.
// copy_cur >= 0: pos/orig are the permuted tmp arrays, and the build copies
// every tmp array back into the step arrays of that parity.
void launch_build_list(const PhysDev& d, const float4* pos, const uint32_t* orig, const uint32_t* items, int copy_cur,
                       bool mixed, cudaStream_t s);
// The bonded kernel of parity `cur` (term forces; ENERGY: block partials)
void launch_bonded(const PhysDev& d, int cur, bool energy, cudaStream_t s);
// The step kernel of parity `cur` (slot cur) or an energy evaluation (slot
// kSlotEval, integrate false), launched with a programmatic dependency on the
// bonded kernel before it.  tail: device-launchable rebuild graph the last
// block launches when a rebuild is due (nullptr: none).
void launch_step(const PhysDev& d, int cur, bool mixed, bool energy, bool integrate, int slot, cudaGraphExec_t tail,
                 cudaStream_t s);

}  // namespace lima
