// Launchers of the physics-semantics kernels (kernels_physics.cu), called by
// the host side in physics_host.cu.
#pragma once
#include <algorithm>

#include "physdev.cuh"

namespace lima {

constexpr int kTB = 256;         // threads per block of the per-particle / per-term kernels
constexpr int kGroup = 8;        // lanes per particle in the list and pair kernels
constexpr int kBuildWarps = 4;   // warps per block of the list build
constexpr int kSlices = 8;       // lanes per particle in the list build (32 / kSlices particles per warp)
constexpr int kMaxTypes = 32;    // LIMA_MAX_ATOM_TYPES

void launch_keys(const PhysDev& d, const float4* pos, cudaStream_t s);
void launch_cell_offsets(const PhysDev& d, const float4* pos, cudaStream_t s);
void launch_permute(const PhysDev& d, int cur, bool mixed, cudaStream_t s);
// items (nullable): slots in cell order when the particles were not re-sorted
void launch_build_list(const PhysDev& d, const float4* pos, const uint32_t* items, cudaStream_t s);
void launch_copy_back(const PhysDev& d, int cur, bool mixed, cudaStream_t s);
// slot: accumulator slot to add energies to; fold_src: slot to fold first (-1: none)
void launch_bonded(const PhysDev& d, int cur, bool energy, int slot, int fold_src, cudaStream_t s);
void launch_list_check(const PhysDev& d, cudaGraphConditionalHandle h, cudaStream_t s);
void launch_pair(const PhysDev& d, int cur, bool mixed, bool energy, bool integrate, int slot, cudaStream_t s);
void launch_finalize(const PhysDev& d, int src, cudaStream_t s);

}  // namespace lima
