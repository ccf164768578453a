// Launchers of the physics-semantics kernels (kernels_physics.cu), called by
// the host side in physics_host.cu.
#pragma once
#include "physdev.cuh"

namespace lima {

constexpr int kTB = 256;      // threads per block
constexpr int kGroup = 8;     // lanes per particle in the pair and list kernels

void launch_keys(const PhysDev& d, int cur, cudaStream_t s);
void launch_permute(const PhysDev& d, int cur, bool mixed, cudaStream_t s);
void launch_build_list(const PhysDev& d, int cur, cudaStream_t s);
void launch_bonded(const PhysDev& d, int cur, bool energy, cudaStream_t s);
void launch_pair(const PhysDev& d, int cur, bool mixed, bool energy, bool integrate, cudaStream_t s);

}  // namespace lima
