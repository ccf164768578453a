// Headless rasterizer buffers and launchers (render.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "lima_abi.h"
#include "physdev.cuh"

namespace lima {

struct RenderBuf {
    bool ready = false;
    int n_slots = 0;
    uint8_t* kind = nullptr;          // [n_slots] ATOM_TYPE per slot
    float4* slot_pos = nullptr;       // [n_slots] positions in the reference's slot layout
    uint32_t* ref_slot = nullptr;     // physics: [n] orig id -> slot
    lima_render_ball* balls[2] = {nullptr, nullptr};   // per slot, then sorted by depth
    float* keys[2] = {nullptr, nullptr};
    uint32_t* vals[2] = {nullptr, nullptr};
    void* sort_tmp = nullptr;
    size_t sort_bytes = 0;
    uint32_t* win = nullptr;          // [pixels] sorted index of the ball on top
    uint8_t* rgb = nullptr;           // [pixels][3]
    size_t img_pixels = 0;
};

// kind: ATOM_TYPE of every slot; ref_slot: physics orig id -> slot (empty for the reference semantics)
bool render_setup(RenderBuf& r, int n_slots, const std::vector<uint8_t>& kind, const std::vector<uint32_t>& ref_slot,
                  std::vector<void*>& allocs, cudaStream_t s);
void render_slot_positions_phys(const RenderBuf& r, const PhysDev& d, int cur, cudaStream_t s);
// balls of r.slot_pos into r.balls[1], sorted by pos.y; returns kernels launched
int render_balls(RenderBuf& r, float L, cudaStream_t s);
// w x h RGB image of r.balls[1] into host_rgb (stream-ordered copy)
bool render_image(RenderBuf& r, int w, int h, uint8_t* host_rgb, std::vector<void*>& allocs, cudaStream_t s);

}  // namespace lima
