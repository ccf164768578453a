// Pair and periodic-boundary math of the physics path, shared by the step
// kernels (kernels_physics.cu) and the frame log (framelog.cu).
#pragma once
#include <cuda_runtime.h>

#include "physdev.cuh"

namespace lima {

// minimum image of one coordinate difference in a cubic box
__device__ __forceinline__ float mimg(float d, float L, float invL) { return d - L * rintf(d * invL); }

// The axes (bit 0 x, 1 y, 2 z) on which a particle lies within r_c of a face
// of the box.  On the other axes every particle within r_c of it (minimum
// image) is so in plain coordinates too, and a pair beyond r_c contributes
// zero either way (a plain coordinate difference is never shorter than its
// minimum image), so its pairs need the minimum image only on these axes.
__device__ __forceinline__ unsigned face_axes(const PhysDev& d, float4 p) {
    const float m = d.rc * 1.0001f + 1e-5f, hi = d.L - m;
    return (p.x < m || p.x > hi ? 1u : 0u) | (p.y < m || p.y > hi ? 2u : 0u) | (p.z < m || p.z > hi ? 4u : 0u);
}

// 1/x by the special-function unit's approximate reciprocal (PTX
// rcp.approx.ftz.f32, relative error within 2^-23); x is a squared pair
// distance, positive and far from the denormal and overflow ranges.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// One pair, branch-free: out-of-cutoff pairs contribute zero through a
// select, the switch is evaluated for every pair (S = 1, S' = 0 below r_on).
// WRAP false: the plain difference is the minimum image (face_axes(i) is 0).
template <bool ENERGY, bool SWITCH, bool WRAP = true>
__device__ __forceinline__ void lj_pair(const PhysDev& d, const float2* __restrict__ row, float4 pi, float4 pj,
                                        float& px, float& py, float& pz, float& e_i, float& w_i) {
    const float dx = WRAP ? mimg(pj.x - pi.x, d.L, d.invL) : pj.x - pi.x;
    const float dy = WRAP ? mimg(pj.y - pi.y, d.L, d.invL) : pj.y - pi.y;
    const float dz = WRAP ? mimg(pj.z - pi.z, d.L, d.invL) : pj.z - pi.z;
    const float r2 = dx * dx + dy * dy + dz * dz;
    const float2 tab = row[__float_as_int(pj.w)];
    const float inv = rcp_approx(r2);
    const float sr2 = tab.x * inv;
    const float sr6 = sr2 * sr2 * sr2;
    float fr = 6.f * tab.y * inv * sr6 * (2.f * sr6 - 1.f);   // F_j / r_vec
    float v = 0.f;
    if (ENERGY || SWITCH) v = tab.y * (sr6 * sr6 - sr6);
    if (SWITCH) {
        // C2 switch in r^2: S = t^3 (10 - 15 t + 6 t^2), t = sat((rc^2 - r^2) / (rc^2 - r_on^2));
        // S = 1 below r_on and S = S' = 0 beyond r_c, so no separate cutoff select
        const float t = __saturatef((d.rc2 - r2) * d.inv_sw_d);
        const float t2 = t * t, omt = 1.f - t;
        const float sw = t2 * t * fmaf(t, fmaf(6.f, t, -15.f), 10.f);
        const float dsw = -60.f * d.inv_sw_d * t2 * omt * omt;   // (dS/dr)/r
        fr = fr * sw - v * dsw;
        v *= sw;
    } else {
        if (ENERGY) {
            const float src2 = tab.x / d.rc2, src6 = src2 * src2 * src2;
            v -= tab.y * (src6 * src6 - src6);
        }
        const bool in = r2 < d.rc2;
        fr = in ? fr : 0.f;
        v = in ? v : 0.f;
    }
    px -= fr * dx;
    py -= fr * dy;
    pz -= fr * dz;
    if (ENERGY) {
        e_i += 0.5f * v;
        w_i += 0.5f * fr * r2;
    }
}

// The step kernel's form of lj_pair: the same force in fewer operations, from
// a table row of (sigma^2, 24 eps).  With s6 = (sigma^2 / r^2)^3 and a = 24 eps s6:
//   6 V   = a s6 - a                      (V = 4 eps s6 (s6 - 1))
//   F/r   = (2 (6 V) + a) / r^2           (= 24 eps s6 (2 s6 - 1) / r^2)
// and with the switch S = t^2 (t P(t)), P = 10 - 15 t + 6 t^2, dS/dr / r =
// -60 isw t^2 (1 - t)^2 (isw = 1 / (rc^2 - r_on^2)):
//   F_s/r = F/r S - V dS/dr / r = t^2 (F/r t P + 10 isw (6 V) (1 - t)^2).
// t = sat(rc^2 isw - r^2 isw) is one fused multiply-add (sw_c0 = rc^2 isw);
// its rounding can leave t ~ 1e-7 just beyond r_c, where S ~ 1e-20.
// WM: the axes that take the minimum image (face_axes of the warp's particles).
template <bool ENERGY, bool SWITCH, int WM>
__device__ __forceinline__ void lj_pair_step(const PhysDev& d, const float2* __restrict__ row, float4 pi, float4 pj,
                                             float& px, float& py, float& pz, float& e_i, float& w_i) {
    const float dx = (WM & 1) ? mimg(pj.x - pi.x, d.L, d.invL) : pj.x - pi.x;
    const float dy = (WM & 2) ? mimg(pj.y - pi.y, d.L, d.invL) : pj.y - pi.y;
    const float dz = (WM & 4) ? mimg(pj.z - pi.z, d.L, d.invL) : pj.z - pi.z;
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    const float2 tab = row[__float_as_int(pj.w)];
    const float inv = rcp_approx(r2);
    const float s2 = tab.x * inv;
    const float s6 = s2 * s2 * s2;
    const float a = tab.y * s6;
    const float v6 = fmaf(a, s6, -a);          // 6 V
    float fr = inv * fmaf(v6, 2.f, a);          // F / r
    float v = 0.f;
    if (SWITCH) {
        const float t = __saturatef(fmaf(r2, -d.inv_sw_d, d.sw_c0));
        const float omt = 1.f - t;
        const float tp = t * fmaf(fmaf(t, 6.f, -15.f), t, 10.f);
        const float t2 = t * t;
        const float z = fmaf(v6 * d.sw_k10, omt * omt, fr * tp);
        if (ENERGY) v = v6 * (1.f / 6.f) * (t2 * tp);
        fr = t2 * z;
    } else {
        const bool in = r2 < d.rc2;
        if (ENERGY) {   // shifted to zero at r_c
            const float src2 = tab.x * d.inv_rc2, src6 = src2 * src2 * src2;
            v = in ? (v6 - tab.y * (src6 * src6 - src6)) * (1.f / 6.f) : 0.f;
        }
        fr = in ? fr : 0.f;
    }
    px = fmaf(-fr, dx, px);
    py = fmaf(-fr, dy, py);
    pz = fmaf(-fr, dz, pz);
    if (ENERGY) {
        e_i += 0.5f * v;
        w_i += 0.5f * fr * r2;
    }
}

}  // namespace lima
