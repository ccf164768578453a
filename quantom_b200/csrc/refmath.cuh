// Device math with the reference's float semantics (LIMA_MD Quantom/Quantom/
// QuantomTypes.cuh:33-168 Float3, Engine.cuh:24-45 LIMAENG, Engine.cu:461-869
// device functions).  Translation units that include this are compiled with
// -fmad=false so that a*b+c is never contracted, matching the reference's
// host-compiled neighbour-list code bit for bit and its kernels to rounding.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lima_abi.h"

namespace refm {

struct F3 {
    float x, y, z;
};

__device__ __forceinline__ F3 mk(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 mk4(float4 v) { return F3{v.x, v.y, v.z}; }
__device__ __forceinline__ float4 to4(F3 a, float w = 0.f) { return make_float4(a.x, a.y, a.z, w); }
__device__ __forceinline__ F3 add(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 sub(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
// Float3::operator*(const double): product in double, narrowed to float.
__device__ __forceinline__ F3 muld(F3 a, double s) {
    return F3{(float)((double)a.x * s), (float)((double)a.y * s), (float)((double)a.z * s)};
}
// The same operator when the scalar is a float: the double product of two
// floats is exact, so narrowing it equals the IEEE float product.
__device__ __forceinline__ F3 mulf(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float len2(F3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
__device__ __forceinline__ float len(F3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
    return F3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ F3 norm(F3 a) {
    float l = len(a);
    if (l != 0.f) return mulf(a, 1.f / l);
    return F3{0.f, 0.f, 0.f};
}
__device__ __forceinline__ float get_angle(F3 a, F3 b) {   // Float3::getAngle, QuantomTypes.cuh:74-83
    float val = dot(a, b) / (len(a) * len(b));
    val = val > 1.f ? 1.f : val;
    val = val < -1.f ? -1.f : val;
    return acosf(val);
}

// LIMAENG::applyHyperpos (Engine.cuh:24-30): the second comparison sees the
// first update, as in the reference.
__device__ __forceinline__ void hyperpos1(float s, float& m, float L, float Lh) {
    m += L * (float)((s - m) > Lh);
    m -= L * (float)((s - m) < -Lh);
}
__device__ __forceinline__ void hyperpos(const F3& s, F3& m, float L, float Lh) {
    hyperpos1(s.x, m.x, L, Lh);
    hyperpos1(s.y, m.y, L, Lh);
    hyperpos1(s.z, m.z, L, Lh);
}
// applyPBC (Engine.cu:461-466)
__device__ __forceinline__ void apply_pbc(F3& p, float L) {
    p.x += L * (float)(p.x < 0.f);
    p.x -= L * (float)(p.x > L);
    p.y += L * (float)(p.y < 0.f);
    p.y -= L * (float)(p.y > L);
    p.z += L * (float)(p.z < 0.f);
    p.z -= L * (float)(p.z > L);
}
// Engine::neighborWithinCutoff (Engine.cu:146-151)
__device__ __forceinline__ bool within(F3 a, F3 b, float C, float offset, float L, float Lh) {
    hyperpos(a, b, L, Lh);
    return len(sub(a, b)) < (C + offset);
}

// calcLJForce (Engine.cu:475-522): force on p0 from p1, no cutoff, no energy.
__device__ __forceinline__ F3 lj_force(F3 p0, F3 p1, float sigma, float epsilon) {
    F3 d = sub(p1, p0);
    float d2 = len2(d);
    float s = sigma * sigma / d2;
    s = s * s * s;
    float fs = 24.f * epsilon * s / d2 * (1.f - 2.f * s);
    return mulf(d, fs);
}
__device__ __forceinline__ float mix_sigma(float a, float b) { return (a + b) * 0.5f; }
__device__ __forceinline__ float eps_arith(float a, float b) { return (a + b) * 0.5f; }   // x*0.5 is exact in either precision
__device__ __forceinline__ float eps_geo(float a, float b) { return sqrtf(a * b); }

// calcPairbondForces (Engine.cu:525-548)
__device__ __forceinline__ void pairbond(F3 a, F3 b, float b0, float kb, F3* res, float& potE) {
    F3 diff = sub(a, b);
    double error = (double)(len(diff) - b0);
    potE = (float)((double)potE + 0.5 * (double)kb * (error * error));
    diff = norm(diff);
    double fs = (double)(-kb) * error;
    res[0] = muld(diff, fs);
    res[1] = muld(muld(diff, fs), -1.0);
}
// calcAnglebondForces (Engine.cu:552-578)
__device__ __forceinline__ void anglebond(F3 l, F3 m, F3 r, float theta0, float k, F3* res, float& potE) {
    F3 v1 = sub(l, m), v2 = sub(r, m);
    F3 n1 = cross(v1, v2), n2 = cross(v2, v1);
    F3 in1 = norm(cross(v1, n2)), in2 = norm(cross(v2, n1));
    double angle = (double)get_angle(v1, v2);
    double error = angle - (double)theta0;
    potE = (float)((double)potE + 0.5 * (double)k * error * error * 0.5);
    double fs = (double)k * error;
    res[0] = muld(in1, fs);
    res[2] = muld(in2, fs);
    res[1] = muld(add(res[0], res[2]), -1.0);
}
// calcDihedralbondForces (Engine.cu:580-637): potE assigned, forces on the
// middle atoms split 50/50.
__device__ __forceinline__ void dihedral(F3 l, F3 lm, F3 rm, F3 r, float phi0, float k, int n, F3* res,
                                         float& potE) {
    F3 n1 = norm(cross(sub(l, lm), sub(rm, lm)));
    F3 n2 = norm(cross(sub(lm, rm), sub(r, rm)));
    float torsion = get_angle(n1, n2);
    if (len(sub(add(l, n1), r)) < len(sub(sub(l, n1), r))) {
        n2.x *= -1.f; n2.y *= -1.f; n2.z *= -1.f;
    } else {
        n1.x *= -1.f; n1.y *= -1.f; n1.z *= -1.f;
    }
    float arg = (float)n * torsion - phi0;
    float fs = k * sinf(arg);
    potE = k * (1.f - cosf(arg));
    res[0] = mulf(n1, fs);
    res[3] = mulf(n2, fs);
    res[1] = mulf(mulf(add(res[0], res[3]), -1.f), 0.5f);
    res[2] = res[1];
}
// integratePosition (Engine.cu:849-869)
__device__ __forceinline__ void integrate(F3& pos, F3& prev, F3 force, double mass, double dt, float lambda,
                                          float L, float Lh) {
    F3 temp = pos;
    hyperpos(pos, prev, L, Lh);
    double mts = dt / mass * dt;
    pos = add(sub(mulf(pos, 2.f), prev), muld(force, mts));
    prev = temp;
    F3 delta = sub(pos, prev);
    pos = add(prev, mulf(delta, lambda));
}
// LJ_Ignores::ignore (Bodies.cuh:191-197)
__device__ __forceinline__ bool ignored(const lima_lj_ignores& ig, int local, int cid) {
    const int n = ig.n_ignores;
    for (int i = 0; i < n; i++)
        if (ig.local_ids[i] == (uint8_t)local && ig.compound_ids[i] == (uint8_t)cid) return true;
    return false;
}

}  // namespace refm
