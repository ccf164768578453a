// Trajectory loss and its parameter gradient on the physics path (adjoint
// of the unrolled velocity-Verlet steps; the algebra is in adjoint.cuh).
//
// Passes over the state of step n (8 lanes per particle over the Verlet list,
// as the forward pair kernel):
//   k_loss_pairs   LJ energy and the RDF-bin occupancies h_b(x_n)
//   k_adj_bonded   per bonded term: its forces as dual numbers along w, so the
//                  tangent is the term's Hessian-vector product; loss gradient
//                  and the bonded-scale derivatives
//   k_adj_pair     per particle: sum over pairs of J_ij (w_i - w_j) with
//                  J = f I + 2 f' d d^T (f(r^2) the switched LJ force / r),
//                  the loss gradient (energy and RDF terms), sigma / epsilon
//                  derivatives chained through Lorentz-Berthelot; updates dL/dx
// Every per-lane sum is FP32; the energies, occupancies and parameter
// derivatives are reduced per block in FP64.
#include <algorithm>
#include <cmath>

#include "adjoint.cuh"
#include "physkern.cuh"
#include "refdev.cuh"

namespace lima {
namespace {

constexpr int kAdjTB = 256;   // 32 particles x kGroup lanes
// Inside a checkpoint segment the pair list is rebuilt in place (particle
// order kept) every kListEpoch steps; the backward pass rebuilds the list of
// each epoch from its first state, which reproduces the forward's lists.
constexpr int kListEpoch = 10;

__device__ __forceinline__ float mimg_a(float d, float L, float invL) { return d - L * rintf(d * invL); }

__device__ __forceinline__ uint32_t nl_at(const PhysDev& d, int i, int k) {
    return nl_word((uint32_t)d.n_pad, (uint32_t)i, (uint32_t)k);
}

__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Quadratic B-spline bins of a distance: bins k0, k0+1, k0+2 with weights w
// and d w / d r (bin b is centred at (b + 1/2) dr).
__device__ __forceinline__ void bspline3(float r, float inv_dr, int& k0, float w[3], float dw[3]) {
    const float u = r * inv_dr - 0.5f;
    const float kc = rintf(u);
    const float t = u - kc;
    k0 = (int)kc - 1;
    w[0] = 0.5f * (0.5f - t) * (0.5f - t);
    w[1] = 0.75f - t * t;
    w[2] = 0.5f * (0.5f + t) * (0.5f + t);
    dw[0] = -(0.5f - t) * inv_dr;
    dw[1] = -2.f * t * inv_dr;
    dw[2] = (0.5f + t) * inv_dr;
}

// Switched LJ with 4 eps factored out: phi = 4 eps * ph, F_i = 4 eps * f * (x_i - x_j).
// Returns ph, f, df/d(r^2) and their sigma derivatives.
struct LJ1 {
    float ph, f, fp, dph_ds, df_ds;
};
__device__ __forceinline__ LJ1 lj1(const PhysDev& d, float r2, float sig2) {
    const float u = 1.f / r2;
    const float s2 = sig2 * u, s6 = s2 * s2 * s2, s12 = s6 * s6;
    const float ph = s12 - s6;
    const float f = 6.f * u * (2.f * s12 - s6);
    const float fp = -6.f * u * u * (14.f * s12 - 4.f * s6);
    const float isig = rsqrtf(sig2);
    const float dph_ds = (12.f * s12 - 6.f * s6) * isig;
    const float df_ds = 6.f * u * (24.f * s12 - 6.f * s6) * isig;
    // C2 switch S(t), t = (rc^2 - r^2) / (rc^2 - r_on^2)
    const float t = __saturatef((d.rc2 - r2) * d.inv_sw_d);
    const float omt = 1.f - t;
    const float S = t * t * t * fmaf(t, fmaf(6.f, t, -15.f), 10.f);
    const float Sp = -30.f * t * t * omt * omt * d.inv_sw_d;
    const float Spp = 60.f * t * omt * (1.f - 2.f * t) * d.inv_sw_d * d.inv_sw_d;
    LJ1 o;
    o.ph = ph * S;
    o.f = f * S - 2.f * ph * Sp;
    o.fp = fp * S + 2.f * f * Sp - 2.f * ph * Spp;
    o.dph_ds = dph_ds * S;
    o.df_ds = df_ds * S - 2.f * dph_ds * Sp;
    return o;
}

struct AdjArgs {
    float dt;
    float le;          // w_energy / (N T) where this state carries a loss term, else 0
    float lr;          // 2 w_rdf / (N T) likewise
    float inv_dr;
    float supp2;       // (r_max + dr)^2
    int n_bins;
    int n_types;
    float4* lam_x;
    const float4* wv;
    float4* adj_term;
    const float* par;  // sigma[n_types], epsilon[n_types], scales
    double* gtheta;
    double2* gterm;    // per bonded term: dL/dc, dL/dk (c = r0 | theta0 | phi0)
};

// --------------------------------------------------------------- loss pass --
// The block's occupancies accumulate in shared memory as 64-bit fixed point
// in units of 2^-32 (each half weight, at most 0.375, converted from FP32;
// integer sums do not depend on their order, so the block's sums are
// deterministic), then go to FP64 once per bin and block.
constexpr double kHistUnit = 1.0 / 4294967296.0;   // 2^-32

__global__ void __launch_bounds__(kAdjTB) k_loss_pairs(PhysDev d, const float4* __restrict__ pos, int n_bins,
                                                       float inv_dr, float supp2, double inv_n,
                                                       double* __restrict__ U_out, double* __restrict__ h_out) {
    __shared__ unsigned long long s_hist[LIMA_LOSS_MAX_BINS];
    __shared__ double s_e[kAdjTB / 32];
    __shared__ float2 s_tab[kMaxTypes * kMaxTypes];
    const int nt2 = d.n_types * d.n_types;
    for (int q = threadIdx.x; q < nt2; q += blockDim.x) s_tab[q] = d.lj_table[q];
    for (int b = threadIdx.x; b < n_bins; b += blockDim.x) s_hist[b] = 0ull;
    __syncthreads();
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) / kGroup;
    const int g = threadIdx.x % kGroup;
    float e = 0.f;
    if (i < d.n) {
        const float4 pi = pos[i];
        const int ti = __float_as_int(pi.w);
        const int cnt = (int)d.nl_cnt[i];
        for (int k = g; k < cnt; k += kGroup) {
            const uint32_t j = nl_load(d, nl_at(d, i, k));
            const float4 pj = pos[j];
            const float dx = mimg_a(pi.x - pj.x, d.L, d.invL), dy = mimg_a(pi.y - pj.y, d.L, d.invL),
                        dz = mimg_a(pi.z - pj.z, d.L, d.invL);
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < d.rc2) {
                const float2 tab = s_tab[ti * d.n_types + __float_as_int(pj.w)];
                e += 0.5f * tab.y * lj1(d, r2, tab.x).ph;
            }
            if (r2 < supp2) {
                int k0;
                float w[3], dw[3];
                bspline3(sqrtf(r2), inv_dr, k0, w, dw);
#pragma unroll
                for (int q = 0; q < 3; q++)
                    if (k0 + q >= 0 && k0 + q < n_bins)   // each pair is seen from both ends: half weight
                        atomicAdd(&s_hist[k0 + q], (unsigned long long)__float2ull_rn(0.5f * w[q] * 4294967296.f));
            }
        }
    }
    // energy: FP64 warp sums, then the block's warps in a fixed order
    const double ew = warp_sum_d((double)e);
    if ((threadIdx.x & 31) == 0) s_e[threadIdx.x >> 5] = ew;
    __syncthreads();
    for (int b = threadIdx.x; b < n_bins; b += blockDim.x)
        if (s_hist[b]) atomicAdd(&h_out[b], (double)s_hist[b] * kHistUnit * inv_n);
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int q = 0; q < kAdjTB / 32; q++) v += s_e[q];
        if (v != 0.0) atomicAdd(U_out, v);
    }
}

// ---------------------------------------------------------- bonded (duals) --
struct Dual {
    float v, t;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.t + b.t}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.t - b.t}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.t}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.v * b.t + a.t * b.v}; }
__device__ __forceinline__ Dual operator*(float s, Dual a) { return {s * a.v, s * a.t}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    const float q = a.v / b.v;
    return {q, (a.t - q * b.t) / b.v};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
    const float s = sqrtf(a.v);
    return {s, 0.5f * a.t / s};
}
__device__ __forceinline__ Dual datan2(Dual y, Dual x) {
    return {atan2f(y.v, x.v), (x.v * y.t - y.v * x.t) / (x.v * x.v + y.v * y.v)};
}
__device__ __forceinline__ Dual dsin(Dual a) { return {sinf(a.v), cosf(a.v) * a.t}; }
__device__ __forceinline__ Dual dcos(Dual a) { return {cosf(a.v), -sinf(a.v) * a.t}; }
__device__ __forceinline__ Dual dmaxf(Dual a, float b) { return a.v > b ? a : Dual{b, 0.f}; }

struct D3 {
    Dual x, y, z;
};
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator-(D3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ D3 operator*(Dual s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ Dual dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// separation b - a (minimum image on the value, tangent passes through)
__device__ __forceinline__ D3 sep(const PhysDev& d, float4 a, float4 wa, float4 b, float4 wb) {
    return {{mimg_a(b.x - a.x, d.L, d.invL), wb.x - wa.x},
            {mimg_a(b.y - a.y, d.L, d.invL), wb.y - wa.y},
            {mimg_a(b.z - a.z, d.L, d.invL), wb.z - wa.z}};
}
__device__ __forceinline__ Dual cst(float v) { return {v, 0.f}; }

// MODE 0: bonded energy of the state into *U_out.  MODE 1: adjoint contributions.
// Every term's forces are F_q = g G_q: a scalar g that carries the constants
// (bond: -k (r - r0); angle: k (theta - theta0); dihedral: dV/dphi =
// -k n sin(n phi - phi0)) times directions G_q that depend on the positions
// only.  The constants' derivatives of the loss at this state are then
//   dL/dc = dt (dg/dc) sum_q w_q . G_q + le dE/dc     (c = r0 | theta0 | phi0, k)
// and go to the term's own FP64 accumulator (one thread per term: no atomics,
// the same order every run).
template <int MODE>
__global__ void __launch_bounds__(kAdjTB) k_adj_bonded(PhysDev d, const float4* __restrict__ po, AdjArgs a,
                                                       int hvp, double* U_out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = d.n_bonds, na = d.n_angles, nd = d.n_dih;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    auto W = [&](int orig) { return (MODE == 1 && hvp) ? a.wv[d.sorted_of_orig[orig]] : zero; };
    int n_at = 0, slot0 = 0;
    bool live = false;
    int at[4] = {0, 0, 0, 0};
    D3 G[4];
    Dual g = cst(0.f), E = cst(0.f);
    float dg_dc = 0.f, dg_dk = 0.f, dE_dc = 0.f, dE_dk = 0.f;
    if (t < nb) {
        live = true;
        const int4 ix = d.bond_idx[t];
        const float2 par = d.bond_par[t];
        at[0] = ix.x, at[1] = ix.y, n_at = 2, slot0 = 2 * t;
        const D3 r = sep(d, po[ix.x], W(ix.x), po[ix.y], W(ix.y));
        const Dual rr = dsqrt(dot(r, r));
        const Dual dr = rr - cst(par.x);
        G[1] = (cst(1.f) / rr) * r;   // F_j = -k (r - r0) r / |r|
        G[0] = -G[1];
        g = (-par.y) * dr;
        E = (0.5f * par.y) * (dr * dr);
        dg_dc = par.y, dg_dk = -dr.v;
        dE_dc = -par.y * dr.v, dE_dk = 0.5f * dr.v * dr.v;
    } else if (t < nb + na) {
        live = true;
        const int q = t - nb;
        const int4 ix = d.angle_idx[q];
        const float2 par = d.angle_par[q];
        at[0] = ix.x, at[1] = ix.y, at[2] = ix.z, n_at = 3, slot0 = 2 * nb + 3 * q;
        const D3 u = sep(d, po[ix.y], W(ix.y), po[ix.x], W(ix.x));   // x_i - x_j
        const D3 v = sep(d, po[ix.y], W(ix.y), po[ix.z], W(ix.z));   // x_k - x_j
        const Dual uu = dot(u, u), vv = dot(v, v);
        const Dual nu = dsqrt(uu), nv = dsqrt(vv);
        const D3 c = cross(u, v);
        const Dual sn = dsqrt(dot(c, c));
        const Dual cs = dot(u, v);
        const Dual th = datan2(sn, cs);
        const Dual dth = th - cst(par.x);
        const Dual inuv = cst(1.f) / (nu * nv);
        const Dual cosv = cs * inuv;
        const Dual is = cst(1.f) / dmaxf(sn * inuv, 1e-6f);
        G[0] = is * (inuv * v - (cosv / uu) * u);
        G[2] = is * (inuv * u - (cosv / vv) * v);
        G[1] = -(G[0] + G[2]);
        g = par.y * dth;
        E = (0.5f * par.y) * (dth * dth);
        dg_dc = -par.y, dg_dk = dth.v;
        dE_dc = -par.y * dth.v, dE_dk = 0.5f * dth.v * dth.v;
    } else if (t < nb + na + nd) {
        live = true;
        const int q = t - nb - na;
        const int4 ix = d.dih_idx[q];
        const float4 par = d.dih_par[q];
        at[0] = ix.x, at[1] = ix.y, at[2] = ix.z, at[3] = ix.w, n_at = 4, slot0 = 2 * nb + 3 * na + 4 * q;
        const D3 b1 = sep(d, po[ix.x], W(ix.x), po[ix.y], W(ix.y));
        const D3 b2 = sep(d, po[ix.y], W(ix.y), po[ix.z], W(ix.z));
        const D3 b3 = sep(d, po[ix.z], W(ix.z), po[ix.w], W(ix.w));
        const D3 m1 = cross(b1, b2), m2 = cross(b2, b3);
        const Dual m1m1 = dot(m1, m1), m2m2 = dot(m2, m2), b2b2 = dot(b2, b2);
        const Dual nb2 = dsqrt(b2b2);
        const Dual phi = datan2(nb2 * dot(b1, m2), dot(m1, m2));
        const Dual arg = par.z * phi - cst(par.x);
        const Dual sa = dsin(arg);
        const D3 hi = (nb2 / m1m1) * m1, hl = -((nb2 / m2m2) * m2);
        const Dual p = dot(b1, b2) / b2b2, r = dot(b3, b2) / b2b2;
        G[0] = hi;
        G[1] = -hi - p * hi + r * hl;
        G[2] = -hl + p * hi - r * hl;
        G[3] = hl;
        g = (-par.y * par.z) * sa;
        E = par.y * (cst(1.f) + dcos(arg));
        const float ca = cosf(arg.v);
        dg_dc = par.y * par.z * ca, dg_dk = -par.z * sa.v;
        dE_dc = par.y * sa.v, dE_dk = 1.f + ca;
    }
    // reductions
    double eu = 0.0;
    if (live) {
        if (MODE == 0) {
            eu = (double)E.v;
        } else {
            float sg = 0.f;   // sum_q w_q . G_q
            for (int q = 0; q < n_at; q++) {
                const float4 wq = W(at[q]);
                const D3 f = g * G[q];
                if (hvp) sg += wq.x * G[q].x.v + wq.y * G[q].y.v + wq.z * G[q].z.v;
                const float4 o = make_float4((hvp ? a.dt * f.x.t : 0.f) - a.le * f.x.v,
                                             (hvp ? a.dt * f.y.t : 0.f) - a.le * f.y.v,
                                             (hvp ? a.dt * f.z.t : 0.f) - a.le * f.z.v, 0.f);
                a.adj_term[slot0 + q] = o;
            }
            double2 acc = a.gterm[t];
            acc.x += (double)(a.dt * dg_dc * sg + a.le * dE_dc);
            acc.y += (double)(a.dt * dg_dk * sg + a.le * dE_dk);
            a.gterm[t] = acc;
        }
    }
    if (MODE == 0) {
        __shared__ double s_b[kAdjTB / 32];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        const double v0 = warp_sum_d(eu);
        if (lane == 0) s_b[w] = v0;
        __syncthreads();
        if (threadIdx.x == 0) {
            double v = 0.0;
            for (int q = 0; q < (int)(blockDim.x >> 5); q++) v += s_b[q];
            if (v != 0.0) atomicAdd(U_out, v);
        }
    }
}

// --------------------------------------------------------------- adjoint ---
// mu = lv + dt lx;  lv <- mu;  w = mu / m
__global__ void k_adj_prep(PhysDev d, AdjArgs a, float4* __restrict__ lam_v, float4* __restrict__ wv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const float4 lx = a.lam_x[i], lv = lam_v[i];
    const float im = d.vel[i].w;
    const float mx = lv.x + a.dt * lx.x, my = lv.y + a.dt * lx.y, mz = lv.z + a.dt * lx.z;
    lam_v[i] = make_float4(mx, my, mz, 0.f);
    wv[i] = make_float4(mx * im, my * im, mz * im, 0.f);
}

template <bool HVP, bool LOSS>
__global__ void __launch_bounds__(kAdjTB) k_adj_pair(PhysDev d, const float4* __restrict__ pos, AdjArgs a,
                                                     const double* __restrict__ hist_n,
                                                     const double* __restrict__ target) {
    __shared__ float2 s_tab[kMaxTypes * kMaxTypes];
    __shared__ float s_c[LIMA_LOSS_MAX_BINS];
    __shared__ float s_par[2 * kMaxTypes];
    __shared__ double s_g[2 * kMaxTypes];
    const int nt = a.n_types;
    for (int q = threadIdx.x; q < nt * nt; q += blockDim.x) s_tab[q] = d.lj_table[q];
    for (int q = threadIdx.x; q < 2 * nt; q += blockDim.x) {
        s_par[q] = a.par[q];
        s_g[q] = 0.0;
    }
    if (LOSS)
        for (int q = threadIdx.x; q < a.n_bins; q += blockDim.x) s_c[q] = (float)(hist_n[q] - target[q]);
    __syncthreads();
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) / kGroup;
    const int g = threadIdx.x % kGroup;
    float hx = 0.f, hy = 0.f, hz = 0.f;   // dt * sum J (w_i - w_j)  (dt applied at the end)
    float fx = 0.f, fy = 0.f, fz = 0.f;   // LJ force on i
    float rx = 0.f, ry = 0.f, rz = 0.f;   // sum G(r) d
    float gs_a = 0.f, ge_a = 0.f;         // parameter derivatives landing on i's type
    float gs_b[kMaxTypes], ge_b[kMaxTypes];
    for (int q = 0; q < nt; q++) gs_b[q] = ge_b[q] = 0.f;
    int ti = 0;
    if (i < d.n) {
        const float4 pi = pos[i];
        ti = __float_as_int(pi.w);
        const float4 wi = HVP ? a.wv[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float eps_a = s_par[nt + ti];
        const int cnt = (int)d.nl_cnt[i];
        for (int k = g; k < cnt; k += kGroup) {
            const uint32_t j = nl_load(d, nl_at(d, i, k));
            const float4 pj = pos[j];
            const float dx = mimg_a(pi.x - pj.x, d.L, d.invL), dy = mimg_a(pi.y - pj.y, d.L, d.invL),
                        dz = mimg_a(pi.z - pj.z, d.L, d.invL);
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 >= d.rc2) continue;
            const int tj = __float_as_int(pj.w);
            const float2 tab = s_tab[ti * nt + tj];
            const float e4 = tab.y;   // 4 eps_ij
            const LJ1 l = lj1(d, r2, tab.x);
            float dsig = 0.f, deps4 = 0.f;   // d/d sigma_ij and d/d (4 eps_ij) of this visit
            if (HVP) {
                const float4 wj = a.wv[j];
                const float ux = wi.x - wj.x, uy = wi.y - wj.y, uz = wi.z - wj.z;
                const float du = dx * ux + dy * uy + dz * uz;
                const float c1 = e4 * l.f, c2 = 2.f * e4 * l.fp * du;
                hx += c1 * ux + c2 * dx;
                hy += c1 * uy + c2 * dy;
                hz += c1 * uz + c2 * dz;
                // half of dt (w_i - w_j) . dF_i/dtheta (the other half comes from j's visit)
                dsig += 0.5f * a.dt * du * e4 * l.df_ds;
                deps4 += 0.5f * a.dt * du * l.f;
            }
            if (LOSS) {
                fx += e4 * l.f * dx;
                fy += e4 * l.f * dy;
                fz += e4 * l.f * dz;
                dsig += 0.5f * a.le * e4 * l.dph_ds;
                deps4 += 0.5f * a.le * l.ph;
                if (a.lr != 0.f && r2 < a.supp2) {
                    const float r = sqrtf(r2);
                    int k0;
                    float w[3], dw[3];
                    bspline3(r, a.inv_dr, k0, w, dw);
                    float G = 0.f;
#pragma unroll
                    for (int q = 0; q < 3; q++)
                        if (k0 + q >= 0 && k0 + q < a.n_bins) G += s_c[k0 + q] * dw[q];
                    G /= r;
                    rx += G * dx;
                    ry += G * dy;
                    rz += G * dz;
                }
            }
            // chain to the per-type parameters: sigma_ij = (s_a + s_b)/2, eps_ij = sqrt(e_a e_b)
            const float eps_ab = 0.25f * e4, eps_b = s_par[nt + tj];
            const float de = 4.f * deps4;   // d/d eps_ij
            gs_a += 0.5f * dsig;
            gs_b[tj] += 0.5f * dsig;
            if (eps_a > 0.f) ge_a += de * eps_ab / (2.f * eps_a);
            if (eps_b > 0.f) ge_b[tj] += de * eps_ab / (2.f * eps_b);
        }
    }
#pragma unroll
    for (int o = kGroup / 2; o > 0; o >>= 1) {
        hx += __shfl_xor_sync(0xffffffffu, hx, o);
        hy += __shfl_xor_sync(0xffffffffu, hy, o);
        hz += __shfl_xor_sync(0xffffffffu, hz, o);
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
        rx += __shfl_xor_sync(0xffffffffu, rx, o);
        ry += __shfl_xor_sync(0xffffffffu, ry, o);
        rz += __shfl_xor_sync(0xffffffffu, rz, o);
    }
    if (i < d.n && g == 0) {
        float bx = 0.f, by = 0.f, bz = 0.f;
        const uint32_t oi = d.orig_of_sorted[i];
        if (oi < (uint32_t)d.n_cp)
            for (uint32_t q = d.bterm_off[oi]; q < d.bterm_off[oi + 1]; q++) {
                const float4 tf = a.adj_term[d.bterm_slot[q]];
                bx += tf.x;
                by += tf.y;
                bz += tf.z;
            }
        float4 lx = a.lam_x[i];
        lx.x += a.dt * hx - a.le * fx + a.lr * rx + bx;
        lx.y += a.dt * hy - a.le * fy + a.lr * ry + by;
        lx.z += a.dt * hz - a.le * fz + a.lr * rz + bz;
        a.lam_x[i] = lx;
    }
    // parameter derivatives: lane -> per-type slots -> block (FP64) -> global
    const int lane = threadIdx.x & 31;
    for (int q = 0; q < nt; q++) {
        float s = gs_b[q] + (q == ti ? gs_a : 0.f);
        float e = ge_b[q] + (q == ti ? ge_a : 0.f);
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_down_sync(0xffffffffu, s, o);
            e += __shfl_down_sync(0xffffffffu, e, o);
        }
        if (lane == 0) {
            if (s != 0.f) atomicAdd(&s_g[q], (double)s);
            if (e != 0.f) atomicAdd(&s_g[nt + q], (double)e);
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 2 * nt; q += blockDim.x)
        if (s_g[q] != 0.0) atomicAdd(&a.gtheta[q], s_g[q]);
}

// ---------------------------------------------------------- state moves ---
__global__ void k_save(PhysDev d, int cur, float4* __restrict__ x, float4* __restrict__ v) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.n) return;
    const uint32_t o = d.orig_of_sorted[k];
    x[o] = d.pos[cur][k];
    v[o] = d.vel[k];
}

// state in orig order; the next rebuild sorts it
__global__ void k_restore(PhysDev d, int cur, const float4* __restrict__ x, const float4* __restrict__ v) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= d.n) return;
    const float4 p = x[o];
    d.pos[cur][o] = p;
    d.vel[o] = v[o];
    d.orig_of_sorted[o] = (uint32_t)o;
    d.sorted_of_orig[o] = (uint32_t)o;
    if (o < d.n_cp) d.pos_orig[cur][o] = p;
}

__global__ void k_to_sorted(PhysDev d, const float4* __restrict__ in, float4* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < d.n) out[k] = in[d.orig_of_sorted[k]];
}

__global__ void k_to_orig(PhysDev d, const float4* __restrict__ in, float4* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < d.n) out[d.orig_of_sorted[k]] = in[k];
}

template <typename T>
T* grow(std::vector<void*>& allocs, size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    allocs.push_back(p);
    return static_cast<T*>(p);
}

bool ensure(const PhysDev& d, AdjBuffers& A, std::vector<void*>& allocs, int n_ckpt, int n_seg, int n_steps,
            int n_bins) {
    const size_t n = (size_t)d.n, np = (size_t)d.n_pad, ncp = (size_t)std::max(d.n_cp, 1);
    if (!A.lam_x) {
        A.lam_x = grow<float4>(allocs, np);
        A.lam_v = grow<float4>(allocs, np);
        A.wv = grow<float4>(allocs, np);
        A.lam_xo = grow<float4>(allocs, n);
        A.lam_vo = grow<float4>(allocs, n);
        A.adj_term = grow<float4>(allocs, (size_t)std::max(d.n_term_slots, 1));
        A.gtheta = grow<double>(allocs, 2 * kMaxTypes + kParKinds);
        A.par = grow<float>(allocs, 2 * kMaxTypes + kParKinds);
        A.cap_terms = std::max(d.n_bonds + d.n_angles + d.n_dih, 1);
        A.gterm = grow<double2>(allocs, (size_t)A.cap_terms);
        if (!A.lam_x || !A.lam_v || !A.wv || !A.lam_xo || !A.lam_vo || !A.adj_term || !A.gtheta || !A.par ||
            !A.gterm)
            return false;
    }
    if (n_ckpt > A.cap_ckpt) {
        A.ck_x = grow<float4>(allocs, n * n_ckpt);
        A.ck_v = grow<float4>(allocs, n * n_ckpt);
        if (!A.ck_x || !A.ck_v) return false;
        A.cap_ckpt = n_ckpt;
    }
    if (n_seg > A.cap_seg) {
        A.seg_x = grow<float4>(allocs, np * n_seg);
        A.seg_xo = grow<float4>(allocs, ncp * n_seg);
        if (!A.seg_x || !A.seg_xo) return false;
        A.cap_seg = n_seg;
    }
    if (n_steps > A.cap_steps || n_bins > A.cap_bins) {
        const int st = std::max(n_steps, A.cap_steps), nb = std::max(n_bins, A.cap_bins);
        A.U = grow<double>(allocs, (size_t)st + 1);
        A.hist = grow<double>(allocs, ((size_t)st + 1) * nb);
        A.target = grow<double>(allocs, nb);
        if (!A.U || !A.hist || !A.target) return false;
        A.cap_steps = st;
        A.cap_bins = nb;
    }
    return true;
}

int read_err(const PhysDev& d, cudaStream_t s) {
    int h = 0;
    cudaMemcpyAsync(&h, d.err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return h;
}

}  // namespace

// ------------------------------------------------------------- parameters --
namespace {
// Groups the loaded terms of one kind into types: the distinct constant sets
// (c, k, n) in ascending order; type_of[t] is term t's type.
void group_terms(const std::vector<float4>& terms, std::vector<int>& type_of, std::vector<float4>& type0) {
    auto less = [](const float4& a, const float4& b) {
        if (a.x != b.x) return a.x < b.x;
        if (a.y != b.y) return a.y < b.y;
        return a.z < b.z;
    };
    type0 = terms;
    std::sort(type0.begin(), type0.end(), less);
    type0.erase(std::unique(type0.begin(), type0.end(),
                            [](const float4& a, const float4& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }),
                type0.end());
    type_of.resize(terms.size());
    for (size_t t = 0; t < terms.size(); t++)
        type_of[t] = (int)(std::lower_bound(type0.begin(), type0.end(), terms[t], less) - type0.begin());
}
}  // namespace

void phys_params_init(const PhysDev& d, const lima_forcefield& ff, PhysParams& pp, cudaStream_t s) {
    pp.n_types = d.n_types;
    pp.sigma.resize(d.n_types);
    pp.epsilon.resize(d.n_types);
    for (int t = 0; t < d.n_types; t++) {
        pp.sigma[t] = ff.particle_parameters[t].sigma;
        pp.epsilon[t] = ff.particle_parameters[t].epsilon;
    }
    pp.scale[0] = pp.scale[1] = pp.scale[2] = 1.0;
    pp.bond0.resize(d.n_bonds);
    pp.angle0.resize(d.n_angles);
    pp.dih0.resize(d.n_dih);
    if (d.n_bonds) cudaMemcpyAsync(pp.bond0.data(), d.bond_par, sizeof(float2) * d.n_bonds, cudaMemcpyDeviceToHost, s);
    if (d.n_angles)
        cudaMemcpyAsync(pp.angle0.data(), d.angle_par, sizeof(float2) * d.n_angles, cudaMemcpyDeviceToHost, s);
    if (d.n_dih) cudaMemcpyAsync(pp.dih0.data(), d.dih_par, sizeof(float4) * d.n_dih, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    std::vector<float4> terms[kParKinds];
    for (const float2& b : pp.bond0) terms[kParBond].push_back(make_float4(b.x, b.y, 0.f, 0.f));
    for (const float2& a : pp.angle0) terms[kParAngle].push_back(make_float4(a.x, a.y, 0.f, 0.f));
    for (const float4& q : pp.dih0) terms[kParDihedral].push_back(make_float4(q.x, q.y, q.z, 0.f));
    for (int k = 0; k < kParKinds; k++) {
        group_terms(terms[k], pp.type_of[k], pp.type0[k]);
        pp.tc[k].resize(pp.type0[k].size());
        pp.tk[k].resize(pp.type0[k].size());
        for (size_t q = 0; q < pp.type0[k].size(); q++) {
            pp.tc[k][q] = pp.type0[k][q].x;
            pp.tk[k][q] = pp.type0[k][q].y;
        }
    }
}

void phys_params_get(const PhysParams& pp, double* theta) {
    const int nt = pp.n_types;
    for (int t = 0; t < nt; t++) {
        theta[t] = pp.sigma[t];
        theta[nt + t] = pp.epsilon[t];
    }
    for (int k = 0; k < kParKinds; k++) theta[2 * nt + k] = pp.scale[k];
    double* o = theta + 2 * nt + kParKinds;
    for (int k = 0; k < kParKinds; k++)
        for (size_t q = 0; q < pp.tc[k].size(); q++) {
            *o++ = pp.tc[k][q];
            *o++ = pp.tk[k][q];
        }
}

int phys_params_set(PhysDev& d, PhysParams& pp, const double* theta, std::string& msg, cudaStream_t s) {
    const int nt = pp.n_types;
    for (int t = 0; t < nt; t++)
        if (!(theta[t] > 0.0) || !(theta[nt + t] >= 0.0) || !std::isfinite(theta[t]) || !std::isfinite(theta[nt + t])) {
            msg = "sigma must be positive and epsilon non-negative (finite)";
            return LIMA_ERR_ARGUMENT;
        }
    for (int k = 0; k < kParKinds; k++)
        if (!(theta[2 * nt + k] >= 0.0) || !std::isfinite(theta[2 * nt + k])) {
            msg = "bonded scales must be finite and non-negative";
            return LIMA_ERR_ARGUMENT;
        }
    const double* tt = theta + 2 * nt + kParKinds;
    for (int k = 0, o = 0; k < kParKinds; k++)
        for (size_t q = 0; q < pp.tc[k].size(); q++, o += 2)
            if (!std::isfinite(tt[o]) || !std::isfinite(tt[o + 1]) || !(tt[o + 1] >= 0.0) ||
                (k == kParBond && !(tt[o] > 0.0))) {
                msg = "bonded type constants must be finite, force constants non-negative and bond lengths positive";
                return LIMA_ERR_ARGUMENT;
            }
    for (int t = 0; t < nt; t++) {
        pp.sigma[t] = theta[t];
        pp.epsilon[t] = theta[nt + t];
    }
    for (int k = 0; k < kParKinds; k++) pp.scale[k] = theta[2 * nt + k];
    for (int k = 0, o = 0; k < kParKinds; k++)
        for (size_t q = 0; q < pp.tc[k].size(); q++, o += 2) {
            pp.tc[k][q] = tt[o];
            pp.tk[k][q] = tt[o + 1];
        }
    std::vector<float2> tab((size_t)nt * nt);
    for (int a = 0; a < nt; a++)
        for (int b = 0; b < nt; b++) {
            const double sg = 0.5 * (pp.sigma[a] + pp.sigma[b]);
            const double ep = std::sqrt(pp.epsilon[a] * pp.epsilon[b]);
            tab[a * nt + b] = make_float2((float)(sg * sg), (float)(4.0 * ep));
        }
    // every term takes its type's constants; the force constant times the kind's scale
    std::vector<float2> bp(pp.bond0), ap(pp.angle0);
    std::vector<float4> dp(pp.dih0);
    for (size_t t = 0; t < bp.size(); t++) {
        const int q = pp.type_of[kParBond][t];
        bp[t] = make_float2((float)pp.tc[kParBond][q], (float)(pp.tk[kParBond][q] * pp.scale[kParBond]));
    }
    for (size_t t = 0; t < ap.size(); t++) {
        const int q = pp.type_of[kParAngle][t];
        ap[t] = make_float2((float)pp.tc[kParAngle][q], (float)(pp.tk[kParAngle][q] * pp.scale[kParAngle]));
    }
    for (size_t t = 0; t < dp.size(); t++) {
        const int q = pp.type_of[kParDihedral][t];
        dp[t].x = (float)pp.tc[kParDihedral][q];
        dp[t].y = (float)(pp.tk[kParDihedral][q] * pp.scale[kParDihedral]);
    }
    cudaMemcpyAsync(d.lj_table, tab.data(), sizeof(float2) * tab.size(), cudaMemcpyHostToDevice, s);
    if (!bp.empty()) cudaMemcpyAsync(d.bond_par, bp.data(), sizeof(float2) * bp.size(), cudaMemcpyHostToDevice, s);
    if (!ap.empty()) cudaMemcpyAsync(d.angle_par, ap.data(), sizeof(float2) * ap.size(), cudaMemcpyHostToDevice, s);
    if (!dp.empty()) cudaMemcpyAsync(d.dih_par, dp.data(), sizeof(float4) * dp.size(), cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    return cudaGetLastError() == cudaSuccess ? LIMA_OK : LIMA_ERR_CUDA;
}

// ------------------------------------------------------------------ passes --
namespace {

struct Runner {
    PhysDev d;           // copy with fixed-period list semantics (stale -> error)
    AdjBuffers& A;
    cudaStream_t s;
    int n_bins;
    float inv_dr, supp2;
    int tb = 256;
    int blocks_n() const { return (d.n + tb - 1) / tb; }
    int blocks_pair() const { return (int)(((size_t)d.n_pad * kGroup + kAdjTB - 1) / kAdjTB); }
    int blocks_terms() const { return std::max(1, (d.n_bonds + d.n_angles + d.n_dih + kAdjTB - 1) / kAdjTB); }

    void save(int cur, int k) { k_save<<<blocks_n(), tb, 0, s>>>(d, cur, A.ck_x + (size_t)k * d.n, A.ck_v + (size_t)k * d.n); }
    void restore(int cur, int k) {
        k_restore<<<blocks_n(), tb, 0, s>>>(d, cur, A.ck_x + (size_t)k * d.n, A.ck_v + (size_t)k * d.n);
        phys_rebuild(d, cur, s);
    }
    // energy and occupancies of the state in parity cur -> U[n], hist[n]
    void loss_pass(int cur, const float4* pos, const float4* po, int n) {
        k_loss_pairs<<<blocks_pair(), kAdjTB, 0, s>>>(d, pos, n_bins, inv_dr, supp2, 1.0 / d.n, A.U + n,
                                                     A.hist + (size_t)n * n_bins);
        AdjArgs a{};
        k_adj_bonded<0><<<blocks_terms(), kAdjTB, 0, s>>>(d, po, a, 0, A.U + n);
        (void)cur;
    }
};

double loss_of(const std::vector<double>& U, const std::vector<double>& H, const std::vector<double>& target, int T,
               int n_bins, int n, double we, double wr) {
    double L = 0.0;
    for (int k = 1; k <= T; k++) {
        double r = 0.0;
        for (int b = 0; b < n_bins; b++) {
            const double c = H[(size_t)k * n_bins + b] - (target.empty() ? 0.0 : target[b]);
            r += c * c;
        }
        L += we * U[k] / n + wr * r;
    }
    return L / T;
}

}  // namespace

int adj_rdf(const PhysDev& d, int cur, AdjBuffers& A, std::vector<void*>& allocs, int n_bins, float r_max, double* h,
            cudaStream_t s, std::string& msg) {
    if (n_bins < 1 || n_bins > LIMA_LOSS_MAX_BINS || !(r_max > 0.f)) {
        msg = "need 1 <= n_bins <= LIMA_LOSS_MAX_BINS and r_max > 0";
        return LIMA_ERR_ARGUMENT;
    }
    const float dr = r_max / n_bins;
    if (r_max + dr > d.rc * (1.f + 1e-6f)) {
        msg = "r_max + r_max/n_bins must not exceed the cutoff";
        return LIMA_ERR_ARGUMENT;
    }
    if (!ensure(d, A, allocs, 1, 1, 1, n_bins)) {
        msg = "cudaMalloc failed for the loss buffers";
        return LIMA_ERR_CUDA;
    }
    Runner R{d, A, s, n_bins, 1.f / dr, (r_max + dr) * (r_max + dr)};
    cudaMemsetAsync(A.hist, 0, sizeof(double) * n_bins, s);
    cudaMemsetAsync(A.U, 0, sizeof(double), s);
    R.loss_pass(cur, d.pos[cur], d.pos_orig[cur], 0);
    cudaMemcpyAsync(h, A.hist, sizeof(double) * n_bins, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return cudaGetLastError() == cudaSuccess ? LIMA_OK : LIMA_ERR_CUDA;
}

int adj_run(const PhysDev& d0, int cur, const PhysParams& pp, AdjBuffers& A, std::vector<void*>& allocs,
            const lima_loss_spec& spec, double* loss, double* grad, cudaStream_t s, std::string& msg) {
    const int T = spec.n_steps;
    if (T < 1 || spec.checkpoint_every < 1 || spec.n_bins < 1 || spec.n_bins > LIMA_LOSS_MAX_BINS ||
        !(spec.r_max > 0.f) || !std::isfinite(spec.w_energy) || !std::isfinite(spec.w_rdf)) {
        msg = "loss spec: need n_steps >= 1, checkpoint_every >= 1, 1 <= n_bins <= 128, r_max > 0, finite weights";
        return LIMA_ERR_ARGUMENT;
    }
    if (spec.w_rdf != 0.0 && !spec.rdf_target) {
        msg = "loss spec: rdf_target is required when w_rdf != 0";
        return LIMA_ERR_ARGUMENT;
    }
    const int nb = spec.n_bins;
    const float dr = spec.r_max / nb;
    if (spec.r_max + dr > d0.rc * (1.f + 1e-6f)) {
        msg = "loss spec: r_max + r_max/n_bins must not exceed the cutoff";
        return LIMA_ERR_ARGUMENT;
    }
    const int C = std::min(spec.checkpoint_every, T);
    const int K = (T + C - 1) / C;
    if (!ensure(d0, A, allocs, K, C + 1, T, nb)) {
        msg = "cudaMalloc failed for the adjoint buffers";
        return LIMA_ERR_CUDA;
    }
    PhysDev d = d0;
    d.dynamic_list = 0;
    Runner R{d, A, s, nb, 1.f / dr, (spec.r_max + dr) * (spec.r_max + dr)};
    std::vector<double> target(nb, 0.0);
    if (spec.rdf_target) target.assign(spec.rdf_target, spec.rdf_target + nb);
    cudaMemcpyAsync(A.target, target.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(A.U, 0, sizeof(double) * (T + 1), s);
    cudaMemsetAsync(A.hist, 0, sizeof(double) * (size_t)(T + 1) * nb, s);
    cudaMemsetAsync(A.gtheta, 0, sizeof(double) * (2 * kMaxTypes + kParKinds), s);
    cudaMemsetAsync(A.gterm, 0, sizeof(double2) * A.cap_terms, s);
    const int nt = pp.n_types;
    std::vector<float> par(2 * nt + kParKinds);
    for (int t = 0; t < nt; t++) {
        par[t] = (float)pp.sigma[t];
        par[nt + t] = (float)pp.epsilon[t];
    }
    for (int k = 0; k < kParKinds; k++) par[2 * nt + k] = (float)pp.scale[k];
    cudaMemcpyAsync(A.par, par.data(), sizeof(float) * par.size(), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(d.err, 0, sizeof(int), s);

    const int start_cur = cur;
    // the first launch or copy that failed, for the error message
    const char* fail_at = nullptr;
    cudaError_t fail_err = cudaSuccess;
    auto note = [&](const char* where) {
        if (fail_at) return;
        const cudaError_t e = cudaPeekAtLastError();
        if (e != cudaSuccess) {
            fail_at = where;
            fail_err = e;
        }
    };
    note("set-up copies");
    // forward: checkpoints at the start of every segment (re-sorted from orig
    // order there, so a recomputation reproduces the trajectory bit for bit)
    R.save(cur, 0);
    note("checkpoint save");
    for (int k = 0; k < K; k++) {
        const bool last = k == K - 1;
        if (grad && last) break;   // the backward pass recomputes the last segment anyway
        R.restore(cur, k);
        note("checkpoint restore and list rebuild");
        const int n0 = k * C, len = std::min(C, T - n0);
        for (int q = 0; q < len; q++) {
            if (q > 0 && q % kListEpoch == 0) phys_rebuild_inplace(d, d.pos[cur], s);
            note("in-place list rebuild");
            phys_step_kernels(d, cur, s, false);
            note("forward step kernels");
            cur ^= 1;
            if (!grad) R.loss_pass(cur, d.pos[cur], d.pos_orig[cur], n0 + q + 1);
            note("loss pass");
        }
        if (!last) R.save(cur, k + 1);
    }
    const double we = spec.w_energy, wr = spec.w_rdf;
    const float le = (float)(we / ((double)d.n * T)), lr = (float)(2.0 * wr / ((double)d.n * T));
    if (grad) {
        cudaMemsetAsync(A.lam_xo, 0, sizeof(float4) * d.n, s);
        cudaMemsetAsync(A.lam_vo, 0, sizeof(float4) * d.n, s);
        cudaMemsetAsync(A.lam_x, 0, sizeof(float4) * d.n_pad, s);
        cudaMemsetAsync(A.lam_v, 0, sizeof(float4) * d.n_pad, s);
        cudaMemsetAsync(A.wv, 0, sizeof(float4) * d.n_pad, s);
        AdjArgs a{};
        a.dt = (float)d.dt;
        a.inv_dr = R.inv_dr;
        a.supp2 = R.supp2;
        a.n_bins = nb;
        a.n_types = nt;
        a.lam_x = A.lam_x;
        a.wv = A.wv;
        a.adj_term = A.adj_term;
        a.par = A.par;
        a.gtheta = A.gtheta;
        a.gterm = A.gterm;
        const int pb = R.blocks_pair(), tbk = R.blocks_terms();
        for (int k = K - 1; k >= 0; k--) {
            const int n0 = k * C, len = std::min(C, T - n0);
            R.restore(cur, k);
            // recompute the segment, keeping every state and its loss terms
            cudaMemcpyAsync(A.seg_x, d.pos[cur], sizeof(float4) * d.n_pad, cudaMemcpyDeviceToDevice, s);
            if (d.n_cp)
                cudaMemcpyAsync(A.seg_xo, d.pos_orig[cur], sizeof(float4) * d.n_cp, cudaMemcpyDeviceToDevice, s);
            for (int q = 0; q < len; q++) {
                if (q > 0 && q % kListEpoch == 0) phys_rebuild_inplace(d, d.pos[cur], s);
                phys_step_kernels(d, cur, s, false);
                cur ^= 1;
                float4* xs = A.seg_x + (size_t)(q + 1) * d.n_pad;
                float4* xo = A.seg_xo + (size_t)(q + 1) * std::max(d.n_cp, 1);
                cudaMemcpyAsync(xs, d.pos[cur], sizeof(float4) * d.n_pad, cudaMemcpyDeviceToDevice, s);
                if (d.n_cp) cudaMemcpyAsync(xo, d.pos_orig[cur], sizeof(float4) * d.n_cp, cudaMemcpyDeviceToDevice, s);
                R.loss_pass(cur, xs, xo, n0 + q + 1);
            }
            k_to_sorted<<<R.blocks_n(), R.tb, 0, s>>>(d, A.lam_xo, A.lam_x);
            k_to_sorted<<<R.blocks_n(), R.tb, 0, s>>>(d, A.lam_vo, A.lam_v);
            // loss term of the segment's last state
            {
                const int q = len;
                a.le = le;
                a.lr = lr;
                const float4* xs = A.seg_x + (size_t)q * d.n_pad;
                const float4* xo = A.seg_xo + (size_t)q * std::max(d.n_cp, 1);
                k_adj_bonded<1><<<tbk, kAdjTB, 0, s>>>(d, xo, a, 0, nullptr);
                k_adj_pair<false, true><<<pb, kAdjTB, 0, s>>>(d, xs, a, A.hist + (size_t)(n0 + q) * nb, A.target);
            }
            int epoch = (len - 1) / kListEpoch;   // the list built last
            for (int q = len - 1; q >= 0; q--) {
                if (q / kListEpoch != epoch) {
                    epoch = q / kListEpoch;
                    phys_rebuild_inplace(d, A.seg_x + (size_t)epoch * kListEpoch * d.n_pad, s);
                }
                const bool has_loss = q >= 1;
                a.le = has_loss ? le : 0.f;
                a.lr = has_loss ? lr : 0.f;
                const float4* xs = A.seg_x + (size_t)q * d.n_pad;
                const float4* xo = A.seg_xo + (size_t)q * std::max(d.n_cp, 1);
                k_adj_prep<<<R.blocks_n(), R.tb, 0, s>>>(d, a, A.lam_v, A.wv);
                k_adj_bonded<1><<<tbk, kAdjTB, 0, s>>>(d, xo, a, 1, nullptr);
                if (has_loss)
                    k_adj_pair<true, true><<<pb, kAdjTB, 0, s>>>(d, xs, a, A.hist + (size_t)(n0 + q) * nb, A.target);
                else
                    k_adj_pair<true, false><<<pb, kAdjTB, 0, s>>>(d, xs, a, nullptr, A.target);
            }
            k_to_orig<<<R.blocks_n(), R.tb, 0, s>>>(d, A.lam_x, A.lam_xo);
            k_to_orig<<<R.blocks_n(), R.tb, 0, s>>>(d, A.lam_v, A.lam_vo);
        }
    }
    // loss value
    std::vector<double> U(T + 1), H((size_t)(T + 1) * nb);
    cudaMemcpyAsync(U.data(), A.U, sizeof(double) * (T + 1), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(H.data(), A.hist, sizeof(double) * H.size(), cudaMemcpyDeviceToHost, s);
    std::vector<double> g(2 * nt, 0.0);
    const int n_terms = d.n_bonds + d.n_angles + d.n_dih;
    std::vector<double2> gt((size_t)n_terms);
    if (grad) {
        cudaMemcpyAsync(g.data(), A.gtheta, sizeof(double) * g.size(), cudaMemcpyDeviceToHost, s);
        if (n_terms) cudaMemcpyAsync(gt.data(), A.gterm, sizeof(double2) * n_terms, cudaMemcpyDeviceToHost, s);
    }
    const int err = read_err(d, s);
    // leave the state as found: restore the first checkpoint into the starting parity
    if (cur != start_cur) cur = start_cur;
    R.restore(cur, 0);
    cudaStreamSynchronize(s);
    note("the passes");
    const cudaError_t last_err = cudaGetLastError();
    if (fail_at || last_err != cudaSuccess) {
        msg = std::string("CUDA error in the loss / adjoint passes (") + (fail_at ? fail_at : "the passes") + "): " +
              cudaGetErrorString(fail_at ? fail_err : last_err);
        return LIMA_ERR_CUDA;
    }
    if (err) {
        cudaMemsetAsync(d.err, 0, sizeof(int), s);
        cudaStreamSynchronize(s);
        msg = (err & ERR_BIT_LIST_STALE) ? "pair list went stale inside a checkpoint segment (raise skin or lower "
                                           "checkpoint_every)"
                                         : "device error during the loss / adjoint passes";
        return LIMA_ERR_NUMERIC;
    }
    *loss = loss_of(U, H, target, T, nb, d.n, we, wr);
    if (grad) {
        for (size_t q = 0; q < g.size(); q++) grad[q] = g[q];
        // bonded constants: the terms' derivatives summed per type in term
        // order; a term's force constant is s_kind * k_type
        double* gs = grad + 2 * nt;
        double* gty = gs + kParKinds;
        for (int q = 0; q < kParKinds + 2 * pp.n_term_types(); q++) gs[q] = 0.0;
        const int base[kParKinds] = {0, d.n_bonds, d.n_bonds + d.n_angles};
        const int cnt[kParKinds] = {d.n_bonds, d.n_angles, d.n_dih};
        for (int k = 0, off = 0; k < kParKinds; off += 2 * (int)pp.tc[k].size(), k++)
            for (int t = 0; t < cnt[k]; t++) {
                const double2 v = gt[base[k] + t];
                const int q = pp.type_of[k][t];
                gs[k] += v.y * pp.tk[k][q];
                gty[off + 2 * q] += v.x;
                gty[off + 2 * q + 1] += v.y * pp.scale[k];
            }
    }
    return LIMA_OK;
}

}  // namespace lima
