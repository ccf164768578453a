// Physics-semantics step: Lorentz-Berthelot LJ with cutoff (+ potential
// switch), harmonic bonds/angles, periodic dihedrals, velocity Verlet with an
// optional Berendsen thermostat.  FP32 forces; in MIXED precision the force
// sums are compensated per 32-neighbour chunk and positions/velocities carry
// FP32 low parts; energy, virial and kinetic-energy reductions and the
// thermostat scalar are FP64.
//
// Per step (two launches, captured in a CUDA graph):
//   k_bonded          one thread per bonded term -> term_force slots (+ energies)
//   k_pair_integrate  one thread per particle (slot order): Verlet-list LJ,
//                     gather of the particle's bonded term forces, kick-drift,
//                     FP64 KE; the last block to finish folds the FP64
//                     accumulators into e_last and computes the next lambda.
// Every nlist_period steps: sort particles by (coarse cell, 4x4x4 Morton
// sub-cell), permute state, rebuild the Verlet list over the 27 coarse cells.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "physdev.cuh"
#include "refdev.cuh"

namespace lima {
namespace {

constexpr int kTB = 256;
constexpr double kR = 8.314462618;   // J/(mol K)

inline float host_int_as_float(int v) {
    float f;
    std::memcpy(&f, &v, sizeof(f));
    return f;
}

__device__ __forceinline__ float mimg(float d, float L, float invL) { return d - L * rintf(d * invL); }

// error-free sum: s + e == a + b exactly
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = a + b;
    const float bp = s - a;
    e = (a - (s - bp)) + (b - bp);
}
// (hi, lo) += x
__device__ __forceinline__ void ds_add(float& hi, float& lo, float x) {
    float s, e;
    two_sum(hi, x + lo, s, e);
    hi = s;
    lo = e;
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void block_add(double* acc, int idx, double v) {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&acc[idx], v);
}

__device__ __forceinline__ uint32_t spread2(uint32_t v) {   // 2-bit value -> bits 0 and 3
    return (v & 1u) | ((v & 2u) << 2);
}

__device__ __forceinline__ void cell_coords(const PhysDev& d, float4 p, int& cx, int& cy, int& cz, uint32_t& sub) {
    const float inv = (float)d.m / d.L;
    float fx = p.x * inv, fy = p.y * inv, fz = p.z * inv;
    cx = min(max((int)fx, 0), d.m - 1);
    cy = min(max((int)fy, 0), d.m - 1);
    cz = min(max((int)fz, 0), d.m - 1);
    uint32_t sx = (uint32_t)min(max((int)((fx - cx) * 4.f), 0), 3);
    uint32_t sy = (uint32_t)min(max((int)((fy - cy) * 4.f), 0), 3);
    uint32_t sz = (uint32_t)min(max((int)((fz - cz) * 4.f), 0), 3);
    sub = (spread2(sx) << 2) | (spread2(sy) << 1) | spread2(sz);
}

// ---------------------------------------------------------------- rebuild ---
__global__ void k_keys(PhysDev d, int cur) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const float4 p = d.pos[cur][i];
    int cx, cy, cz;
    uint32_t sub;
    cell_coords(d, p, cx, cy, cz, sub);
    d.keys[0][i] = ((uint32_t)((cx * d.m + cy) * d.m + cz) << 6) | sub;
    d.vals[0][i] = i;
}

__global__ void k_permute(PhysDev d, int cur, int mixed) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.n) return;
    const uint32_t src = d.vals[1][k];
    const float4 p = d.pos[cur][src];
    d.pos_tmp[k] = p;
    d.vel_tmp[k] = d.vel[src];
    if (mixed) {
        d.posc_tmp[k] = d.posc[src];
        d.velc_tmp[k] = d.velc[src];
    }
    const uint32_t o = d.orig_of_sorted[src];
    d.orig_tmp[k] = o;
    d.sorted_of_orig[o] = k;
    d.xref[k] = p;
    const uint32_t c = d.keys[1][k] >> 6;
    if (k == 0 || (d.keys[1][k - 1] >> 6) != c) d.cstart[c] = k;
    if (k == d.n - 1 || (d.keys[1][k + 1] >> 6) != c) d.cend[c] = k + 1;
}

__device__ __forceinline__ bool excluded(const PhysDev& d, uint32_t oi, uint32_t oj) {
    for (uint32_t q = d.excl_off[oi]; q < d.excl_off[oi + 1]; q++)
        if (d.excl_ids[q] == oj) return true;
    return false;
}

__global__ void __launch_bounds__(kTB) k_build_list(PhysDev d, int cur) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const float4 pi = d.pos[cur][i];
    const uint32_t oi = d.orig_of_sorted[i];
    const bool cpi = oi < (uint32_t)d.n_cp && d.excl_off[oi + 1] > d.excl_off[oi];
    int cx, cy, cz;
    uint32_t sub;
    cell_coords(d, pi, cx, cy, cz, sub);
    const int m = d.m;
    int cnt = 0;
    const int ncell = m >= 3 ? 27 : m * m * m;
    for (int q = 0; q < ncell; q++) {
        int c;
        if (m >= 3) {
            const int dx = q / 9 - 1, dy = (q / 3) % 3 - 1, dz = q % 3 - 1;
            c = (((cx + dx + m) % m) * m + ((cy + dy + m) % m)) * m + ((cz + dz + m) % m);
        } else {
            c = q;
        }
        const uint32_t b = d.cstart[c], e = d.cend[c];
        for (uint32_t j = b; j < e; j++) {
            if ((int)j == i) continue;
            const float4 pj = d.pos[cur][j];
            const float dx = mimg(pj.x - pi.x, d.L, d.invL);
            const float dy = mimg(pj.y - pi.y, d.L, d.invL);
            const float dz = mimg(pj.z - pi.z, d.L, d.invL);
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 >= d.rlist2) continue;
            if (cpi) {
                const uint32_t oj = d.orig_of_sorted[j];
                if (oj < (uint32_t)d.n_cp && excluded(d, oi, oj)) continue;
            }
            if (cnt < d.nl_cap) d.nl[(size_t)cnt * d.n_pad + i] = j;
            cnt++;
        }
    }
    d.nl_cnt[i] = min(cnt, d.nl_cap);
    if (cnt > d.nl_cap) atomicOr(d.err, ERR_BIT_PHYS_LIST_OVERFLOW);
}

// ----------------------------------------------------------------- bonded ---
template <bool ENERGY>
__global__ void __launch_bounds__(kTB) k_bonded(PhysDev d, int cur) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double eb = 0.0, ea = 0.0, ed = 0.0, vir = 0.0;
    const float L = d.L, iL = d.invL;
    auto P = [&](int orig) { return d.pos[cur][d.sorted_of_orig[orig]]; };
    if (t < d.n_bonds) {
        const int4 ix = d.bond_idx[t];
        const float2 par = d.bond_par[t];
        const float4 a = P(ix.x), b = P(ix.y);
        const float rx = mimg(b.x - a.x, L, iL), ry = mimg(b.y - a.y, L, iL), rz = mimg(b.z - a.z, L, iL);
        const float rr = sqrtf(rx * rx + ry * ry + rz * rz);
        const float dr = rr - par.x;
        const float f = -par.y * dr / rr;   // F_j = f * r
        d.term_force[2 * t + 0] = make_float4(-f * rx, -f * ry, -f * rz, 0.f);
        d.term_force[2 * t + 1] = make_float4(f * rx, f * ry, f * rz, 0.f);
        if (ENERGY) {
            eb = 0.5 * (double)par.y * (double)dr * (double)dr;
            vir = (double)(f * rr * rr);
        }
    } else if (t < d.n_bonds + d.n_angles) {
        const int a_ = t - d.n_bonds;
        const int4 ix = d.angle_idx[a_];
        const float2 par = d.angle_par[a_];
        const float4 pi = P(ix.x), pj = P(ix.y), pk = P(ix.z);
        const float ux = mimg(pi.x - pj.x, L, iL), uy = mimg(pi.y - pj.y, L, iL), uz = mimg(pi.z - pj.z, L, iL);
        const float vx = mimg(pk.x - pj.x, L, iL), vy = mimg(pk.y - pj.y, L, iL), vz = mimg(pk.z - pj.z, L, iL);
        const float uu = ux * ux + uy * uy + uz * uz, vv = vx * vx + vy * vy + vz * vz;
        const float nu = sqrtf(uu), nv = sqrtf(vv);
        const float cx_ = uy * vz - uz * vy, cy_ = uz * vx - ux * vz, cz_ = ux * vy - uy * vx;
        const float sn = sqrtf(cx_ * cx_ + cy_ * cy_ + cz_ * cz_);
        const float cs = ux * vx + uy * vy + uz * vz;
        const float th = atan2f(sn, cs);
        const float dth = th - par.x;
        const float c = cs / (nu * nv);
        const float s = fmaxf(sn / (nu * nv), 1e-6f);
        const float g = par.y * dth / s;   // dV/dtheta / sin
        const float inuv = 1.f / (nu * nv);
        const float fix = g * (vx * inuv - c * ux / uu), fiy = g * (vy * inuv - c * uy / uu), fiz = g * (vz * inuv - c * uz / uu);
        const float fkx = g * (ux * inuv - c * vx / vv), fky = g * (uy * inuv - c * vy / vv), fkz = g * (uz * inuv - c * vz / vv);
        const int base = 2 * d.n_bonds + 3 * a_;
        d.term_force[base + 0] = make_float4(fix, fiy, fiz, 0.f);
        d.term_force[base + 1] = make_float4(-fix - fkx, -fiy - fky, -fiz - fkz, 0.f);
        d.term_force[base + 2] = make_float4(fkx, fky, fkz, 0.f);
        if (ENERGY) {
            ea = 0.5 * (double)par.y * (double)dth * (double)dth;
            vir = (double)(ux * fix + uy * fiy + uz * fiz + vx * fkx + vy * fky + vz * fkz);
        }
    } else if (t < d.n_bonds + d.n_angles + d.n_dih) {
        const int q = t - d.n_bonds - d.n_angles;
        const int4 ix = d.dih_idx[q];
        const float4 par = d.dih_par[q];
        const float4 xi = P(ix.x), xj = P(ix.y), xk = P(ix.z), xl = P(ix.w);
        const float b1x = mimg(xj.x - xi.x, L, iL), b1y = mimg(xj.y - xi.y, L, iL), b1z = mimg(xj.z - xi.z, L, iL);
        const float b2x = mimg(xk.x - xj.x, L, iL), b2y = mimg(xk.y - xj.y, L, iL), b2z = mimg(xk.z - xj.z, L, iL);
        const float b3x = mimg(xl.x - xk.x, L, iL), b3y = mimg(xl.y - xk.y, L, iL), b3z = mimg(xl.z - xk.z, L, iL);
        const float m1x = b1y * b2z - b1z * b2y, m1y = b1z * b2x - b1x * b2z, m1z = b1x * b2y - b1y * b2x;
        const float m2x = b2y * b3z - b2z * b3y, m2y = b2z * b3x - b2x * b3z, m2z = b2x * b3y - b2y * b3x;
        const float m1m1 = m1x * m1x + m1y * m1y + m1z * m1z, m2m2 = m2x * m2x + m2y * m2y + m2z * m2z;
        const float b2b2 = b2x * b2x + b2y * b2y + b2z * b2z;
        const float nb2 = sqrtf(b2b2);
        const float m1m2 = m1x * m2x + m1y * m2y + m1z * m2z;
        const float xx = b1x * m2x + b1y * m2y + b1z * m2z;
        const float phi = atan2f(nb2 * xx, m1m2);
        const float nn = par.z;
        float sv, cv;
        sincosf(nn * phi - par.x, &sv, &cv);
        const float dVdphi = -par.y * nn * sv;
        const float gi = dVdphi * nb2 / m1m1, gl = -dVdphi * nb2 / m2m2;
        const float fix = gi * m1x, fiy = gi * m1y, fiz = gi * m1z;
        const float flx = gl * m2x, fly = gl * m2y, flz = gl * m2z;
        const float p = (b1x * b2x + b1y * b2y + b1z * b2z) / b2b2;
        const float r = (b3x * b2x + b3y * b2y + b3z * b2z) / b2b2;
        const float fjx = -fix - p * fix + r * flx, fjy = -fiy - p * fiy + r * fly, fjz = -fiz - p * fiz + r * flz;
        const float fkx = -flx + p * fix - r * flx, fky = -fly + p * fiy - r * fly, fkz = -flz + p * fiz - r * flz;
        const int base = 2 * d.n_bonds + 3 * d.n_angles + 4 * q;
        d.term_force[base + 0] = make_float4(fix, fiy, fiz, 0.f);
        d.term_force[base + 1] = make_float4(fjx, fjy, fjz, 0.f);
        d.term_force[base + 2] = make_float4(fkx, fky, fkz, 0.f);
        d.term_force[base + 3] = make_float4(flx, fly, flz, 0.f);
        if (ENERGY) {
            ed = (double)par.y * (1.0 + (double)cv);
            vir = (double)(b1x * fjx + b1y * fjy + b1z * fjz + (b1x + b2x) * fkx + (b1y + b2y) * fky + (b1z + b2z) * fkz +
                           (b1x + b2x + b3x) * flx + (b1y + b2y + b3y) * fly + (b1z + b2z + b3z) * flz);
        }
    }
    if (ENERGY) {
        block_add(d.acc, LIMA_E_BOND, eb);
        block_add(d.acc, LIMA_E_ANGLE, ea);
        block_add(d.acc, LIMA_E_DIHEDRAL, ed);
        block_add(d.acc, LIMA_E_VIRIAL, vir);
    }
}

// ------------------------------------------------------- pair + integrate ---
template <bool MIXED, bool ENERGY, bool INTEGRATE>
__global__ void __launch_bounds__(kTB) k_pair_integrate(PhysDev d, int cur) {
    extern __shared__ float2 s_tab[];
    const int nt2 = d.n_types * d.n_types;
    for (int q = threadIdx.x; q < nt2; q += blockDim.x) s_tab[q] = d.lj_table[q];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ke = 0.0, elj = 0.0, vir = 0.0;
    if (i < d.n) {
        const float4 pi = d.pos[cur][i];
        const int ti = __float_as_int(pi.w);
        const float2* row = &s_tab[ti * d.n_types];
        const float L = d.L, iL = d.invL, rc2 = d.rc2;
        float fx = 0.f, fy = 0.f, fz = 0.f, cxx = 0.f, cyy = 0.f, czz = 0.f;
        float e_i = 0.f, w_i = 0.f;
        const int cnt = d.nl_cnt[i];
        const uint32_t* nl = d.nl + i;
        int k = 0;
        while (k < cnt) {
            const int kend = MIXED ? min(cnt, k + 32) : cnt;
            float px = 0.f, py = 0.f, pz = 0.f;
            for (; k < kend; k++) {
                const uint32_t j = __ldg(&nl[(size_t)k * d.n_pad]);
                const float4 pj = d.pos[cur][j];
                const float dx = mimg(pj.x - pi.x, L, iL);
                const float dy = mimg(pj.y - pi.y, L, iL);
                const float dz = mimg(pj.z - pi.z, L, iL);
                const float r2 = dx * dx + dy * dy + dz * dz;
                if (r2 < rc2) {
                    const float2 tab = row[__float_as_int(pj.w)];
                    const float inv = __frcp_rn(r2);
                    const float sr2 = tab.x * inv;
                    const float sr6 = sr2 * sr2 * sr2;
                    float fr = 6.f * tab.y * inv * sr6 * (2.f * sr6 - 1.f);   // F_j / r_vec
                    float v = 0.f;
                    if (ENERGY || d.use_switch) v = tab.y * (sr6 * sr6 - sr6);
                    if (d.use_switch && r2 > d.ron2) {
                        const float a = rc2 - r2;
                        const float sw = a * a * (rc2 + 2.f * r2 - 3.f * d.ron2) * d.inv_sw_den;
                        const float dsw = 12.f * a * (d.ron2 - r2) * d.inv_sw_den;   // (dS/dr)/r
                        fr = fr * sw - v * dsw;
                        v *= sw;
                    } else if (ENERGY && !d.use_switch) {
                        const float src2 = tab.x / rc2, src6 = src2 * src2 * src2;
                        v -= tab.y * (src6 * src6 - src6);
                    }
                    px -= fr * dx;
                    py -= fr * dy;
                    pz -= fr * dz;
                    if (ENERGY) {
                        e_i += 0.5f * v;
                        w_i += 0.5f * fr * r2;
                    }
                }
            }
            if (MIXED) {
                ds_add(fx, cxx, px);
                ds_add(fy, cyy, py);
                ds_add(fz, czz, pz);
            } else {
                fx += px;
                fy += py;
                fz += pz;
            }
        }
        // bonded contributions of this particle
        const uint32_t oi = d.orig_of_sorted[i];
        if (oi < (uint32_t)d.n_cp) {
            float bx = 0.f, by = 0.f, bz = 0.f;
            for (uint32_t q = d.bterm_off[oi]; q < d.bterm_off[oi + 1]; q++) {
                const float4 tf = d.term_force[d.bterm_slot[q]];
                bx += tf.x;
                by += tf.y;
                bz += tf.z;
            }
            if (MIXED) {
                ds_add(fx, cxx, bx);
                ds_add(fy, cyy, by);
                ds_add(fz, czz, bz);
            } else {
                fx += bx;
                fy += by;
                fz += bz;
            }
        }
        if (MIXED) {
            fx += cxx;
            fy += cyy;
            fz += czz;
        }
        d.force[i] = make_float4(fx, fy, fz, ENERGY ? e_i : 0.f);
        if (ENERGY) {
            elj = (double)e_i;
            vir = (double)w_i;
        }
        // velocity Verlet as kick-drift over half-step velocities
        const float4 v = d.vel[i];
        const float im = v.w;
        const float h = (float)(0.5 * d.dt);
        const float ax = fx * im, ay = fy * im, az = fz * im;
        if (MIXED) {
            float4 vc = d.velc[i];
            float vhx = v.x, vhy = v.y, vhz = v.z;
            ds_add(vhx, vc.x, ax * h);
            ds_add(vhy, vc.y, ay * h);
            ds_add(vhz, vc.z, az * h);
            const double vx = (double)vhx + vc.x, vy = (double)vhy + vc.y, vz = (double)vhz + vc.z;
            ke = 0.5 / (double)im * (vx * vx + vy * vy + vz * vz);
            if (INTEGRATE) {
                const float lam = *d.lambda;
                if (lam != 1.f) {   // scale the (hi, lo) pair: exact product error kept in lo
                    float p = lam * vhx; vc.x = fmaf(lam, vhx, -p) + lam * vc.x; vhx = p;
                    p = lam * vhy; vc.y = fmaf(lam, vhy, -p) + lam * vc.y; vhy = p;
                    p = lam * vhz; vc.z = fmaf(lam, vhz, -p) + lam * vc.z; vhz = p;
                }
                ds_add(vhx, vc.x, ax * h);
                ds_add(vhy, vc.y, ay * h);
                ds_add(vhz, vc.z, az * h);
                float4 pc = d.posc[i];
                const float dtf = (float)d.dt;
                float x = pi.x, y = pi.y, z = pi.z;
                // position += v*dt, with the product's rounding error kept
                float t = vhx * dtf; ds_add(x, pc.x, t); pc.x += fmaf(vhx, dtf, -t) + vc.x * dtf;
                t = vhy * dtf; ds_add(y, pc.y, t); pc.y += fmaf(vhy, dtf, -t) + vc.y * dtf;
                t = vhz * dtf; ds_add(z, pc.z, t); pc.z += fmaf(vhz, dtf, -t) + vc.z * dtf;
                if (x < 0.f) ds_add(x, pc.x, L); else if (x >= L) ds_add(x, pc.x, -L);
                if (y < 0.f) ds_add(y, pc.y, L); else if (y >= L) ds_add(y, pc.y, -L);
                if (z < 0.f) ds_add(z, pc.z, L); else if (z >= L) ds_add(z, pc.z, -L);
                if (x >= L) x -= L;
                if (y >= L) y -= L;
                if (z >= L) z -= L;
                d.pos[cur ^ 1][i] = make_float4(x, y, z, pi.w);
                d.posc[i] = pc;
                d.vel[i] = make_float4(vhx, vhy, vhz, im);
                d.velc[i] = vc;
                const float4 xr = d.xref[i];
                const float ddx = mimg(x - xr.x, L, iL), ddy = mimg(y - xr.y, L, iL), ddz = mimg(z - xr.z, L, iL);
                if (ddx * ddx + ddy * ddy + ddz * ddz > d.half_skin2) atomicOr(d.err, ERR_BIT_PHYS_LIST_OVERFLOW);
                if (!(x == x) || !(y == y) || !(z == z)) atomicOr(d.err, ERR_BIT_NAN);
            }
        } else {
            float vx = v.x + ax * h, vy = v.y + ay * h, vz = v.z + az * h;
            ke = 0.5 / (double)im * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
            if (INTEGRATE) {
                const float lam = *d.lambda;
                vx = lam * vx + ax * h;
                vy = lam * vy + ay * h;
                vz = lam * vz + az * h;
                const float dtf = (float)d.dt;
                float x = pi.x + vx * dtf, y = pi.y + vy * dtf, z = pi.z + vz * dtf;
                x += (x < 0.f) ? L : ((x >= L) ? -L : 0.f);
                y += (y < 0.f) ? L : ((y >= L) ? -L : 0.f);
                z += (z < 0.f) ? L : ((z >= L) ? -L : 0.f);
                if (x >= L) x -= L;
                if (y >= L) y -= L;
                if (z >= L) z -= L;
                d.pos[cur ^ 1][i] = make_float4(x, y, z, pi.w);
                d.vel[i] = make_float4(vx, vy, vz, im);
                const float4 xr = d.xref[i];
                const float ddx = mimg(x - xr.x, L, iL), ddy = mimg(y - xr.y, L, iL), ddz = mimg(z - xr.z, L, iL);
                if (ddx * ddx + ddy * ddy + ddz * ddz > d.half_skin2) atomicOr(d.err, ERR_BIT_PHYS_LIST_OVERFLOW);
                if (!(x == x) || !(y == y) || !(z == z)) atomicOr(d.err, ERR_BIT_NAN);
            }
        }
    }
    block_add(d.acc, LIMA_E_KINETIC, ke);
    if (ENERGY) {
        block_add(d.acc, LIMA_E_LJ, elj);
        block_add(d.acc, LIMA_E_VIRIAL, vir);
    }
    // last block: fold FP64 accumulators, temperature, next lambda
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(d.done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        volatile double* acc = d.acc;
        const double kin = acc[LIMA_E_KINETIC];
        const double temp = 2.0 * kin / (3.0 * (double)d.n * kR);
        d.e_last[LIMA_E_KINETIC] = kin;
        d.e_last[LIMA_E_TEMPERATURE] = temp;
        if (ENERGY) {
            d.e_last[LIMA_E_LJ] = acc[LIMA_E_LJ];
            d.e_last[LIMA_E_BOND] = acc[LIMA_E_BOND];
            d.e_last[LIMA_E_ANGLE] = acc[LIMA_E_ANGLE];
            d.e_last[LIMA_E_DIHEDRAL] = acc[LIMA_E_DIHEDRAL];
            d.e_last[LIMA_E_VIRIAL] = acc[LIMA_E_VIRIAL];
            d.e_last[LIMA_E_TOTAL] = acc[LIMA_E_LJ] + acc[LIMA_E_BOND] + acc[LIMA_E_ANGLE] + acc[LIMA_E_DIHEDRAL] + kin;
        }
        for (int q = 0; q < LIMA_E_COUNT; q++) acc[q] = 0.0;
        if (INTEGRATE) {
            float lam = 1.f;
            if (d.thermostat == LIMA_THERMOSTAT_BERENDSEN && temp > 0.0)
                lam = (float)sqrt(1.0 + d.dt / d.tau_t * (d.t_target / temp - 1.0));
            *d.lambda = lam;
            *d.t_prev = temp;
        }
        __threadfence();
        *d.done = 0;
    }
}

template <bool MIXED, bool ENERGY, bool INTEGRATE>
void launch_pair(const PhysDev& d, int cur, cudaStream_t s) {
    const int nb = (d.n + kTB - 1) / kTB;
    const size_t smem = sizeof(float2) * d.n_types * d.n_types;
    k_pair_integrate<MIXED, ENERGY, INTEGRATE><<<nb, kTB, smem, s>>>(d, cur);
}

void launch_bonded(const PhysDev& d, int cur, bool energy, cudaStream_t s) {
    const int nterms = d.n_bonds + d.n_angles + d.n_dih;
    if (nterms == 0) return;
    const int nb = (nterms + kTB - 1) / kTB;
    if (energy)
        k_bonded<true><<<nb, kTB, 0, s>>>(d, cur);
    else
        k_bonded<false><<<nb, kTB, 0, s>>>(d, cur);
}

template <typename T>
T* dalloc(std::vector<void*>& allocs, size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
    allocs.push_back(p);
    return static_cast<T*>(p);
}

}  // namespace

// ===================================================================== host ==
int phys_setup(const PhysHost& h, PhysDev& d, cudaStream_t s, std::vector<void*>& allocs, std::string& msg) {
    const lima_params& p = *h.params;
    if (p.thermostat == LIMA_THERMOSTAT_REFERENCE) {
        msg = "the reference thermostat belongs to reference semantics";
        return LIMA_ERR_UNSUPPORTED;
    }
    std::memset(&d, 0, sizeof(d));
    d.n_c = h.n_c;
    d.n_s = h.n_s;
    std::vector<int> base(h.n_c + 1, 0);
    for (int c = 0; c < h.n_c; c++) base[c + 1] = base[c] + h.comps[c].n_particles;
    d.n_cp = base[h.n_c];
    d.n = d.n_cp + h.n_s;
    if (d.n < 2) {
        msg = "physics semantics needs at least two particles";
        return LIMA_ERR_ARGUMENT;
    }
    d.n_pad = (d.n + 31) / 32 * 32;
    d.L = p.box_len;
    d.invL = 1.f / p.box_len;
    d.rc = p.cutoff;
    d.rc2 = p.cutoff * p.cutoff;
    d.rlist = p.cutoff + p.skin;
    d.rlist2 = d.rlist * d.rlist;
    d.half_skin2 = 0.25f * p.skin * p.skin;
    d.use_switch = p.switch_on < p.cutoff ? 1 : 0;
    const float ron = d.use_switch ? p.switch_on : p.cutoff;
    d.ron2 = ron * ron;
    d.inv_sw_den = d.use_switch ? 1.f / ((d.rc2 - d.ron2) * (d.rc2 - d.ron2) * (d.rc2 - d.ron2)) : 0.f;
    d.dt = p.dt;
    d.precision = p.precision;
    d.thermostat = p.thermostat;
    d.t_target = p.t_target;
    d.tau_t = p.tau_t;

    // types and the Lorentz-Berthelot table
    int max_type = 0;
    for (int c = 0; c < h.n_c; c++)
        for (int t = 0; t < h.comps[c].n_particles; t++) max_type = std::max<int>(max_type, h.comps[c].atom_types[t]);
    d.n_types = max_type + 1;
    for (int t = 0; t < d.n_types; t++) {
        const auto& pp = h.ff->particle_parameters[t];
        if (!(pp.mass > 0.f) || !(pp.sigma > 0.f) || !(pp.epsilon >= 0.f)) {
            msg = "force field entry for a used type has non-positive mass/sigma or negative epsilon";
            return LIMA_ERR_ARGUMENT;
        }
    }
    std::vector<float2> tab(d.n_types * d.n_types);
    for (int a = 0; a < d.n_types; a++)
        for (int b = 0; b < d.n_types; b++) {
            const auto& A = h.ff->particle_parameters[a];
            const auto& B = h.ff->particle_parameters[b];
            const double sg = 0.5 * ((double)A.sigma + (double)B.sigma);
            const double ep = std::sqrt((double)A.epsilon * (double)B.epsilon);
            tab[a * d.n_types + b] = make_float2((float)(sg * sg), (float)(4.0 * ep));
        }
    // exclusions (LJ_Ignores -> orig ids)
    std::vector<std::vector<uint32_t>> excl(d.n);
    for (int c = 0; c < h.n_c; c++)
        for (int t = 0; t < h.comps[c].n_particles; t++) {
            const lima_lj_ignores& ig = h.comps[c].lj_ignore_list[t];
            for (int q = 0; q < ig.n_ignores; q++) {
                const int oc = ig.compound_ids[q], ol = ig.local_ids[q];
                if (oc >= h.n_c || ol >= h.comps[oc].n_particles) {
                    msg = "LJ_Ignores entry refers to a missing particle";
                    return LIMA_ERR_ARGUMENT;
                }
                excl[base[c] + t].push_back(base[oc] + ol);
            }
        }
    std::vector<uint32_t> eoff(d.n + 1, 0), eids;
    for (int i = 0; i < d.n; i++) {
        eoff[i + 1] = eoff[i] + excl[i].size();
        eids.insert(eids.end(), excl[i].begin(), excl[i].end());
    }
    // bonded terms with orig ids (compounds, then bridges)
    std::vector<int4> bidx, aidx, didx;
    std::vector<float2> bpar, apar;
    std::vector<float4> dpar;
    for (int c = 0; c < h.n_c; c++) {
        const lima_compound& cp = h.comps[c];
        const int o = base[c];
        for (int b = 0; b < cp.n_singlebonds; b++) {
            const auto& t = cp.singlebonds[b];
            bidx.push_back(make_int4(o + t.atom_indexes[0], o + t.atom_indexes[1], 0, 0));
            bpar.push_back(make_float2(t.b0, t.kb));
        }
        for (int b = 0; b < cp.n_anglebonds; b++) {
            const auto& t = cp.anglebonds[b];
            aidx.push_back(make_int4(o + t.atom_indexes[0], o + t.atom_indexes[1], o + t.atom_indexes[2], 0));
            apar.push_back(make_float2(t.theta_0, t.k_theta));
        }
        for (int b = 0; b < cp.n_dihedrals; b++) {
            const auto& t = cp.dihedrals[b];
            didx.push_back(make_int4(o + t.atom_indexes[0], o + t.atom_indexes[1], o + t.atom_indexes[2], o + t.atom_indexes[3]));
            dpar.push_back(make_float4(t.phi_0, t.k_phi, (float)t.n, 0.f));
        }
    }
    for (int b = 0; b < h.n_b; b++) {
        const lima_compound_bridge_compact& br = h.bridges[b];
        auto g = [&](uint32_t local) {
            const auto& r = br.particle_refs[local];
            return base[r.compound_id] + r.local_id_compound;
        };
        for (int q = 0; q < br.n_singlebonds; q++) {
            const auto& t = br.singlebonds[q];
            bidx.push_back(make_int4(g(t.atom_indexes[0]), g(t.atom_indexes[1]), 0, 0));
            bpar.push_back(make_float2(t.b0, t.kb));
        }
        for (int q = 0; q < br.n_anglebonds; q++) {
            const auto& t = br.anglebonds[q];
            aidx.push_back(make_int4(g(t.atom_indexes[0]), g(t.atom_indexes[1]), g(t.atom_indexes[2]), 0));
            apar.push_back(make_float2(t.theta_0, t.k_theta));
        }
        for (int q = 0; q < br.n_dihedrals; q++) {
            const auto& t = br.dihedrals[q];
            didx.push_back(make_int4(g(t.atom_indexes[0]), g(t.atom_indexes[1]), g(t.atom_indexes[2]), g(t.atom_indexes[3])));
            dpar.push_back(make_float4(t.phi_0, t.k_phi, (float)t.n, 0.f));
        }
    }
    d.n_bonds = (int)bidx.size();
    d.n_angles = (int)aidx.size();
    d.n_dih = (int)didx.size();
    d.n_term_slots = 2 * d.n_bonds + 3 * d.n_angles + 4 * d.n_dih;
    std::vector<std::vector<uint32_t>> slots(d.n_cp);
    for (int b = 0; b < d.n_bonds; b++) {
        slots[bidx[b].x].push_back(2 * b);
        slots[bidx[b].y].push_back(2 * b + 1);
    }
    for (int a = 0; a < d.n_angles; a++) {
        const int base_ = 2 * d.n_bonds + 3 * a;
        slots[aidx[a].x].push_back(base_);
        slots[aidx[a].y].push_back(base_ + 1);
        slots[aidx[a].z].push_back(base_ + 2);
    }
    for (int q = 0; q < d.n_dih; q++) {
        const int base_ = 2 * d.n_bonds + 3 * d.n_angles + 4 * q;
        slots[didx[q].x].push_back(base_);
        slots[didx[q].y].push_back(base_ + 1);
        slots[didx[q].z].push_back(base_ + 2);
        slots[didx[q].w].push_back(base_ + 3);
    }
    std::vector<uint32_t> boff(d.n_cp + 1, 0), bslot;
    for (int i = 0; i < d.n_cp; i++) {
        boff[i + 1] = boff[i] + slots[i].size();
        bslot.insert(bslot.end(), slots[i].begin(), slots[i].end());
    }

    // sort grid and list capacity
    d.m = std::max(1, (int)std::floor(d.L / d.rlist));
    while (d.m > 1 && d.L / d.m < d.rlist) d.m--;
    d.coarse = d.L / d.m;
    const double rho = d.n / ((double)d.L * d.L * d.L);
    const double expect = 4.0 / 3.0 * M_PI * (double)d.rlist * d.rlist * d.rlist * rho;
    d.nl_cap = std::min(d.n, (int)((1.6 * expect + 96) / 32 + 1) * 32);
    if (d.nl_cap < 32) d.nl_cap = 32;

    try {
        for (int b = 0; b < 2; b++) d.pos[b] = dalloc<float4>(allocs, d.n_pad);
        d.vel = dalloc<float4>(allocs, d.n_pad);
        d.posc = dalloc<float4>(allocs, d.n_pad);
        d.velc = dalloc<float4>(allocs, d.n_pad);
        d.xref = dalloc<float4>(allocs, d.n_pad);
        d.force = dalloc<float4>(allocs, d.n_pad);
        d.orig_of_sorted = dalloc<uint32_t>(allocs, d.n_pad);
        d.sorted_of_orig = dalloc<uint32_t>(allocs, d.n);
        d.lj_table = dalloc<float2>(allocs, tab.size());
        for (int b = 0; b < 2; b++) {
            d.keys[b] = dalloc<uint32_t>(allocs, d.n);
            d.vals[b] = dalloc<uint32_t>(allocs, d.n);
        }
        const size_t ncell = (size_t)d.m * d.m * d.m;
        d.cstart = dalloc<uint32_t>(allocs, ncell);
        d.cend = dalloc<uint32_t>(allocs, ncell);
        d.pos_tmp = dalloc<float4>(allocs, d.n);
        d.vel_tmp = dalloc<float4>(allocs, d.n);
        d.posc_tmp = dalloc<float4>(allocs, d.n);
        d.velc_tmp = dalloc<float4>(allocs, d.n);
        d.orig_tmp = dalloc<uint32_t>(allocs, d.n);
        d.nl = dalloc<uint32_t>(allocs, (size_t)d.nl_cap * d.n_pad);
        d.nl_cnt = dalloc<uint32_t>(allocs, d.n_pad);
        d.excl_off = dalloc<uint32_t>(allocs, eoff.size());
        d.excl_ids = dalloc<uint32_t>(allocs, eids.size());
        d.bond_idx = dalloc<int4>(allocs, bidx.size());
        d.bond_par = dalloc<float2>(allocs, bpar.size());
        d.angle_idx = dalloc<int4>(allocs, aidx.size());
        d.angle_par = dalloc<float2>(allocs, apar.size());
        d.dih_idx = dalloc<int4>(allocs, didx.size());
        d.dih_par = dalloc<float4>(allocs, dpar.size());
        d.bterm_off = dalloc<uint32_t>(allocs, boff.size());
        d.bterm_slot = dalloc<uint32_t>(allocs, bslot.size());
        d.term_force = dalloc<float4>(allocs, d.n_term_slots);
        d.acc = dalloc<double>(allocs, LIMA_E_COUNT);
        d.e_last = dalloc<double>(allocs, LIMA_E_COUNT);
        d.t_prev = dalloc<double>(allocs, 1);
        d.lambda = dalloc<float>(allocs, 1);
        d.done = dalloc<unsigned int>(allocs, 1);
        d.err = dalloc<int>(allocs, 1);
        cub::DeviceRadixSort::SortPairs(nullptr, d.sort_tmp_bytes, d.keys[0], d.keys[1], d.vals[0], d.vals[1], d.n, 0,
                                        32, s);
        d.sort_tmp = dalloc<uint8_t>(allocs, d.sort_tmp_bytes);
    } catch (const std::exception& e) {
        msg = std::string("device allocation failed: ") + e.what();
        return LIMA_ERR_CUDA;
    }
    auto up = [&](void* dst, const void* src, size_t bytes) {
        if (bytes) cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    };
    up(d.lj_table, tab.data(), sizeof(float2) * tab.size());
    up(d.excl_off, eoff.data(), sizeof(uint32_t) * eoff.size());
    up(d.excl_ids, eids.data(), sizeof(uint32_t) * eids.size());
    up(d.bond_idx, bidx.data(), sizeof(int4) * bidx.size());
    up(d.bond_par, bpar.data(), sizeof(float2) * bpar.size());
    up(d.angle_idx, aidx.data(), sizeof(int4) * aidx.size());
    up(d.angle_par, apar.data(), sizeof(float2) * apar.size());
    up(d.dih_idx, didx.data(), sizeof(int4) * didx.size());
    up(d.dih_par, dpar.data(), sizeof(float4) * dpar.size());
    up(d.bterm_off, boff.data(), sizeof(uint32_t) * boff.size());
    up(d.bterm_slot, bslot.data(), sizeof(uint32_t) * bslot.size());
    cudaMemsetAsync(d.acc, 0, sizeof(double) * LIMA_E_COUNT, s);
    cudaMemsetAsync(d.e_last, 0, sizeof(double) * LIMA_E_COUNT, s);
    cudaMemsetAsync(d.t_prev, 0, sizeof(double), s);
    cudaMemsetAsync(d.done, 0, sizeof(unsigned int), s);
    cudaMemsetAsync(d.err, 0, sizeof(int), s);
    cudaMemsetAsync(d.nl_cnt, 0, sizeof(uint32_t) * d.n_pad, s);
    cudaMemsetAsync(d.force, 0, sizeof(float4) * d.n_pad, s);
    set_device_float(d.lambda, 1.f, s);
    phys_upload_state(h, d, 0, s);
    return cudaGetLastError() == cudaSuccess ? 0 : LIMA_ERR_CUDA;
}

// Host state (reference layout) -> device, in orig order (sorted = identity
// until the next rebuild).  Velocities from the Stormer pair: v = (x - x_prev)/dt.
void phys_upload_state(const PhysHost& h, PhysDev& d, int cur, cudaStream_t s) {
    std::vector<float4> pos(d.n_pad), vel(d.n_pad), zero(d.n_pad, make_float4(0, 0, 0, 0));
    std::vector<uint32_t> ident(d.n_pad);
    const float L = d.L;
    auto wrap = [&](double x) {
        x = std::fmod(x, (double)L);
        if (x < 0) x += L;
        float f = (float)x;
        if (f >= L) f = 0.f;
        return f;
    };
    auto mimg = [&](double dd) { return dd - L * std::nearbyint(dd / L); };
    int k = 0;
    for (int c = 0; c < h.n_c; c++)
        for (int t = 0; t < h.comps[c].n_particles; t++, k++) {
            const lima_float3 x = h.states[c].positions[t], xp = h.comps[c].prev_positions[t];
            const int type = h.comps[c].atom_types[t];
            pos[k] = make_float4(wrap(x.x), wrap(x.y), wrap(x.z), host_int_as_float(type));
            const float im = 1.f / h.ff->particle_parameters[type].mass;
            vel[k] = make_float4((float)(mimg((double)x.x - xp.x) / d.dt), (float)(mimg((double)x.y - xp.y) / d.dt),
                                 (float)(mimg((double)x.z - xp.z) / d.dt), im);
        }
    const float im_sol = 1.f / h.ff->particle_parameters[LIMA_ATOMTYPE_SOL].mass;
    for (int si = 0; si < h.n_s; si++, k++) {
        const lima_float3 x = h.sols[si].pos, xp = h.sols[si].pos_tsub1;
        pos[k] = make_float4(wrap(x.x), wrap(x.y), wrap(x.z), host_int_as_float(LIMA_ATOMTYPE_SOL));
        vel[k] = make_float4((float)(mimg((double)x.x - xp.x) / d.dt), (float)(mimg((double)x.y - xp.y) / d.dt),
                             (float)(mimg((double)x.z - xp.z) / d.dt), im_sol);
    }
    for (int i = d.n; i < d.n_pad; i++) {
        pos[i] = make_float4(0, 0, 0, host_int_as_float(0));
        vel[i] = make_float4(0, 0, 0, 0);
    }
    for (int i = 0; i < d.n_pad; i++) ident[i] = i < d.n ? i : 0xffffffffu;
    cudaMemcpyAsync(d.pos[cur], pos.data(), sizeof(float4) * d.n_pad, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d.vel, vel.data(), sizeof(float4) * d.n_pad, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d.posc, zero.data(), sizeof(float4) * d.n_pad, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d.velc, zero.data(), sizeof(float4) * d.n_pad, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d.orig_of_sorted, ident.data(), sizeof(uint32_t) * d.n_pad, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d.sorted_of_orig, ident.data(), sizeof(uint32_t) * d.n, cudaMemcpyHostToDevice, s);
    set_device_float(d.lambda, 1.f, s);
    cudaStreamSynchronize(s);
}

void phys_rebuild(PhysDev& d, int cur, cudaStream_t s) {
    const int nb = (d.n + kTB - 1) / kTB;
    const size_t ncell = (size_t)d.m * d.m * d.m;
    const bool mixed = d.precision == LIMA_PRECISION_MIXED;
    k_keys<<<nb, kTB, 0, s>>>(d, cur);
    size_t bytes = d.sort_tmp_bytes;
    int end_bit = 6;
    while ((1ull << end_bit) < (unsigned long long)ncell * 64ull) end_bit++;
    cub::DeviceRadixSort::SortPairs(d.sort_tmp, bytes, d.keys[0], d.keys[1], d.vals[0], d.vals[1], d.n, 0, end_bit, s);
    cudaMemsetAsync(d.cstart, 0, sizeof(uint32_t) * ncell, s);
    cudaMemsetAsync(d.cend, 0, sizeof(uint32_t) * ncell, s);
    k_permute<<<nb, kTB, 0, s>>>(d, cur, mixed ? 1 : 0);
    cudaMemcpyAsync(d.pos[cur], d.pos_tmp, sizeof(float4) * d.n, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d.vel, d.vel_tmp, sizeof(float4) * d.n, cudaMemcpyDeviceToDevice, s);
    if (mixed) {
        cudaMemcpyAsync(d.posc, d.posc_tmp, sizeof(float4) * d.n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(d.velc, d.velc_tmp, sizeof(float4) * d.n, cudaMemcpyDeviceToDevice, s);
    }
    cudaMemcpyAsync(d.orig_of_sorted, d.orig_tmp, sizeof(uint32_t) * d.n, cudaMemcpyDeviceToDevice, s);
    k_build_list<<<nb, kTB, 0, s>>>(d, cur);
}

void phys_prime(PhysDev&, int, cudaStream_t) {}

void phys_step_kernels(const PhysDev& d, int cur, cudaStream_t s, bool energy) {
    launch_bonded(d, cur, energy, s);
    const bool mixed = d.precision == LIMA_PRECISION_MIXED;
    if (mixed) {
        if (energy) launch_pair<true, true, true>(d, cur, s);
        else launch_pair<true, false, true>(d, cur, s);
    } else {
        if (energy) launch_pair<false, true, true>(d, cur, s);
        else launch_pair<false, false, true>(d, cur, s);
    }
}

void phys_energy_now(PhysDev& d, int cur, cudaStream_t s) {
    launch_bonded(d, cur, true, s);
    if (d.precision == LIMA_PRECISION_MIXED)
        launch_pair<true, true, false>(d, cur, s);
    else
        launch_pair<false, true, false>(d, cur, s);
}

namespace {
struct Snapshot {
    std::vector<float4> pos, posc, vel, velc, force;
    std::vector<uint32_t> orig;
};
Snapshot snapshot(const PhysDev& d, int cur, bool want_force) {
    Snapshot sn;
    sn.pos.resize(d.n);
    sn.vel.resize(d.n);
    sn.orig.resize(d.n);
    cudaMemcpy(sn.pos.data(), d.pos[cur], sizeof(float4) * d.n, cudaMemcpyDeviceToHost);
    cudaMemcpy(sn.vel.data(), d.vel, sizeof(float4) * d.n, cudaMemcpyDeviceToHost);
    cudaMemcpy(sn.orig.data(), d.orig_of_sorted, sizeof(uint32_t) * d.n, cudaMemcpyDeviceToHost);
    if (d.precision == LIMA_PRECISION_MIXED) {
        sn.posc.resize(d.n);
        sn.velc.resize(d.n);
        cudaMemcpy(sn.posc.data(), d.posc, sizeof(float4) * d.n, cudaMemcpyDeviceToHost);
        cudaMemcpy(sn.velc.data(), d.velc, sizeof(float4) * d.n, cudaMemcpyDeviceToHost);
    }
    if (want_force) {
        sn.force.resize(d.n);
        cudaMemcpy(sn.force.data(), d.force, sizeof(float4) * d.n, cudaMemcpyDeviceToHost);
    }
    return sn;
}
// orig -> (position, previous position = x - v dt), full precision sum of hi+lo
void orig_state(const PhysDev& d, const Snapshot& sn, std::vector<double>& x, std::vector<double>& xp) {
    x.assign(3 * (size_t)d.n, 0.0);
    xp.assign(3 * (size_t)d.n, 0.0);
    const bool mixed = !sn.posc.empty();
    for (int k = 0; k < d.n; k++) {
        const uint32_t o = sn.orig[k];
        const float4 p = sn.pos[k], v = sn.vel[k];
        double px = p.x, py = p.y, pz = p.z, vx = v.x, vy = v.y, vz = v.z;
        if (mixed) {
            px += sn.posc[k].x; py += sn.posc[k].y; pz += sn.posc[k].z;
            vx += sn.velc[k].x; vy += sn.velc[k].y; vz += sn.velc[k].z;
        }
        x[3 * o] = px; x[3 * o + 1] = py; x[3 * o + 2] = pz;
        xp[3 * o] = px - vx * d.dt; xp[3 * o + 1] = py - vy * d.dt; xp[3 * o + 2] = pz - vz * d.dt;
    }
}
}  // namespace

// compound positions in the reference's convention: particle 0 in the box,
// the others as the image nearest to it (Engine.cu:993-996)
void phys_read_compounds(const PhysDev& d, int cur, const lima_compound* comps, float4* pos_out, float4* prev_out) {
    Snapshot sn = snapshot(d, cur, false);
    std::vector<double> x, xp;
    orig_state(d, sn, x, xp);
    const double L = d.L;
    int o = 0;
    for (int c = 0; c < d.n_c; c++) {
        const int n = comps[c].n_particles;
        const double* p0 = &x[3 * (size_t)o];
        for (int t = 0; t < n; t++) {
            const double* pt = &x[3 * (size_t)(o + t)];
            const double* qt = &xp[3 * (size_t)(o + t)];
            double q[3], r[3];
            for (int k = 0; k < 3; k++) {
                double dd = pt[k] - p0[k];
                dd -= L * std::nearbyint(dd / L);
                q[k] = t == 0 ? pt[k] : p0[k] + dd;
                r[k] = q[k] - (pt[k] - qt[k]);
            }
            pos_out[c * 64 + t] = make_float4((float)q[0], (float)q[1], (float)q[2], 0.f);
            prev_out[c * 64 + t] = make_float4((float)r[0], (float)r[1], (float)r[2], 0.f);
        }
        o += n;
    }
}

void phys_read_solvents(const PhysDev& d, int cur, float4* pos_out, float4* prev_out) {
    Snapshot sn = snapshot(d, cur, false);
    std::vector<double> x, xp;
    orig_state(d, sn, x, xp);
    for (int si = 0; si < d.n_s; si++) {
        const size_t o = 3 * (size_t)(d.n_cp + si);
        pos_out[si] = make_float4((float)x[o], (float)x[o + 1], (float)x[o + 2], 0.f);
        prev_out[si] = make_float4((float)xp[o], (float)xp[o + 1], (float)xp[o + 2], 0.f);
    }
}

void phys_read_forces(const PhysDev& d, const lima_compound* comps, float4* fc, float4* fs) {
    Snapshot sn = snapshot(d, 0, true);
    std::vector<float4> by_orig(d.n);
    for (int k = 0; k < d.n; k++) by_orig[sn.orig[k]] = sn.force[k];
    int o = 0;
    for (int c = 0; c < d.n_c; c++) {
        for (int t = 0; t < 64; t++) fc[c * 64 + t] = make_float4(0, 0, 0, 0);
        for (int t = 0; t < comps[c].n_particles; t++) fc[c * 64 + t] = by_orig[o + t];
        o += comps[c].n_particles;
    }
    for (int si = 0; si < d.n_s; si++) fs[si] = by_orig[d.n_cp + si];
}

void phys_read_energies(const PhysDev& d, double* totals, double* per_particle, const lima_compound* comps, int n_c,
                        int n_s) {
    if (totals) cudaMemcpy(totals, d.e_last, sizeof(double) * LIMA_E_COUNT, cudaMemcpyDeviceToHost);
    if (per_particle) {
        Snapshot sn = snapshot(d, 0, true);
        std::vector<double> by_orig(d.n);
        for (int k = 0; k < d.n; k++) by_orig[sn.orig[k]] = sn.force[k].w;
        std::memset(per_particle, 0, sizeof(double) * ((size_t)n_c * 64 + n_s));
        int o = 0;
        for (int c = 0; c < n_c; c++) {
            for (int t = 0; t < comps[c].n_particles; t++) per_particle[c * 64 + t] = by_orig[o + t];
            o += comps[c].n_particles;
        }
        for (int si = 0; si < n_s; si++) per_particle[(size_t)n_c * 64 + si] = by_orig[d.n_cp + si];
    }
}

}  // namespace lima
