// Physics-semantics step kernels: Lorentz-Berthelot LJ with cutoff
// (+ potential switch), harmonic bonds/angles, periodic dihedrals, velocity
// Verlet with an optional Berendsen thermostat.  FP32 forces; in MIXED
// precision the force sums are compensated (every 8 pairs per lane and across
// lanes) and positions/velocities carry FP32 low parts; energy, virial and
// kinetic-energy reductions and the thermostat scalar are FP64, summed in a
// fixed order (run-to-run identical).
//
// Layout: particles sorted by cell (side >= r_list/2, x-major), so the
// kGroup = 8 lanes of the 4 particles a warp handles share a cell and read
// largely the same neighbours — the position gathers of a warp hit L1.
//
// Per step, one launch (captured in a CUDA graph):
//   k_step   8 lanes per particle walk its Verlet list (blocked so the
//            lanes of consecutive particles read one line), branch-free LJ +
//            switch; a compound particle's lanes also evaluate the bonded
//            terms it takes part in and keep its role's force; partial forces
//            reduced with warp shuffles; lane 0 kicks, drifts and gives the
//            kinetic energy.  Each block sums its FP64 values in a fixed
//            order into a partial; the block that finishes last adds the
//            partials in block order, sets the next step's Berendsen scalar
//            and, when a particle moved more than skin/2, tail-launches the
//            rebuild graph, which runs before the next step.
// Rebuild (a device-launchable graph, or host launches): k_sort_count,
// k_sort_scan, k_sort_fill, k_sort_order (a stable counting sort by cell),
// k_permute (every per-slot array into the new order, through tmp arrays)
// and k_build_list — one warp per 8 particles over the columns of their
// 5x5x5 cell neighbourhood that their bounding box can reach, which also
// copies the permuted arrays back.
#include "physdev.cuh"
#include "physkern.cuh"
#include "physmath.cuh"
#include "refdev.cuh"

namespace lima {
namespace {

constexpr double kR = 8.314462618;   // J/(mol K)

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

// lane 0 receives the warp's sum; the order of the additions is fixed
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void cell_xyz(const PhysDev& d, float4 p, int& cx, int& cy, int& cz) {
    const float inv = (float)d.m / d.L;
    cx = min(max((int)(p.x * inv), 0), d.m - 1);
    cy = min(max((int)(p.y * inv), 0), d.m - 1);
    cz = min(max((int)(p.z * inv), 0), d.m - 1);
}

__device__ __forceinline__ bool excluded(const PhysDev& d, uint32_t oi, uint32_t oj) {
    for (uint32_t q = d.excl_off[oi]; q < d.excl_off[oi + 1]; q++)
        if (d.excl_ids[q] == oj) return true;
    return false;
}

}  // namespace

// ----------------------------------------------------- counting sort by cell ---
// Cell of every slot and its arrival rank in the cell (atomic, so the ranks
// are put in slot order by k_sort_order).
__global__ void k_sort_count(PhysDev d, const float4* __restrict__ pos) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    int cx, cy, cz;
    cell_xyz(d, pos[i], cx, cy, cz);
    const uint32_t c = (uint32_t)((cx * d.m + cy) * d.m + cz);
    d.cell_key[i] = c;
    d.cell_rank[i] = atomicAdd(&d.ccount[c], 1u);
}

// One block: exclusive scan of the cell occupancies into cstart (cstart[n_cells]
// = n); the occupancies are reset to zero for the next sort.  Thread t owns a
// contiguous run of cells.
__global__ void __launch_bounds__(kScanThreads) k_sort_scan(PhysDev d) {
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int per = (d.n_cells + kScanThreads - 1) / kScanThreads;
    const int b = t * per, e = min(d.n_cells, b + per);
    uint32_t sum = 0u;
    for (int c = b; c < e; c++) sum += d.ccount[c];
    uint32_t x = sum;   // inclusive scan over the warp
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {   // kScanThreads / 32 == 32 warp totals
        uint32_t v = s_warp[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        s_warp[lane] = v;
    }
    __syncthreads();
    uint32_t run = (w ? s_warp[w - 1] : 0u) + x - sum;
    for (int c = b; c < e; c++) {
        const uint32_t k = d.ccount[c];
        d.cstart[c] = run;
        d.ccount[c] = 0u;
        run += k;
    }
    if (t == 0) d.cstart[d.n_cells] = (uint32_t)d.n;
}

__global__ void k_sort_fill(PhysDev d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    d.order[d.cstart[d.cell_key[i]] + d.cell_rank[i]] = (uint32_t)i;
}

// One warp per cell: the cell's slots (in arrival order from k_sort_fill) put
// in ascending order, which makes the sort stable and the new order a
// function of the positions and the old order only.  Each lane ranks its slot
// by counting the smaller ones; cells of more than 32 particles are sorted by
// lane 0 (insertion sort).
__global__ void k_sort_order(PhysDev d) {
    const int lane = threadIdx.x & 31;
    const int c = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (c >= d.n_cells) return;
    const uint32_t b = d.cstart[c], n = d.cstart[c + 1] - b;
    if (n <= 1u) return;
    if (n <= 32u) {
        const uint32_t v = (uint32_t)lane < n ? d.order[b + lane] : 0xffffffffu;
        uint32_t rank = 0u;
        for (uint32_t k = 0; k < n; k++) rank += __shfl_sync(0xffffffffu, v, (int)k) < v ? 1u : 0u;
        __syncwarp();
        if ((uint32_t)lane < n) d.order[b + rank] = v;
        return;
    }
    if (lane != 0) return;
    for (uint32_t k = b + 1; k < b + n; k++) {
        const uint32_t v = d.order[k];
        uint32_t j = k;
        while (j > b && d.order[j - 1] > v) {
            d.order[j] = d.order[j - 1];
            j--;
        }
        d.order[j] = v;
    }
}

// Every per-slot array gathered into cell order (tmp arrays); reference
// positions of the list; the orig <-> slot maps.
__global__ void k_permute(PhysDev d, int cur, int mixed) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.n) return;
    const uint32_t src = d.order[k];
    const float4 p = d.pos[cur][src];
    d.pos_tmp[0][k] = p;
    d.pos_tmp[1][k] = d.pos[cur ^ 1][src];
    d.vel_tmp[k] = d.vel[src];
    d.force_tmp[k] = d.force[src];
    if (mixed) {
        d.posc_tmp[k] = d.posc[src];
        d.velc_tmp[k] = d.velc[src];
    }
    const uint32_t o = d.orig_of_sorted[src];
    d.orig_tmp[k] = o;
    d.sorted_of_orig[o] = k;
    d.xref[k] = p;
}

__global__ void k_set_xref(PhysDev d, const float4* __restrict__ pos) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < d.n) d.xref[k] = pos[k];
}


// Verlet-list build: one warp per 8 consecutive particles of the cell order,
// 4 lanes per particle (lane = 4 p + s).  The warp's particles are taken in
// groups that share a home column (cells (x, y, *)) and a z-window of at most
// m-4 cells; lanes outside the current group idle.  For a group, each of the
// 25 columns around it is culled when the xy gap between the group's bounding
// box and the column exceeds r_list, and otherwise contributes the cells that
// the group's z-range, widened by the reach sqrt(r_list^2 - gap^2), overlaps:
// one or two contiguous slot ranges of the cell order (at most m cells).  The
// ranges are walked as one stream of candidates, 32 at a time: each lane
// fetches one (the next batch while the current one is tested), shifts it
// into the home frame by whole box lengths and stages it in shared memory.
// Slice s of a particle tests candidates s, s+4, ..., drops itself and
// bonded exclusions, and the slices' hit masks are merged with xor-shuffles;
// each lane then writes its hits at their rank in the merged mask, so rows
// list their neighbours in candidate order (deterministic).  Boxes with fewer
// than 5 cells per side stream all particles with the minimum image.
// pos/orig: positions and orig ids by slot.  items (nullable): the cell order
// as a list of slots when the particles were not moved into it (in-place
// rebuild).  copy_cur >= 0: the particles were permuted into the tmp arrays
// (pos = pos_tmp[0], orig = orig_tmp); the build also copies every slot back
// into the step arrays of parity copy_cur (the rebuild's last copy).
namespace {

constexpr int kBuildSlices = 4;                  // lanes per particle
constexpr int kBuildPerWarp = 32 / kBuildSlices; // particles per warp
constexpr int kMaxRanges = 50;                   // 25 columns, one or two slot ranges each

struct BuildSmem {
    float4 cand[32];                 // staged candidates: shifted position, w = slot | compound bit
    int rstart[kMaxRanges + 1];      // first stream index of range r; rstart[kMaxRanges] = stream length
    int rbase[kMaxRanges];           // first cell-order position of range r
    float rsx[kMaxRanges], rsy[kMaxRanges], rsz[kMaxRanges];   // shift of range r
};

static_assert(kGroup == 8, "the list build writes blocks of 8 entries");

// candidate f of the stream (shifted position, w = slot | compound bit), or a
// NaN sentinel past its end (fails the distance test).  r: the lane's current
// range, advanced past the ranges that end at or before f (f only grows).
__device__ __forceinline__ float4 fetch_cand(const PhysDev& d, const BuildSmem* sm, const float4* __restrict__ pos,
                                             const uint32_t* __restrict__ orig, const uint32_t* __restrict__ items,
                                             int f, int total, bool any_ex, int& r) {
    if (f >= total) {
        const float nan = __int_as_float(0x7fc00000);
        return make_float4(nan, nan, nan, __uint_as_float(0u));
    }
    while (sm->rstart[r + 1] <= f) r++;   // rstart[kMaxRanges] = total > f
    const int q = sm->rbase[r] + (f - sm->rstart[r]);
    const int j = items ? (int)items[q] : q;
    const float4 p = pos[j];
    uint32_t tag = (uint32_t)j;
    if (any_ex && orig[j] < (uint32_t)d.n_cp) tag |= 0x80000000u;
    return make_float4(p.x + sm->rsx[r], p.y + sm->rsy[r], p.z + sm->rsz[r], __uint_as_float(tag));
}

// The group's candidate stream (ranges set up in sm) against every member's particle.
template <bool MIN_IMAGE>
__device__ __forceinline__ void scan_stream(const PhysDev& d, const float4* __restrict__ pos,
                                            const uint32_t* __restrict__ orig, const uint32_t* __restrict__ items,
                                            BuildSmem* sm, int total, bool mine, bool any_ex, int i, float4 pi,
                                            uint32_t oi, bool ex, int lane, int sub, int& cnt) {
    int r = 0;
    float4 nxt = fetch_cand(d, sm, pos, orig, items, lane, total, any_ex, r);
    for (int t0 = 0; t0 < total; t0 += 32) {
        __syncwarp();
        sm->cand[lane] = nxt;
        __syncwarp();
        nxt = fetch_cand(d, sm, pos, orig, items, t0 + 32 + lane, total, any_ex, r);   // in flight during the tests
        uint32_t hm = 0u;
        if (mine) {
#pragma unroll
            for (int t = 0; t < 32 / kBuildSlices; t++) {
                const int c = kBuildSlices * t + sub;
                const float4 q = sm->cand[c];
                float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
                if (MIN_IMAGE) {
                    dx = mimg(dx, d.L, d.invL);
                    dy = mimg(dy, d.L, d.invL);
                    dz = mimg(dz, d.L, d.invL);
                }
                const bool hit = dx * dx + dy * dy + dz * dz < d.rlist2 &&
                                 (__float_as_uint(q.w) & 0x7fffffffu) != (uint32_t)i;   // not itself
                hm |= (hit ? 1u : 0u) << c;
            }
            if (ex)   // a compound particle drops its bonded exclusions
                for (uint32_t b = hm; b; b &= b - 1u) {
                    const int c = __ffs(b) - 1;
                    const uint32_t tag = __float_as_uint(sm->cand[c].w);
                    if ((tag >> 31) && excluded(d, oi, orig[tag & 0x7fffffffu])) hm &= ~(1u << c);
                }
        }
        uint32_t all = hm;   // the particle's hits (its 4 slices are lanes 4p .. 4p+3)
        all |= __shfl_xor_sync(0xffffffffu, all, 1);
        all |= __shfl_xor_sync(0xffffffffu, all, 2);
        // hit of rank k goes to entry cnt + k; slice s writes ranks s, s + 4, ...
        // (entry e of particle i at nl_word, below 2^32 because the list is
        // smaller than 16 GB)
        uint32_t b = all;
        for (int k = 0; k < sub && b; k++) b &= b - 1u;
        for (uint32_t e = (uint32_t)(cnt + sub); b; e += kBuildSlices) {
            const int c = __ffs(b) - 1;
            if (e < (uint32_t)d.nl_cap)
                nl_store(d, nl_word((uint32_t)d.n_pad, (uint32_t)i, e), __float_as_uint(sm->cand[c].w) & 0x7fffffffu);
#pragma unroll
            for (int q = 0; q < kBuildSlices; q++) b &= b - 1u;
        }
        cnt += __popc(all);
    }
}

}  // namespace

__global__ void __launch_bounds__(kBuildWarps * 32) k_build_list(PhysDev d, const float4* __restrict__ pos,
                                                                 const uint32_t* __restrict__ orig,
                                                                 const uint32_t* __restrict__ items, int copy_cur,
                                                                 int mixed) {
    __shared__ BuildSmem s_build[kBuildWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int pl = lane / kBuildSlices, sub = lane % kBuildSlices;
    const int gw = blockIdx.x * kBuildWarps + w;
    if (copy_cur >= 0) {   // the rebuild's copy of the permuted tmp arrays into the step arrays
        if (gw == 0 && lane == 0) *d.need_rebuild = 0;
        for (int k = gw * 32 + lane; k < d.n; k += gridDim.x * kBuildWarps * 32) {
            d.pos[copy_cur][k] = d.pos_tmp[0][k];
            d.pos[copy_cur ^ 1][k] = d.pos_tmp[1][k];
            d.vel[k] = d.vel_tmp[k];
            d.force[k] = d.force_tmp[k];
            if (mixed) {
                d.posc[k] = d.posc_tmp[k];
                d.velc[k] = d.velc_tmp[k];
            }
            d.orig_of_sorted[k] = d.orig_tmp[k];
        }
    }
    const int base = gw * kBuildPerWarp;
    if (base >= d.n) return;   // the whole warp
    BuildSmem* sm = &s_build[w];
    const int qi = base + pl;   // position in the cell order
    const bool have = qi < d.n;
    const int i = have ? (items ? (int)items[qi] : qi) : 0;   // slot
    const float4 pi = have ? pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t oi = have ? orig[i] : 0u;
    const bool ex = have && oi < (uint32_t)d.n_cp && d.excl_off[oi + 1] > d.excl_off[oi];
    const bool any_ex = __any_sync(0xffffffffu, ex);
    int cnt = 0;
    const int m = d.m;

    if (m < 5) {   // one range: every particle, minimum image
        if (lane == 0) {
            sm->rstart[0] = 0;
            sm->rbase[0] = 0;
            sm->rsx[0] = sm->rsy[0] = sm->rsz[0] = 0.f;
            for (int r = 1; r <= kMaxRanges; r++) sm->rstart[r] = d.n;
        }
        __syncwarp();
        scan_stream<true>(d, pos, orig, items, sm, d.n, have, any_ex, i, pi, oi, ex, lane, sub, cnt);
    } else {
        const float cs = d.L / (float)m;   // cell side
        int cx = -1, cy = -1, cz = 0;
        if (have) cell_xyz(d, pi, cx, cy, cz);
        // one bit per particle, at its slice-0 lane
        unsigned todo = __ballot_sync(0xffffffffu, have && sub == 0);
        while (todo) {   // warp-uniform: todo is the same in every lane
            const int lead = __ffs(todo) - 1;
            const int hx = __shfl_sync(0xffffffffu, cx, lead);
            const int hy = __shfl_sync(0xffffffffu, cy, lead);
            const int hz0 = __shfl_sync(0xffffffffu, cz, lead);
            const bool mine = ((todo >> (pl * kBuildSlices)) & 1u) && cx == hx && cy == hy && cz <= hz0 + (m - 5);
            todo &= ~__ballot_sync(0xffffffffu, mine && sub == 0);
            int hz1 = mine ? cz : -1;   // the group's top cell
            float bxl = mine ? pi.x : 3.4e38f, bxh = mine ? pi.x : -3.4e38f;
            float byl = mine ? pi.y : 3.4e38f, byh = mine ? pi.y : -3.4e38f;
            float bzl = mine ? pi.z : 3.4e38f, bzh = mine ? pi.z : -3.4e38f;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                hz1 = max(hz1, __shfl_xor_sync(0xffffffffu, hz1, o));
                bxl = fminf(bxl, __shfl_xor_sync(0xffffffffu, bxl, o));
                bxh = fmaxf(bxh, __shfl_xor_sync(0xffffffffu, bxh, o));
                byl = fminf(byl, __shfl_xor_sync(0xffffffffu, byl, o));
                byh = fmaxf(byh, __shfl_xor_sync(0xffffffffu, byh, o));
                bzl = fminf(bzl, __shfl_xor_sync(0xffffffffu, bzl, o));
                bzh = fmaxf(bzh, __shfl_xor_sync(0xffffffffu, bzh, o));
            }
            // lane c < 25: column (hx + c / 5 - 2, hy + c % 5 - 2), ranges 2c and 2c + 1
            int b0 = 0, l0 = 0, b1 = 0, l1 = 0;
            float sx = 0.f, sy = 0.f, sz0 = 0.f, sz1 = 0.f;
            if (lane < 25) {
                const int ox = lane / 5 - 2, oy = lane % 5 - 2;
                const float cxl = (float)(hx + ox) * cs, cxh = cxl + cs;   // unwrapped, home frame
                const float cyl = (float)(hy + oy) * cs, cyh = cyl + cs;
                const float gx = fmaxf(0.f, fmaxf(cxl - bxh, bxl - cxh));
                const float gy = fmaxf(0.f, fmaxf(cyl - byh, byl - cyh));
                const float g2 = gx * gx + gy * gy;
                if (g2 < d.rlist2 * 1.0001f) {   // the margin covers cell rounding
                    int x = hx + ox, y = hy + oy;
                    if (x < 0) { x += m; sx = -d.L; } else if (x >= m) { x -= m; sx = d.L; }
                    if (y < 0) { y += m; sy = -d.L; } else if (y >= m) { y -= m; sy = d.L; }
                    const int col = (x * m + y) * m;
                    // cells within the reach of the group's z-range (unwrapped; at
                    // most m of them: the group spans <= m - 4 cells)
                    const float reach = sqrtf(fmaxf(d.rlist2 - g2, 0.f)) + 1e-4f * cs;
                    const int u0 = max((int)floorf((bzl - reach) / cs), hz0 - 2);
                    const int u1 = min((int)floorf((bzh + reach) / cs), hz1 + 2);
                    if (u0 < 0) {
                        b0 = (int)d.cstart[col + u0 + m];
                        l0 = (int)d.cstart[col + m] - b0;
                        sz0 = -d.L;
                        b1 = (int)d.cstart[col];
                        l1 = (int)d.cstart[col + u1 + 1] - b1;
                    } else if (u1 >= m) {
                        b0 = (int)d.cstart[col + u0];
                        l0 = (int)d.cstart[col + m] - b0;
                        b1 = (int)d.cstart[col];
                        l1 = (int)d.cstart[col + u1 - m + 1] - b1;
                        sz1 = d.L;
                    } else if (u1 >= u0) {
                        b0 = (int)d.cstart[col + u0];
                        l0 = (int)d.cstart[col + u1 + 1] - b0;
                    }
                }
            }
            // stream offsets: inclusive scan of the per-column lengths
            const int len = l0 + l1;
            int incl = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            __syncwarp();   // the previous group's readers of sm are done
            if (lane < 25) {
                const int st = incl - len;
                sm->rstart[2 * lane] = st;
                sm->rstart[2 * lane + 1] = st + l0;
                sm->rbase[2 * lane] = b0;
                sm->rbase[2 * lane + 1] = b1;
                sm->rsx[2 * lane] = sm->rsx[2 * lane + 1] = sx;
                sm->rsy[2 * lane] = sm->rsy[2 * lane + 1] = sy;
                sm->rsz[2 * lane] = sz0;
                sm->rsz[2 * lane + 1] = sz1;
            }
            if (lane == 0) sm->rstart[kMaxRanges] = total;
            __syncwarp();
            scan_stream<false>(d, pos, orig, items, sm, total, mine, any_ex, i, pi, oi, ex, lane, sub, cnt);
        }
    }
    if (have && sub == 0) {
        d.nl_cnt[i] = (uint32_t)min(cnt, d.nl_cap);
        if (cnt > d.nl_cap) {
            atomicOr(d.err, ERR_BIT_PHYS_LIST_OVERFLOW);
            atomicMax(d.nl_need, cnt);
        }
    }
}

// ------------------------------------------------------------- bonded terms ---
// The bonded terms read the orig-ordered compound positions (pos_orig), none
// of the arrays a list rebuild re-sorts.  MIXED: every bond vector is
// (b_hi - a_hi) + (b_lo - a_lo), so the stiff bonded forces see the (hi, lo)
// positions, not their FP32 rounding.
namespace {

// programmatic dependent launch: let the next kernel of the stream start /
// wait until the kernels this one depends on have finished and their writes
// are visible (a no-op without a programmatic dependency)
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

#if LIMA_STAGED_LIST
// Bulk copies global -> shared memory completing on an mbarrier (the copy
// engine, not the threads, moves the bytes).  Sources are this GPU's own
// memory, and each copy lands in the issuing block's shared memory only.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// waits for the phase of `parity` to complete; false after the iteration limit
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (int it = 0; it < (1 << 20); it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// orders this thread's earlier generic-proxy shared accesses (after a block
// barrier: the block's) before its following bulk-copy writes
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
#endif  // LIMA_STAGED_LIST

// lane 0 receives the warp's sum of v[0..K); then thread 0 adds the warps in
// order into out[0..K) (fixed order)
template <int K>
__device__ __forceinline__ void block_sums_fixed(double (&v)[K], double* out) {
    __shared__ double s_b[kTB / 32][K];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < K; q++) {
        const double x = warp_sum(v[q]);
        if (lane == 0) s_b[w][q] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < K; q++) {
            double t = 0.0;
            for (int k = 0; k < (int)(blockDim.x / 32); k++) t += s_b[k][q];
            out[q] = t;
        }
}

}  // namespace

// One thread per bonded term: the forces on its atoms into its term_force
// slots (w: each atom's share of the term's energy).  The step kernel that
// follows is launched programmatically and starts right away; only the lanes
// that gather these slots wait for this kernel.  ENERGY: per-block FP64 sums
// of the bond, angle and dihedral energies and the virial into bpart.
template <bool ENERGY, bool MIXED>
__global__ void __launch_bounds__(kTB) k_bonded(PhysDev d, int cur) {
    pdl_launch_dependents();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double eb = 0.0, ea = 0.0, ed = 0.0, vir = 0.0;
    const float L = d.L, iL = d.invL;
    const float4* __restrict__ po = d.pos_orig[cur];
    const float4* __restrict__ pc = d.posc_orig[cur];
    // minimum-image vector from particle a to particle b (orig ids)
    auto V = [&](int a, int b, float& x, float& y, float& z) {
        const float4 pa = po[a], pb = po[b];
        x = mimg(pb.x - pa.x, L, iL);
        y = mimg(pb.y - pa.y, L, iL);
        z = mimg(pb.z - pa.z, L, iL);
        if (MIXED) {
            const float4 ca = pc[a], cb = pc[b];
            x += cb.x - ca.x;
            y += cb.y - ca.y;
            z += cb.z - ca.z;
        }
    };
    if (t < d.n_bonds) {
        const int4 ix = d.bond_idx[t];
        const float2 par = d.bond_par[t];
        float rx, ry, rz;
        V(ix.x, ix.y, rx, ry, rz);
        const float rr = sqrtf(rx * rx + ry * ry + rz * rz);
        const float dr = rr - par.x;
        const float f = -par.y * dr / rr;   // F_j = f * r
        if (ENERGY) {
            eb = 0.5 * (double)par.y * (double)dr * (double)dr;
            vir = (double)(f * rr * rr);
        }
        // w: each atom's share of the term's energy (per-particle potential energy)
        const float sh = ENERGY ? (float)(0.5 * eb) : 0.f;
        d.term_force[2 * t + 0] = make_float4(-f * rx, -f * ry, -f * rz, sh);
        d.term_force[2 * t + 1] = make_float4(f * rx, f * ry, f * rz, sh);
    } else if (t < d.n_bonds + d.n_angles) {
        const int a_ = t - d.n_bonds;
        const int4 ix = d.angle_idx[a_];
        const float2 par = d.angle_par[a_];
        float ux, uy, uz, vx, vy, vz;
        V(ix.y, ix.x, ux, uy, uz);
        V(ix.y, ix.z, vx, vy, vz);
        const float uu = ux * ux + uy * uy + uz * uz, vv = vx * vx + vy * vy + vz * vz;
        const float nu = sqrtf(uu), nv = sqrtf(vv);
        const float cx_ = uy * vz - uz * vy, cy_ = uz * vx - ux * vz, cz_ = ux * vy - uy * vx;
        const float sn = sqrtf(cx_ * cx_ + cy_ * cy_ + cz_ * cz_);
        const float cs = ux * vx + uy * vy + uz * vz;
        const float th = atan2f(sn, cs);
        const float dth = th - par.x;
        const float inuv = 1.f / (nu * nv);
        const float cosv = cs * inuv;
        const float s = fmaxf(sn * inuv, 1e-6f);
        const float gk = par.y * dth / s;   // (dV/dtheta) / sin(theta)
        const float fix = gk * (vx * inuv - cosv * ux / uu), fiy = gk * (vy * inuv - cosv * uy / uu),
                    fiz = gk * (vz * inuv - cosv * uz / uu);
        const float fkx = gk * (ux * inuv - cosv * vx / vv), fky = gk * (uy * inuv - cosv * vy / vv),
                    fkz = gk * (uz * inuv - cosv * vz / vv);
        if (ENERGY) {
            ea = 0.5 * (double)par.y * (double)dth * (double)dth;
            vir = (double)(ux * fix + uy * fiy + uz * fiz + vx * fkx + vy * fky + vz * fkz);
        }
        const float sh = ENERGY ? (float)(ea / 3.0) : 0.f;
        const int base = 2 * d.n_bonds + 3 * a_;
        d.term_force[base + 0] = make_float4(fix, fiy, fiz, sh);
        d.term_force[base + 1] = make_float4(-fix - fkx, -fiy - fky, -fiz - fkz, sh);
        d.term_force[base + 2] = make_float4(fkx, fky, fkz, sh);
    } else if (t < d.n_bonds + d.n_angles + d.n_dih) {
        const int q = t - d.n_bonds - d.n_angles;
        const int4 ix = d.dih_idx[q];
        const float4 par = d.dih_par[q];
        float b1x, b1y, b1z, b2x, b2y, b2z, b3x, b3y, b3z;
        V(ix.x, ix.y, b1x, b1y, b1z);
        V(ix.y, ix.z, b2x, b2y, b2z);
        V(ix.z, ix.w, b3x, b3y, b3z);
        const float m1x = b1y * b2z - b1z * b2y, m1y = b1z * b2x - b1x * b2z, m1z = b1x * b2y - b1y * b2x;
        const float m2x = b2y * b3z - b2z * b3y, m2y = b2z * b3x - b2x * b3z, m2z = b2x * b3y - b2y * b3x;
        const float m1m1 = m1x * m1x + m1y * m1y + m1z * m1z, m2m2 = m2x * m2x + m2y * m2y + m2z * m2z;
        const float b2b2 = b2x * b2x + b2y * b2y + b2z * b2z;
        const float nb2 = sqrtf(b2b2);
        const float m1m2 = m1x * m2x + m1y * m2y + m1z * m2z;
        const float xx = b1x * m2x + b1y * m2y + b1z * m2z;
        const float phi = atan2f(nb2 * xx, m1m2);   // IUPAC dihedral angle
        const float nn = par.z;
        float sv, cv;
        sincosf(nn * phi - par.x, &sv, &cv);
        const float dVdphi = -par.y * nn * sv;     // V = k (1 + cos(n phi - phi0))
        const float gi = dVdphi * nb2 / m1m1, gl = -dVdphi * nb2 / m2m2;
        const float fix = gi * m1x, fiy = gi * m1y, fiz = gi * m1z;
        const float flx = gl * m2x, fly = gl * m2y, flz = gl * m2z;
        const float p = (b1x * b2x + b1y * b2y + b1z * b2z) / b2b2;
        const float r = (b3x * b2x + b3y * b2y + b3z * b2z) / b2b2;
        const float fjx = -fix - p * fix + r * flx, fjy = -fiy - p * fiy + r * fly, fjz = -fiz - p * fiz + r * flz;
        const float fkx = -flx + p * fix - r * flx, fky = -fly + p * fiy - r * fly, fkz = -flz + p * fiz - r * flz;
        if (ENERGY) ed = (double)par.y * (1.0 + (double)cv);
        const float sh = ENERGY ? (float)(0.25 * ed) : 0.f;
        const int base = 2 * d.n_bonds + 3 * d.n_angles + 4 * q;
        d.term_force[base + 0] = make_float4(fix, fiy, fiz, sh);
        d.term_force[base + 1] = make_float4(fjx, fjy, fjz, sh);
        d.term_force[base + 2] = make_float4(fkx, fky, fkz, sh);
        d.term_force[base + 3] = make_float4(flx, fly, flz, sh);
        if (ENERGY) {
            vir = (double)(b1x * fjx + b1y * fjy + b1z * fjz + (b1x + b2x) * fkx + (b1y + b2y) * fky +
                           (b1z + b2z) * fkz + (b1x + b2x + b3x) * flx + (b1y + b2y + b3y) * fly +
                           (b1z + b2z + b3z) * flz);
        }
    }
    if (ENERGY) {
        double v[4] = {eb, ea, ed, vir};
        block_sums_fixed<4>(v, d.bpart + (size_t)blockIdx.x * 4);
    }
}

namespace {

// The FP64 sums of a step kernel (kinetic energy; with ENERGY also the LJ
// energy and virial), per block in a fixed order, then over the blocks by the
// block that finishes last (in block order).  That block adds the bonded
// kernel's block partials (ENERGY), folds the totals into e_last and the next
// Berendsen scalar and, when a rebuild is due and `tail` is set, launches it.
// TAIL: this kernel may launch the rebuild graph; a kernel that holds a
// device-side graph launch must itself run inside a graph, so the direct
// launches use the variant without it.
template <bool ENERGY, bool INTEGRATE, bool TAIL>
__device__ __forceinline__ void finish_sums(const PhysDev& d, int slot, cudaGraphExec_t tail, double (&v)[kRed]) {
    __shared__ double s_red[kTB / 32][kRed];
    __shared__ int s_last;
    constexpr int nq = ENERGY ? kRed : 1;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < nq; q++) {
        const double x = warp_sum(v[q]);
        if (lane == 0) s_red[w][q] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < nq; q++) {
            double t = 0.0;
            for (int k = 0; k < kTB / 32; k++) t += s_red[k][q];
            d.part[(size_t)blockIdx.x * kRedStride + q] = t;
        }
        __threadfence();
        s_last = atomicAdd(d.done, 1u) == gridDim.x - 1u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double a[kRed];
#pragma unroll
    for (int q = 0; q < nq; q++) a[q] = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < nq; q++) a[q] += __ldcg(&d.part[(size_t)b * kRedStride + q]);
#pragma unroll
    for (int q = 0; q < nq; q++) {
        const double x = warp_sum(a[q]);
        if (lane == 0) s_red[w][q] = x;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double tot[kRed] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < nq; q++)
        for (int k = 0; k < kTB / 32; k++) tot[q] += s_red[k][q];
    const double kin = tot[0];
    const double temp = 2.0 * kin / (3.0 * (double)d.n * kR);
    d.e_last[LIMA_E_KINETIC] = kin;
    d.e_last[LIMA_E_TEMPERATURE] = temp;
    if (ENERGY) {
        // the bonded kernel's block partials (bond, angle, dihedral, virial), in block order
        pdl_wait();
        double bs[4] = {0.0, 0.0, 0.0, 0.0};
        const int nbb = bonded_blocks(d);
        for (int b = 0; b < nbb; b++)
#pragma unroll
            for (int q = 0; q < 4; q++) bs[q] += __ldcg(&d.bpart[(size_t)b * 4 + q]);
        d.e_last[LIMA_E_LJ] = tot[1];
        d.e_last[LIMA_E_BOND] = bs[0];
        d.e_last[LIMA_E_ANGLE] = bs[1];
        d.e_last[LIMA_E_DIHEDRAL] = bs[2];
        d.e_last[LIMA_E_VIRIAL] = tot[2] + bs[3];
        d.e_last[LIMA_E_TOTAL] = tot[1] + bs[0] + bs[1] + bs[2] + kin;
    }
    if (slot < 2) {
        float lam = 1.f;
        if (d.thermostat == LIMA_THERMOSTAT_BERENDSEN && temp > 0.0)
            lam = (float)sqrt(1.0 + d.dt / d.tau_t * (d.t_target / temp - 1.0));
        d.lambda[slot ^ 1] = lam;
    }
    *d.done = 0u;   // for the next launch
    if (TAIL && INTEGRATE && tail != nullptr && *(volatile int*)d.need_rebuild) {
        if (cudaGraphLaunch(tail, cudaStreamGraphTailLaunch) == cudaSuccess)
            *d.rebuild_count += 1ull;
        else
            atomicOr(d.err, ERR_BIT_REBUILD_LAUNCH);
    }
}

}  // namespace

// ------------------------------------------------------------------ the step ---
// (lj_pair_step: physmath.cuh)
// The four ids of one chunk column (nl_word): one 8-byte load of 16-bit ids
// or one 16-byte load of 32-bit ids.
template <typename ID>
struct ChunkIds;
template <>
struct ChunkIds<uint16_t> {
    using V = uint2;
    static __device__ __forceinline__ void split(V v, uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& e) {
        a = v.x & 0xffffu;
        b = v.x >> 16;
        c = v.y & 0xffffu;
        e = v.y >> 16;
    }
};
template <>
struct ChunkIds<uint32_t> {
    using V = uint4;
    static __device__ __forceinline__ void split(V v, uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& e) {
        a = v.x;
        b = v.y;
        c = v.z;
        e = v.w;
    }
};

// One lane's entries of its particle's Verlet list: `rows` entries, four per
// chunk column (col: the lane's column of chunk 0; cstride: vectors between
// chunks), each chunk one vector load and four position gathers in flight.
// In the last, partial chunk the words past the lane's count are not ids
// (the gathers for them re-read the first entry and are not evaluated).
// MIXED: compensated sums every two chunks (8 pairs).  WM: the axes that take
// the minimum image.  The plain FP32 walk loads each chunk's ids one chunk
// ahead (the mixed walk, and the energies of an unswitched cutoff, have no
// registers to spare for it).
template <bool MIXED, bool ENERGY, bool SWITCH, int WM, typename ID>
__device__ __forceinline__ void pair_rows(const PhysDev& d, const float2* row, float4 pi, const float4* __restrict__ pos,
                                          const typename ChunkIds<ID>::V* __restrict__ col, uint32_t cstride, int rows,
                                          float& fx, float& fy, float& fz, float& cxx, float& cyy, float& czz,
                                          float& e_i, float& w_i) {
    constexpr bool kAhead = !MIXED && (SWITCH || !ENERGY);
    const int full = rows >> 2, tail = rows & 3;
    const int nch = full + (tail ? 1 : 0);
    uint32_t off = 0;
    int c = 0;
    typename ChunkIds<ID>::V nxt{};
    if (kAhead && nch > 0) nxt = __ldg(col);
    while (c < full) {
        const int cend = MIXED ? min(full, c + 2) : full;
        float px = 0.f, py = 0.f, pz = 0.f;
        for (; c < cend; c++, off += cstride) {
            uint32_t j0, j1, j2, j3;
            ChunkIds<ID>::split(kAhead ? nxt : __ldg(col + off), j0, j1, j2, j3);
            if (kAhead && c + 1 < nch) nxt = __ldg(col + off + cstride);
            const float4 p0 = __ldg(pos + j0), p1 = __ldg(pos + j1), p2 = __ldg(pos + j2), p3 = __ldg(pos + j3);
            lj_pair_step<ENERGY, SWITCH, WM>(d, row, pi, p0, px, py, pz, e_i, w_i);
            lj_pair_step<ENERGY, SWITCH, WM>(d, row, pi, p1, px, py, pz, e_i, w_i);
            lj_pair_step<ENERGY, SWITCH, WM>(d, row, pi, p2, px, py, pz, e_i, w_i);
            lj_pair_step<ENERGY, SWITCH, WM>(d, row, pi, p3, px, py, pz, e_i, w_i);
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
    if (tail) {
        uint32_t j0, j1, j2, j3;
        ChunkIds<ID>::split(kAhead ? nxt : __ldg(col + off), j0, j1, j2, j3);
        const float4 p0 = __ldg(pos + j0);
        const float4 p1 = __ldg(pos + (tail > 1 ? j1 : j0));
        const float4 p2 = __ldg(pos + (tail > 2 ? j2 : j0));
        float px = 0.f, py = 0.f, pz = 0.f;
        lj_pair_step<ENERGY, SWITCH, WM>(d, row, pi, p0, px, py, pz, e_i, w_i);
        if (tail > 1) lj_pair_step<ENERGY, SWITCH, WM>(d, row, pi, p1, px, py, pz, e_i, w_i);
        if (tail > 2) lj_pair_step<ENERGY, SWITCH, WM>(d, row, pi, p2, px, py, pz, e_i, w_i);
        (void)j3;
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
}

#if LIMA_STAGED_LIST
// One lane's entries of one staged group of list chunks: entry q of the lane
// at srow[(q / 4) * kChunkWords + q % 4] (shared memory; srow = the lane's
// column of the group's first chunk); MIXED: one compensated sum per group.
constexpr int kStageChunks = kStageRows / 4;   // list chunks per staged group
constexpr int kChunkWords = kTB * 4;           // words of one chunk of a block's 32 particles
__device__ __forceinline__ int staged_at(int q) { return (q >> 2) * kChunkWords + (q & 3); }
template <bool MIXED, bool ENERGY, bool SWITCH, int WM>
__device__ __forceinline__ void pair_staged(const PhysDev& d, const float2* row, float4 pi,
                                            const float4* __restrict__ pos, const uint32_t* srow, int nq, float& fx,
                                            float& fy, float& fz, float& cxx, float& cyy, float& czz, float& e_i,
                                            float& w_i) {
    float px = 0.f, py = 0.f, pz = 0.f;
    // staged ids are clamped into the position array (a wrong id stays a wrong force, not a stray read)
    const uint32_t lim = (uint32_t)d.n_pad - 1u;
    int q = 0;
    for (; q + 3 < nq; q += 4) {
        const uint32_t j0 = min(srow[staged_at(q)], lim), j1 = min(srow[staged_at(q + 1)], lim);
        const uint32_t j2 = min(srow[staged_at(q + 2)], lim), j3 = min(srow[staged_at(q + 3)], lim);
        const float4 p0 = __ldg(pos + j0), p1 = __ldg(pos + j1), p2 = __ldg(pos + j2), p3 = __ldg(pos + j3);
        lj_pair_step<ENERGY, SWITCH, WM>(d, row, pi, p0, px, py, pz, e_i, w_i);
        lj_pair_step<ENERGY, SWITCH, WM>(d, row, pi, p1, px, py, pz, e_i, w_i);
        lj_pair_step<ENERGY, SWITCH, WM>(d, row, pi, p2, px, py, pz, e_i, w_i);
        lj_pair_step<ENERGY, SWITCH, WM>(d, row, pi, p3, px, py, pz, e_i, w_i);
    }
    for (; q < nq; q++)
        lj_pair_step<ENERGY, SWITCH, WM>(d, row, pi, __ldg(pos + min(srow[staged_at(q)], lim)), px, py, pz, e_i, w_i);
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

// The block's list chunks through shared memory: chunk q of the block's 32
// particles is four contiguous kilobytes of the list (nl_word: lane t of the
// block reads words 4t .. 4t + 3 of each chunk), so each chunk is one bulk
// copy.  Groups of kStageChunks chunks (kStageRows rows) alternate between
// two buffers: thread 0 issues group s + 1 while the block evaluates group
// s, and a block barrier after each group frees its buffer for group s + 2.  Waits are bounded; one that runs out sets
// ERR_BIT_TILE_TIMEOUT and ends the issuing, and thread 0 waits (bounded) for
// the copies already issued before the block moves on.
template <bool MIXED, bool ENERGY, bool SWITCH>
__device__ __forceinline__ void pair_walk_staged(const PhysDev& d, const float2* row, float4 pi,
                                                 const float4* __restrict__ pos, int rows, bool active, unsigned wm,
                                                 float& fx, float& fy, float& fz, float& cxx, float& cyy, float& czz,
                                                 float& e_i, float& w_i) {
    __shared__ __align__(128) uint32_t s_stage[2][kStageChunks][kChunkWords];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ int s_rows, s_fail;
    if (threadIdx.x == 0) {
        s_rows = 0;
        s_fail = 0;
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (active && threadIdx.x % kStepLanes == 0) atomicMax(&s_rows, rows);
    __syncthreads();
    const int bchunks = (s_rows + 3) / 4;
    const int nst = (bchunks + kStageChunks - 1) / kStageChunks;
    // chunk 0 of this block's particles: particle i0 = blockIdx.x * 32, word i0 * 32
    const uint32_t* src0 = d.nl + (size_t)blockIdx.x * kChunkWords;
    const size_t stride = (size_t)d.n_pad * kListChunk;   // words between chunks
    int issued = 0;   // thread 0: groups issued
    auto issue = [&](int st) {
        const int c0 = st * kStageChunks, nc = min(kStageChunks, bchunks - c0);
        uint64_t* bar = &s_bar[st & 1];
        fence_proxy_async_smem();
        mbar_expect_tx(bar, (uint32_t)(nc * kChunkWords * sizeof(uint32_t)));
        for (int q = 0; q < nc; q++)
            bulk_g2s(&s_stage[st & 1][q][0], src0 + (size_t)(c0 + q) * stride, kChunkWords * sizeof(uint32_t), bar);
        issued = st + 1;
    };
    if (threadIdx.x == 0 && nst > 0) issue(0);
    for (int st = 0; st < nst; st++) {
        if (threadIdx.x == 0 && st + 1 < nst && !*(volatile int*)&s_fail) issue(st + 1);
        const bool got = !*(volatile int*)&s_fail && mbar_wait_bounded(&s_bar[st & 1], (uint32_t)(st >> 1) & 1u);
        if (!got && !*(volatile int*)&s_fail) {
            s_fail = 1;
            atomicOr(d.err, ERR_BIT_TILE_TIMEOUT);
        }
        const int nq = got ? max(0, min(kStageRows, rows - st * kStageRows)) : 0;
        const uint32_t* srow = &s_stage[st & 1][0][threadIdx.x * 4];
#define LIMA_STAGED_CALL(WM) \
    pair_staged<MIXED, ENERGY, SWITCH, WM>(d, row, pi, pos, srow, nq, fx, fy, fz, cxx, cyy, czz, e_i, w_i)
        switch (wm) {
            case 0: LIMA_STAGED_CALL(0); break;
            case 1: LIMA_STAGED_CALL(1); break;
            case 2: LIMA_STAGED_CALL(2); break;
            case 4: LIMA_STAGED_CALL(4); break;
            default: LIMA_STAGED_CALL(7); break;
        }
#undef LIMA_STAGED_CALL
        __syncthreads();
    }
    // after a timeout: the groups issued and not yet seen complete
    if (threadIdx.x == 0 && s_fail)
        for (int st = max(0, issued - 2); st < issued; st++) mbar_wait_bounded(&s_bar[st & 1], (uint32_t)(st >> 1) & 1u);
    __syncthreads();
}
#endif  // LIMA_STAGED_LIST

template <bool MIXED, bool ENERGY, bool INTEGRATE, bool SWITCH, bool TAIL, typename ID>
__device__ __forceinline__ void step_body(const PhysDev& d, int cur, int slot, cudaGraphExec_t tail) {
    // the LJ table as lj_pair_step reads it: (sigma^2, 24 eps)
    extern __shared__ float2 s_tab[];
    const int nt2 = d.n_types * d.n_types;
    for (int q = threadIdx.x; q < nt2; q += blockDim.x) {
        const float2 t = d.lj_table[q];
        s_tab[q] = make_float2(t.x, 6.f * t.y);
    }
    __syncthreads();
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) / kStepLanes;
    const int g = threadIdx.x % kStepLanes;
    const bool active = i < d.n;
    // FP64 sums of this thread: kinetic energy, LJ energy, LJ virial
    double red[kRed] = {0.0, 0.0, 0.0};
    const float4* __restrict__ pos = d.pos[cur];
    const float4 pi = active ? pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float2* row = &s_tab[__float_as_int(pi.w) * d.n_types];
    float fx = 0.f, fy = 0.f, fz = 0.f, cxx = 0.f, cyy = 0.f, czz = 0.f;
    float e_i = 0.f, w_i = 0.f;
    const int cnt = active ? (int)d.nl_cnt[i] : 0;
    // this lane's entries: g, g + 8, g + 16, ... below cnt
    const int rows = cnt > g ? (cnt - g + kStepLanes - 1) / kStepLanes : 0;
    // the axes that take the minimum image: those on which some particle of the
    // warp lies within r_c of a face (one axis alone, or all three)
    const unsigned wm = __reduce_or_sync(0xffffffffu, active ? face_axes(d, pi) : 0u);
#if LIMA_STAGED_LIST
    pair_walk_staged<MIXED, ENERGY, SWITCH>(d, row, pi, pos, rows, active, wm, fx, fy, fz, cxx, cyy, czz, e_i, w_i);
#else
    // the lane's column of chunk 0 (nl_word with k = g), chunks n_pad * 8 vectors apart
    using V = typename ChunkIds<ID>::V;
    const V* __restrict__ col = reinterpret_cast<const V*>(d.nl) + (uint32_t)i * kGroup + g;
    const uint32_t cstride = (uint32_t)d.n_pad * kGroup;
    {   // the warp's list chunks into L2 at once: chunk q of its 4 particles is
        // 4 x 32 contiguous ids, one bulk prefetch per lane q (no completion to wait for)
        const int wch = ((int)__reduce_max_sync(0xffffffffu, (unsigned)rows) + 3) / 4;
        const int lane = threadIdx.x & 31;
        if (lane < wch) {
            const uint32_t i0 = (blockIdx.x * blockDim.x + (threadIdx.x & ~31u)) / kStepLanes;
            const char* a = reinterpret_cast<const char*>(d.nl) + ((size_t)lane * d.n_pad + i0) * kListChunk * sizeof(ID);
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((unsigned)(4 * kListChunk * sizeof(ID)))
                         : "memory");
        }
    }
#define LIMA_ROWS_CALL(WM) \
    pair_rows<MIXED, ENERGY, SWITCH, WM, ID>(d, row, pi, pos, col, cstride, rows, fx, fy, fz, cxx, cyy, czz, e_i, w_i)
    switch (wm) {
        case 0: LIMA_ROWS_CALL(0); break;
        case 1: LIMA_ROWS_CALL(1); break;
        case 2: LIMA_ROWS_CALL(2); break;
        case 4: LIMA_ROWS_CALL(4); break;
        default: LIMA_ROWS_CALL(7); break;
    }
#undef LIMA_ROWS_CALL
#endif
    // reduce the kStepLanes lanes of this particle (warp shuffles)
#pragma unroll
    for (int o = kStepLanes / 2; o > 0; o >>= 1) {
        if (MIXED) {
            const float ox = __shfl_xor_sync(0xffffffffu, fx, o), oy = __shfl_xor_sync(0xffffffffu, fy, o),
                        oz = __shfl_xor_sync(0xffffffffu, fz, o);
            const float ocx = __shfl_xor_sync(0xffffffffu, cxx, o), ocy = __shfl_xor_sync(0xffffffffu, cyy, o),
                        ocz = __shfl_xor_sync(0xffffffffu, czz, o);
            float s, e;
            two_sum(fx, ox, s, e); fx = s; cxx += ocx + e;
            two_sum(fy, oy, s, e); fy = s; cyy += ocy + e;
            two_sum(fz, oz, s, e); fz = s; czz += ocz + e;
        } else {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
        }
        if (ENERGY) {
            e_i += __shfl_xor_sync(0xffffffffu, e_i, o);
            w_i += __shfl_xor_sync(0xffffffffu, w_i, o);
        }
    }
    const uint32_t oi = active ? d.orig_of_sorted[i] : 0xffffffffu;
    if (active && g == 0) {
        float e_b = 0.f;
        if (oi < (uint32_t)d.n_cp) {
            // the bonded kernel's forces on this particle (it runs beside this
            // kernel's list walk; wait for it only here)
            pdl_wait();
            float bx = 0.f, by = 0.f, bz = 0.f, bw = 0.f;
            for (uint32_t q = d.bterm_off[oi]; q < d.bterm_off[oi + 1]; q++) {
                const float4 tf = __ldcg(&d.term_force[d.bterm_slot[q]]);
                bx += tf.x;
                by += tf.y;
                bz += tf.z;
                bw += tf.w;
            }
            e_b = bw;
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
        // w: the particle's potential energy, its LJ pair halves plus its bonded-term shares
        d.force[i] = make_float4(fx, fy, fz, ENERGY ? e_i + e_b : 0.f);
        if (ENERGY) {
            red[1] = (double)e_i;
            red[2] = (double)w_i;
        }
        // velocity Verlet as kick-drift over half-step velocities
        const float4 v = d.vel[i];
        const float im = v.w;
        const float h = (float)(0.5 * d.dt);
        const float ax = fx * im, ay = fy * im, az = fz * im;
        const float L = d.L, iL = d.invL;
        if (MIXED) {
            float4 vc = d.velc[i];
            float vhx = v.x, vhy = v.y, vhz = v.z;
            ds_add(vhx, vc.x, ax * h);
            ds_add(vhy, vc.y, ay * h);
            ds_add(vhz, vc.z, az * h);
            const double vx = (double)vhx + vc.x, vy = (double)vhy + vc.y, vz = (double)vhz + vc.z;
            red[0] = 0.5 / (double)im * (vx * vx + vy * vy + vz * vz);
            if (INTEGRATE) {
                const float lam = d.lambda[slot];
                if (lam != 1.f) {   // scale (hi, lo): keep the product's rounding error in lo
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
                float tt = vhx * dtf; ds_add(x, pc.x, tt); pc.x += fmaf(vhx, dtf, -tt) + vc.x * dtf;
                tt = vhy * dtf; ds_add(y, pc.y, tt); pc.y += fmaf(vhy, dtf, -tt) + vc.y * dtf;
                tt = vhz * dtf; ds_add(z, pc.z, tt); pc.z += fmaf(vhz, dtf, -tt) + vc.z * dtf;
                if (x < 0.f) ds_add(x, pc.x, L); else if (x >= L) ds_add(x, pc.x, -L);
                if (y < 0.f) ds_add(y, pc.y, L); else if (y >= L) ds_add(y, pc.y, -L);
                if (z < 0.f) ds_add(z, pc.z, L); else if (z >= L) ds_add(z, pc.z, -L);
                if (x >= L) x -= L;
                if (y >= L) y -= L;
                if (z >= L) z -= L;
                d.pos[cur ^ 1][i] = make_float4(x, y, z, pi.w);
                if (oi < (uint32_t)d.n_cp) {
                    d.pos_orig[cur ^ 1][oi] = make_float4(x, y, z, pi.w);
                    d.posc_orig[cur ^ 1][oi] = pc;
                }
                d.posc[i] = pc;
                d.vel[i] = make_float4(vhx, vhy, vhz, im);
                d.velc[i] = vc;
                const float4 xr = d.xref[i];
                const float ddx = mimg(x - xr.x, L, iL), ddy = mimg(y - xr.y, L, iL), ddz = mimg(z - xr.z, L, iL);
                if (ddx * ddx + ddy * ddy + ddz * ddz > d.half_skin2) {
                    if (d.dynamic_list) atomicExch(d.need_rebuild, 1);
                    else atomicOr(d.err, ERR_BIT_LIST_STALE);
                }
                if (!(x == x) || !(y == y) || !(z == z)) atomicOr(d.err, ERR_BIT_NAN);
            }
        } else {
            float vx = v.x + ax * h, vy = v.y + ay * h, vz = v.z + az * h;
            red[0] = 0.5 / (double)im * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
            if (INTEGRATE) {
                const float lam = d.lambda[slot];
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
                if (oi < (uint32_t)d.n_cp) d.pos_orig[cur ^ 1][oi] = make_float4(x, y, z, pi.w);
                d.vel[i] = make_float4(vx, vy, vz, im);
                const float4 xr = d.xref[i];
                const float ddx = mimg(x - xr.x, L, iL), ddy = mimg(y - xr.y, L, iL), ddz = mimg(z - xr.z, L, iL);
                if (ddx * ddx + ddy * ddy + ddz * ddz > d.half_skin2) {
                    if (d.dynamic_list) atomicExch(d.need_rebuild, 1);
                    else atomicOr(d.err, ERR_BIT_LIST_STALE);
                }
                if (!(x == x) || !(y == y) || !(z == z)) atomicOr(d.err, ERR_BIT_NAN);
            }
        }
    }
    finish_sums<ENERGY, INTEGRATE, TAIL>(d, slot, tail, red);
}

// FP32: at most 48 registers, 5 blocks of 256 per SM.  Mixed keeps the
// compiler's own choice (a 5-block bound slowed it).
// ID: the list's slot-id type (uint16_t when the slots fit, else uint32_t).
template <bool ENERGY, bool INTEGRATE, bool SWITCH, bool TAIL, typename ID>
__global__ void __launch_bounds__(kTB, 5) k_step(PhysDev d, int cur, int slot, cudaGraphExec_t tail) {
    step_body<false, ENERGY, INTEGRATE, SWITCH, TAIL, ID>(d, cur, slot, tail);
}
template <bool ENERGY, bool INTEGRATE, bool SWITCH, bool TAIL, typename ID>
__global__ void __launch_bounds__(kTB) k_step_mixed(PhysDev d, int cur, int slot, cudaGraphExec_t tail) {
    step_body<true, ENERGY, INTEGRATE, SWITCH, TAIL, ID>(d, cur, slot, tail);
}

// ---------------------------------------------------------------- launchers --
namespace {

// The step kernel with a programmatic dependency on the kernel before it in
// the stream (the bonded kernel): it may start before that one has finished
// and waits for it only where it reads its results.
template <typename K>
void launch_programmatic(K kernel, const PhysDev& d, int cur, int slot, cudaGraphExec_t tail, size_t smem,
                         cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)step_blocks(d));
    cfg.blockDim = dim3(kTB);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, d, cur, slot, tail);
}

template <bool MIXED, bool ENERGY, bool INTEGRATE, bool TAIL, typename ID>
void step_variant_id(const PhysDev& d, int cur, int slot, cudaGraphExec_t tail, cudaStream_t s) {
    const size_t smem = sizeof(float2) * d.n_types * d.n_types;
    if (MIXED && d.use_switch)
        launch_programmatic(k_step_mixed<ENERGY, INTEGRATE, true, TAIL, ID>, d, cur, slot, tail, smem, s);
    else if (MIXED)
        launch_programmatic(k_step_mixed<ENERGY, INTEGRATE, false, TAIL, ID>, d, cur, slot, tail, smem, s);
    else if (d.use_switch)
        launch_programmatic(k_step<ENERGY, INTEGRATE, true, TAIL, ID>, d, cur, slot, tail, smem, s);
    else
        launch_programmatic(k_step<ENERGY, INTEGRATE, false, TAIL, ID>, d, cur, slot, tail, smem, s);
}

template <bool MIXED, bool ENERGY, bool INTEGRATE, bool TAIL>
void step_variant(const PhysDev& d, int cur, int slot, cudaGraphExec_t tail, cudaStream_t s) {
    if (d.nl16)
        step_variant_id<MIXED, ENERGY, INTEGRATE, TAIL, uint16_t>(d, cur, slot, tail, s);
    else
        step_variant_id<MIXED, ENERGY, INTEGRATE, TAIL, uint32_t>(d, cur, slot, tail, s);
}

template <bool MIXED, bool ENERGY, bool INTEGRATE>
void step_tail(const PhysDev& d, int cur, int slot, cudaGraphExec_t tail, cudaStream_t s) {
    if (tail)
        step_variant<MIXED, ENERGY, INTEGRATE, true>(d, cur, slot, tail, s);
    else
        step_variant<MIXED, ENERGY, INTEGRATE, false>(d, cur, slot, nullptr, s);
}

}  // namespace

void launch_sort(const PhysDev& d, const float4* pos, cudaStream_t s) {
    k_sort_count<<<(d.n + kTB - 1) / kTB, kTB, 0, s>>>(d, pos);
    k_sort_scan<<<1, kScanThreads, 0, s>>>(d);
    k_sort_fill<<<(d.n + kTB - 1) / kTB, kTB, 0, s>>>(d);
    k_sort_order<<<(int)(((size_t)d.n_cells * 32 + kTB - 1) / kTB), kTB, 0, s>>>(d);
}

void launch_permute(const PhysDev& d, int cur, bool mixed, cudaStream_t s) {
    k_permute<<<(d.n + kTB - 1) / kTB, kTB, 0, s>>>(d, cur, mixed ? 1 : 0);
}

void launch_set_xref(const PhysDev& d, const float4* pos, cudaStream_t s) {
    k_set_xref<<<(d.n + kTB - 1) / kTB, kTB, 0, s>>>(d, pos);
}

bool list_ids_16bit(int n_pad) { return !kStagedList && n_pad <= 65536; }

void launch_build_list(const PhysDev& d, const float4* pos, const uint32_t* orig, const uint32_t* items, int copy_cur,
                       bool mixed, cudaStream_t s) {
    const int warps = (d.n + 7) / 8;   // 8 particles per warp
    k_build_list<<<(warps + kBuildWarps - 1) / kBuildWarps, kBuildWarps * 32, 0, s>>>(d, pos, orig, items, copy_cur,
                                                                                    mixed ? 1 : 0);
}

namespace {
// position and half-step velocity of orig id o in FP64 (hi + lo)
__device__ __forceinline__ void state_of_orig(const PhysDev& d, int cur, uint32_t o, double* x, double* v) {
    const uint32_t k = d.sorted_of_orig[o];
    const float4 p = d.pos[cur][k], w = d.vel[k];
    x[0] = p.x; x[1] = p.y; x[2] = p.z;
    v[0] = w.x; v[1] = w.y; v[2] = w.z;
    if (d.precision == LIMA_PRECISION_MIXED) {
        const float4 pc = d.posc[k], wc = d.velc[k];
        x[0] += pc.x; x[1] += pc.y; x[2] += pc.z;
        v[0] += wc.x; v[1] += wc.y; v[2] += wc.z;
    }
}

// one thread per compound slot (c, t)
__global__ void k_read_compounds(PhysDev d, int cur, lima_compound_state* __restrict__ states,
                                 lima_float3* __restrict__ prev) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= d.n_c * LIMA_MAX_COMPOUND_PARTICLES) return;
    const int c = q / LIMA_MAX_COMPOUND_PARTICLES, t = q % LIMA_MAX_COMPOUND_PARTICLES;
    const uint32_t b = d.cp_base[c];
    const int n = (int)(d.cp_base[c + 1] - b);
    lima_float3 a = {0.f, 0.f, 0.f}, r = {0.f, 0.f, 0.f};
    if (t < n) {
        double x[3], v[3], x0[3], vv[3];
        state_of_orig(d, cur, b + t, x, v);
        state_of_orig(d, cur, b, x0, vv);
        const double L = d.L;
        double qq[3];
        for (int k = 0; k < 3; k++) {
            double dd = x[k] - x0[k];
            dd -= L * nearbyint(dd / L);
            qq[k] = t == 0 ? x[k] : x0[k] + dd;
        }
        a = lima_float3{(float)qq[0], (float)qq[1], (float)qq[2]};
        r = lima_float3{(float)(qq[0] - v[0] * d.dt), (float)(qq[1] - v[1] * d.dt), (float)(qq[2] - v[2] * d.dt)};
    }
    if (states) {
        states[c].positions[t] = a;
        if (t == 0) {
            // the count and the struct's padding bytes
            uint32_t* tail = reinterpret_cast<uint32_t*>(&states[c].n_particles);
            *tail = (uint32_t)n;
        }
    }
    if (prev) prev[q] = r;
}

__global__ void k_read_solvents(PhysDev d, int cur, lima_solvent* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.n_s) return;
    double x[3], v[3];
    state_of_orig(d, cur, (uint32_t)(d.n_cp + s), x, v);
    out[s].pos = lima_float3{(float)x[0], (float)x[1], (float)x[2]};
    out[s].pos_tsub1 = lima_float3{(float)(x[0] - v[0] * d.dt), (float)(x[1] - v[1] * d.dt), (float)(x[2] - v[2] * d.dt)};
}
}  // namespace

void launch_read_compounds(const PhysDev& d, int cur, lima_compound_state* states, lima_float3* prev, cudaStream_t s) {
    const int n = d.n_c * LIMA_MAX_COMPOUND_PARTICLES;
    if (n > 0) k_read_compounds<<<(n + kTB - 1) / kTB, kTB, 0, s>>>(d, cur, states, prev);
}

void launch_read_solvents(const PhysDev& d, int cur, lima_solvent* out, cudaStream_t s) {
    if (d.n_s > 0) k_read_solvents<<<(d.n_s + kTB - 1) / kTB, kTB, 0, s>>>(d, cur, out);
}

void launch_bonded(const PhysDev& d, int cur, bool energy, cudaStream_t s) {
    const int nb = bonded_blocks(d);
    const bool mixed = d.precision == LIMA_PRECISION_MIXED;
    if (energy && mixed)
        k_bonded<true, true><<<nb, kTB, 0, s>>>(d, cur);
    else if (energy)
        k_bonded<true, false><<<nb, kTB, 0, s>>>(d, cur);
    else if (mixed)
        k_bonded<false, true><<<nb, kTB, 0, s>>>(d, cur);
    else
        k_bonded<false, false><<<nb, kTB, 0, s>>>(d, cur);
}

void launch_step(const PhysDev& d, int cur, bool mixed, bool energy, bool integrate, int slot, cudaGraphExec_t tail,
                 cudaStream_t s) {
    if (mixed) {
        if (!integrate) step_variant<true, true, false, false>(d, cur, slot, nullptr, s);
        else if (energy) step_tail<true, true, true>(d, cur, slot, tail, s);
        else step_tail<true, false, true>(d, cur, slot, tail, s);
    } else {
        if (!integrate) step_variant<false, true, false, false>(d, cur, slot, nullptr, s);
        else if (energy) step_tail<false, true, true>(d, cur, slot, tail, s);
        else step_tail<false, false, true>(d, cur, slot, tail, s);
    }
}

}  // namespace lima
