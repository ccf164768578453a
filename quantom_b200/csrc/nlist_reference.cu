// Neighbour-list build with the reference's semantics, on the device.
//
// The reference rebuilds its lists on the host every 200 steps in a detached
// thread (Engine::handleNLISTS / updateNeighborLists / cullDistantNeighbors,
// Quantom/Quantom/Engine.cu:88-287): O(N^2) candidate loops, cull-by-
// swap-remove, hash-table de-duplication.  As sets, its result is:
//   solvent-solvent   {i<j : within(pos_i, pos_j, C + C)}           (:198, :264)
//   compound-solvent  {(c,s) : within(key_c, pos_s, C + (r_c + C))} (:182, :231)
//   compound-compound {i<j : (prev(i,j) and within(key_i, key_j, C + ((r_i + r_j) + C)))
//                             or within(key_i, key_j, C + ((r_i + r_i) + C))}  (:168, :243-246)
// where within() is neighborWithinCutoff (:146-151) — minimum image by
// applyHyperpos, then sqrtf(x*x+y*y+z*z) < limit in float — always evaluated
// with the lower id first, r = confining_particle_sphere and key_c the key
// particle's position.  Here: a uniform cell grid (cells >= 2C) and one warp
// per solvent for solvent-solvent, one block per compound for compound-solvent,
// one thread per compound for compound-compound.  This file is compiled with
// -fmad=false, so the distance test is bit-identical to the host code.  Lists
// come out sorted ascending (the reference's order after a build from empty
// lists).  Overflow sets an error bit instead of exit(1) (Bodies.cuh:215-245).
#include "refdev.cuh"
#include "refmath.cuh"

namespace lima {
using namespace refm;

namespace {

// cell of a coordinate's periodic image in [0, L): a position a little
// outside the box (as loaded, before the first step wraps it) still lands in
// the cell its neighbours search
__device__ __forceinline__ int cell_of(float x, float L, float cell, int m) {
    x -= L * floorf(x / L);
    int c = (int)(x / cell);
    return c < 0 ? 0 : (c >= m ? m - 1 : c);
}

__global__ void k_cell_count(RefDev d, int cur) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.n_s) return;
    float4 p = d.spos[cur][s];
    int k = (cell_of(p.x, d.L, d.cell, d.m) * d.m + cell_of(p.y, d.L, d.cell, d.m)) * d.m + cell_of(p.z, d.L, d.cell, d.m);
    d.sol_cell[s] = k;
    atomicAdd(&d.cell_count[k], 1u);
}

// exclusive scan of n counts by one block of 1024 threads
__global__ void k_scan(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int n) {
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < n; base += blockDim.x) {
        int i = base + threadIdx.x;
        uint32_t v = i < n ? in[i] : 0;
        uint32_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t t = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            warp_tot[lane] = t;   // inclusive over warps
        }
        __syncthreads();
        uint32_t before = (w ? warp_tot[w - 1] : 0) + carry;
        if (i < n) out[i] = before + x - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = before + x;
        __syncthreads();
    }
}

__global__ void k_cell_fill(RefDev d) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.n_s) return;
    uint32_t k = d.sol_cell[s];
    uint32_t slot = d.cell_start[k] + atomicAdd(&d.cell_fill[k], 1u);
    d.cell_items[slot] = s;
}

// One warp per solvent.  Candidates from the 27 surrounding cells are tested
// with the reference's float expression, collected in shared memory, sorted
// ascending (bitonic, in the warp) and written column-major:
// ss_ids[k * n_s + i] so that the force kernel's per-thread reads coalesce.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_ss_list(RefDev d, int cur, int cap_pow2) {
    extern __shared__ uint32_t sbuf[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i = blockIdx.x * WARPS + w;
    if (i >= d.n_s) return;
    uint32_t* buf = sbuf + w * cap_pow2;
    const F3 pi = mk4(d.spos[cur][i]);
    const int m = d.m;
    const int span = m >= 3 ? 1 : 0;
    const int cx = cell_of(pi.x, d.L, d.cell, m), cy = cell_of(pi.y, d.L, d.cell, m), cz = cell_of(pi.z, d.L, d.cell, m);
    int cnt = 0;
    for (int dx = -span; dx <= span; dx++)
        for (int dy = -span; dy <= span; dy++)
            for (int dz = -span; dz <= span; dz++) {
                const int k = (((cx + dx + m) % m) * m + ((cy + dy + m) % m)) * m + ((cz + dz + m) % m);
                const uint32_t start = d.cell_start[k], count = d.cell_count[k];
                for (uint32_t b = 0; b < count; b += 32) {
                    bool ok = false;
                    uint32_t j = 0;
                    if (b + lane < count) {
                        j = d.cell_items[start + b + lane];
                        if ((int)j != i) {
                            const F3 pj = mk4(d.spos[cur][j]);
                            ok = ((int)j > i) ? within(pi, pj, d.C, d.C, d.L, d.Lh) : within(pj, pi, d.C, d.C, d.L, d.Lh);
                        }
                    }
                    const unsigned bal = __ballot_sync(0xffffffffu, ok);
                    const int pos = cnt + __popc(bal & ((1u << lane) - 1u));
                    if (ok && pos < cap_pow2) buf[pos] = j;
                    cnt += __popc(bal);
                }
            }
    const int kept = cnt < cap_pow2 ? cnt : cap_pow2;
    int P = 32;
    while (P < kept) P <<= 1;
    for (int t = kept + lane; t < P; t += 32) buf[t] = 0xffffffffu;
    __syncwarp();
    for (int k = 2; k <= P; k <<= 1)
        for (int jj = k >> 1; jj > 0; jj >>= 1) {
            for (int t = lane; t < P; t += 32) {
                const int ixj = t ^ jj;
                if (ixj > t) {
                    const uint32_t a = buf[t], b = buf[ixj];
                    const bool up = (t & k) == 0;
                    if ((a > b) == up) {
                        buf[t] = b;
                        buf[ixj] = a;
                    }
                }
            }
            __syncwarp();
        }
    const int out = kept < d.ss_cap ? kept : d.ss_cap;
    for (int t = lane; t < out; t += 32) d.ss_ids[(size_t)t * d.n_s + i] = buf[t];
    if (lane == 0) {
        d.ss_cnt[i] = out;
        if (cnt > d.ss_cap) atomicOr(d.err, ERR_BIT_SS_OVERFLOW);
    }
}

// One block per compound; solvents scanned in ascending id order with an
// ordered block-wide compaction, so the row comes out sorted.
__global__ void __launch_bounds__(256) k_cs_list(RefDev d, int cur) {
    __shared__ uint32_t warp_cnt[8];
    __shared__ int total;
    const int c = blockIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const lima_compound& cp = d.comps[c];
    const F3 key = mk4(d.cpos[cur][c * kMaxCP + cp.key_particle_index]);
    const float off = cp.confining_particle_sphere + d.C;
    if (threadIdx.x == 0) total = 0;
    __syncthreads();
    for (int base = 0; base < d.n_s; base += 256) {
        const int s = base + threadIdx.x;
        bool ok = false;
        if (s < d.n_s) ok = within(key, mk4(d.spos[cur][s]), d.C, off, d.L, d.Lh);
        const unsigned bal = __ballot_sync(0xffffffffu, ok);
        if (lane == 0) warp_cnt[w] = __popc(bal);
        __syncthreads();
        int before = total;
        for (int q = 0; q < w; q++) before += warp_cnt[q];
        const int pos = before + __popc(bal & ((1u << lane) - 1u));
        if (ok && pos < d.cs_cap) d.cs_ids[(size_t)c * d.cs_cap + pos] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = total;
            for (int q = 0; q < 8; q++) t += warp_cnt[q];
            total = t;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        d.cs_cnt[c] = total < d.cs_cap ? total : d.cs_cap;
        if (total > d.cs_cap) atomicOr(d.err, ERR_BIT_CS_OVERFLOW);
    }
}

// One block, thread i builds compound i's list (ascending); previous
// membership is read before any thread overwrites it.
__global__ void k_cc_list(RefDev d, int cur) {
    const int i = threadIdx.x;
    const int n = d.n_c;
    int cnt = 0;
    bool overflow = false;
    if (i < n) {
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            const int lo = i < j ? i : j, hi = i < j ? j : i;
            const lima_compound& a = d.comps[lo];
            const lima_compound& b = d.comps[hi];
            const F3 klo = mk4(d.cpos[cur][lo * kMaxCP + a.key_particle_index]);
            const F3 khi = mk4(d.cpos[cur][hi * kMaxCP + b.key_particle_index]);
            const float rlo = a.confining_particle_sphere, rhi = b.confining_particle_sphere;
            const bool keep = d.cc_prev[lo * n + hi] && within(klo, khi, d.C, rlo + rhi + d.C, d.L, d.Lh);
            const bool add = within(klo, khi, d.C, rlo + rlo + d.C, d.L, d.Lh);
            if (keep || add) {
                if (cnt < kMaxCP) d.cc_ids[i * kMaxCP + cnt] = j;
                else overflow = true;
                cnt++;
            }
        }
    }
    __syncthreads();
    if (i < n) {
        const int kept = cnt < kMaxCP ? cnt : kMaxCP;
        d.cc_cnt[i] = kept;
        for (int j = 0; j < n; j++) d.cc_prev[i * n + j] = 0;
        for (int q = 0; q < kept; q++) d.cc_prev[i * n + d.cc_ids[i * kMaxCP + q]] = 1;
        if (overflow) atomicOr(d.err, ERR_BIT_CC_OVERFLOW);
    }
}

}  // namespace

void ref_build_nlists(const RefDev& d, int cur, cudaStream_t s) {
    if (d.n_s > 0) {
        const int ncells = d.m * d.m * d.m;
        cudaMemsetAsync(d.cell_count, 0, sizeof(uint32_t) * ncells, s);
        cudaMemsetAsync(d.cell_fill, 0, sizeof(uint32_t) * ncells, s);
        const int tb = 256, nb = (d.n_s + tb - 1) / tb;
        k_cell_count<<<nb, tb, 0, s>>>(d, cur);
        k_scan<<<1, 1024, 0, s>>>(d.cell_count, d.cell_start, ncells);
        k_cell_fill<<<nb, tb, 0, s>>>(d);
        int cap2 = 32;
        while (cap2 < d.ss_cap) cap2 <<= 1;
        constexpr int W = 4;
        k_ss_list<W><<<(d.n_s + W - 1) / W, W * 32, W * cap2 * sizeof(uint32_t), s>>>(d, cur, cap2);
    }
    if (d.n_c > 0) {
        if (d.n_s > 0) k_cs_list<<<d.n_c, 256, 0, s>>>(d, cur);
        k_cc_list<<<1, ((d.n_c + 31) / 32) * 32, 0, s>>>(d, cur);
    }
}

}  // namespace lima

// ---------------------------------------------------------------------------
// Solvent-solvent list build that allocates no memory.
//
// Who needs it: a caller that owns its device memory and cannot hand the
// library an allocation: a host that reserved the device's memory up front,
// or a stepping loop that must not call cudaMalloc/cudaFree, which can block
// on work queued on other streams and can fail once that memory is spoken
// for.  Such a caller cannot create a lima_ctx, whose buffers lima_finish_box
// allocates.  This entry point runs the same kernels as the context's build
// (k_cell_count, k_scan, k_cell_fill, k_ss_list) on caller-owned device
// buffers.  Its cell grid and the staged float4 positions live in
// g_noalloc_scratch, one file-scope device array of kNaScratchBytes
// (1,966,080 bytes): at most LIMA_NOALLOC_MAX_SOLVENTS solvents and a grid of
// at most 32^3 cells.  A coarser grid leaves the sorted lists unchanged.
//
// The array is shared by every call on a device, so calls that overlap in
// time (other streams, other host threads) race.
#include <cmath>
#include <cstdio>
#include <mutex>

namespace {
constexpr int kNaMaxM = 32;
constexpr size_t kNaPosBytes = static_cast<size_t>(LIMA_NOALLOC_MAX_SOLVENTS) * sizeof(float4);
constexpr size_t kNaItemBytes = static_cast<size_t>(LIMA_NOALLOC_MAX_SOLVENTS) * sizeof(uint32_t);
constexpr size_t kNaCellBytes = static_cast<size_t>(kNaMaxM) * kNaMaxM * kNaMaxM * sizeof(uint32_t);
// regions: pos4 | cell_items | sol_cell | cell_count | cell_start | cell_fill (each a multiple of 256 B)
constexpr size_t kNaScratchBytes = kNaPosBytes + 2 * kNaItemBytes + 3 * kNaCellBytes;
static_assert(kNaPosBytes % 256 == 0 && kNaItemBytes % 256 == 0 && kNaCellBytes % 256 == 0, "region alignment");
constexpr int kNaMaxDevices = 64;
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaScratchBytes];

namespace lima {
namespace {

std::mutex g_na_mu;
void* g_na_addr[kNaMaxDevices] = {};

__global__ void k_na_stage(const lima_solvent* __restrict__ sol, float4* __restrict__ pos, int n) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) {
        const lima_float3 p = sol[s].pos;
        pos[s] = make_float4(p.x, p.y, p.z, 0.f);
    }
}

lima_status na_fail(char* err, size_t err_len, lima_status st, const char* msg) {
    if (err && err_len) std::snprintf(err, err_len, "%s", msg);
    return st;
}

}  // namespace
}  // namespace lima

extern "C" lima_status lima_ss_nlist_noalloc(const lima_solvent* d_solvents, int n_solvents, float box_len,
                                             float cutoff, int capacity, uint32_t* d_ids, uint32_t* d_counts,
                                             int* d_overflow, void* stream, char* err, size_t err_len) {
    using namespace lima;
    char msg[160];
    if (err && err_len) err[0] = '\0';
    if (n_solvents < 1) return na_fail(err, err_len, LIMA_ERR_ARGUMENT, "n_solvents must be at least 1");
    if (n_solvents > LIMA_NOALLOC_MAX_SOLVENTS) {
        std::snprintf(msg, sizeof msg, "n_solvents %d exceeds the no-allocation maximum of %d", n_solvents,
                      LIMA_NOALLOC_MAX_SOLVENTS);
        return na_fail(err, err_len, LIMA_ERR_CAPACITY, msg);
    }
    if (capacity < 32 || capacity > 2048)
        return na_fail(err, err_len, LIMA_ERR_CAPACITY, "capacity outside 32..2048");
    if (!(box_len > 0.f) || !std::isfinite(box_len) || !(cutoff > 0.f) || !std::isfinite(cutoff))
        return na_fail(err, err_len, LIMA_ERR_ARGUMENT, "box_len and cutoff must be positive and finite");
    if (!d_solvents || !d_ids || !d_counts || !d_overflow)
        return na_fail(err, err_len, LIMA_ERR_ARGUMENT, "null device buffer");
    if ((reinterpret_cast<uintptr_t>(d_solvents) | reinterpret_cast<uintptr_t>(d_ids) |
         reinterpret_cast<uintptr_t>(d_counts) | reinterpret_cast<uintptr_t>(d_overflow)) & 3u)
        return na_fail(err, err_len, LIMA_ERR_ARGUMENT, "device buffers must be 4-byte aligned");

    // scratch address on the current device, looked up on the first call there
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return na_fail(err, err_len, LIMA_ERR_CUDA, "cudaGetDevice failed");
    if (dev < 0 || dev >= kNaMaxDevices) return na_fail(err, err_len, LIMA_ERR_UNSUPPORTED, "device ordinal >= 64");
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_na_mu);
        if (!g_na_addr[dev]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                std::snprintf(msg, sizeof msg, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
                return na_fail(err, err_len, LIMA_ERR_CUDA, msg);
            }
            g_na_addr[dev] = p;
        }
        base = static_cast<unsigned char*>(g_na_addr[dev]);
    }

    RefDev d{};
    d.n_s = n_solvents;
    d.L = box_len;
    d.Lh = box_len / 2.f;
    d.C = cutoff;
    // the context's grid rule (cells no smaller than the list radius C + C), capped at 32 per side
    const float radius = d.C + d.C;
    int m = static_cast<int>(std::floor(d.L / (radius * 1.0001f)));
    if (m < 3) m = 1;
    while (m > 1 && d.L / static_cast<float>(m) < radius) m--;
    if (m < 3) m = 1;
    if (m > kNaMaxM) m = kNaMaxM;
    d.m = m;
    d.cell = d.L / static_cast<float>(m);
    const int ncells = m * m * m;
    float4* pos4 = reinterpret_cast<float4*>(base);
    d.spos[0] = d.spos[1] = pos4;
    d.cell_items = reinterpret_cast<uint32_t*>(base + kNaPosBytes);
    d.sol_cell = reinterpret_cast<uint32_t*>(base + kNaPosBytes + kNaItemBytes);
    d.cell_count = reinterpret_cast<uint32_t*>(base + kNaPosBytes + 2 * kNaItemBytes);
    d.cell_start = reinterpret_cast<uint32_t*>(base + kNaPosBytes + 2 * kNaItemBytes + kNaCellBytes);
    d.cell_fill = reinterpret_cast<uint32_t*>(base + kNaPosBytes + 2 * kNaItemBytes + 2 * kNaCellBytes);
    d.ss_ids = d_ids;
    d.ss_cnt = d_counts;
    d.ss_cap = capacity;
    d.err = d_overflow;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // start at zero: the per-cell counters (atomic counts and fill cursors) and the overflow flag
    cudaError_t e = cudaMemsetAsync(d.cell_count, 0, sizeof(uint32_t) * ncells, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d.cell_fill, 0, sizeof(uint32_t) * ncells, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_overflow, 0, sizeof(int), s);
    if (e != cudaSuccess) {
        std::snprintf(msg, sizeof msg, "cudaMemsetAsync: %s", cudaGetErrorString(e));
        return na_fail(err, err_len, LIMA_ERR_CUDA, msg);
    }
    const int tb = 256, nb = (n_solvents + tb - 1) / tb;
    k_na_stage<<<nb, tb, 0, s>>>(d_solvents, pos4, n_solvents);
    k_cell_count<<<nb, tb, 0, s>>>(d, 0);
    k_scan<<<1, 1024, 0, s>>>(d.cell_count, d.cell_start, ncells);
    k_cell_fill<<<nb, tb, 0, s>>>(d);
    int cap2 = 32;
    while (cap2 < capacity) cap2 <<= 1;
    constexpr int W = 4;
    k_ss_list<W><<<(n_solvents + W - 1) / W, W * 32, W * cap2 * sizeof(uint32_t), s>>>(d, 0, cap2);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::snprintf(msg, sizeof msg, "kernel launch: %s", cudaGetErrorString(e));
        return na_fail(err, err_len, LIMA_ERR_CUDA, msg);
    }
    return LIMA_OK;
}
