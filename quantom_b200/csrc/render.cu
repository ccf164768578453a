// Headless rasterizer: the reference's Rasterizer (Rasterizer.cu:12-294) and
// the picture its display draws from it (DisplayV2.cpp:13-51), as CUDA
// kernels into device buffers.  There is no window: lima_render returns the
// RenderBall list, lima_render_image an RGB image.
//
//   k_slot_pos   physics: positions of the sorted particle arrays into the
//                reference's slot layout (compound c particle l at c*64 + l,
//                solvents after), compounds in the image of their particle 0
//   k_balls      per slot: atom type -> colour and radius, position ->
//                normalised device coordinates (Rasterizer.cu:229-251); the
//                depth key is the normalised y
//   cub radix sort of the keys (stable, slots fed in reverse order so equal
//                depths keep descending slot order), k_gather_balls into that
//                order (the reference's host merge sort by pos.y,
//                Rasterizer.cu:254-293)
//   k_splat      one warp per ball over its pixel bounding box: each covered
//                pixel keeps the smallest sorted index (atomicMin), i.e. the
//                ball the display draws last (it draws from the back,
//                DisplayV2.cpp:41-47)
//   k_shade      per pixel: the winning ball's colour times the triangle
//                fan's Gouraud light, 0.5 at the centre and (1 + sin a) / 2
//                on the rim, i.e. 0.5 + 0.5 * dy / R
// Every product and sum is an explicitly rounded operation (no contraction),
// so the C restatement in the oracle reproduces the output bit for bit.
#include <cub/device/device_radix_sort.cuh>

#include "render.cuh"

namespace lima {
namespace {

constexpr int kRT = 256;

// ATOM_TYPE (QuantomTypes.cuh:16)
enum : uint8_t { AT_NONE = 0, AT_O = 1, AT_C = 2, AT_P = 3, AT_N = 4, AT_H = 5, AT_SOL = 6, AT_S = 7 };

__device__ __forceinline__ void type_color(uint8_t t, int* c) {   // getColor, Rasterizer.cu:168-189
    int r = 0, g = 0, b = 0;
    switch (t) {
        case AT_SOL: r = 0x03; g = 0xa9; b = 0xf4; break;
        case AT_H: r = 0xF1; g = 0xF1; b = 0xF1; break;
        case AT_O: r = 0xE0; g = 0x20; b = 0x20; break;
        case AT_C: r = 0x30; g = 0x10; b = 0x90; break;
        case AT_P: r = 0xFC; g = 0xF7; b = 0x5E; break;
        case AT_N: r = 0x2E; g = 0x8B; b = 0x57; break;
        case AT_NONE: r = 0xF2; g = 0xE5; b = 0xD9; break;
        default: break;
    }
    c[0] = r;
    c[1] = g;
    c[2] = b;
}

__device__ __forceinline__ float type_radius(uint8_t t) {   // getRadius, Rasterizer.cu:191-213
    switch (t) {
        case AT_H: return 0.04f;
        case AT_C: return 0.1f;
        case AT_N: return 0.1f;
        case AT_O: return 0.12f;
        case AT_SOL: return 0.08f;
        case AT_P: return 0.15f;
        default: return 1.f;
    }
}

__global__ void k_slot_pos(PhysDev d, int cur, const uint32_t* __restrict__ ref_slot, float4* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.n) return;
    const uint32_t o = d.orig_of_sorted[k];
    const uint32_t slot = ref_slot[o];
    float4 p = d.pos[cur][k];
    const uint32_t l = slot % LIMA_MAX_COMPOUND_PARTICLES;
    if (o < (uint32_t)d.n_cp && l != 0) {
        const float4 p0 = d.pos[cur][d.sorted_of_orig[o - l]];
        const double L = (double)d.L;
        double dd = (double)p.x - (double)p0.x;
        dd -= L * rint(dd / L);
        p.x = (float)((double)p0.x + dd);
        dd = (double)p.y - (double)p0.y;
        dd -= L * rint(dd / L);
        p.y = (float)((double)p0.y + dd);
        dd = (double)p.z - (double)p0.z;
        dd -= L * rint(dd / L);
        p.z = (float)((double)p0.z + dd);
    }
    out[slot] = p;
}

__global__ void k_balls(const float4* __restrict__ pos, const uint8_t* __restrict__ kind, int n, float L,
                        lima_render_ball* __restrict__ balls, float* __restrict__ keys, uint32_t* __restrict__ vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t t = kind[i];
    // an empty compound slot sits at the box origin (the reference leaves it unset)
    const float4 p = t == AT_NONE ? make_float4(0.f, 0.f, 0.f, 0.f) : pos[i];
    lima_render_ball b;
    int c[3];
    type_color(t, c);
    // radius / (1 + y * 0.001) in nm, then a quarter of it (Rasterizer.cu:236-240)
    const float rad = __fdiv_rn(type_radius(t), __fadd_rn(1.f, __fmul_rn(p.y, 0.001f)));
    b.radius = __fmul_rn(0.25f, rad);
    // (x / L - 0.5) * 1.8 in double (Rasterizer.cu:241-243)
    const double dl = (double)L;
    b.pos.x = (float)(__dmul_rn(__dadd_rn(__ddiv_rn((double)p.x, dl), -0.5), 1.8));
    b.pos.y = (float)(__dmul_rn(__dadd_rn(__ddiv_rn((double)p.y, dl), -0.5), 1.8));
    b.pos.z = (float)(__dmul_rn(__dadd_rn(__ddiv_rn((double)p.z, dl), -0.5), 1.8));
    b.color[0] = c[0];
    b.color[1] = c[1];
    b.color[2] = c[2];
    b.disable = t == AT_NONE ? 1 : 0;
    b.pad[0] = b.pad[1] = b.pad[2] = 0;
    balls[i] = b;
    // slots enter the stable sort in reverse order: equal depths come out in
    // descending slot order, as the reference's merge, which takes the right
    // half's ball on a tie (Rasterizer.cu:254-271), leaves them
    keys[n - 1 - i] = b.pos.y;
    vals[n - 1 - i] = (uint32_t)i;
}

__global__ void k_gather_balls(const lima_render_ball* __restrict__ in, const uint32_t* __restrict__ order, int n,
                               lima_render_ball* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[order[i]];
}

// pixel centre (px, py) in normalised device coordinates: x right, y up
__device__ __forceinline__ float ndc_x(int px, int w) {
    return __fadd_rn(__fdiv_rn((float)(2 * px + 1), (float)w), -1.f);
}
__device__ __forceinline__ float ndc_y(int py, int h) {
    return __fadd_rn(1.f, -__fdiv_rn((float)(2 * py + 1), (float)h));
}

__device__ __forceinline__ bool covers(const lima_render_ball& b, float x, float y) {
    const float dx = __fadd_rn(x, -b.pos.x), dy = __fadd_rn(y, -b.pos.z);
    return __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)) <= __fmul_rn(b.radius, b.radius);
}

__global__ void k_splat(const lima_render_ball* __restrict__ balls, int n, int w, int h, uint32_t* __restrict__ win) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (warp >= n) return;
    const lima_render_ball b = balls[warp];
    if (b.disable) return;
    // pixel box of the disc (one pixel of margin; the test per pixel is exact)
    const float hw = 0.5f * (float)w, hh = 0.5f * (float)h;
    int x0 = (int)floorf((b.pos.x - b.radius + 1.f) * hw) - 1, x1 = (int)ceilf((b.pos.x + b.radius + 1.f) * hw) + 1;
    int y0 = (int)floorf((1.f - b.pos.z - b.radius) * hh) - 1, y1 = (int)ceilf((1.f - b.pos.z + b.radius) * hh) + 1;
    x0 = max(x0, 0);
    y0 = max(y0, 0);
    x1 = min(x1, w - 1);
    y1 = min(y1, h - 1);
    if (x0 > x1 || y0 > y1) return;
    const int bw = x1 - x0 + 1;
    const int np = bw * (y1 - y0 + 1);
    for (int q = lane; q < np; q += 32) {
        const int px = x0 + q % bw, py = y0 + q / bw;
        if (covers(b, ndc_x(px, w), ndc_y(py, h))) atomicMin(&win[(size_t)py * w + px], (uint32_t)warp);
    }
}

__global__ void k_shade(const lima_render_ball* __restrict__ balls, const uint32_t* __restrict__ win, int w, int h,
                        uint8_t* __restrict__ rgb) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= w * h) return;
    const uint32_t k = win[p];
    uint8_t* o = rgb + 3 * (size_t)p;
    if (k == 0xffffffffu) {   // glClear: black
        o[0] = o[1] = o[2] = 0;
        return;
    }
    const lima_render_ball b = balls[k];
    const float dy = __fadd_rn(ndc_y(p / w, h), -b.pos.z);
    const float light = __fadd_rn(0.5f, __fmul_rn(0.5f, __fdiv_rn(dy, b.radius)));
    // Int3 * float = floor per channel (QuantomTypes.cuh:27), then glColor3ub
    for (int q = 0; q < 3; q++) o[q] = (uint8_t)(int)floorf(__fmul_rn((float)b.color[q], light));
}

template <typename T>
T* alloc(std::vector<void*>& allocs, size_t n) {
    void* ptr = nullptr;
    if (cudaMalloc(&ptr, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    allocs.push_back(ptr);
    return static_cast<T*>(ptr);
}

}  // namespace

bool render_setup(RenderBuf& r, int n_slots, const std::vector<uint8_t>& kind, const std::vector<uint32_t>& ref_slot,
                  std::vector<void*>& allocs, cudaStream_t s) {
    if (r.ready) return true;
    r.n_slots = n_slots;
    r.kind = alloc<uint8_t>(allocs, n_slots);
    r.slot_pos = alloc<float4>(allocs, n_slots);
    r.balls[0] = alloc<lima_render_ball>(allocs, n_slots);
    r.balls[1] = alloc<lima_render_ball>(allocs, n_slots);
    for (int b = 0; b < 2; b++) {
        r.keys[b] = alloc<float>(allocs, n_slots);
        r.vals[b] = alloc<uint32_t>(allocs, n_slots);
    }
    r.ref_slot = ref_slot.empty() ? nullptr : alloc<uint32_t>(allocs, ref_slot.size());
    if (!r.kind || !r.slot_pos || !r.balls[0] || !r.balls[1] || !r.keys[0] || !r.keys[1] || !r.vals[0] || !r.vals[1] ||
        (!ref_slot.empty() && !r.ref_slot))
        return false;
    cub::DeviceRadixSort::SortPairs(nullptr, r.sort_bytes, r.keys[0], r.keys[1], r.vals[0], r.vals[1], n_slots, 0, 32,
                                    s);
    r.sort_tmp = alloc<uint8_t>(allocs, r.sort_bytes);
    if (!r.sort_tmp) return false;
    cudaMemcpyAsync(r.kind, kind.data(), n_slots, cudaMemcpyHostToDevice, s);
    if (r.ref_slot)
        cudaMemcpyAsync(r.ref_slot, ref_slot.data(), sizeof(uint32_t) * ref_slot.size(), cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    r.ready = true;
    return true;
}

void render_slot_positions_phys(const RenderBuf& r, const PhysDev& d, int cur, cudaStream_t s) {
    cudaMemsetAsync(r.slot_pos, 0, sizeof(float4) * r.n_slots, s);
    k_slot_pos<<<(d.n + kRT - 1) / kRT, kRT, 0, s>>>(d, cur, r.ref_slot, r.slot_pos);
}

int render_balls(RenderBuf& r, float L, cudaStream_t s) {
    const int n = r.n_slots;
    const int nb = (n + kRT - 1) / kRT;
    k_balls<<<nb, kRT, 0, s>>>(r.slot_pos, r.kind, n, L, r.balls[0], r.keys[0], r.vals[0]);
    size_t bytes = r.sort_bytes;
    cub::DeviceRadixSort::SortPairs(r.sort_tmp, bytes, r.keys[0], r.keys[1], r.vals[0], r.vals[1], n, 0, 32, s);
    k_gather_balls<<<nb, kRT, 0, s>>>(r.balls[0], r.vals[1], n, r.balls[1]);
    return 2;
}

bool render_image(RenderBuf& r, int w, int h, uint8_t* host_rgb, std::vector<void*>& allocs, cudaStream_t s) {
    const size_t np = (size_t)w * h;
    if (np > r.img_pixels) {
        r.win = alloc<uint32_t>(allocs, np);
        r.rgb = alloc<uint8_t>(allocs, 3 * np);
        if (!r.win || !r.rgb) return false;
        r.img_pixels = np;
    }
    cudaMemsetAsync(r.win, 0xff, sizeof(uint32_t) * np, s);
    const int n = r.n_slots;
    k_splat<<<(int)(((size_t)n * 32 + kRT - 1) / kRT), kRT, 0, s>>>(r.balls[1], n, w, h, r.win);
    k_shade<<<(int)((np + kRT - 1) / kRT), kRT, 0, s>>>(r.balls[1], r.win, w, h, r.rgb);
    cudaMemcpyAsync(host_rgb, r.rgb, 3 * np, cudaMemcpyDeviceToHost, s);
    return true;
}

}  // namespace lima
