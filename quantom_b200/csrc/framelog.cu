// Frame log of the physics path (framelog.cuh).
//
//   k_log_frame  one thread per particle: position (traj_buffer) and
//                potential energy (potE_buffer) into the reference slot of
//                the particle; compound particles also their position into
//                the train record (data_GAN value 0); thread 0 the frame's
//                FP64 energies from the step's accumulator slot and the
//                reference's 10-float log line of particle 0 (outdata).
//                With no per-particle array logged, one block writes the
//                energies and that line.  Its last block moves the device
//                ring position on, so a step graph can hold the frame.
//   k_log_train  8 lanes per compound particle over its Verlet list: the LJ
//                force from solvent neighbours only (data_GAN value 1,
//                Engine.cu:1034 force_LJ_sol), reduced with warp shuffles
#include <algorithm>
#include <cstring>
#include <type_traits>

#include "framelog.cuh"
#include "physkern.cuh"
#include "physmath.cuh"
#include "refdev.cuh"
#include "refmath.cuh"

namespace lima {
namespace {

// the ring position of the frame being written
__device__ __forceinline__ int ring_pos(const FrameLogDev& g) {
    return (int)(__ldcg(g.frame_ctr) % (unsigned long long)g.ring);
}

// one particle's entries of frame r
__device__ __forceinline__ void log_frame_particle(const PhysDev& d, const FrameLogDev& g, int cur, int r, int k) {
    const uint32_t o = d.orig_of_sorted[k];
    const uint32_t slot = g.ref_slot[o];
    float4 p = d.pos[cur][k];
    const float4 f = d.force[k];
    const uint32_t l = slot % LIMA_MAX_COMPOUND_PARTICLES;
    if (o < (uint32_t)d.n_cp && l != 0) {
        // a compound's particles in the periodic image of its particle 0, as the
        // reference keeps them (applyHyperpos, Engine.cu:996) and lima_get_compound_states
        // returns them: p0 + minimum image of (p - p0), in double
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
    if (g.traj) {
        float* t = g.traj + ((size_t)r * g.n_slots + slot) * 3;
        t[0] = p.x;
        t[1] = p.y;
        t[2] = p.z;
    }
    if (g.potE) g.potE[(size_t)r * g.n_slots + slot] = (double)f.w;
    if (g.train && o < (uint32_t)d.n_cp) {
        float* t = g.train + ((size_t)r * g.n_train + slot) * (kTrainValues * 3);
        t[0] = p.x;
        t[1] = p.y;
        t[2] = p.z;
    }
    if (o == 0 && g.logdata) {
        // the reference's outdata line of compound 0 particle 0 (Engine.cu:1022-1029):
        // speed over the step, kinetic energy, potential energy, |force|
        const float4 v = d.vel[k];   // velocity of the half step just taken, w = 1/m
        const float v2 = v.x * v.x + v.y * v.y + v.z * v.z;
        float* l = g.logdata + (size_t)r * kLogDataFloats;
        l[0] = sqrtf(v2);
        l[1] = 0.5f * v2 / v.w;
        l[2] = f.w;
        l[3] = sqrtf(f.x * f.x + f.y * f.y + f.z * f.z);
        for (int q = 4; q < kLogDataFloats; q++) l[q] = 0.f;
    }
}

// per_particle 0 (no per-particle arrays logged): one block, whose thread 0
// writes the energies and the log line of particle 0
__global__ void __launch_bounds__(kTB) k_log_frame(PhysDev d, FrameLogDev g, int cur, int per_particle) {
    const int k = per_particle ? (int)(blockIdx.x * blockDim.x + threadIdx.x)
                               : (threadIdx.x == 0 ? (int)d.sorted_of_orig[0] : d.n);
    const int r = ring_pos(g);
    if (blockIdx.x == 0 && threadIdx.x == 0 && g.energies) {   // the step kernel's FP64 totals of the logged step
        double* e = g.energies + (size_t)r * LIMA_E_COUNT;
        for (int q = 0; q < LIMA_E_COUNT; q++) e[q] = d.e_last[q];
    }
    if (k < d.n) log_frame_particle(d, g, cur, r, k);
    // the last block to finish moves the ring on (every block has read r)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(g.blocks_done, 1u) == gridDim.x - 1u) {
            *g.blocks_done = 0u;
            *g.frame_ctr += 1ull;
        }
    }
}

template <bool SWITCH>
__global__ void __launch_bounds__(kTB) k_log_train(PhysDev d, FrameLogDev g, int cur) {
    const int r = ring_pos(g);   // k_log_frame of the same frame runs after this kernel
    extern __shared__ float2 s_tab[];
    const int nt2 = d.n_types * d.n_types;
    for (int q = threadIdx.x; q < nt2; q += blockDim.x) s_tab[q] = d.lj_table[q];
    __syncthreads();
    const int o = (blockIdx.x * blockDim.x + threadIdx.x) / kGroup;
    const int lane = threadIdx.x % kGroup;
    const bool active = o < d.n_cp;
    float fx = 0.f, fy = 0.f, fz = 0.f, e = 0.f, w = 0.f;
    if (active) {
        const int i = (int)d.sorted_of_orig[o];
        const float4* __restrict__ pos = d.pos[cur];
        const float4 pi = pos[i];
        const float2* row = &s_tab[__float_as_int(pi.w) * d.n_types];
        const int cnt = (int)d.nl_cnt[i];
        for (int k = lane; k < cnt; k += kGroup) {
            const uint32_t j = nl_load(d, nl_word((uint32_t)d.n_pad, (uint32_t)i, (uint32_t)k));
            if (d.orig_of_sorted[j] < (uint32_t)d.n_cp) continue;   // solvent neighbours only
            lj_pair<false, SWITCH>(d, row, pi, pos[j], fx, fy, fz, e, w);
        }
    }
#pragma unroll
    for (int q = kGroup / 2; q > 0; q >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, q);
        fy += __shfl_xor_sync(0xffffffffu, fy, q);
        fz += __shfl_xor_sync(0xffffffffu, fz, q);
    }
    if (active && lane == 0) {
        float* t = g.train + ((size_t)r * g.n_train + g.ref_slot[o]) * (kTrainValues * 3) + 3;
        t[0] = fx;
        t[1] = fy;
        t[2] = fz;
    }
}

// ---- reference semantics -----------------------------------------------------
// The reference's own per-step log, read from the state its step leaves
// (positions after the integration, compound particles in the image of their
// particle 0): traj_buffer and potE_buffer of every slot (Engine.cu:1007-1013,
// 1136-1145; solvents log potE 0, as the reference computes none for them),
// data_GAN of the compound slots (position, or (-1, -1, -1) past n_particles,
// and the LJ force from solvents, Engine.cu:1030-1040) and the outdata line of
// compound 0 particle 0 (speed and kinetic energy over the step, its potE and
// |force|, Engine.cu:1016-1029).  `after`: the parity holding the positions
// after the step.
__global__ void __launch_bounds__(kTB) k_log_ref_frame(RefDev d, FrameLogDev g, int after, int r) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n_slots) return;
    const bool comp = k < g.n_train;
    const float4 p = comp ? d.cpos[after][k] : d.spos[after][k - g.n_train];
    if (g.traj) {
        float* t = g.traj + ((size_t)r * g.n_slots + k) * 3;
        t[0] = p.x;
        t[1] = p.y;
        t[2] = p.z;
    }
    if (g.potE) g.potE[(size_t)r * g.n_slots + k] = comp ? d.potE[k] : 0.0;
    if (comp && g.train) {
        const int c = k / LIMA_MAX_COMPOUND_PARTICLES, l = k % LIMA_MAX_COMPOUND_PARTICLES;
        const bool live = l < d.comps[c].n_particles;
        const float4 f = d.force_ljsol[k];
        float* t = g.train + ((size_t)r * g.n_train + k) * (kTrainValues * 3);
        t[0] = live ? p.x : -1.f;
        t[1] = live ? p.y : -1.f;
        t[2] = live ? p.z : -1.f;
        t[3] = live ? f.x : 0.f;
        t[4] = live ? f.y : 0.f;
        t[5] = live ? f.z : 0.f;
        for (int q = 6; q < kTrainValues * 3; q++) t[q] = 0.f;
    }
    if (k == 0 && g.logdata) {
        float* l = g.logdata + (size_t)r * kLogDataFloats;
        for (int q = 0; q < kLogDataFloats; q++) l[q] = 0.f;
        if (g.n_train > 0) {
            // Engine.cu:1016-1029: speed and kinetic energy from the position
            // and the previous position (in its image), potE, |force|
            refm::F3 a = refm::mk4(p), b = refm::mk4(d.cprev[0]);
            refm::hyperpos(a, b, d.L, d.Lh);
            const float dist = refm::len(refm::sub(a, b));
            l[0] = dist / (float)d.dt;
            const float vel = (float)((double)(dist * 0.5f) / d.dt);
            l[1] = (float)(0.5 * (double)d.pp[d.comps[0].atom_types[0]].mass * (double)vel * (double)vel);
            l[2] = (float)d.potE[0];
            l[3] = refm::len(refm::mk4(d.force_c[0]));
        }
    }
}

// The frame's energies: the reference computes no LJ energy; its bonded
// potE summed over the compound slots (fixed order, one block), as
// lima_get_energies reports it, and the last reference-thermostat temperature.
__global__ void __launch_bounds__(kTB) k_log_ref_energy(RefDev d, FrameLogDev g, int r) {
    __shared__ double s_sum[kTB];
    const int ncp = d.n_c * LIMA_MAX_COMPOUND_PARTICLES;
    double a = 0.0;
    for (int k = threadIdx.x; k < ncp; k += blockDim.x) a += d.potE[k];
    s_sum[threadIdx.x] = a;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) s_sum[threadIdx.x] += s_sum[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0 && g.energies) {
        double* e = g.energies + (size_t)r * LIMA_E_COUNT;
        for (int q = 0; q < LIMA_E_COUNT; q++) e[q] = 0.0;
        e[LIMA_E_BOND] = s_sum[0];
        e[LIMA_E_TOTAL] = s_sum[0];
        e[LIMA_E_TEMPERATURE] = *d.ke_accum;
    }
}

// a device buffer of the frame log, from the process's stream-ordered pool
template <typename T>
T* grow(FrameLog& g, size_t n) {
    void* ptr = pool_alloc(std::max<size_t>(n, 1) * sizeof(T), g.stream);
    if (!ptr) return nullptr;
    g.dallocs.push_back(ptr);
    return static_cast<T*>(ptr);
}

// byte offsets of the arrays of one ring (device ring and pinned staging alike)
struct Sections {
    size_t traj, potE, train, energies, logdata, total;
};

Sections sections(const FrameLogDev& g, int frames) {
    Sections s{};
    const size_t f = (size_t)frames;
    size_t o = 0;
    s.traj = o;
    if (g.traj) o += f * g.n_slots * 3 * sizeof(float);
    o = (o + 15) & ~(size_t)15;
    s.potE = o;
    if (g.potE) o += f * g.n_slots * sizeof(double);
    o = (o + 15) & ~(size_t)15;
    s.train = o;
    if (g.train) o += f * g.n_train * kTrainValues * 3 * sizeof(float);
    o = (o + 15) & ~(size_t)15;
    s.energies = o;
    o += f * LIMA_E_COUNT * sizeof(double);
    s.logdata = o;
    o += f * kLogDataFloats * sizeof(float);
    s.total = o;
    return s;
}

// frames [0, count) of the device ring -> pinned buffer b, stream-ordered
void copy_ring(FrameLog& g, int b, int count, cudaStream_t s) {
    const FrameLogDev& v = g.dev;
    const Sections R = sections(v, v.ring);   // device ring and staging share the full-ring layout
    char* dst = static_cast<char*>(g.pinned[b]);
    const size_t c = (size_t)count;
    if (v.traj) cudaMemcpyAsync(dst + R.traj, v.traj, c * v.n_slots * 3 * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (v.potE) cudaMemcpyAsync(dst + R.potE, v.potE, c * v.n_slots * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (v.train)
        cudaMemcpyAsync(dst + R.train, v.train, c * v.n_train * kTrainValues * 3 * sizeof(float),
                        cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(dst + R.energies, v.energies, c * LIMA_E_COUNT * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(dst + R.logdata, v.logdata, c * kLogDataFloats * sizeof(float), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(g.done[b], s);
}

// `count` frames laid out as a full ring at src (host memory) -> the host store
void append_frames(FrameLog& g, const char* src, int count) {
    const FrameLogDev& v = g.dev;
    const Sections R = sections(v, v.ring);
    auto append = [&](auto& vec, size_t off, size_t n) {
        using T = typename std::decay_t<decltype(vec)>::value_type;
        const T* p = reinterpret_cast<const T*>(src + off);
        vec.insert(vec.end(), p, p + n);
    };
    const size_t c = (size_t)count;
    if (v.traj) append(g.traj, R.traj, c * v.n_slots * 3);
    if (v.potE) append(g.potE, R.potE, c * v.n_slots);
    if (v.train) append(g.train, R.train, c * v.n_train * kTrainValues * 3);
    append(g.energies, R.energies, c * LIMA_E_COUNT);
    append(g.logdata, R.logdata, c * kLogDataFloats);
}

// pinned buffer b (copy finished) -> the host store
void absorb(FrameLog& g, int b) {
    const int count = g.pending[b];
    if (!count) return;
    cudaEventSynchronize(g.done[b]);
    append_frames(g, static_cast<const char*>(g.pinned[b]), count);
    g.steps.insert(g.steps.end(), g.buf_steps[b].begin(), g.buf_steps[b].end());
    g.buf_steps[b].clear();
    g.pending[b] = 0;
}

// The two pinned staging rings, allocated when a ring first fills (a short
// run whose frames fit in the device ring never needs them).  Both rings are
// one allocation: a pinned allocation costs far more than its size.
bool ensure_pinned(FrameLog& g) {
    if (g.pinned[0]) return true;
    const size_t stride = (g.ring_bytes + 255) & ~static_cast<size_t>(255);
    g.pinned[0] = pinned_alloc(2 * stride);
    if (!g.pinned[0]) return false;
    g.pinned[1] = static_cast<char*>(g.pinned[0]) + stride;
    for (int b = 0; b < 2; b++)
        if (cudaEventCreateWithFlags(&g.done[b], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
    return true;
}

// the frames in the device ring -> the host store, waiting for the stream
// (no staging rings: a readback, or pinned memory ran out)
void drain_sync(FrameLog& g, cudaStream_t s) {
    if (!g.in_ring) return;
    std::vector<char> buf(g.ring_bytes);
    const FrameLogDev& v = g.dev;
    const Sections R = sections(v, v.ring);
    const size_t c = (size_t)g.in_ring;
    char* dst = buf.data();
    if (v.traj) cudaMemcpyAsync(dst + R.traj, v.traj, c * v.n_slots * 3 * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (v.potE) cudaMemcpyAsync(dst + R.potE, v.potE, c * v.n_slots * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (v.train)
        cudaMemcpyAsync(dst + R.train, v.train, c * v.n_train * kTrainValues * 3 * sizeof(float),
                        cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(dst + R.energies, v.energies, c * LIMA_E_COUNT * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(dst + R.logdata, v.logdata, c * kLogDataFloats * sizeof(float), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    append_frames(g, dst, g.in_ring);
    g.steps.insert(g.steps.end(), g.ring_steps.begin(), g.ring_steps.end());
    g.ring_steps.clear();
    g.in_ring = 0;
    cudaMemsetAsync(v.frame_ctr, 0, sizeof(unsigned long long), s);
}

// the frames in the device ring -> the next pinned buffer (absorbing what it held first)
void drain(FrameLog& g, cudaStream_t s) {
    if (!g.in_ring) return;
    if (!ensure_pinned(g)) {
        drain_sync(g, s);
        return;
    }
    const int b = g.next_buf;
    absorb(g, b);
    copy_ring(g, b, g.in_ring, s);
    g.pending[b] = g.in_ring;
    g.buf_steps[b].swap(g.ring_steps);
    g.ring_steps.clear();
    g.in_ring = 0;
    g.next_buf ^= 1;
    cudaMemsetAsync(g.dev.frame_ctr, 0, sizeof(unsigned long long), s);   // after the copy, in stream order
}

}  // namespace

void framelog_free(FrameLog& g) {
    for (int b = 0; b < 2; b++)
        if (g.pending[b] && g.done[b]) cudaEventSynchronize(g.done[b]);   // copies still in flight
    for (void* p : g.dallocs) pool_free(p, g.stream);
    if (!g.dallocs.empty()) cudaStreamSynchronize(g.stream);
    g.dallocs.clear();
    pinned_free(g.pinned[0]);   // one allocation holds both staging rings
    g.pinned[0] = g.pinned[1] = nullptr;
    for (auto& e : g.done)
        if (e) {
            cudaEventDestroy(e);
            e = nullptr;
        }
    g = FrameLog{};
}

void framelog_start(FrameLog& g, int n_s, const std::vector<int>& n_compound_particles, const lima_log_params& p,
                    cudaStream_t s, std::string& msg, int& status) {
    framelog_free(g);
    g.stream = s;
    status = LIMA_OK;
    const int n_c = (int)n_compound_particles.size();
    FrameLogDev& v = g.dev;
    v.flags = p.flags;
    v.ring = p.ring_frames;
    v.n_train = n_c * LIMA_MAX_COMPOUND_PARTICLES;
    v.n_slots = v.n_train + n_s;
    int n = n_s;
    for (int c = 0; c < n_c; c++) n += n_compound_particles[c];
    std::vector<uint32_t> slot(std::max(n, 1));
    int o = 0;
    for (int c = 0; c < n_c; c++)
        for (int l = 0; l < n_compound_particles[c]; l++) slot[o++] = (uint32_t)(c * LIMA_MAX_COMPOUND_PARTICLES + l);
    for (int s = 0; s < n_s; s++) slot[o++] = (uint32_t)(v.n_train + s);
    const size_t f = (size_t)v.ring;
    uint32_t* ref_slot = grow<uint32_t>(g, slot.size());
    v.traj = (p.flags & LIMA_LOG_TRAJ) ? grow<float>(g, f * v.n_slots * 3) : nullptr;
    v.potE = (p.flags & LIMA_LOG_POTE) ? grow<double>(g, f * v.n_slots) : nullptr;
    v.train = (p.flags & LIMA_LOG_TRAIN) && n_c ? grow<float>(g, f * v.n_train * kTrainValues * 3) : nullptr;
    v.energies = grow<double>(g, f * LIMA_E_COUNT);
    v.logdata = grow<float>(g, f * kLogDataFloats);
    v.frame_ctr = grow<unsigned long long>(g, 1);
    v.blocks_done = grow<unsigned int>(g, 1);
    const Sections R = sections(v, v.ring);
    g.ring_bytes = R.total;
    bool ok = ref_slot && v.energies && v.logdata && v.frame_ctr && v.blocks_done &&
              (!(p.flags & LIMA_LOG_TRAJ) || v.traj) && (!(p.flags & LIMA_LOG_POTE) || v.potE) &&
              (!(p.flags & LIMA_LOG_TRAIN) || !n_c || v.train);
    if (!ok) {
        const cudaStream_t st = g.stream;
        framelog_free(g);
        cudaGetLastError();
        g.stream = st;
        msg = "frame log: out of device memory for the ring";
        status = LIMA_ERR_CUDA;
        return;
    }
    v.ref_slot = ref_slot;
    // set-up copies in the engine's stream order; the host arrays live until the sync below
    cudaMemcpyAsync(ref_slot, slot.data(), sizeof(uint32_t) * slot.size(), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(v.frame_ctr, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(v.blocks_done, 0, sizeof(unsigned int), s);
    if (v.traj) cudaMemsetAsync(v.traj, 0, f * v.n_slots * 3 * sizeof(float), s);
    if (v.potE) cudaMemsetAsync(v.potE, 0, f * v.n_slots * sizeof(double), s);
    std::vector<float> pad;
    if (v.train) {
        // padding particles of a compound: position (-1, -1, -1) (Engine.cu:1036-1037), zero force
        pad.assign((size_t)v.n_train * kTrainValues * 3, 0.f);
        for (int c = 0; c < n_c; c++)
            for (int l = n_compound_particles[c]; l < LIMA_MAX_COMPOUND_PARTICLES; l++)
                for (int q = 0; q < 3; q++) pad[((size_t)c * LIMA_MAX_COMPOUND_PARTICLES + l) * kTrainValues * 3 + q] = -1.f;
        for (size_t r = 0; r < f; r++)
            cudaMemcpyAsync(v.train + r * pad.size(), pad.data(), sizeof(float) * pad.size(), cudaMemcpyHostToDevice, s);
    }
    cudaStreamSynchronize(s);
    g.every = p.every;
    g.on = true;
}

int framelog_launch(const FrameLog& g, const PhysDev& d, int cur, cudaStream_t s) {
    const FrameLogDev& v = g.dev;
    int launched = 1;
    if (v.train && d.n_cp > 0) {   // before k_log_frame, which moves the ring position on
        const int nb = (int)(((size_t)d.n_cp * kGroup + kTB - 1) / kTB);
        const size_t smem = sizeof(float2) * d.n_types * d.n_types;
        if (d.use_switch)
            k_log_train<true><<<nb, kTB, smem, s>>>(d, v, cur);
        else
            k_log_train<false><<<nb, kTB, smem, s>>>(d, v, cur);
        launched++;
    }
    const bool per_particle = v.traj || v.potE || v.train;
    k_log_frame<<<per_particle ? (d.n + kTB - 1) / kTB : 1, per_particle ? kTB : 32, 0, s>>>(d, v, cur,
                                                                                         per_particle ? 1 : 0);
    return launched;
}

void framelog_note(FrameLog& g, uint64_t step, cudaStream_t s) {
    g.ring_steps.push_back(step);
    g.in_ring++;
    g.frames_logged++;
    if (g.in_ring == g.dev.ring) drain(g, s);
}

int framelog_record(FrameLog& g, const PhysDev& d, int cur, uint64_t step, cudaStream_t s) {
    const int launched = framelog_launch(g, d, cur, s);
    framelog_note(g, step, s);
    return launched;
}

int framelog_record_ref(FrameLog& g, const RefDev& d, int after, uint64_t step, cudaStream_t s) {
    const FrameLogDev& v = g.dev;
    const int r = g.in_ring;
    k_log_ref_frame<<<(v.n_slots + kTB - 1) / kTB, kTB, 0, s>>>(d, v, after, r);
    k_log_ref_energy<<<1, kTB, 0, s>>>(d, v, r);
    g.ring_steps.push_back(step);
    g.in_ring++;
    g.frames_logged++;
    if (g.in_ring == v.ring) drain(g, s);
    return 2;
}

void framelog_flush(FrameLog& g, cudaStream_t s) {
    // the older pending buffer first, then the frames still in the device ring
    if (g.pinned[0]) {
        absorb(g, g.next_buf);
        absorb(g, g.next_buf ^ 1);
    }
    drain_sync(g, s);
}

}  // namespace lima
