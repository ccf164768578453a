// Host engine and C-ABI (include/lima_abi.h) of the B200 LIMA_MD step path.
//
// Replaces the reference's Engine (Quantom/Quantom/Engine.cuh:109-208,
// Engine.cu:9-451) and the Box set-up it relies on
// (BoxBuilder::finishBox, BoxBuilder.cu:73-145):
//   * no managed memory: the box is uploaded once into device buffers laid
//     out for coalesced access (refdev.cuh / physdev.cuh);
//   * the per-step host work of Engine::hostMaster (neighbour lists on a
//     detached std::thread every 200 steps, thermostat every 40) runs on the
//     device in stream order, so lima_step never synchronises with the host;
//   * a plain step is captured once into a CUDA graph per buffer parity and
//     replayed;
//   * errors come back as status codes, never exit() (Engine.cuh:47-55,
//     Bodies.cuh:243).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "adjoint.cuh"
#include "framelog.cuh"
#include "render.cuh"
#include "lima_abi.h"
#include "physdev.cuh"
#include "refdev.cuh"

namespace {

struct LimaFail {
    lima_status st;
    std::string msg;
};

[[noreturn]] void fail(lima_status st, const std::string& msg) { throw LimaFail{st, msg}; }

void cuda_ok(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(LIMA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

struct lima_ctx {
    lima_params p{};
    std::string err;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // host copies of the box (the caller keeps its own arrays)
    lima_forcefield ff{};
    bool ff_set = false;
    std::vector<lima_compound> comps;
    std::vector<lima_compound_state> states;
    std::vector<lima_compound_bridge_compact> bridges;
    std::vector<lima_solvent> sols;
    bool finished = false;
    uint64_t step = 0;
    uint64_t last_nlist_step = 0;
    int cur = 0;
    int n_particles_total = 0;
    std::vector<void*> dallocs;
    std::vector<void*> pool_allocs;   // physics buffers from the process-wide pool (freed on the stream)
    lima::RefDev ref{};
    lima::PhysDev phys{};
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    // physics with dynamic lists: [parity][plain, energy, energy + frame log]
    // step graphs, each with the rebuild as a device tail launch
    cudaGraphExec_t dgraph[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    int dgraph_kernels[3] = {0, 0, 0};
    uint64_t host_rebuilds = 0;   // list builds launched by the host (creation, set_state, build_nlist, ...)
    // physics: differentiable parameters and the loss / adjoint buffers
    lima::PhysParams params;
    lima::AdjBuffers adj;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    lima::StepFork fork;       // reference semantics: solvent kernel beside the compound kernels
    bool timed = false;
    bool lambda_pending_reset = false;
    float ref_temperature = 0.f;
    uint64_t launches = 0;     // kernels of this library launched by this context
    int graph_kernels = 0;     // kernels in one replay of a step graph
    lima::FrameLog log;        // physics: frames recorded every log.every steps
    // physics readbacks: device copies of the reference's state structs (pool)
    void* read_stage = nullptr;
    lima::RenderBuf render;    // headless rasterizer buffers (allocated by the first lima_render)

    template <typename T>
    T* dalloc(size_t n) {
        void* ptr = nullptr;
        cuda_ok(cudaMalloc(&ptr, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
        dallocs.push_back(ptr);
        return static_cast<T*>(ptr);
    }
    ~lima_ctx() {
        lima::framelog_free(log);
        lima::phys_free_rebuild(phys);
        for (auto& g : graph)
            if (g) cudaGraphExecDestroy(g);
        for (auto& row : dgraph)
            for (auto& g : row)
                if (g) cudaGraphExecDestroy(g);
        for (void* ptr : dallocs) cudaFree(ptr);
        for (void* ptr : pool_allocs) lima::pool_free(ptr, stream);
        if (!pool_allocs.empty()) cudaStreamSynchronize(stream);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (fork.fork) cudaEventDestroy(fork.fork);
        if (fork.join) cudaEventDestroy(fork.join);
        if (fork.join2) cudaEventDestroy(fork.join2);
        if (fork.side) cudaStreamDestroy(fork.side);
        if (fork.side2) cudaStreamDestroy(fork.side2);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

namespace {

template <typename F>
lima_status guarded(lima_ctx* c, F&& f) {
    if (!c) return LIMA_ERR_ARGUMENT;
    try {
        f();
        return LIMA_OK;
    } catch (const LimaFail& e) {
        c->err = e.msg;
        return e.st;
    } catch (const std::exception& e) {
        c->err = e.what();
        return LIMA_ERR_ARGUMENT;
    }
}

// the message is built only when the check fails (the box checks run per particle)
void need(bool cond, lima_status st, const char* msg) {
    if (!cond) fail(st, msg);
}
void need(bool cond, lima_status st, const std::string& msg) {
    if (!cond) fail(st, msg);
}

float4 f4(const lima_float3& v) { return make_float4(v.x, v.y, v.z, 0.f); }

// ---------------------------------------------------------------------------
// validation of the reference layout the caller hands over
void validate_box(lima_ctx* c) {
    need(c->ff_set, LIMA_ERR_STATE, "lima_set_forcefield must come before lima_finish_box");
    const int nc = static_cast<int>(c->comps.size());
    need(nc <= LIMA_MAX_COMPOUNDS, LIMA_ERR_ARGUMENT, "more than 255 compounds (LJ_Ignores stores uint8 compound ids)");
    for (int i = 0; i < nc; i++) {
        const lima_compound& cp = c->comps[i];
        const int n = cp.n_particles;
        need(n >= 1 && n <= LIMA_MAX_COMPOUND_PARTICLES, LIMA_ERR_ARGUMENT, "compound n_particles outside 1..64");
        need(c->states[i].n_particles == cp.n_particles, LIMA_ERR_ARGUMENT, "CompoundState.n_particles != Compound.n_particles");
        need(cp.n_singlebonds <= LIMA_MAX_PAIRBONDS && cp.n_anglebonds <= LIMA_MAX_ANGLEBONDS &&
                 cp.n_dihedrals <= LIMA_MAX_DIHEDRALS,
             LIMA_ERR_ARGUMENT, "bonded term count beyond the Compound capacity");
        need(cp.key_particle_index >= 0 && cp.key_particle_index < n, LIMA_ERR_ARGUMENT, "key_particle_index out of range");
        for (int t = 0; t < n; t++) {
            need(cp.atom_types[t] < LIMA_MAX_ATOM_TYPES, LIMA_ERR_ARGUMENT, "atom type >= 32");
            need(cp.lj_ignore_list[t].n_ignores <= LIMA_LJ_IGNORES_MAX, LIMA_ERR_ARGUMENT, "LJ_Ignores.n_ignores > 32");
        }
        for (int b = 0; b < cp.n_singlebonds; b++)
            for (int k = 0; k < 2; k++) need(cp.singlebonds[b].atom_indexes[k] < (uint32_t)n, LIMA_ERR_ARGUMENT, "bond atom index out of range");
        for (int b = 0; b < cp.n_anglebonds; b++)
            for (int k = 0; k < 3; k++) need(cp.anglebonds[b].atom_indexes[k] < (uint32_t)n, LIMA_ERR_ARGUMENT, "angle atom index out of range");
        for (int b = 0; b < cp.n_dihedrals; b++)
            for (int k = 0; k < 4; k++) need(cp.dihedrals[b].atom_indexes[k] < (uint32_t)n, LIMA_ERR_ARGUMENT, "dihedral atom index out of range");
    }
    for (const auto& br : c->bridges) {
        need(br.n_particles >= 0 && br.n_particles <= LIMA_MAX_PARTICLES_IN_BRIDGE, LIMA_ERR_ARGUMENT, "bridge n_particles outside 0..32");
        need(br.n_singlebonds <= LIMA_MAX_SINGLEBONDS_IN_BRIDGE && br.n_anglebonds <= LIMA_MAX_ANGLEBONDS_IN_BRIDGE &&
                 br.n_dihedrals <= LIMA_MAX_DIHEDRALBONDS_IN_BRIDGE,
             LIMA_ERR_ARGUMENT, "bridge term count beyond capacity");
        for (int t = 0; t < br.n_particles; t++) {
            const auto& r = br.particle_refs[t];
            need(r.compound_id >= 0 && r.compound_id < nc, LIMA_ERR_ARGUMENT, "bridge compound id out of range");
            need(r.local_id_compound >= 0 && r.local_id_compound < c->comps[r.compound_id].n_particles,
                 LIMA_ERR_ARGUMENT, "bridge local id out of range");
        }
        for (int b = 0; b < br.n_singlebonds; b++)
            for (int k = 0; k < 2; k++) need(br.singlebonds[b].atom_indexes[k] < (uint32_t)br.n_particles, LIMA_ERR_ARGUMENT, "bridge bond index out of range");
        for (int b = 0; b < br.n_anglebonds; b++)
            for (int k = 0; k < 3; k++) need(br.anglebonds[b].atom_indexes[k] < (uint32_t)br.n_particles, LIMA_ERR_ARGUMENT, "bridge angle index out of range");
        for (int b = 0; b < br.n_dihedrals; b++)
            for (int k = 0; k < 4; k++) need(br.dihedrals[b].atom_indexes[k] < (uint32_t)br.n_particles, LIMA_ERR_ARGUMENT, "bridge dihedral index out of range");
    }
    for (const auto& s : c->sols) {
        const float L = c->p.box_len;
        // the reference loads positions as given and wraps them after the first
        // integration (applyPBC, Engine.cu:461-466); any image within one box
        // length of [0, box_len] is accepted
        need(s.pos.x >= -L && s.pos.x <= 2.f * L && s.pos.y >= -L && s.pos.y <= 2.f * L && s.pos.z >= -L &&
                 s.pos.z <= 2.f * L,
             LIMA_ERR_ARGUMENT, "solvent position more than one box length outside [0, box_len]");
    }
}

// ---------------------------------------------------------------------------
// reference semantics
void ref_setup(lima_ctx* c) {
    lima::RefDev& d = c->ref;
    const int nc = static_cast<int>(c->comps.size()), ns = static_cast<int>(c->sols.size());
    const int nb = static_cast<int>(c->bridges.size());
    d.n_c = nc;
    d.n_s = ns;
    d.n_b = nb;
    d.L = c->p.box_len;
    d.Lh = c->p.box_len / 2.f;
    d.C = c->p.ref_cutoff > 0.f ? c->p.ref_cutoff : c->p.cutoff / 2.f;
    d.dt = c->p.dt;
    cudaStream_t s = c->stream;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        if (bytes) cuda_ok(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "upload");
    };
    lima_compound* dcomps = c->dalloc<lima_compound>(nc);
    up(dcomps, c->comps.data(), sizeof(lima_compound) * nc);
    d.comps = dcomps;
    lima_compound_bridge_compact* dbr = c->dalloc<lima_compound_bridge_compact>(nb);
    up(dbr, c->bridges.data(), sizeof(lima_compound_bridge_compact) * nb);
    d.bridges = dbr;
    lima_particle_parameters* dpp = c->dalloc<lima_particle_parameters>(LIMA_MAX_ATOM_TYPES);
    up(dpp, c->ff.particle_parameters, sizeof(lima_forcefield));
    d.pp = dpp;

    const size_t ncp = static_cast<size_t>(nc) * lima::kMaxCP;
    std::vector<float4> hpos(ncp, make_float4(0, 0, 0, 0)), hprev(ncp, make_float4(0, 0, 0, 0)),
        hbr(ncp, make_float4(0, 0, 0, 0));
    for (int i = 0; i < nc; i++)
        for (int t = 0; t < c->comps[i].n_particles; t++) {
            hpos[i * lima::kMaxCP + t] = f4(c->states[i].positions[t]);
            hprev[i * lima::kMaxCP + t] = f4(c->comps[i].prev_positions[t]);
            hbr[i * lima::kMaxCP + t] = f4(c->comps[i].forces[t]);
        }
    for (int b = 0; b < 2; b++) {
        d.cpos[b] = c->dalloc<float4>(ncp);
        up(d.cpos[b], hpos.data(), sizeof(float4) * ncp);
    }
    d.cprev = c->dalloc<float4>(ncp);
    up(d.cprev, hprev.data(), sizeof(float4) * ncp);
    d.cbridge = c->dalloc<float4>(ncp);
    up(d.cbridge, hbr.data(), sizeof(float4) * ncp);
    std::vector<float4> sp(ns), spr(ns);
    for (int i = 0; i < ns; i++) {
        sp[i] = f4(c->sols[i].pos);
        spr[i] = f4(c->sols[i].pos_tsub1);
    }
    for (int b = 0; b < 2; b++) {
        d.spos[b] = c->dalloc<float4>(ns);
        d.sprev[b] = c->dalloc<float4>(ns);
        up(d.spos[b], sp.data(), sizeof(float4) * ns);
        up(d.sprev[b], spr.data(), sizeof(float4) * ns);
    }
    d.ss_cap = c->p.solvent_list_capacity;
    d.cs_cap = c->p.compound_list_capacity;
    d.ss_ids = c->dalloc<uint32_t>(static_cast<size_t>(ns) * d.ss_cap);
    d.ss_cnt = c->dalloc<uint32_t>(ns);
    d.cs_ids = c->dalloc<uint32_t>(static_cast<size_t>(nc) * d.cs_cap);
    d.cs_cnt = c->dalloc<uint32_t>(nc);
    d.cc_ids = c->dalloc<uint32_t>(ncp);
    d.cc_cnt = c->dalloc<uint32_t>(nc);
    d.cc_prev = c->dalloc<uint8_t>(static_cast<size_t>(nc) * nc);
    cuda_ok(cudaMemsetAsync(d.ss_cnt, 0, sizeof(uint32_t) * std::max(ns, 1), s), "memset");
    cuda_ok(cudaMemsetAsync(d.cs_cnt, 0, sizeof(uint32_t) * std::max(nc, 1), s), "memset");
    cuda_ok(cudaMemsetAsync(d.cc_cnt, 0, sizeof(uint32_t) * std::max(nc, 1), s), "memset");
    cuda_ok(cudaMemsetAsync(d.cc_prev, 0, std::max<size_t>(1, static_cast<size_t>(nc) * nc), s), "memset");
    const float radius = d.C + d.C;
    int m = static_cast<int>(std::floor(d.L / (radius * 1.0001f)));
    if (m < 3) m = 1;
    while (m > 1 && d.L / static_cast<float>(m) < radius) m--;
    if (m < 3) m = 1;
    d.m = m;
    d.cell = d.L / static_cast<float>(m);
    const size_t ncell = static_cast<size_t>(m) * m * m;
    d.cell_count = c->dalloc<uint32_t>(ncell);
    d.cell_start = c->dalloc<uint32_t>(ncell);
    d.cell_fill = c->dalloc<uint32_t>(ncell);
    d.cell_items = c->dalloc<uint32_t>(ns);
    d.sol_cell = c->dalloc<uint32_t>(ns);
    d.n_chunks = (d.cs_cap + lima::kCsChunk - 1) / lima::kCsChunk;
    d.cs_partial = c->dalloc<float4>(static_cast<size_t>(nc) * d.n_chunks * lima::kMaxCP);
    d.cc_partial = c->dalloc<float4>(static_cast<size_t>(nc) * (1 + lima::kMaxCP) * lima::kMaxCP);
    {   // enough lanes per solvent to fill the SMs, at most one wave of 1,024 threads per SM
        int dev = 0, n_sm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        // the loop over the compounds: up to two waves of 1,024 threads per SM
        d.sol_lanes = 1;
        while (d.sol_lanes < 16 && static_cast<size_t>(ns) * d.sol_lanes * 2 <= static_cast<size_t>(n_sm) * 2048)
            d.sol_lanes *= 2;
        // the list loop: one lane per solvent, gathers pipelined (it runs
        // beside the loop over the compounds, which fills the SMs' issue slots)
        d.sol_list_lanes = 1;
        // LIMA_SOLVENT_LANES / LIMA_SOLVENT_LIST_LANES = 1|2|4|8|16 override the
        // choices (results do not depend on them)
        auto lanes_env = [](const char* name, int& out) {
            if (const char* e = std::getenv(name)) {
                const int w = std::atoi(e);
                if (w == 1 || w == 2 || w == 4 || w == 8 || w == 16) out = w;
            }
        };
        lanes_env("LIMA_SOLVENT_LANES", d.sol_lanes);
        lanes_env("LIMA_SOLVENT_LIST_LANES", d.sol_list_lanes);
        // blocks of 32-128 threads, at least two blocks per SM where the solvents allow
        d.sol_list_block = 128;
        while (d.sol_list_block > 32 &&
               static_cast<size_t>(ns) * d.sol_list_lanes < static_cast<size_t>(d.sol_list_block) * n_sm * 2)
            d.sol_list_block /= 2;
    }
    d.sol_force = c->dalloc<float4>(ns);
    d.sol_acc = c->dalloc<float4>(ns);
    d.sol_image = c->dalloc<float4>(ns);
    d.force_c = c->dalloc<float4>(ncp);
    d.force_s = c->dalloc<float4>(ns);
    d.potE = c->dalloc<double>(ncp);
    d.force_ljsol = c->dalloc<float4>(ncp);
    cuda_ok(cudaMemsetAsync(d.force_ljsol, 0, sizeof(float4) * std::max<size_t>(ncp, 1), s), "memset");
    cuda_ok(cudaMemsetAsync(d.force_c, 0, sizeof(float4) * std::max<size_t>(ncp, 1), s), "memset");
    cuda_ok(cudaMemsetAsync(d.force_s, 0, sizeof(float4) * std::max(ns, 1), s), "memset");
    cuda_ok(cudaMemsetAsync(d.potE, 0, sizeof(double) * std::max<size_t>(ncp, 1), s), "memset");
    d.lambda = c->dalloc<float>(1);
    lima::set_device_float(d.lambda, 1.f, s);
    d.err = c->dalloc<int>(1);
    cuda_ok(cudaMemsetAsync(d.err, 0, sizeof(int), s), "memset");
    d.csnap = c->dalloc<float4>(ncp);
    d.ssnap = c->dalloc<float4>(ns);
    d.ke_accum = c->dalloc<double>(1);
    {   // per-atom bonded contribution lists (see RefDev::bt_off)
        std::vector<uint32_t> off(static_cast<size_t>(nc) * 65 + 1, 0);
        std::vector<uint16_t> code;
        for (int i = 0; i < nc; i++) {
            const lima_compound& cp = c->comps[i];
            for (int t = 0; t < lima::kMaxCP; t++) {
                off[i * 65 + t] = static_cast<uint32_t>(code.size());
                for (int b = 0; b < cp.n_singlebonds; b++)
                    for (int k = 0; k < 2; k++)
                        if (static_cast<int>(cp.singlebonds[b].atom_indexes[k]) == t) code.push_back((0 << 14) | (b << 2) | k);
                for (int b = 0; b < cp.n_anglebonds; b++)
                    for (int k = 0; k < 3; k++)
                        if (static_cast<int>(cp.anglebonds[b].atom_indexes[k]) == t) code.push_back((1 << 14) | (b << 2) | k);
                for (int b = 0; b < cp.n_dihedrals; b++)
                    for (int k = 0; k < 4; k++)
                        if (static_cast<int>(cp.dihedrals[b].atom_indexes[k]) == t) code.push_back((2 << 14) | (b << 2) | k);
            }
            off[i * 65 + 64] = static_cast<uint32_t>(code.size());
        }
        off[static_cast<size_t>(nc) * 65] = static_cast<uint32_t>(code.size());
        d.bt_off = c->dalloc<uint32_t>(off.size());
        d.bt_code = c->dalloc<uint16_t>(code.size());
        up(d.bt_off, off.data(), sizeof(uint32_t) * off.size());
        up(d.bt_code, code.data(), sizeof(uint16_t) * code.size());
        cuda_ok(cudaStreamSynchronize(s), "upload");
    }
    c->n_particles_total = ns;
    for (const auto& cp : c->comps) c->n_particles_total += cp.n_particles;
}

void capture_graphs(lima_ctx* c, void (*launch)(lima_ctx*, int)) {
    for (int parity = 0; parity < 2; parity++) {
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        launch(c, parity);
        if (cudaStreamEndCapture(c->stream, &g) != cudaSuccess || !g) {
            cudaGetLastError();
            return;
        }
        if (cudaGraphInstantiate(&c->graph[parity], g, 0) != cudaSuccess) {
            cudaGetLastError();
            c->graph[parity] = nullptr;
        }
        cudaGraphDestroy(g);
    }
}

void ref_launch_step(lima_ctx* c, int parity) {
    c->graph_kernels = lima::ref_step_kernels(c->ref, parity, c->stream, nullptr, &c->fork);
}
void phys_launch_step(lima_ctx* c, int parity) {
    c->graph_kernels = lima::phys_step_kernels(c->phys, parity, c->stream);
}

void check_device_errors(lima_ctx* c) {
    int* err_ptr = c->p.semantics == LIMA_SEMANTICS_REFERENCE ? c->ref.err : c->phys.err;
    int h = 0;
    cuda_ok(cudaMemcpyAsync(&h, err_ptr, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "read error flags");
    cuda_ok(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    if (h) {
        cuda_ok(cudaMemsetAsync(err_ptr, 0, sizeof(int), c->stream), "memset");
        cuda_ok(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
        std::string m;
        if (h & lima::ERR_BIT_SS_OVERFLOW) m += "solvent-solvent list overflow; ";
        if (h & lima::ERR_BIT_CS_OVERFLOW) m += "compound-solvent list overflow; ";
        if (h & lima::ERR_BIT_CC_OVERFLOW) m += "compound-compound list overflow; ";
        if (h & lima::ERR_BIT_PHYS_LIST_OVERFLOW) m += "pair list overflow; ";
        if (h & lima::ERR_BIT_LIST_STALE)
            m += "pair list went stale: a particle moved more than skin/2 between rebuilds (raise skin or lower "
                 "nlist_period); ";
        if (h & lima::ERR_BIT_TILE_TIMEOUT) m += "shared-memory staging wait timed out; ";
        if (h & lima::ERR_BIT_REBUILD_LAUNCH) m += "the device could not launch a due pair-list rebuild; ";
        if (h & lima::ERR_BIT_NAN) m += "NaN position; ";
        if (h & lima::ERR_BIT_CRITICAL_FORCE) m += "critical force (|F| > 2e12); ";
        const bool cap = h & (lima::ERR_BIT_SS_OVERFLOW | lima::ERR_BIT_CS_OVERFLOW | lima::ERR_BIT_CC_OVERFLOW |
                              lima::ERR_BIT_PHYS_LIST_OVERFLOW);
        fail(cap ? LIMA_ERR_CAPACITY : LIMA_ERR_NUMERIC, m);
    }
}

void sync_checked(lima_ctx* c) {
    cuda_ok(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    cuda_ok(cudaGetLastError(), "kernel launch");
    check_device_errors(c);
}

void ref_nlist_now(lima_ctx* c) {
    lima::ref_build_nlists(c->ref, c->cur, c->stream);
    c->launches += (c->ref.n_s > 0 ? 4 : 0) + (c->ref.n_c > 0 ? (c->ref.n_s > 0 ? 2 : 1) : 0);
    c->last_nlist_step = c->step;
}

// One step.  prof (nullable): [0] before any list rebuild, [1] after it, then
// the frame-log kernels of a logged step, captured into its step graph
struct LogCapture {
    const lima::FrameLog* log;
    const lima::PhysDev* d;
    int cur;
};
int capture_frame_log(void* ctx, cudaStream_t s) {
    const LogCapture* lc = static_cast<const LogCapture*>(ctx);
    return lima::framelog_launch(*lc->log, *lc->d, lc->cur, s);
}

// the four per-kernel-group events of ref_step_kernels / phys_step_kernels;
// with prof the step is launched directly instead of through the graph.
void one_step(lima_ctx* c, cudaEvent_t* prof) {
    const int period = std::max(1, c->p.nlist_period);
    const bool rebuild = c->step > 0 && c->step - c->last_nlist_step >= static_cast<uint64_t>(period);
    // profiling a dynamic list: the host reads the rebuild request before the first event
    const bool dyn_rebuild = prof && c->p.semantics == LIMA_SEMANTICS_PHYSICS && c->phys.dynamic_list &&
                             lima::phys_rebuild_pending(c->phys, c->stream);
    if (prof) cuda_ok(cudaEventRecord(prof[0], c->stream), "cudaEventRecord");
    if (c->p.semantics == LIMA_SEMANTICS_REFERENCE) {
        lima::RefDev& d = c->ref;
        if (rebuild) ref_nlist_now(c);
        if (prof) cuda_ok(cudaEventRecord(prof[1], c->stream), "cudaEventRecord");
        if (c->graph[c->cur] && !prof) {
            cuda_ok(cudaGraphLaunch(c->graph[c->cur], c->stream), "cudaGraphLaunch");
            c->launches += c->graph_kernels;
        } else {
            c->launches += lima::ref_step_kernels(d, c->cur, c->stream, prof ? prof + 2 : nullptr, &c->fork);
        }
        c->cur ^= 1;
        if (c->log.on && (c->step % static_cast<uint64_t>(c->log.every)) == 0)
            c->launches += lima::framelog_record_ref(c->log, d, c->cur, c->step, c->stream);
        c->step++;
        if (c->lambda_pending_reset) {
            lima::set_device_float(d.lambda, 1.f, c->stream);
            c->launches++;
            c->lambda_pending_reset = false;
        }
        if (c->p.thermostat == LIMA_THERMOSTAT_REFERENCE) {
            const int tp = std::max(3, c->p.thermostat_period);
            const uint64_t k = c->step % tp;
            if (k == static_cast<uint64_t>(tp - 2)) {
                lima::ref_thermostat_snapshot(d, c->cur, c->stream);
                c->launches++;
            }
            if (k == 0 && c->step >= 2) {
                lima::ref_thermostat_update(d, c->cur, c->n_particles_total, static_cast<float>(c->p.t_target),
                                            c->step > 20, c->stream);
                c->launches += 2;
                c->lambda_pending_reset = true;   // applied for one step (Engine.cu:67-69)
            }
        }
    } else if (c->phys.dynamic_list) {
        const bool logged = c->log.on && (c->step % static_cast<uint64_t>(c->log.every)) == 0;
        const bool energy = logged || (c->p.energy_period > 0 && (c->step % c->p.energy_period) == 0);
        if (!prof) {
            // a logged step records its frame inside the step graph (the frame
            // kernels take their ring position from the device)
            const int v = logged ? 2 : (energy ? 1 : 0);
            cudaGraphExec_t& g = c->dgraph[c->cur][v];
            if (!g) {   // instantiated on first use: a short run pays only for the variants it steps
                LogCapture lc{&c->log, &c->phys, c->cur};
                const int k = lima::phys_capture_dynamic(c->phys, c->cur, energy, c->stream, &g,
                                                         logged ? capture_frame_log : nullptr, &lc);
                need(k > 0, LIMA_ERR_CUDA, "cannot build the step graph of a dynamic pair list");
                c->dgraph_kernels[v] = k;
            }
            cuda_ok(cudaGraphLaunch(g, c->stream), "cudaGraphLaunch");
            c->launches += c->dgraph_kernels[v];
            if (logged) lima::framelog_note(c->log, c->step, c->stream);
        } else {   // profiling: the same kernels launched directly, the rebuild decided on the host
            if (dyn_rebuild) {
                lima::phys_rebuild(c->phys, c->cur, c->stream);
                c->launches += lima::kRebuildKernels;
                c->host_rebuilds++;
            }
            cuda_ok(cudaEventRecord(prof[1], c->stream), "cudaEventRecord");
            c->launches += lima::phys_step_kernels(c->phys, c->cur, c->stream, energy, prof + 2);
            cuda_ok(cudaEventRecord(prof[5], c->stream), "cudaEventRecord");
        }
        if (logged && prof) c->launches += lima::framelog_record(c->log, c->phys, c->cur, c->step, c->stream);
        c->cur ^= 1;
        c->step++;
    } else {
        if (rebuild) {
            lima::phys_rebuild(c->phys, c->cur, c->stream);
            c->launches += lima::kRebuildKernels;
            c->host_rebuilds++;
            c->last_nlist_step = c->step;
        }
        if (prof) cuda_ok(cudaEventRecord(prof[1], c->stream), "cudaEventRecord");
        const bool logged = c->log.on && (c->step % static_cast<uint64_t>(c->log.every)) == 0;
        const bool energy = logged || (c->p.energy_period > 0 && (c->step % c->p.energy_period) == 0);
        if (energy || !c->graph[c->cur] || prof) {
            c->launches += lima::phys_step_kernels(c->phys, c->cur, c->stream, energy, prof ? prof + 2 : nullptr);
            if (prof) cuda_ok(cudaEventRecord(prof[5], c->stream), "cudaEventRecord");
        } else {
            cuda_ok(cudaGraphLaunch(c->graph[c->cur], c->stream), "cudaGraphLaunch");
            c->launches += c->graph_kernels;
        }
        if (logged) c->launches += lima::framelog_record(c->log, c->phys, c->cur, c->step, c->stream);
        c->cur ^= 1;
        c->step++;
    }
}

}  // namespace

// ===========================================================================
extern "C" {

void lima_default_params(lima_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->box_len = 7.f;
    p->cutoff = 1.4f;
    p->ref_cutoff = 0.f;
    p->skin = 0.1f;
    p->switch_on = 1.0f;
    p->dt = 1e-7;
    p->nlist_period = 200;
    p->semantics = LIMA_SEMANTICS_REFERENCE;
    p->precision = LIMA_PRECISION_FP32;
    p->thermostat = LIMA_THERMOSTAT_NONE;
    p->t_target = 310.0;
    p->tau_t = 1e-4;
    p->thermostat_period = 40;
    p->energy_period = 0;
    p->solvent_list_capacity = 512;
    p->compound_list_capacity = 8192;
    p->device = 0;
    p->stream = nullptr;
}

lima_status lima_create(const lima_params* params, lima_ctx** out) {
    if (!params || !out) return LIMA_ERR_ARGUMENT;
    *out = nullptr;
    auto* c = new lima_ctx();
    c->p = *params;
    lima_status st = guarded(c, [&] {
        const lima_params& p = c->p;
        need(p.box_len > 0.f, LIMA_ERR_ARGUMENT, "box_len must be positive");
        need(p.dt > 0.0, LIMA_ERR_ARGUMENT, "dt must be positive");
        need(p.semantics == LIMA_SEMANTICS_REFERENCE || p.semantics == LIMA_SEMANTICS_PHYSICS, LIMA_ERR_ARGUMENT,
             "unknown semantics");
        need(p.precision == LIMA_PRECISION_FP32 || p.precision == LIMA_PRECISION_MIXED, LIMA_ERR_ARGUMENT,
             "unknown precision");
        need(p.thermostat >= 0 && p.thermostat <= 2, LIMA_ERR_ARGUMENT, "unknown thermostat");
        need(p.solvent_list_capacity >= 32 && p.solvent_list_capacity <= 2048, LIMA_ERR_ARGUMENT,
             "solvent_list_capacity outside 32..2048");
        need(p.compound_list_capacity >= 64 && p.compound_list_capacity <= (1 << 20), LIMA_ERR_ARGUMENT,
             "compound_list_capacity outside 64..2^20");
        need(p.cutoff > 0.f || p.ref_cutoff > 0.f, LIMA_ERR_ARGUMENT, "cutoff must be positive");
        if (p.semantics == LIMA_SEMANTICS_PHYSICS) {
            need(p.cutoff > 0.f && p.skin >= 0.f && 2.f * (p.cutoff + p.skin) <= p.box_len, LIMA_ERR_ARGUMENT,
                 "physics semantics needs 2*(cutoff+skin) <= box_len");
        }
        int ndev = 0;
        cuda_ok(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
        need(p.device >= 0 && p.device < ndev, LIMA_ERR_ARGUMENT, "no such CUDA device");
        cuda_ok(cudaSetDevice(p.device), "cudaSetDevice");
        if (p.stream) {
            c->stream = static_cast<cudaStream_t>(p.stream);
        } else {
            cuda_ok(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            c->own_stream = true;
        }
        cuda_ok(cudaEventCreate(&c->ev0), "cudaEventCreate");
        cuda_ok(cudaEventCreate(&c->ev1), "cudaEventCreate");
        if (p.semantics == LIMA_SEMANTICS_REFERENCE) {   // the solvent kernels' side streams
            cuda_ok(cudaStreamCreateWithFlags(&c->fork.side, cudaStreamNonBlocking), "cudaStreamCreate");
            cuda_ok(cudaEventCreateWithFlags(&c->fork.fork, cudaEventDisableTiming), "cudaEventCreate");
            cuda_ok(cudaEventCreateWithFlags(&c->fork.join, cudaEventDisableTiming), "cudaEventCreate");
            cuda_ok(cudaStreamCreateWithFlags(&c->fork.side2, cudaStreamNonBlocking), "cudaStreamCreate");
            cuda_ok(cudaEventCreateWithFlags(&c->fork.join2, cudaEventDisableTiming), "cudaEventCreate");
        }
    });
    if (st != LIMA_OK) {
        fprintf(stderr, "lima_create: %s\n", c->err.c_str());
        delete c;
        return st;
    }
    *out = c;
    return LIMA_OK;
}

void lima_destroy(lima_ctx* ctx) {
    if (!ctx) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    delete ctx;
}

const char* lima_last_error(const lima_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

lima_status lima_set_forcefield(lima_ctx* c, const lima_forcefield* ff) {
    return guarded(c, [&] {
        need(ff != nullptr, LIMA_ERR_ARGUMENT, "null forcefield");
        need(!c->finished, LIMA_ERR_STATE, "box already finished");
        c->ff = *ff;
        c->ff_set = true;
    });
}

lima_status lima_load_compounds(lima_ctx* c, const lima_compound* compounds, const lima_compound_state* states,
                                int n) {
    return guarded(c, [&] {
        need(!c->finished, LIMA_ERR_STATE, "box already finished");
        need(n >= 0 && n <= LIMA_MAX_COMPOUNDS, LIMA_ERR_ARGUMENT, "n_compounds outside 0..255");
        need(n == 0 || (compounds && states), LIMA_ERR_ARGUMENT, "null compound arrays");
        c->comps.assign(compounds, compounds + n);
        c->states.assign(states, states + n);
    });
}

lima_status lima_load_bridges(lima_ctx* c, const lima_compound_bridge_compact* bridges, int n) {
    return guarded(c, [&] {
        need(!c->finished, LIMA_ERR_STATE, "box already finished");
        need(n >= 0 && n <= 4 * LIMA_MAX_COMPOUNDS, LIMA_ERR_ARGUMENT, "n_bridges out of range");
        need(n == 0 || bridges, LIMA_ERR_ARGUMENT, "null bridge array");
        c->bridges.assign(bridges, bridges + n);
    });
}

lima_status lima_load_solvents(lima_ctx* c, const lima_solvent* solvents, uint32_t n) {
    return guarded(c, [&] {
        need(!c->finished, LIMA_ERR_STATE, "box already finished");
        need(n == 0 || solvents, LIMA_ERR_ARGUMENT, "null solvent array");
        need(n <= (1u << 26), LIMA_ERR_ARGUMENT, "more than 2^26 solvents");
        c->sols.assign(solvents, solvents + n);
    });
}

lima_status lima_finish_box(lima_ctx* c) {
    return guarded(c, [&] {
        need(!c->finished, LIMA_ERR_STATE, "box already finished");
        validate_box(c);
        cuda_ok(cudaSetDevice(c->p.device), "cudaSetDevice");
        if (c->p.semantics == LIMA_SEMANTICS_REFERENCE) {
            ref_setup(c);
            ref_nlist_now(c);
            sync_checked(c);
            capture_graphs(c, ref_launch_step);
        } else {
            lima::PhysHost h;
            h.params = &c->p;
            h.ff = &c->ff;
            h.comps = c->comps.data();
            h.states = c->states.data();
            h.n_c = static_cast<int>(c->comps.size());
            h.bridges = c->bridges.data();
            h.n_b = static_cast<int>(c->bridges.size());
            h.sols = c->sols.data();
            h.n_s = static_cast<int>(c->sols.size());
            std::string msg;
            const int rc = lima::phys_setup(h, c->phys, c->stream, c->pool_allocs, msg);
            if (rc != 0) fail(static_cast<lima_status>(rc), msg);
            lima::phys_rebuild(c->phys, c->cur, c->stream);
            // a solute denser than the box average can overflow the first list:
            // grow the capacity to the measured longest row once, and rebuild
            if (lima::phys_fit_list(c->phys, c->stream, c->pool_allocs)) {
                lima::phys_rebuild(c->phys, c->cur, c->stream);
                c->launches += lima::kRebuildKernels;
                c->host_rebuilds++;
            }
            lima::phys_prime(c->phys, c->cur, c->stream);
            c->host_rebuilds++;
            sync_checked(c);
            lima::phys_params_init(c->phys, c->ff, c->params, c->stream);
            if (c->phys.dynamic_list) {
                std::string rmsg;
                const int rrc = lima::phys_capture_rebuild(c->phys, c->stream, rmsg);
                if (rrc != 0) fail(static_cast<lima_status>(rrc), rmsg);
                // the step graphs themselves are instantiated on first use (one_step)
            } else {
                capture_graphs(c, phys_launch_step);
            }
            c->n_particles_total = c->phys.n;
        }
        sync_checked(c);
        c->finished = true;
    });
}

lima_status lima_step(lima_ctx* c, int n_steps) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        need(n_steps >= 0, LIMA_ERR_ARGUMENT, "negative step count");
        cuda_ok(cudaEventRecord(c->ev0, c->stream), "cudaEventRecord");
        for (int i = 0; i < n_steps; i++) one_step(c, nullptr);
        cuda_ok(cudaEventRecord(c->ev1, c->stream), "cudaEventRecord");
        cuda_ok(cudaGetLastError(), "kernel launch");
        c->timed = true;
    });
}

lima_status lima_profile_steps(lima_ctx* c, int n_steps, float* ms) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        need(n_steps > 0 && ms != nullptr, LIMA_ERR_ARGUMENT, "need n_steps > 0 and an output array");
        cudaEvent_t ev[6];
        for (auto& e : ev) cuda_ok(cudaEventCreate(&e), "cudaEventCreate");
        double acc[LIMA_PROF_COUNT] = {0, 0, 0, 0, 0};
        lima_status st = LIMA_OK;
        std::string msg;
        try {
            for (int i = 0; i < n_steps; i++) {
                one_step(c, ev);
                if (c->p.semantics == LIMA_SEMANTICS_REFERENCE)
                    cuda_ok(cudaEventRecord(ev[5], c->stream), "cudaEventRecord");
                cuda_ok(cudaEventSynchronize(ev[5]), "cudaEventSynchronize");
                float t[5];
                for (int k = 0; k < 5; k++) cuda_ok(cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]), "cudaEventElapsedTime");
                acc[LIMA_PROF_NLIST] += t[0];
                if (c->p.semantics == LIMA_SEMANTICS_REFERENCE) {
                    acc[LIMA_PROF_BONDED] += t[2];     // bridges
                    acc[LIMA_PROF_COMPOUND] += t[3];   // compound<-solvent chunks + compound kernel
                    acc[LIMA_PROF_PAIR] += t[4];       // solvent kernel
                } else {
                    acc[LIMA_PROF_BONDED] += t[2];
                    acc[LIMA_PROF_PAIR] += t[3];       // pair + integrate
                }
                float tot = 0.f;
                cuda_ok(cudaEventElapsedTime(&tot, ev[0], ev[5]), "cudaEventElapsedTime");
                acc[LIMA_PROF_TOTAL] += tot;
            }
        } catch (const LimaFail& e) {
            st = e.st;
            msg = e.msg;
        }
        for (auto& e : ev) cudaEventDestroy(e);
        if (st != LIMA_OK) fail(st, msg);
        // the profiled steps ran outside the step graphs, so a rebuild the last
        // one asked for is still due: run it before the next step
        if (c->p.semantics == LIMA_SEMANTICS_PHYSICS && c->phys.dynamic_list &&
            lima::phys_rebuild_pending(c->phys, c->stream)) {
            lima::phys_rebuild(c->phys, c->cur, c->stream);
            c->launches += lima::kRebuildKernels;
            c->host_rebuilds++;
        }
        for (int k = 0; k < LIMA_PROF_COUNT; k++) ms[k] = static_cast<float>(acc[k] / n_steps);
        sync_checked(c);
    });
}

lima_status lima_get_kernel_launches(lima_ctx* c, uint64_t* count) {
    return guarded(c, [&] {
        need(count != nullptr, LIMA_ERR_ARGUMENT, "null count");
        *count = c->launches;
        if (c->finished && c->p.semantics == LIMA_SEMANTICS_PHYSICS && c->phys.dynamic_list)
            *count += lima::phys_device_rebuilds(c->phys, c->stream) * lima::kRebuildKernels;
    });
}

lima_status lima_synchronize(lima_ctx* c) {
    return guarded(c, [&] { sync_checked(c); });
}

lima_status lima_get_step(lima_ctx* c, uint64_t* step) {
    return guarded(c, [&] {
        need(step != nullptr, LIMA_ERR_ARGUMENT, "null step");
        *step = c->step;
    });
}

lima_status lima_get_last_step_ms(lima_ctx* c, float* ms) {
    return guarded(c, [&] {
        need(ms != nullptr, LIMA_ERR_ARGUMENT, "null ms");
        need(c->timed, LIMA_ERR_STATE, "no lima_step has run");
        cuda_ok(cudaEventSynchronize(c->ev1), "cudaEventSynchronize");
        cuda_ok(cudaEventElapsedTime(ms, c->ev0, c->ev1), "cudaEventElapsedTime");
    });
}

lima_status lima_set_thermostat_scalar(lima_ctx* c, float scalar) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        need(c->p.semantics == LIMA_SEMANTICS_REFERENCE, LIMA_ERR_UNSUPPORTED,
             "the thermostat scalar belongs to reference semantics");
        need(std::isfinite(scalar) && scalar > 0.f, LIMA_ERR_ARGUMENT, "thermostat scalar must be finite and positive");
        lima::set_device_float(c->ref.lambda, scalar, c->stream);
        c->lambda_pending_reset = true;
    });
}

namespace {
// physics semantics: device copies of the reference's state structs (one pool
// block per context, made by the first read)
struct PhysStage {
    lima_compound_state* states;
    lima_float3* prev;
    lima_solvent* sols;
};
PhysStage phys_stage(lima_ctx* c) {
    const size_t nc = c->comps.size(), ns = c->sols.size();
    const size_t b_states = (nc * sizeof(lima_compound_state) + 255) & ~size_t(255);
    const size_t b_prev = (nc * lima::kMaxCP * sizeof(lima_float3) + 255) & ~size_t(255);
    if (!c->read_stage) {
        c->read_stage = lima::pool_alloc(b_states + b_prev + ns * sizeof(lima_solvent), c->stream);
        need(c->read_stage != nullptr, LIMA_ERR_CUDA, "cannot allocate the readback buffer");
        c->pool_allocs.push_back(c->read_stage);
    }
    uint8_t* b = static_cast<uint8_t*>(c->read_stage);
    return {reinterpret_cast<lima_compound_state*>(b), reinterpret_cast<lima_float3*>(b + b_states),
            reinterpret_cast<lima_solvent*>(b + b_states + b_prev)};
}
}  // namespace

lima_status lima_get_compound_states(lima_ctx* c, lima_compound_state* states, lima_float3* prev) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        sync_checked(c);
        const int nc = static_cast<int>(c->comps.size());
        const size_t ncp = static_cast<size_t>(nc) * lima::kMaxCP;
        if (c->p.semantics == LIMA_SEMANTICS_PHYSICS) {
            // one kernel writes the structs on the device; one copy each into the caller's arrays
            if (nc == 0 || (!states && !prev)) return;
            const PhysStage st = phys_stage(c);
            lima::launch_read_compounds(c->phys, c->cur, states ? st.states : nullptr, prev ? st.prev : nullptr,
                                        c->stream);
            if (states)
                cudaMemcpyAsync(states, st.states, sizeof(lima_compound_state) * nc, cudaMemcpyDeviceToHost, c->stream);
            if (prev) cudaMemcpyAsync(prev, st.prev, sizeof(lima_float3) * ncp, cudaMemcpyDeviceToHost, c->stream);
            sync_checked(c);
            return;
        }
        std::vector<float4> hp(ncp), hq(ncp);
        cuda_ok(cudaMemcpy(hp.data(), c->ref.cpos[c->cur], sizeof(float4) * ncp, cudaMemcpyDeviceToHost), "D2H");
        cuda_ok(cudaMemcpy(hq.data(), c->ref.cprev, sizeof(float4) * ncp, cudaMemcpyDeviceToHost), "D2H");
        for (int i = 0; i < nc; i++) {
            if (states) {
                std::memset(&states[i], 0, sizeof(lima_compound_state));
                states[i].n_particles = c->comps[i].n_particles;
            }
            for (int t = 0; t < lima::kMaxCP; t++) {
                const bool live = t < c->comps[i].n_particles;
                const float4 a = hp[i * lima::kMaxCP + t], b = hq[i * lima::kMaxCP + t];
                if (states && live) states[i].positions[t] = lima_float3{a.x, a.y, a.z};
                if (prev) prev[i * lima::kMaxCP + t] = live ? lima_float3{b.x, b.y, b.z} : lima_float3{0.f, 0.f, 0.f};
            }
        }
    });
}

lima_status lima_get_solvents(lima_ctx* c, lima_solvent* sols) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        need(sols != nullptr || c->sols.empty(), LIMA_ERR_ARGUMENT, "null solvent array");
        sync_checked(c);
        const int ns = static_cast<int>(c->sols.size());
        if (ns == 0) return;
        if (c->p.semantics == LIMA_SEMANTICS_PHYSICS) {
            const PhysStage st = phys_stage(c);
            lima::launch_read_solvents(c->phys, c->cur, st.sols, c->stream);
            cudaMemcpyAsync(sols, st.sols, sizeof(lima_solvent) * ns, cudaMemcpyDeviceToHost, c->stream);
            sync_checked(c);
            return;
        }
        std::vector<float4> a(ns), b(ns);
        cuda_ok(cudaMemcpy(a.data(), c->ref.spos[c->cur], sizeof(float4) * ns, cudaMemcpyDeviceToHost), "D2H");
        cuda_ok(cudaMemcpy(b.data(), c->ref.sprev[c->cur], sizeof(float4) * ns, cudaMemcpyDeviceToHost), "D2H");
        for (int i = 0; i < ns; i++) {
            sols[i].pos = lima_float3{a[i].x, a[i].y, a[i].z};
            sols[i].pos_tsub1 = lima_float3{b[i].x, b[i].y, b[i].z};
        }
    });
}

lima_status lima_get_positions(lima_ctx* c, float* cxyz, float* sxyz) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        sync_checked(c);
        const int nc = static_cast<int>(c->comps.size()), ns = static_cast<int>(c->sols.size());
        const size_t ncp = static_cast<size_t>(nc) * lima::kMaxCP;
        const bool phys = c->p.semantics == LIMA_SEMANTICS_PHYSICS;
        if (cxyz && nc > 0) {
            std::vector<float4> hp(ncp);
            if (phys) {
                // the same values lima_get_compound_states gives
                std::vector<lima_compound_state> st(nc);
                const PhysStage g = phys_stage(c);
                lima::launch_read_compounds(c->phys, c->cur, g.states, nullptr, c->stream);
                cudaMemcpyAsync(st.data(), g.states, sizeof(lima_compound_state) * nc, cudaMemcpyDeviceToHost, c->stream);
                sync_checked(c);
                for (size_t k = 0; k < ncp; k++) {
                    const lima_float3 v = st[k / lima::kMaxCP].positions[k % lima::kMaxCP];
                    hp[k] = make_float4(v.x, v.y, v.z, 0.f);
                }
            } else {
                cuda_ok(cudaMemcpy(hp.data(), c->ref.cpos[c->cur], sizeof(float4) * ncp, cudaMemcpyDeviceToHost), "D2H");
            }
            for (int i = 0; i < nc; i++)
                for (int t = 0; t < lima::kMaxCP; t++) {
                    const size_t k = static_cast<size_t>(i) * lima::kMaxCP + t;
                    const bool live = t < c->comps[i].n_particles;
                    cxyz[3 * k] = live ? hp[k].x : 0.f;
                    cxyz[3 * k + 1] = live ? hp[k].y : 0.f;
                    cxyz[3 * k + 2] = live ? hp[k].z : 0.f;
                }
        }
        if (sxyz && ns > 0) {
            if (phys) {
                std::vector<lima_solvent> sv(ns);
                const PhysStage g = phys_stage(c);
                lima::launch_read_solvents(c->phys, c->cur, g.sols, c->stream);
                cudaMemcpyAsync(sv.data(), g.sols, sizeof(lima_solvent) * ns, cudaMemcpyDeviceToHost, c->stream);
                sync_checked(c);
                for (int i = 0; i < ns; i++) {
                    sxyz[3 * i] = sv[i].pos.x;
                    sxyz[3 * i + 1] = sv[i].pos.y;
                    sxyz[3 * i + 2] = sv[i].pos.z;
                }
            } else {
                std::vector<float4> a(ns);
                cuda_ok(cudaMemcpy(a.data(), c->ref.spos[c->cur], sizeof(float4) * ns, cudaMemcpyDeviceToHost), "D2H");
                for (int i = 0; i < ns; i++) {
                    sxyz[3 * i] = a[i].x;
                    sxyz[3 * i + 1] = a[i].y;
                    sxyz[3 * i + 2] = a[i].z;
                }
            }
        }
    });
}

lima_status lima_set_state(lima_ctx* c, const lima_compound_state* states, const lima_float3* prev,
                           const lima_solvent* sols) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        sync_checked(c);
        const int nc = static_cast<int>(c->comps.size()), ns = static_cast<int>(c->sols.size());
        for (int i = 0; i < nc; i++) {
            if (states) c->states[i] = states[i];
            if (prev)
                for (int t = 0; t < c->comps[i].n_particles; t++) c->comps[i].prev_positions[t] = prev[i * lima::kMaxCP + t];
        }
        if (sols) std::memcpy(c->sols.data(), sols, sizeof(lima_solvent) * ns);
        if (c->p.semantics == LIMA_SEMANTICS_REFERENCE) {
            const size_t ncp = static_cast<size_t>(nc) * lima::kMaxCP;
            std::vector<float4> hp(ncp, make_float4(0, 0, 0, 0)), hq(ncp, make_float4(0, 0, 0, 0));
            for (int i = 0; i < nc; i++)
                for (int t = 0; t < c->comps[i].n_particles; t++) {
                    hp[i * lima::kMaxCP + t] = f4(c->states[i].positions[t]);
                    hq[i * lima::kMaxCP + t] = f4(c->comps[i].prev_positions[t]);
                }
            std::vector<float4> sp(ns), spr(ns);
            for (int i = 0; i < ns; i++) {
                sp[i] = f4(c->sols[i].pos);
                spr[i] = f4(c->sols[i].pos_tsub1);
            }
            cuda_ok(cudaMemcpy(c->ref.cpos[c->cur], hp.data(), sizeof(float4) * ncp, cudaMemcpyHostToDevice), "H2D");
            cuda_ok(cudaMemcpy(c->ref.cprev, hq.data(), sizeof(float4) * ncp, cudaMemcpyHostToDevice), "H2D");
            cuda_ok(cudaMemcpy(c->ref.spos[c->cur], sp.data(), sizeof(float4) * ns, cudaMemcpyHostToDevice), "H2D");
            cuda_ok(cudaMemcpy(c->ref.sprev[c->cur], spr.data(), sizeof(float4) * ns, cudaMemcpyHostToDevice), "H2D");
        } else {
            lima::PhysHost h;
            h.params = &c->p;
            h.ff = &c->ff;
            h.comps = c->comps.data();
            h.states = c->states.data();
            h.n_c = nc;
            h.bridges = c->bridges.data();
            h.n_b = static_cast<int>(c->bridges.size());
            h.sols = c->sols.data();
            h.n_s = ns;
            lima::phys_upload_state(h, c->phys, c->cur, c->stream);
            lima::phys_rebuild(c->phys, c->cur, c->stream);
            lima::phys_prime(c->phys, c->cur, c->stream);
            c->launches += lima::kRebuildKernels;
            c->host_rebuilds++;
            c->last_nlist_step = c->step;
        }
        sync_checked(c);
    });
}

lima_status lima_get_forces(lima_ctx* c, lima_float3* fc, lima_float3* fs) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        sync_checked(c);
        const int nc = static_cast<int>(c->comps.size()), ns = static_cast<int>(c->sols.size());
        const size_t ncp = static_cast<size_t>(nc) * lima::kMaxCP;
        std::vector<float4> a(ncp), b(ns);
        if (c->p.semantics == LIMA_SEMANTICS_REFERENCE) {
            cuda_ok(cudaMemcpy(a.data(), c->ref.force_c, sizeof(float4) * ncp, cudaMemcpyDeviceToHost), "D2H");
            cuda_ok(cudaMemcpy(b.data(), c->ref.force_s, sizeof(float4) * ns, cudaMemcpyDeviceToHost), "D2H");
        } else {
            lima::phys_read_forces(c->phys, c->comps.data(), a.data(), b.data());
        }
        if (fc)
            for (size_t i = 0; i < ncp; i++) fc[i] = lima_float3{a[i].x, a[i].y, a[i].z};
        if (fs)
            for (int i = 0; i < ns; i++) fs[i] = lima_float3{b[i].x, b[i].y, b[i].z};
    });
}

lima_status lima_compute_energies(lima_ctx* c) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        need(c->p.semantics == LIMA_SEMANTICS_PHYSICS, LIMA_ERR_UNSUPPORTED,
             "the reference computes no LJ energy; reference semantics report potE of the last step");
        if (c->phys.dynamic_list && lima::phys_rebuild_pending(c->phys, c->stream)) {
            lima::phys_rebuild(c->phys, c->cur, c->stream);
            c->launches += lima::kRebuildKernels;
            c->host_rebuilds++;
        }
        lima::phys_energy_now(c->phys, c->cur, c->stream);
        c->launches += 2;
        sync_checked(c);
    });
}

lima_status lima_get_energies(lima_ctx* c, double* totals, double* per_particle) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        sync_checked(c);
        const int nc = static_cast<int>(c->comps.size()), ns = static_cast<int>(c->sols.size());
        const size_t ncp = static_cast<size_t>(nc) * lima::kMaxCP;
        if (c->p.semantics == LIMA_SEMANTICS_REFERENCE) {
            std::vector<double> pe(ncp);
            cuda_ok(cudaMemcpy(pe.data(), c->ref.potE, sizeof(double) * ncp, cudaMemcpyDeviceToHost), "D2H");
            if (per_particle) {
                std::memcpy(per_particle, pe.data(), sizeof(double) * ncp);
                std::memset(per_particle + ncp, 0, sizeof(double) * ns);
            }
            if (totals) {
                std::memset(totals, 0, sizeof(double) * LIMA_E_COUNT);
                double sum = 0;
                for (int i = 0; i < nc; i++)
                    for (int t = 0; t < lima::kMaxCP; t++) sum += pe[i * lima::kMaxCP + t];
                totals[LIMA_E_BOND] = sum;   // the reference's bonded potE (its only energy)
                totals[LIMA_E_TOTAL] = sum;
                double temp = 0;
                cuda_ok(cudaMemcpy(&temp, c->ref.ke_accum, sizeof(double), cudaMemcpyDeviceToHost), "D2H");
                totals[LIMA_E_TEMPERATURE] = temp;
            }
        } else {
            lima::phys_read_energies(c->phys, totals, per_particle, c->comps.data(), nc, ns);
        }
    });
}

lima_status lima_build_nlist(lima_ctx* c) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        if (c->p.semantics == LIMA_SEMANTICS_REFERENCE) {
            ref_nlist_now(c);
        } else {
            lima::phys_rebuild(c->phys, c->cur, c->stream);
            c->launches += lima::kRebuildKernels;
            c->host_rebuilds++;
            c->last_nlist_step = c->step;
        }
        sync_checked(c);
    });
}

namespace {
void need_physics(lima_ctx* c) {
    need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
    need(c->p.semantics == LIMA_SEMANTICS_PHYSICS, LIMA_ERR_UNSUPPORTED,
         "parameters and gradients belong to physics semantics");
}
void need_gradable(lima_ctx* c) {
    need_physics(c);
    need(c->p.precision == LIMA_PRECISION_FP32, LIMA_ERR_UNSUPPORTED, "the loss / adjoint passes run in plain FP32");
    need(c->p.thermostat == LIMA_THERMOSTAT_NONE, LIMA_ERR_UNSUPPORTED,
         "the loss / adjoint passes integrate NVE (thermostat none)");
    need(c->phys.use_switch, LIMA_ERR_UNSUPPORTED, "the loss / adjoint passes need the potential switch");
}
}  // namespace

lima_status lima_get_param_count(lima_ctx* c, int* n) {
    return guarded(c, [&] {
        need(n != nullptr, LIMA_ERR_ARGUMENT, "null count");
        need_physics(c);
        *n = c->params.count();
    });
}

lima_status lima_get_param_layout(lima_ctx* c, int* counts) {
    return guarded(c, [&] {
        need(counts != nullptr, LIMA_ERR_ARGUMENT, "null counts");
        need_physics(c);
        counts[0] = c->params.n_types;
        for (int k = 0; k < lima::kParKinds; k++) counts[1 + k] = static_cast<int>(c->params.tc[k].size());
    });
}

lima_status lima_get_bonded_types(lima_ctx* c, int kind, int* n_terms, int* type_of) {
    return guarded(c, [&] {
        need(kind >= 0 && kind < lima::kParKinds, LIMA_ERR_ARGUMENT, "kind must be 0 (bond), 1 (angle) or 2 (dihedral)");
        need(n_terms != nullptr, LIMA_ERR_ARGUMENT, "null count");
        need_physics(c);
        const auto& v = c->params.type_of[kind];
        *n_terms = static_cast<int>(v.size());
        if (type_of) std::copy(v.begin(), v.end(), type_of);
    });
}

lima_status lima_get_params(lima_ctx* c, double* theta) {
    return guarded(c, [&] {
        need(theta != nullptr, LIMA_ERR_ARGUMENT, "null parameter vector");
        need_physics(c);
        lima::phys_params_get(c->params, theta);
    });
}

lima_status lima_set_params(lima_ctx* c, const double* theta) {
    return guarded(c, [&] {
        need(theta != nullptr, LIMA_ERR_ARGUMENT, "null parameter vector");
        need_physics(c);
        sync_checked(c);
        std::string msg;
        const int st = lima::phys_params_set(c->phys, c->params, theta, msg, c->stream);
        if (st != LIMA_OK) fail(static_cast<lima_status>(st), msg);
        for (int t = 0; t < c->params.n_types; t++) {
            c->ff.particle_parameters[t].sigma = static_cast<float>(c->params.sigma[t]);
            c->ff.particle_parameters[t].epsilon = static_cast<float>(c->params.epsilon[t]);
        }
    });
}

lima_status lima_loss(lima_ctx* c, const lima_loss_spec* spec, double* loss) {
    return guarded(c, [&] {
        need(spec != nullptr && loss != nullptr, LIMA_ERR_ARGUMENT, "null spec or output");
        need_gradable(c);
        sync_checked(c);
        std::string msg;
        const int st = lima::adj_run(c->phys, c->cur, c->params, c->adj, c->dallocs, *spec, loss, nullptr, c->stream, msg);
        if (st != LIMA_OK) fail(static_cast<lima_status>(st), msg);
        c->host_rebuilds += 1;
        sync_checked(c);
    });
}

lima_status lima_grad(lima_ctx* c, const lima_loss_spec* spec, double* loss, double* grad) {
    return guarded(c, [&] {
        need(spec != nullptr && loss != nullptr && grad != nullptr, LIMA_ERR_ARGUMENT, "null spec or output");
        need_gradable(c);
        sync_checked(c);
        std::string msg;
        const int st = lima::adj_run(c->phys, c->cur, c->params, c->adj, c->dallocs, *spec, loss, grad, c->stream, msg);
        if (st != LIMA_OK) fail(static_cast<lima_status>(st), msg);
        c->host_rebuilds += 1;
        sync_checked(c);
    });
}

lima_status lima_rdf(lima_ctx* c, int n_bins, float r_max, double* h) {
    return guarded(c, [&] {
        need(h != nullptr, LIMA_ERR_ARGUMENT, "null output");
        need_physics(c);
        sync_checked(c);
        std::string msg;
        const int st = lima::adj_rdf(c->phys, c->cur, c->adj, c->dallocs, n_bins, r_max, h, c->stream, msg);
        if (st != LIMA_OK) fail(static_cast<lima_status>(st), msg);
    });
}

// ------------------------------------------------------------ frame log ---
lima_status lima_log_start(lima_ctx* c, const lima_log_params* p) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        need(p != nullptr, LIMA_ERR_ARGUMENT, "null log params");
        need(p->every >= 1, LIMA_ERR_ARGUMENT, "log every must be >= 1");
        need(p->ring_frames >= 1 && p->ring_frames <= 65536, LIMA_ERR_ARGUMENT, "ring_frames outside 1..65536");
        need((p->flags & ~(LIMA_LOG_TRAJ | LIMA_LOG_POTE | LIMA_LOG_TRAIN)) == 0, LIMA_ERR_ARGUMENT,
             "unknown log flags");
        sync_checked(c);
        // the logged-step graphs hold the old log's buffers
        for (auto& row : c->dgraph)
            if (row[2]) {
                cudaGraphExecDestroy(row[2]);
                row[2] = nullptr;
            }
        std::vector<int> np;
        for (const auto& cp : c->comps) np.push_back(cp.n_particles);
        std::string msg;
        int st = LIMA_OK;
        lima::framelog_start(c->log, static_cast<int>(c->sols.size()), np, *p, c->stream, msg, st);
        if (st != LIMA_OK) fail(static_cast<lima_status>(st), msg);
        sync_checked(c);
    });
}

lima_status lima_log_stop(lima_ctx* c) {
    return guarded(c, [&] {
        if (!c->log.on) return;
        lima::framelog_flush(c->log, c->stream);
        c->log.on = false;
        sync_checked(c);
    });
}

lima_status lima_log_count(lima_ctx* c, uint64_t* n) {
    return guarded(c, [&] {
        need(n != nullptr, LIMA_ERR_ARGUMENT, "null count");
        if (c->log.dev.ring) lima::framelog_flush(c->log, c->stream);
        sync_checked(c);
        *n = c->log.steps.size();
    });
}

lima_status lima_log_read(lima_ctx* c, uint64_t first, uint64_t count, uint64_t* steps, double* energies, float* traj,
                          double* potE, float* train, float* logdata) {
    return guarded(c, [&] {
        if (c->log.dev.ring) lima::framelog_flush(c->log, c->stream);
        sync_checked(c);
        const lima::FrameLog& g = c->log;
        const uint64_t nf = g.steps.size();
        need(first <= nf && count <= nf - first, LIMA_ERR_ARGUMENT, "frames outside what was recorded");
        need(!traj || g.dev.traj, LIMA_ERR_ARGUMENT, "positions were not recorded (LIMA_LOG_TRAJ)");
        need(!potE || g.dev.potE, LIMA_ERR_ARGUMENT, "potential energies were not recorded (LIMA_LOG_POTE)");
        need(!train || g.dev.train, LIMA_ERR_ARGUMENT, "train data were not recorded (LIMA_LOG_TRAIN)");
        const size_t ns = (size_t)g.dev.n_slots, nt = (size_t)g.dev.n_train * lima::kTrainValues * 3;
        if (steps) std::copy(g.steps.begin() + first, g.steps.begin() + first + count, steps);
        if (energies)
            std::copy(g.energies.begin() + first * LIMA_E_COUNT, g.energies.begin() + (first + count) * LIMA_E_COUNT,
                      energies);
        if (traj) std::copy(g.traj.begin() + first * ns * 3, g.traj.begin() + (first + count) * ns * 3, traj);
        if (potE) std::copy(g.potE.begin() + first * ns, g.potE.begin() + (first + count) * ns, potE);
        if (train) std::copy(g.train.begin() + first * nt, g.train.begin() + (first + count) * nt, train);
        if (logdata)
            std::copy(g.logdata.begin() + first * lima::kLogDataFloats,
                      g.logdata.begin() + (first + count) * lima::kLogDataFloats, logdata);
    });
}

}  // extern "C"

namespace {
// Analyzer::analyzeEnergy (Analyzer.cu:33-207) on the recorded frames of a
// reference-semantics run: for frame f with neighbours f - 1 and f + 1, per
// particle the frame's potE and the kinetic energy of calcKineticEnergy
// (Engine.cuh:32-45) over the positions two frames apart, with the solvent
// mass for every particle as the reference's kernels use it; averaged over the
// solvents and over the compound particles, and those two averages weighed by
// their particle counts.  One Float3 per analysable frame (frames - 3, as the
// reference analyses steps - 3); sums in double.
std::vector<float> analyze_energy(lima_ctx* c, const lima::FrameLog& g) {
    const size_t nf = g.steps.size(), slots = g.dev.n_slots, ntr = g.dev.n_train;
    const int nc = static_cast<int>(c->comps.size()), ns = static_cast<int>(c->sols.size());
    int ncp = 0;
    for (const auto& cp : c->comps) ncp += cp.n_particles;
    const double mass = c->ff.particle_parameters[LIMA_ATOMTYPE_SOL].mass;
    const double dt = c->p.dt * static_cast<double>(g.every);
    const float L = c->p.box_len, Lh = 0.5f * L;
    auto ke = [&](const float* a, const float* b) {   // calcKineticEnergy(a, b): b moved into a's image
        float bb[3];
        for (int q = 0; q < 3; q++) {
            bb[q] = b[q];
            if (bb[q] - a[q] > Lh) bb[q] -= L;
            else if (bb[q] - a[q] < -Lh) bb[q] += L;
        }
        const float dx = a[0] - bb[0], dy = a[1] - bb[1], dz = a[2] - bb[2];
        const float vel = static_cast<float>(static_cast<double>(std::sqrt(dx * dx + dy * dy + dz * dz) * 0.5f) / dt);
        return static_cast<float>(0.5 * mass * static_cast<double>(vel) * static_cast<double>(vel));
    };
    std::vector<float> out;
    const size_t n_an = nf >= 4 ? nf - 3 : 0;
    for (size_t k = 0; k < n_an; k++) {
        const size_t f = k + 1;
        const float* xm = &g.traj[(f - 1) * slots * 3];
        const float* xp = &g.traj[(f + 1) * slots * 3];
        const double* pe = &g.potE[f * slots];
        double sol[3] = {0, 0, 0}, cmp[3] = {0, 0, 0};
        for (int s = 0; s < ns; s++) {
            const size_t i = ntr + s;
            const double k_e = ke(&xp[3 * i], &xm[3 * i]);
            sol[0] += pe[i];
            sol[1] += k_e;
            sol[2] += pe[i] + k_e;
        }
        for (int ci = 0; ci < nc; ci++)
            for (int t = 0; t < c->comps[ci].n_particles; t++) {
                const size_t i = static_cast<size_t>(ci) * LIMA_MAX_COMPOUND_PARTICLES + t;
                const double k_e = ke(&xp[3 * i], &xm[3 * i]);
                cmp[0] += pe[i];
                cmp[1] += k_e;
                cmp[2] += pe[i] + k_e;
            }
        const double n_tot = static_cast<double>(ns + ncp);
        for (int q = 0; q < 3; q++) {
            const double avg_s = ns ? sol[q] / ns : 0.0, avg_c = ncp ? cmp[q] / ncp : 0.0;
            out.push_back(static_cast<float>((avg_s * ns + avg_c * ncp) / n_tot));
        }
    }
    return out;
}
}  // namespace

extern "C" {

lima_status lima_log_write(lima_ctx* c, const char* dir) {
    return guarded(c, [&] {
        need(dir != nullptr, LIMA_ERR_ARGUMENT, "null directory");
        if (c->log.dev.ring) lima::framelog_flush(c->log, c->stream);
        sync_checked(c);
        const lima::FrameLog& g = c->log;
        const size_t nf = g.steps.size();
        need(nf > 0, LIMA_ERR_STATE, "no frames recorded");
        auto dump = [&](const char* name, const void* data, size_t bytes) {
            const std::string path = std::string(dir) + "/" + name;
            FILE* f = std::fopen(path.c_str(), "wb");
            need(f != nullptr, LIMA_ERR_ARGUMENT, "cannot open " + path);
            const size_t w = bytes ? std::fwrite(data, 1, bytes, f) : 0;
            std::fclose(f);
            need(w == bytes, LIMA_ERR_ARGUMENT, "short write to " + path);
        };
        // Environment.cpp:130: logging_data, 10 floats per step
        dump("logdata.bin", g.logdata.data(), g.logdata.size() * sizeof(float));
        std::vector<float> energy, temperature(nf);
        for (size_t f = 0; f < nf; f++) temperature[f] = static_cast<float>(g.energies[f * LIMA_E_COUNT + LIMA_E_TEMPERATURE]);
        if (c->p.semantics == LIMA_SEMANTICS_PHYSICS) {
            // Analyzer::analyzeEnergy (Analyzer.cu:177-183): per step the mean per particle of
            // (potential, kinetic, total) energy as a Float3; here from the step's FP64 sums
            const double n = static_cast<double>(c->phys.n);
            energy.resize(nf * 3);
            for (size_t f = 0; f < nf; f++) {
                const double* e = &g.energies[f * LIMA_E_COUNT];
                const double pot = e[LIMA_E_LJ] + e[LIMA_E_BOND] + e[LIMA_E_ANGLE] + e[LIMA_E_DIHEDRAL];
                energy[3 * f + 0] = static_cast<float>(pot / n);
                energy[3 * f + 1] = static_cast<float>(e[LIMA_E_KINETIC] / n);
                energy[3 * f + 2] = static_cast<float>(e[LIMA_E_TOTAL] / n);
            }
        } else {
            need(g.dev.traj && g.dev.potE, LIMA_ERR_STATE, "the energy analysis needs traj and potE frames");
            energy = analyze_energy(c, g);
        }
        dump("energy.bin", energy.data(), energy.size() * sizeof(float));
        dump("temperature.bin", temperature.data(), temperature.size() * sizeof(float));
        // Environment.cpp:137-141: data_GAN of every step
        if (g.dev.train) dump("sim_traindata.bin", g.train.data(), g.train.size() * sizeof(float));
        if (g.dev.traj) dump("traj.bin", g.traj.data(), g.traj.size() * sizeof(float));
        if (g.dev.potE) dump("potE.bin", g.potE.data(), g.potE.size() * sizeof(double));
    });
}

// ----------------------------------------------------------- rasterizer ---
namespace {
// balls of the current state into c->render.balls[1] (device), sorted by depth
void render_now(lima_ctx* c) {
    lima::RenderBuf& r = c->render;
    const int nc = static_cast<int>(c->comps.size()), ns = static_cast<int>(c->sols.size());
    const int n_slots = nc * lima::kMaxCP + ns;
    if (!r.ready) {
        // ATOM_TYPE per slot: compound particles by atom_color_types (RAS_getTypeFromIndex,
        // Rasterizer.cu:126-146), solvents SOL, empty slots NONE (QuantomTypes.cuh:16)
        static const uint8_t by_color[7] = {6, 2, 1, 4, 5, 3, 6};
        std::vector<uint8_t> kind(n_slots, 0);
        for (int cc = 0; cc < nc; cc++)
            for (int l = 0; l < c->comps[cc].n_particles; l++) {
                const int t = c->comps[cc].atom_color_types[l];
                kind[cc * lima::kMaxCP + l] = t < 7 ? by_color[t] : 0;
            }
        for (int s = 0; s < ns; s++) kind[nc * lima::kMaxCP + s] = 6;
        std::vector<uint32_t> ref_slot;
        if (c->p.semantics == LIMA_SEMANTICS_PHYSICS) {
            for (int cc = 0; cc < nc; cc++)
                for (int l = 0; l < c->comps[cc].n_particles; l++) ref_slot.push_back(cc * lima::kMaxCP + l);
            for (int s = 0; s < ns; s++) ref_slot.push_back(nc * lima::kMaxCP + s);
        }
        need(lima::render_setup(r, n_slots, kind, ref_slot, c->dallocs, c->stream), LIMA_ERR_CUDA,
             "rasterizer: out of device memory");
    }
    if (c->p.semantics == LIMA_SEMANTICS_PHYSICS) {
        lima::render_slot_positions_phys(r, c->phys, c->cur, c->stream);
        c->launches++;
    } else {
        if (nc)
            cuda_ok(cudaMemcpyAsync(r.slot_pos, c->ref.cpos[c->cur], sizeof(float4) * nc * lima::kMaxCP,
                                    cudaMemcpyDeviceToDevice, c->stream),
                    "cudaMemcpyAsync");
        if (ns)
            cuda_ok(cudaMemcpyAsync(r.slot_pos + nc * lima::kMaxCP, c->ref.spos[c->cur], sizeof(float4) * ns,
                                    cudaMemcpyDeviceToDevice, c->stream),
                    "cudaMemcpyAsync");
    }
    c->launches += lima::render_balls(r, c->p.box_len, c->stream);
}
}  // namespace

lima_status lima_render(lima_ctx* c, lima_render_ball* balls) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        need(balls != nullptr, LIMA_ERR_ARGUMENT, "null ball array");
        sync_checked(c);
        render_now(c);
        cuda_ok(cudaMemcpyAsync(balls, c->render.balls[1], sizeof(lima_render_ball) * c->render.n_slots,
                                cudaMemcpyDeviceToHost, c->stream),
                "cudaMemcpyAsync");
        sync_checked(c);
    });
}

lima_status lima_render_image(lima_ctx* c, int width, int height, uint8_t* rgb) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        need(rgb != nullptr, LIMA_ERR_ARGUMENT, "null image");
        need(width >= 1 && width <= 16384 && height >= 1 && height <= 16384, LIMA_ERR_ARGUMENT,
             "image size outside 1..16384");
        sync_checked(c);
        render_now(c);
        need(lima::render_image(c->render, width, height, rgb, c->dallocs, c->stream), LIMA_ERR_CUDA,
             "rasterizer: out of device memory for the image");
        c->launches += 2;
        sync_checked(c);
    });
}

lima_status lima_get_rebuild_count(lima_ctx* c, uint64_t* count) {
    return guarded(c, [&] {
        need(count != nullptr, LIMA_ERR_ARGUMENT, "null count");
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        need(c->p.semantics == LIMA_SEMANTICS_PHYSICS, LIMA_ERR_UNSUPPORTED,
             "reference semantics rebuild every nlist_period steps");
        *count = c->host_rebuilds + (c->phys.dynamic_list ? lima::phys_device_rebuilds(c->phys, c->stream) : 0);
    });
}

lima_status lima_get_nlist(lima_ctx* c, int which, uint32_t* offsets, uint32_t* ids, uint32_t* total) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        need(offsets != nullptr, LIMA_ERR_ARGUMENT, "null offsets");
        if (c->p.semantics == LIMA_SEMANTICS_PHYSICS) {
            need(which == LIMA_NL_PAIR, LIMA_ERR_UNSUPPORTED,
                 "physics semantics keeps one Verlet list (LIMA_NL_PAIR); entity lists belong to reference semantics");
            sync_checked(c);
            const uint32_t tot = lima::phys_read_list(c->phys, offsets, ids);
            if (total) *total = tot;
            return;
        }
        need(which >= 0 && which <= 3, LIMA_ERR_ARGUMENT, "unknown list selector");
        sync_checked(c);
        const lima::RefDev& d = c->ref;
        const int nc = d.n_c, ns = d.n_s;
        std::vector<uint32_t> cnt, rows;
        auto fetch = [&](const uint32_t* dcnt, const uint32_t* dids, int n, size_t cap, bool colmajor) {
            cnt.resize(n);
            rows.resize(static_cast<size_t>(n) * cap);
            if (n) {
                cuda_ok(cudaMemcpy(cnt.data(), dcnt, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost), "D2H");
                cuda_ok(cudaMemcpy(rows.data(), dids, sizeof(uint32_t) * n * cap, cudaMemcpyDeviceToHost), "D2H");
            }
            (void)colmajor;
        };
        uint32_t pos = 0;
        if (which == LIMA_NL_COMPOUND_COMPOUND || which == LIMA_NL_COMPOUND_SOLVENT) {
            const bool cc = which == LIMA_NL_COMPOUND_COMPOUND;
            const size_t cap = cc ? lima::kMaxCP : d.cs_cap;
            fetch(cc ? d.cc_cnt : d.cs_cnt, cc ? d.cc_ids : d.cs_ids, nc, cap, false);
            for (int i = 0; i < nc; i++) {
                offsets[i] = pos;
                if (ids)
                    for (uint32_t k = 0; k < cnt[i]; k++) ids[pos + k] = rows[i * cap + k];
                pos += cnt[i];
            }
            offsets[nc] = pos;
        } else if (which == LIMA_NL_SOLVENT_SOLVENT) {
            fetch(d.ss_cnt, d.ss_ids, ns, d.ss_cap, true);
            for (int i = 0; i < ns; i++) {
                offsets[i] = pos;
                if (ids)
                    for (uint32_t k = 0; k < cnt[i]; k++) ids[pos + k] = rows[static_cast<size_t>(k) * ns + i];
                pos += cnt[i];
            }
            offsets[ns] = pos;
        } else {   // solvent -> compound: the transpose of compound -> solvent
            fetch(d.cs_cnt, d.cs_ids, nc, d.cs_cap, false);
            std::vector<std::vector<uint32_t>> tr(ns);
            for (int cidx = 0; cidx < nc; cidx++)
                for (uint32_t k = 0; k < cnt[cidx]; k++) tr[rows[static_cast<size_t>(cidx) * d.cs_cap + k]].push_back(cidx);
            for (int i = 0; i < ns; i++) {
                offsets[i] = pos;
                if (ids)
                    for (size_t k = 0; k < tr[i].size(); k++) ids[pos + k] = tr[i][k];
                pos += static_cast<uint32_t>(tr[i].size());
            }
            offsets[ns] = pos;
        }
        if (total) *total = pos;
    });
}

lima_status lima_set_nlist(lima_ctx* c, int which, const uint32_t* offsets, const uint32_t* ids) {
    return guarded(c, [&] {
        need(c->finished, LIMA_ERR_STATE, "lima_finish_box has not run");
        need(c->p.semantics == LIMA_SEMANTICS_REFERENCE, LIMA_ERR_UNSUPPORTED, "lists can be set in reference semantics only");
        need(offsets != nullptr && ids != nullptr, LIMA_ERR_ARGUMENT, "null list arrays");
        need(which != LIMA_NL_SOLVENT_COMPOUND, LIMA_ERR_UNSUPPORTED, "solvent->compound lists are derived from compound->solvent");
        sync_checked(c);
        lima::RefDev& d = c->ref;
        const int n = (which == LIMA_NL_SOLVENT_SOLVENT) ? d.n_s : d.n_c;
        const int idmax = (which == LIMA_NL_COMPOUND_SOLVENT || which == LIMA_NL_SOLVENT_SOLVENT) ? d.n_s : d.n_c;
        const size_t cap = which == LIMA_NL_COMPOUND_COMPOUND ? lima::kMaxCP
                                                              : (which == LIMA_NL_COMPOUND_SOLVENT ? d.cs_cap : d.ss_cap);
        std::vector<uint32_t> cnt(n), rows(static_cast<size_t>(n) * cap, 0);
        for (int i = 0; i < n; i++) {
            need(offsets[i + 1] >= offsets[i], LIMA_ERR_ARGUMENT, "offsets not monotone");
            const uint32_t k = offsets[i + 1] - offsets[i];
            need(k <= cap, LIMA_ERR_CAPACITY, "list longer than its capacity");
            cnt[i] = k;
            for (uint32_t q = 0; q < k; q++) {
                const uint32_t id = ids[offsets[i] + q];
                need(id < static_cast<uint32_t>(idmax), LIMA_ERR_ARGUMENT, "list id out of range");
                if (which == LIMA_NL_SOLVENT_SOLVENT)
                    rows[static_cast<size_t>(q) * n + i] = id;
                else
                    rows[i * cap + q] = id;
            }
        }
        uint32_t* dcnt = which == LIMA_NL_COMPOUND_COMPOUND ? d.cc_cnt : (which == LIMA_NL_COMPOUND_SOLVENT ? d.cs_cnt : d.ss_cnt);
        uint32_t* dids = which == LIMA_NL_COMPOUND_COMPOUND ? d.cc_ids : (which == LIMA_NL_COMPOUND_SOLVENT ? d.cs_ids : d.ss_ids);
        if (n) {
            cuda_ok(cudaMemcpy(dcnt, cnt.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice), "H2D");
            cuda_ok(cudaMemcpy(dids, rows.data(), sizeof(uint32_t) * rows.size(), cudaMemcpyHostToDevice), "H2D");
        }
        if (which == LIMA_NL_COMPOUND_COMPOUND && n) {
            std::vector<uint8_t> bm(static_cast<size_t>(n) * n, 0);
            for (int i = 0; i < n; i++)
                for (uint32_t q = 0; q < cnt[i]; q++) bm[static_cast<size_t>(i) * n + rows[i * cap + q]] = 1;
            cuda_ok(cudaMemcpy(d.cc_prev, bm.data(), bm.size(), cudaMemcpyHostToDevice), "H2D");
        }
    });
}

}  // extern "C"
