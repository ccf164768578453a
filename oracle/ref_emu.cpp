// Oracle build of the REFERENCE engine for the host CPU.  Test infrastructure:
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load the
// library this file builds (oracle/_ref/libref_lima.so); the product never does.
//
// It compiles the reference's own per-step code — Quantom/Quantom/Engine.cu
// (kernels compoundBridgeKernel/compoundKernel/solventForceKernel at
// Engine.cu:880-1223, device math at Engine.cu:461-869, host neighbour-list
// code at Engine.cu:146-287) and the headers it includes — from a temporary
// copy made by oracle/build_ref.sh, and runs the three kernels on the host
// with a small CUDA-block emulator:
//   * every CUDA thread of a block is a fiber with its own stack;
//   * __syncthreads() yields to the block scheduler, which resumes every fiber
//     of the block in threadIdx order until each reaches the barrier (or
//     returns), then releases the barrier;
//   * __shared__ variables are per-OS-thread statics (ref_shim/cuda_runtime.h);
//   * blocks of compoundKernel/solventForceKernel run in parallel over a pool
//     of std::threads (they write disjoint outputs); compoundBridgeKernel runs its
//     blocks in order, because two bridges may write the same particle.
//
// Deviations from running the reference on a GPU, all deliberate:
//   * host IEEE float arithmetic with no FMA contraction (-ffp-contract=off),
//     the semantics of the reference's host neighbour-list code; the GPU build
//     of the reference contracts a*b+c into FMAs inside the kernels;
//   * NeighborList::loadData's double increment (Bodies.cuh:280-283) is
//     removed in the copy, so compoundKernel sees every solvent neighbour
//     instead of stale shared memory for half of them;
//   * BOX_LEN/CUTOFF are runtime values and list capacities are raised
//     (ref_shim/Constants.cuh).
#include "cuda_runtime.h"

#include <vector>
#include <string>
#include <memory>
#include <stdexcept>
#include <atomic>
#include <thread>

#define private public
#include "Engine.cu"
#include "Rasterizer.cu"
#undef private

float BOX_LEN = 7.f;
float BOX_LEN_HALF = 3.5f;
float CUTOFF = 0.7f;

thread_local uint3 threadIdx = {0, 0, 0};
thread_local uint3 blockIdx = {0, 0, 0};
thread_local dim3 blockDim(1, 1, 1);
thread_local dim3 gridDim(1, 1, 1);

// ---------------------------------------------------------------- fibers ----
extern "C" void lima_emu_switch(void** save_sp, void* to_sp);

namespace {

enum FiberState { F_READY = 0, F_BARRIER = 1, F_DONE = 2 };
constexpr size_t kFiberStack = 256 * 1024;

using KernelFn = void (*)(Box*);

struct Fiber {
    void* sp = nullptr;
    int state = F_READY;
    char* stack = nullptr;
};

struct Runner {
    std::vector<Fiber> fibers;
    void* sched_sp = nullptr;
    int cur = 0;
    KernelFn fn = nullptr;
    Box* arg = nullptr;
    bool aborted = false;
    ~Runner() {
        for (auto& f : fibers) std::free(f.stack);
    }
};

thread_local Runner* tl_runner = nullptr;
thread_local bool tl_in_fiber = false;
thread_local int tl_kernel_kind = 0;  // 1 compoundKernel, 2 solventForceKernel, 3 bridge

// Set when a fiber called exit(); read by the launch after the kernel.
int g_exit_code = 0;
bool g_exit_called = false;

[[noreturn]] void fiber_main() {
    Runner* r = tl_runner;
    r->fn(r->arg);
    r->fibers[r->cur].state = F_DONE;
    lima_emu_switch(&r->fibers[r->cur].sp, r->sched_sp);
    __builtin_unreachable();
}

// Frame layout must match lima_emu_switch (ref_switch.S): from the lowest
// address: [mxcsr|fpu cw][r15][r14][r13][r12][rbx][rbp][return address].
void* prep_fiber_stack(char* base, size_t size) {
    uintptr_t top = (reinterpret_cast<uintptr_t>(base) + size) & ~static_cast<uintptr_t>(15);
    uint64_t* sp = reinterpret_cast<uint64_t*>(top);
    *--sp = 0;                                             // fake caller return address
    *--sp = reinterpret_cast<uint64_t>(&fiber_main);       // consumed by `ret`
    for (int i = 0; i < 6; i++) *--sp = 0;                 // rbp rbx r12 r13 r14 r15
    --sp;
    uint32_t* csr = reinterpret_cast<uint32_t*>(sp);
    csr[0] = 0x1F80;                                       // MXCSR default
    reinterpret_cast<uint16_t*>(csr)[2] = 0x037F;          // x87 control word default
    return sp;
}

// Runs one block to completion.  Returns false if a fiber called exit().
bool run_block(Runner& r, KernelFn fn, Box* arg, unsigned bidx, unsigned nthreads, unsigned ngrid) {
    if (r.fibers.size() < nthreads) {
        size_t old = r.fibers.size();
        r.fibers.resize(nthreads);
        for (size_t i = old; i < nthreads; i++) r.fibers[i].stack = static_cast<char*>(std::malloc(kFiberStack));
    }
    r.fn = fn;
    r.arg = arg;
    r.aborted = false;
    blockIdx = {bidx, 0, 0};
    blockDim = dim3(nthreads, 1, 1);
    gridDim = dim3(ngrid, 1, 1);
    for (unsigned t = 0; t < nthreads; t++) {
        r.fibers[t].sp = prep_fiber_stack(r.fibers[t].stack, kFiberStack);
        r.fibers[t].state = F_READY;
    }
    tl_runner = &r;
    for (;;) {
        bool any = false;
        for (unsigned t = 0; t < nthreads; t++) {
            if (r.fibers[t].state == F_DONE) continue;
            any = true;
            r.fibers[t].state = F_READY;
            r.cur = static_cast<int>(t);
            threadIdx = {t, 0, 0};
            tl_in_fiber = true;
            lima_emu_switch(&r.sched_sp, r.fibers[t].sp);
            tl_in_fiber = false;
            if (r.aborted) {
                tl_runner = nullptr;
                return false;
            }
        }
        if (!any) break;
    }
    tl_runner = nullptr;
    return true;
}

bool launch(KernelFn fn, int kind, unsigned grid, unsigned block, Box* box, bool parallel, int n_threads) {
    if (!parallel || n_threads <= 1 || grid <= 1) {
        Runner r;
        tl_kernel_kind = kind;
        bool ok = true;
        for (unsigned b = 0; b < grid && ok; b++) ok = run_block(r, fn, box, b, block, grid);
        tl_kernel_kind = 0;
        return ok;
    }
    std::atomic<unsigned> next{0};
    std::atomic<bool> ok{true};
    auto worker = [&]() {
        Runner r;
        tl_kernel_kind = kind;
        for (;;) {
            unsigned b = next.fetch_add(1);
            if (b >= grid || !ok.load()) break;
            if (!run_block(r, fn, box, b, block, grid)) ok.store(false);
        }
        tl_kernel_kind = 0;
    };
    const int nt = static_cast<int>(std::min<unsigned>(static_cast<unsigned>(n_threads), grid));
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
    return ok.load();
}

struct RefExit {
    int code;
};

int g_n_threads = 1;

// Total force handed to integratePosition, per particle of the last step.
std::vector<Float3>* g_forces_c = nullptr;
std::vector<Float3>* g_forces_s = nullptr;

}  // namespace

void __syncthreads() {
    Runner* r = tl_runner;
    if (!r || !tl_in_fiber) return;
    Fiber& f = r->fibers[r->cur];
    f.state = F_BARRIER;
    lima_emu_switch(&f.sp, r->sched_sp);
}

[[noreturn]] void lima_ref_exit(int code) {
    if (tl_in_fiber && tl_runner) {
        Runner* r = tl_runner;
        g_exit_called = true;
        g_exit_code = code;
        r->aborted = true;
        Fiber& f = r->fibers[r->cur];
        f.state = F_DONE;
        lima_emu_switch(&f.sp, r->sched_sp);
        __builtin_unreachable();
    }
    throw RefExit{code};
}

void lima_ref_force_hook(int p_index, const Float3* force) {
    if (tl_kernel_kind == 1 && g_forces_c) {
        (*g_forces_c)[blockIdx.x * MAX_COMPOUND_PARTICLES + threadIdx.x] = *force;
    } else if (tl_kernel_kind == 2 && g_forces_s) {
        (*g_forces_s)[p_index - MAX_COMPOUND_PARTICLES] = *force;
    }
}

// Engine::step (Engine.cu:400-451) contains <<<>>> launches, which g++ cannot
// parse; the build script removes it from the copy and this definition takes
// its place, with the same order of kernels and buffer swaps.
void Engine::step() {
    Box* box = simulation->box;
    if (box->bridge_bundle->n_bridges > 0)
        launch(compoundBridgeKernel, 3, box->bridge_bundle->n_bridges, MAX_PARTICLES_IN_BRIDGE, box, false, 1);
    if (simulation->n_compounds > 0)
        launch(compoundKernel, 1, box->n_compounds, THREADS_PER_COMPOUNDBLOCK, box, true, g_n_threads);
    if (simulation->n_solvents > 0)
        launch(solventForceKernel, 2, simulation->blocks_per_solventkernel, THREADS_PER_SOLVENTBLOCK, box, true,
               g_n_threads);
    std::swap(box->compound_state_array, box->compound_state_array_next);
    std::swap(box->solvents, box->solvents_next);
    simulation->incStep();
}

// ------------------------------------------------------------- C API -------
namespace {

struct RefCtx {
    std::unique_ptr<Simulation> sim;
    std::unique_ptr<Engine> engine;
    NListDataCollection* nldc = nullptr;
    std::vector<Float3> forces_c, forces_s;
    std::string err;
    int n_threads = 1;
    // owned allocations
    std::vector<void*> allocs;
    ~RefCtx() {
        for (void* p : allocs) std::free(p);
        if (nldc) {
            delete[] nldc->compoundstates;
            delete[] nldc->solvents;
            delete[] nldc->compound_neighborlists;
            delete[] nldc->solvent_neighborlists;
            ::operator delete(static_cast<void*>(nldc));
        }
        if (sim) {
            delete[] sim->compounds_host;
            delete sim->box;
        }
    }
    template <typename T>
    T* alloc(size_t n) {
        void* p = std::calloc(n ? n : 1, sizeof(T));
        allocs.push_back(p);
        return static_cast<T*>(p);
    }
};

template <typename F>
int guarded(RefCtx* c, F&& f) {
    try {
        g_exit_called = false;
        int rc = f();
        if (g_exit_called) {
            c->err = "reference called exit(" + std::to_string(g_exit_code) + ") inside a kernel";
            return -2;
        }
        return rc;
    } catch (const RefExit& e) {
        c->err = "reference called exit(" + std::to_string(e.code) + ")";
        return -2;
    } catch (const std::exception& e) {
        c->err = e.what();
        return -3;
    }
}

}  // namespace

extern "C" {

// Layout facts of the reference structs as this build sees them, so tests can
// check that the C-ABI's structs are byte-compatible.
long ref_layout(int which) {
    switch (which) {
        case 0: return sizeof(Float3);
        case 1: return sizeof(Solvent);
        case 2: return sizeof(CompoundState);
        case 3: return sizeof(Compound);
        case 4: return sizeof(NeighborList);
        case 5: return sizeof(LJ_Ignores);
        case 6: return sizeof(PairBond);
        case 7: return sizeof(AngleBond);
        case 8: return sizeof(DihedralBond);
        case 9: return sizeof(CompoundBridgeCompact);
        case 10: return sizeof(ForceField);
        case 11: return sizeof(ParticleRefCompact);
        case 20: return offsetof(Compound, prev_positions);
        case 21: return offsetof(Compound, forces);
        case 22: return offsetof(Compound, atom_types);
        case 23: return offsetof(Compound, atom_color_types);
        case 24: return offsetof(Compound, lj_ignore_list);
        case 25: return offsetof(Compound, particle_global_ids);
        case 26: return offsetof(Compound, center_of_mass);
        case 27: return offsetof(Compound, n_singlebonds);
        case 28: return offsetof(Compound, singlebonds);
        case 29: return offsetof(Compound, n_anglebonds);
        case 30: return offsetof(Compound, anglebonds);
        case 31: return offsetof(Compound, n_dihedrals);
        case 32: return offsetof(Compound, dihedrals);
        case 33: return offsetof(Compound, key_particle_index);
        case 34: return offsetof(Compound, confining_particle_sphere);
        case 40: return offsetof(CompoundBridgeCompact, particle_refs);
        case 41: return offsetof(CompoundBridgeCompact, atom_types);
        case 42: return offsetof(CompoundBridgeCompact, n_particles);
        case 43: return offsetof(CompoundBridgeCompact, n_singlebonds);
        case 44: return offsetof(CompoundBridgeCompact, singlebonds);
        case 45: return offsetof(CompoundBridgeCompact, n_anglebonds);
        case 46: return offsetof(CompoundBridgeCompact, anglebonds);
        case 47: return offsetof(CompoundBridgeCompact, n_dihedrals);
        case 48: return offsetof(CompoundBridgeCompact, dihedrals);
        case 50: return offsetof(DihedralBond, n);
        case 51: return offsetof(DihedralBond, atom_indexes);
        case 60: return NEIGHBORLIST_MAX_COMPOUNDS;
        case 61: return NEIGHBORLIST_MAX_SOLVENTS;
        case 62: return MAX_SOLVENTS;
        case 63: return MAX_COMPOUNDS;
        case 64: return MAX_COMPOUND_PARTICLES;
        case 65: return COMPOUNDBRIDGES_IN_BUNDLE;
        default: return -1;
    }
}

void* ref_create(float box_len, float cutoff, double dt, int n_threads) {
    BOX_LEN = box_len;
    BOX_LEN_HALF = box_len / 2.f;
    CUTOFF = cutoff;
    auto* c = new RefCtx();
    c->n_threads = n_threads > 0 ? n_threads : 1;
    g_n_threads = c->n_threads;
    c->sim.reset(new Simulation());
    c->sim->box->dt = dt;
    return c;
}

void ref_destroy(void* h) { delete static_cast<RefCtx*>(h); }

const char* ref_last_error(void* h) { return static_cast<RefCtx*>(h)->err.c_str(); }

int ref_set_threads(void* h, int n) {
    auto* c = static_cast<RefCtx*>(h);
    c->n_threads = n > 0 ? n : 1;
    g_n_threads = c->n_threads;
    return 0;
}

// Loads a box in the reference layout.  Mirrors BoxBuilder::finishBox
// (BoxBuilder.cu:73-145) for the parts the step path reads.
int ref_load(void* h, const void* forcefield, int n_c, const void* compounds, const void* states, int n_s,
             const void* solvents, int n_b, const void* bridges) {
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&]() -> int {
        if (n_c < 0 || n_c > MAX_COMPOUNDS || n_s < 0 || n_s > MAX_SOLVENTS || n_b < 0 ||
            n_b > COMPOUNDBRIDGES_IN_BUNDLE) {
            c->err = "size outside the reference layout";
            return -1;
        }
        Simulation* sim = c->sim.get();
        Box* box = sim->box;
        std::memcpy(&forcefield_device, forcefield, sizeof(ForceField));
        c->engine.reset(new Engine());
        c->engine->forcefield_host = forcefield_device;
        c->engine->simulation = sim;

        box->n_compounds = n_c;
        box->n_solvents = static_cast<uint16_t>(n_s);
        box->compounds = c->alloc<Compound>(n_c);
        if (n_c) std::memcpy(box->compounds, compounds, sizeof(Compound) * n_c);
        box->compound_state_array = c->alloc<CompoundState>(MAX_COMPOUNDS);
        box->compound_state_array_next = c->alloc<CompoundState>(MAX_COMPOUNDS);
        if (n_c) std::memcpy(box->compound_state_array, states, sizeof(CompoundState) * n_c);
        std::memcpy(box->compound_state_array_next, box->compound_state_array, sizeof(CompoundState) * MAX_COMPOUNDS);
        box->compound_neighborlists = c->alloc<NeighborList>(MAX_COMPOUNDS);
        box->solvent_neighborlists = c->alloc<NeighborList>(n_s + 1);
        box->solvents = c->alloc<Solvent>(n_s + 1);
        box->solvents_next = c->alloc<Solvent>(n_s + 1);
        if (n_s) std::memcpy(box->solvents, solvents, sizeof(Solvent) * n_s);
        std::memcpy(box->solvents_next, box->solvents, sizeof(Solvent) * n_s);
        box->bridge_bundle = c->alloc<CompoundBridgeBundleCompact>(1);
        box->bridge_bundle->n_bridges = n_b;
        if (n_b) std::memcpy(box->bridge_bundle->compound_bridges, bridges, sizeof(CompoundBridgeCompact) * n_b);
        box->step = 0;
        box->critical_error_encountered = false;
        box->thermostat_scalar = 1.f;

        sim->n_compounds = n_c;
        sim->n_bridges = n_b;
        sim->n_solvents = n_s;
        sim->blocks_per_solventkernel = static_cast<int>(std::ceil(static_cast<float>(n_s) / THREADS_PER_SOLVENTBLOCK));
        sim->compounds_host = new Compound[n_c > 0 ? n_c : 1];
        for (int i = 0; i < n_c; i++) sim->compounds_host[i] = box->compounds[i];
        sim->total_particles_upperbound = n_c * MAX_COMPOUND_PARTICLES + n_s;
        box->total_particles_upperbound = sim->total_particles_upperbound;
        uint32_t tpu = sim->total_particles_upperbound;
        box->potE_buffer = c->alloc<double>(static_cast<size_t>(tpu) * STEPS_PER_LOGTRANSFER);
        box->traj_buffer = c->alloc<Float3>(static_cast<size_t>(tpu) * STEPS_PER_LOGTRANSFER);
        box->outdata = c->alloc<float>(10 * STEPS_PER_LOGTRANSFER);
        box->data_GAN = c->alloc<Float3>(static_cast<size_t>(N_DATAGAN_VALUES) * MAX_COMPOUND_PARTICLES *
                                         (n_c > 0 ? n_c : 1) * STEPS_PER_TRAINDATATRANSFER);

        // NListDataCollection(Simulation*) (Engine.cuh:63-72), built in place so
        // that its fixed-size arrays live on the heap.
        void* raw = ::operator new(sizeof(NListDataCollection));
        std::memset(raw, 0, sizeof(NListDataCollection));
        auto* nl = static_cast<NListDataCollection*>(raw);
        nl->n_compounds = n_c;
        nl->n_solvents = n_s;
        nl->compoundstates = new CompoundState[n_c > 0 ? n_c : 1];
        nl->solvents = new Solvent[n_s > 0 ? n_s : 1];
        nl->compound_neighborlists = new NeighborList[MAX_COMPOUNDS];
        nl->solvent_neighborlists = new NeighborList[n_s > 0 ? n_s : 1];
        c->nldc = nl;
        c->engine->nlist_data_collection = nl;

        c->forces_c.assign(static_cast<size_t>(n_c) * MAX_COMPOUND_PARTICLES, Float3(0.f));
        c->forces_s.assign(static_cast<size_t>(n_s), Float3(0.f));
        return 0;
    });
}

// One synchronous neighbour-list update exactly as Engine::handleNLISTS does it
// with async=false (Engine.cu:92-111): offload positions, cull + add on the
// host (updateNeighborLists), push the lists to the box.
int ref_update_nlists(void* h) {
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&]() -> int {
        Engine* e = c->engine.get();
        Simulation* sim = c->sim.get();
        e->offloadPositionDataNLIST(sim);
        int timing = 0;
        Engine::updateNeighborLists(sim, c->nldc, &e->updated_neighborlists_ready, &timing);
        if (e->updated_neighborlists_ready) e->pushNlistsToDevice();
        return 0;
    });
}

// CSR export of the box's lists.  which: 0 compound->compound,
// 1 compound->solvent, 2 solvent->compound, 3 solvent->solvent.  Call with
// ids == NULL to get offsets (n_entities + 1 ints); ids in list order.
int ref_get_nlist_csr(void* h, int which, int* offsets, int* ids) {
    auto* c = static_cast<RefCtx*>(h);
    Box* box = c->sim->box;
    const bool comp = which < 2;
    const int n = comp ? static_cast<int>(box->n_compounds) : static_cast<int>(box->n_solvents);
    const NeighborList* lists = comp ? box->compound_neighborlists : box->solvent_neighborlists;
    int pos = 0;
    for (int i = 0; i < n; i++) {
        const NeighborList& L = lists[i];
        const bool want_comp = (which == 0 || which == 2);
        const int cnt = want_comp ? L.n_compound_neighbors : L.n_solvent_neighbors;
        const uint16_t* src = want_comp ? L.neighborcompound_ids : L.neighborsolvent_ids;
        if (offsets) offsets[i] = pos;
        if (ids)
            for (int k = 0; k < cnt; k++) ids[pos + k] = src[k];
        pos += cnt;
    }
    if (offsets) offsets[n] = pos;
    return pos;
}

// Replaces the box's lists (and the host collection's copies) by CSR input,
// preserving the given order; used to hand a previous list state to the
// reference's incremental update.
int ref_set_nlist_csr(void* h, int which, const int* offsets, const int* ids) {
    auto* c = static_cast<RefCtx*>(h);
    Box* box = c->sim->box;
    const bool comp = which < 2;
    const int n = comp ? static_cast<int>(box->n_compounds) : static_cast<int>(box->n_solvents);
    NeighborList* lists = comp ? box->compound_neighborlists : box->solvent_neighborlists;
    NeighborList* host = comp ? c->nldc->compound_neighborlists : c->nldc->solvent_neighborlists;
    const bool want_comp = (which == 0 || which == 2);
    const int cap = want_comp ? NEIGHBORLIST_MAX_COMPOUNDS : NEIGHBORLIST_MAX_SOLVENTS;
    for (int i = 0; i < n; i++) {
        const int cnt = offsets[i + 1] - offsets[i];
        if (cnt > cap) {
            c->err = "list longer than the reference capacity";
            return -1;
        }
        for (NeighborList* L : {&lists[i], &host[i]}) {
            if (want_comp) {
                L->n_compound_neighbors = static_cast<uint16_t>(cnt);
                for (int k = 0; k < cnt; k++) L->neighborcompound_ids[k] = static_cast<uint16_t>(ids[offsets[i] + k]);
            } else {
                L->n_solvent_neighbors = static_cast<uint16_t>(cnt);
                for (int k = 0; k < cnt; k++) L->neighborsolvent_ids[k] = static_cast<uint16_t>(ids[offsets[i] + k]);
            }
        }
    }
    return 0;
}

// n_steps of Engine::step with a fixed thermostat scalar and no list update.
int ref_step(void* h, int n_steps, float thermostat_scalar) {
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&]() -> int {
        g_forces_c = &c->forces_c;
        g_forces_s = &c->forces_s;
        g_n_threads = c->n_threads;
        for (int s = 0; s < n_steps; s++) {
            c->sim->box->thermostat_scalar = thermostat_scalar;
            c->engine->step();
            if (g_exit_called) break;
        }
        g_forces_c = nullptr;
        g_forces_s = nullptr;
        return c->sim->box->critical_error_encountered ? 1 : 0;
    });
}

int ref_get_state(void* h, void* compounds_out, void* states_out, void* solvents_out) {
    auto* c = static_cast<RefCtx*>(h);
    Box* box = c->sim->box;
    if (compounds_out) std::memcpy(compounds_out, box->compounds, sizeof(Compound) * box->n_compounds);
    if (states_out) std::memcpy(states_out, box->compound_state_array, sizeof(CompoundState) * box->n_compounds);
    if (solvents_out) std::memcpy(solvents_out, box->solvents, sizeof(Solvent) * box->n_solvents);
    return 0;
}

int ref_get_forces(void* h, float* fc, float* fs) {
    auto* c = static_cast<RefCtx*>(h);
    if (fc) std::memcpy(fc, c->forces_c.data(), sizeof(Float3) * c->forces_c.size());
    if (fs) std::memcpy(fs, c->forces_s.data(), sizeof(Float3) * c->forces_s.size());
    return 0;
}

// Per-particle potE the kernels logged for the most recent step
// (potE_buffer slot (step-1) % STEPS_PER_LOGTRANSFER, Engine.cu:1012,1141,1218).
int ref_get_potE(void* h, double* out) {
    auto* c = static_cast<RefCtx*>(h);
    Box* box = c->sim->box;
    if (box->step == 0) return -1;
    const uint32_t tpu = box->total_particles_upperbound;
    const size_t off = static_cast<size_t>((box->step - 1) % STEPS_PER_LOGTRANSFER) * tpu;
    std::memcpy(out, box->potE_buffer + off, sizeof(double) * tpu);
    return 0;
}

// The reference's logging buffers of the most recent step: traj_buffer and
// potE_buffer slot (step-1) % STEPS_PER_LOGTRANSFER (total_particles_upperbound
// entries), outdata (10 floats) and data_GAN slot (step-1) %
// STEPS_PER_TRAINDATATRANSFER (N_DATAGAN_VALUES Float3 per compound particle
// slot); Engine.cu:1007-1040, 1136-1145.  Any output may be NULL.
int ref_get_log(void* h, double* potE, float* traj, float* outdata, float* gan) {
    auto* c = static_cast<RefCtx*>(h);
    Box* box = c->sim->box;
    if (box->step == 0) return -1;
    const uint32_t tpu = box->total_particles_upperbound;
    const size_t s_log = static_cast<size_t>((box->step - 1) % STEPS_PER_LOGTRANSFER);
    const size_t s_gan = static_cast<size_t>((box->step - 1) % STEPS_PER_TRAINDATATRANSFER);
    if (potE) std::memcpy(potE, box->potE_buffer + s_log * tpu, sizeof(double) * tpu);
    if (traj) std::memcpy(traj, box->traj_buffer + s_log * tpu, sizeof(Float3) * tpu);
    if (outdata) std::memcpy(outdata, box->outdata + s_log * 10, sizeof(float) * 10);
    const size_t ng = static_cast<size_t>(N_DATAGAN_VALUES) * MAX_COMPOUND_PARTICLES * box->n_compounds;
    if (gan) std::memcpy(gan, box->data_GAN + s_gan * ng, sizeof(Float3) * ng);
    return 0;
}

int ref_get_step(void* h) { return static_cast<int>(static_cast<RefCtx*>(h)->sim->box->step); }

// The reference's RenderBall list of the current box, as Rasterizer::render
// (Rasterizer.cu:12-27) makes it: loadCompoundatomsKernel over n_compounds
// blocks of MAX_COMPOUND_PARTICLES threads, loadSolventatomsKernel over
// ceil(n_solvents / 100) blocks of 100, processAtomsKernel over
// ceil(upper / 64) blocks of 64 (upper = total_particles_upperbound,
// BoxBuilder.cu:78), then mergeSortAPI over the first `upper` balls.  The
// kernels have no barriers or shared memory, so their threads run one after
// another.  The atom buffer is zero-filled where the reference leaves device
// memory unset (positions of the empty compound slots, the padding up to a
// whole block); its last block reads and writes past `upper`, so both
// buffers are a whole number of blocks long.  `out` receives `upper` balls.
int ref_render(void* h, void* out) {
    auto* c = static_cast<RefCtx*>(h);
    Simulation* sim = c->sim.get();
    Box* box = sim->box;
    const int nc = box->n_compounds, ns = box->n_solvents;
    const int upper = nc * MAX_COMPOUND_PARTICLES + ns;
    if (upper <= 0) return -1;
    const int blocks = (int)ceil((float)upper / (float)RAS_THREADS_PER_BLOCK);
    const size_t cap = (size_t)blocks * RAS_THREADS_PER_BLOCK;
    RenderAtom* atoms = static_cast<RenderAtom*>(std::calloc(cap, sizeof(RenderAtom)));
    RenderBall* balls = static_cast<RenderBall*>(std::calloc(cap, sizeof(RenderBall)));
    if (!atoms || !balls) {
        std::free(atoms);
        std::free(balls);
        return -1;
    }
    auto run = [](unsigned grid, unsigned block, auto&& body) {
        blockDim = dim3(block, 1, 1);
        gridDim = dim3(grid, 1, 1);
        for (unsigned b = 0; b < grid; b++)
            for (unsigned t = 0; t < block; t++) {
                blockIdx = {b, 0, 0};
                threadIdx = {t, 0, 0};
                body();
            }
    };
    if (nc > 0) run(nc, MAX_COMPOUND_PARTICLES, [&] { loadCompoundatomsKernel(box, atoms); });
    if (ns > 0) {
        const int sb = (int)ceil((float)ns / (float)THREADS_PER_LOADSOLVENTSATOMSKERNEL);
        const int off = nc * MAX_COMPOUND_PARTICLES;
        run(sb, THREADS_PER_LOADSOLVENTSATOMSKERNEL, [&] { loadSolventatomsKernel(box, atoms, off); });
    }
    run(blocks, RAS_THREADS_PER_BLOCK, [&] { processAtomsKernel(atoms, balls); });
    mergeSortAPI(balls, upper);
    std::memcpy(out, balls, sizeof(RenderBall) * (size_t)upper);
    std::free(atoms);
    std::free(balls);
    return 0;
}

}  // extern "C"
