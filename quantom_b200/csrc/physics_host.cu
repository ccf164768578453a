// Host side of the physics-semantics path: set-up from the reference layout,
// list rebuilds, step launches and readback (kernels in kernels_physics.cu).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#include "physdev.cuh"
#include "physkern.cuh"
#include "refdev.cuh"

namespace lima {
namespace {

inline float host_int_as_float(int v) {
    float f;
    std::memcpy(&f, &v, sizeof(f));
    return f;
}

// One device allocation carved into 256-byte aligned pieces: a pass with
// base 0 sums the sizes, a second pass over the allocation hands out pointers.
struct Arena {
    uintptr_t base = 0;
    size_t off = 0;
    template <typename T>
    T* take(size_t n) {
        off = (off + 255) & ~static_cast<size_t>(255);
        T* p = reinterpret_cast<T*>(base + off);
        off += std::max<size_t>(n, 1) * sizeof(T);
        return p;
    }
};

}  // namespace

void* pool_alloc(size_t bytes, cudaStream_t s) {
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(mu);
        if ((int)pools.size() <= dev) pools.resize(dev + 1, nullptr);
        if (!pools[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            if (cudaMemPoolCreate(&pools[dev], &props) != cudaSuccess) {
                cudaGetLastError();
                pools[dev] = nullptr;
                return nullptr;
            }
            uint64_t keep = UINT64_MAX;   // freed blocks stay with the pool
            cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        }
        pool = pools[dev];
    }
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, std::max<size_t>(bytes, 1), pool, s) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void pool_free(void* p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

namespace {
struct PinnedCache {
    std::mutex mu;
    std::multimap<size_t, void*> idle;       // freed blocks by size
    std::unordered_map<void*, size_t> size;  // every block handed out
};
PinnedCache& pinned_cache() {
    static PinnedCache* c = new PinnedCache();   // lives to process exit (blocks are reused, not returned)
    return *c;
}
}  // namespace

void* pinned_alloc(size_t bytes) {
    bytes = std::max<size_t>(bytes, 1);
    PinnedCache& c = pinned_cache();
    {
        std::lock_guard<std::mutex> lock(c.mu);
        auto it = c.idle.lower_bound(bytes);
        if (it != c.idle.end() && it->first <= 2 * bytes) {   // reuse a block of at most twice the size
            void* p = it->second;
            c.idle.erase(it);
            return p;
        }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(c.mu);
    c.size[p] = bytes;
    return p;
}

void pinned_free(void* p) {
    if (!p) return;
    PinnedCache& c = pinned_cache();
    std::lock_guard<std::mutex> lock(c.mu);
    auto it = c.size.find(p);
    if (it != c.size.end()) c.idle.emplace(it->second, p);
}

namespace {

template <typename T>
T* dalloc(std::vector<void*>& allocs, size_t n, cudaStream_t s) {
    void* p = pool_alloc(std::max<size_t>(n, 1) * sizeof(T), s);
    if (!p) throw std::runtime_error("device allocation failed");
    allocs.push_back(p);
    return static_cast<T*>(p);
}

}  // namespace

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
    d.dynamic_list = p.nlist_period <= 0 ? 1 : 0;
    d.use_switch = p.switch_on < p.cutoff ? 1 : 0;
    const float ron = d.use_switch ? p.switch_on : p.cutoff;
    d.ron2 = ron * ron;
    d.inv_sw_d = d.use_switch ? 1.f / (d.rc2 - d.ron2) : 0.f;
    d.sw_c0 = d.rc2 * d.inv_sw_d;
    d.sw_k10 = 10.f * d.inv_sw_d;
    d.inv_rc2 = 1.f / d.rc2;
    d.dt = p.dt;
    d.precision = p.precision;
    d.thermostat = p.thermostat;
    d.t_target = p.t_target;
    d.tau_t = p.tau_t;

    // types and the Lorentz-Berthelot table (sigma^2, 4 eps)
    int max_type = 0;
    for (int c = 0; c < h.n_c; c++)
        for (int t = 0; t < h.comps[c].n_particles; t++) max_type = std::max<int>(max_type, h.comps[c].atom_types[t]);
    d.n_types = max_type + 1;
    for (int t = 0; t < d.n_types; t++) {
        const auto& pp = h.ff->particle_parameters[t];
        const bool used = t == LIMA_ATOMTYPE_SOL ? h.n_s > 0 : true;
        if (used && (!(pp.mass > 0.f) || !(pp.sigma > 0.f) || !(pp.epsilon >= 0.f))) {
            msg = "force-field entry of a used type has non-positive mass/sigma or negative epsilon";
            return LIMA_ERR_ARGUMENT;
        }
    }
    std::vector<float2> tab(d.n_types * d.n_types);
    for (int a = 0; a < d.n_types; a++)
        for (int b = 0; b < d.n_types; b++) {
            const auto& A = h.ff->particle_parameters[a];
            const auto& B = h.ff->particle_parameters[b];
            const double sg = 0.5 * ((double)A.sigma + (double)B.sigma);
            const double ep = std::sqrt(std::max(0.0, (double)A.epsilon * (double)B.epsilon));
            tab[a * d.n_types + b] = make_float2((float)(sg * sg), (float)(4.0 * ep));
        }
    // exclusions (LJ_Ignores -> orig ids; solvents have none)
    std::vector<std::vector<uint32_t>> excl(d.n_cp);
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
        eoff[i + 1] = eoff[i] + (i < d.n_cp ? (uint32_t)excl[i].size() : 0u);
        if (i < d.n_cp) eids.insert(eids.end(), excl[i].begin(), excl[i].end());
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
            didx.push_back(make_int4(o + t.atom_indexes[0], o + t.atom_indexes[1], o + t.atom_indexes[2],
                                     o + t.atom_indexes[3]));
            dpar.push_back(make_float4(t.phi_0, t.k_phi, (float)t.n, 0.f));
        }
    }
    for (int b = 0; b < h.n_b; b++) {
        const lima_compound_bridge_compact& br = h.bridges[b];
        auto gid = [&](uint32_t local) {
            const auto& r = br.particle_refs[local];
            return base[r.compound_id] + r.local_id_compound;
        };
        for (int q = 0; q < br.n_singlebonds; q++) {
            const auto& t = br.singlebonds[q];
            bidx.push_back(make_int4(gid(t.atom_indexes[0]), gid(t.atom_indexes[1]), 0, 0));
            bpar.push_back(make_float2(t.b0, t.kb));
        }
        for (int q = 0; q < br.n_anglebonds; q++) {
            const auto& t = br.anglebonds[q];
            aidx.push_back(make_int4(gid(t.atom_indexes[0]), gid(t.atom_indexes[1]), gid(t.atom_indexes[2]), 0));
            apar.push_back(make_float2(t.theta_0, t.k_theta));
        }
        for (int q = 0; q < br.n_dihedrals; q++) {
            const auto& t = br.dihedrals[q];
            didx.push_back(make_int4(gid(t.atom_indexes[0]), gid(t.atom_indexes[1]), gid(t.atom_indexes[2]),
                                     gid(t.atom_indexes[3])));
            dpar.push_back(make_float4(t.phi_0, t.k_phi, (float)t.n, 0.f));
        }
    }
    d.n_bonds = (int)bidx.size();
    d.n_angles = (int)aidx.size();
    d.n_dih = (int)didx.size();
    d.n_term_slots = 2 * d.n_bonds + 3 * d.n_angles + 4 * d.n_dih;
    std::vector<std::vector<uint32_t>> slots(std::max(d.n_cp, 1));
    for (int b = 0; b < d.n_bonds; b++) {
        slots[bidx[b].x].push_back(2 * b);
        slots[bidx[b].y].push_back(2 * b + 1);
    }
    for (int a = 0; a < d.n_angles; a++) {
        const int b0 = 2 * d.n_bonds + 3 * a;
        slots[aidx[a].x].push_back(b0);
        slots[aidx[a].y].push_back(b0 + 1);
        slots[aidx[a].z].push_back(b0 + 2);
    }
    for (int q = 0; q < d.n_dih; q++) {
        const int b0 = 2 * d.n_bonds + 3 * d.n_angles + 4 * q;
        slots[didx[q].x].push_back(b0);
        slots[didx[q].y].push_back(b0 + 1);
        slots[didx[q].z].push_back(b0 + 2);
        slots[didx[q].w].push_back(b0 + 3);
    }
    std::vector<uint32_t> boff(d.n_cp + 1, 0), bslot;
    for (int i = 0; i < d.n_cp; i++) {
        boff[i + 1] = boff[i] + (uint32_t)slots[i].size();
        bslot.insert(bslot.end(), slots[i].begin(), slots[i].end());
    }

    // cell grid (side >= rlist/2: the 5x5x5 neighbourhood covers rlist) and
    // Verlet-list capacity
    const float half = 0.5f * d.rlist;
    d.m = std::max(1, (int)std::floor(d.L / half));
    while (d.m > 1 && d.L / d.m < half) d.m--;
    d.n_cells = d.m * d.m * d.m;
    const double rho = d.n / ((double)d.L * d.L * d.L);
    const double expect = 4.0 / 3.0 * M_PI * (double)d.rlist * d.rlist * d.rlist * rho;
    d.nl_cap = std::min(nl_round_cap(d.n), nl_round_cap((int)(1.6 * expect + 96)));
    d.nl_cap = std::max(d.nl_cap, kListChunk);
    d.nl16 = list_ids_16bit(d.n_pad) ? 1 : 0;

    // every fixed-size buffer in one allocation; the list separately (it may grow)
    // the topology arrays first and together: the host builds their image
    // with the same offsets and uploads it in one copy
    auto carve_topology = [&](Arena& a) {
        d.cp_base = a.take<uint32_t>((size_t)h.n_c + 1);
        d.lj_table = a.take<float2>(tab.size());
        d.excl_off = a.take<uint32_t>(eoff.size());
        d.excl_ids = a.take<uint32_t>(eids.size());
        d.bond_idx = a.take<int4>(bidx.size());
        d.bond_par = a.take<float2>(bpar.size());
        d.angle_idx = a.take<int4>(aidx.size());
        d.angle_par = a.take<float2>(apar.size());
        d.dih_idx = a.take<int4>(didx.size());
        d.dih_par = a.take<float4>(dpar.size());
        d.bterm_off = a.take<uint32_t>(boff.size());
        d.bterm_slot = a.take<uint32_t>(bslot.size());
    };
    size_t topo_bytes = 0;
    auto carve = [&](Arena& a) {
        carve_topology(a);
        topo_bytes = a.off;
        for (int b = 0; b < 2; b++) d.pos[b] = a.take<float4>(d.n_pad);
        d.vel = a.take<float4>(d.n_pad);
        d.posc = a.take<float4>(d.n_pad);
        d.velc = a.take<float4>(d.n_pad);
        d.xref = a.take<float4>(d.n_pad);
        d.force = a.take<float4>(d.n_pad);
        for (int b = 0; b < 2; b++) d.pos_orig[b] = a.take<float4>(std::max(1, d.n_cp));
        for (int b = 0; b < 2; b++) d.posc_orig[b] = a.take<float4>(std::max(1, d.n_cp));
        d.orig_of_sorted = a.take<uint32_t>(d.n_pad);
        d.sorted_of_orig = a.take<uint32_t>(d.n);
        d.cell_key = a.take<uint32_t>(d.n);
        d.cell_rank = a.take<uint32_t>(d.n);
        d.ccount = a.take<uint32_t>(d.n_cells);
        d.order = a.take<uint32_t>(d.n);
        d.cstart = a.take<uint32_t>((size_t)d.n_cells + 1);
        for (int b = 0; b < 2; b++) d.pos_tmp[b] = a.take<float4>(d.n);
        d.vel_tmp = a.take<float4>(d.n);
        d.posc_tmp = a.take<float4>(d.n);
        d.velc_tmp = a.take<float4>(d.n);
        d.force_tmp = a.take<float4>(d.n);
        d.orig_tmp = a.take<uint32_t>(d.n);
        d.nl_cnt = a.take<uint32_t>(d.n_pad);
        d.nl_need = a.take<int>(1);
        d.term_force = a.take<float4>(d.n_term_slots);
        d.part = a.take<double>((size_t)step_blocks(d) * kRedStride);
        d.bpart = a.take<double>((size_t)bonded_blocks(d) * 4);
        d.done = a.take<unsigned int>(1);
        d.e_last = a.take<double>(LIMA_E_COUNT);
        d.lambda = a.take<float>(2);
        d.err = a.take<int>(1);
        d.need_rebuild = a.take<int>(1);
        d.rebuild_count = a.take<unsigned long long>(1);
    };
    try {
        Arena plan;
        carve(plan);
        Arena real;
        real.base = reinterpret_cast<uintptr_t>(dalloc<uint8_t>(allocs, plan.off, s));
        carve(real);
        d.nl = reinterpret_cast<uint32_t*>(dalloc<uint8_t>(allocs, (size_t)d.nl_cap * d.n_pad * nl_entry_bytes(d), s));
    } catch (const std::exception& e) {
        msg = std::string("device allocation failed: ") + e.what();
        return LIMA_ERR_CUDA;
    }
    // the topology image: each array at the offset its device copy has
    {
        std::vector<uint8_t> img(topo_bytes, 0);
        const uintptr_t dev0 = reinterpret_cast<uintptr_t>(d.cp_base);
        auto put = [&](const void* dst, const void* src, size_t bytes) {
            if (bytes) std::memcpy(img.data() + (reinterpret_cast<uintptr_t>(dst) - dev0), src, bytes);
        };
        std::vector<uint32_t> cbase(base.begin(), base.end());
        put(d.cp_base, cbase.data(), sizeof(uint32_t) * cbase.size());
        put(d.lj_table, tab.data(), sizeof(float2) * tab.size());
        put(d.excl_off, eoff.data(), sizeof(uint32_t) * eoff.size());
        put(d.excl_ids, eids.data(), sizeof(uint32_t) * eids.size());
        put(d.bond_idx, bidx.data(), sizeof(int4) * bidx.size());
        put(d.bond_par, bpar.data(), sizeof(float2) * bpar.size());
        put(d.angle_idx, aidx.data(), sizeof(int4) * aidx.size());
        put(d.angle_par, apar.data(), sizeof(float2) * apar.size());
        put(d.dih_idx, didx.data(), sizeof(int4) * didx.size());
        put(d.dih_par, dpar.data(), sizeof(float4) * dpar.size());
        put(d.bterm_off, boff.data(), sizeof(uint32_t) * boff.size());
        put(d.bterm_slot, bslot.data(), sizeof(uint32_t) * bslot.size());
        cudaMemcpyAsync(d.cp_base, img.data(), topo_bytes, cudaMemcpyHostToDevice, s);   // pageable: copied at the call
    }
    cudaMemsetAsync(d.ccount, 0, sizeof(uint32_t) * d.n_cells, s);
    cudaMemsetAsync(d.done, 0, sizeof(unsigned int), s);
    cudaMemsetAsync(d.e_last, 0, sizeof(double) * LIMA_E_COUNT, s);
    cudaMemsetAsync(d.err, 0, sizeof(int), s);
    cudaMemsetAsync(d.need_rebuild, 0, sizeof(int), s);
    cudaMemsetAsync(d.rebuild_count, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(d.nl_cnt, 0, sizeof(uint32_t) * d.n_pad, s);
    cudaMemsetAsync(d.nl_need, 0, sizeof(int), s);
    cudaMemsetAsync(d.force, 0, sizeof(float4) * d.n_pad, s);
    phys_upload_state(h, d, 0, s);
    return cudaGetLastError() == cudaSuccess ? 0 : LIMA_ERR_CUDA;
}

// Host state (reference layout) -> device, in orig order (the next rebuild
// sorts).  Half-step velocities from the Stormer pair: v = (x - x_prev)/dt.
// Positions are wrapped into [0, L) in double and rounded to FP32; mixed
// precision keeps what the rounding dropped (of the position and of the
// velocity) in the low words, so its state starts at the input itself.
void phys_upload_state(const PhysHost& h, PhysDev& d, int cur, cudaStream_t s) {
    // staged in one pinned block (pageable sources would each take a driver
    // staging pass); plain host memory when no pinned block can be had
    const size_t np = (size_t)d.n_pad;
    const size_t bytes = np * (4 * sizeof(float4) + sizeof(uint32_t));
    void* block = pinned_alloc(bytes);
    std::vector<uint8_t> fallback;
    if (!block) {
        fallback.resize(bytes);
        block = fallback.data();
    }
    float4* pos = static_cast<float4*>(block);
    float4* vel = pos + np;
    float4* posc = vel + np;
    float4* velc = posc + np;
    uint32_t* ident = reinterpret_cast<uint32_t*>(velc + np);
    const float L = d.L;
    const bool mixed = d.precision == LIMA_PRECISION_MIXED;
    // the coordinate in [0, L) as FP32 plus its rounding residual (hi + lo = x mod L)
    auto wrap = [&](double x, float& lo) {
        if (!(x >= 0.0 && x < (double)L)) {   // most inputs are inside the box already
            x = std::fmod(x, (double)L);
            if (x < 0) x += L;
        }
        float f = (float)x;
        if (f >= L) {   // rounded up onto the face: the image at 0
            f = 0.f;
            x -= L;
        }
        lo = mixed ? (float)(x - (double)f) : 0.f;
        return f;
    };
    auto split = [&](double v, float& lo) {
        const float f = (float)v;
        lo = mixed ? (float)(v - (double)f) : 0.f;
        return f;
    };
    auto mimg = [&](double dd) { return std::fabs(dd) <= 0.5 * L ? dd : dd - L * std::nearbyint(dd / L); };
    auto put = [&](int k, const lima_float3& x, const lima_float3& xp, int type, float im) {
        float lx, ly, lz, ux, uy, uz;
        const float px = wrap(x.x, lx), py = wrap(x.y, ly), pz = wrap(x.z, lz);
        pos[k] = make_float4(px, py, pz, host_int_as_float(type));
        posc[k] = make_float4(lx, ly, lz, 0.f);
        const float vx = split(mimg((double)x.x - xp.x) / d.dt, ux), vy = split(mimg((double)x.y - xp.y) / d.dt, uy),
                    vz = split(mimg((double)x.z - xp.z) / d.dt, uz);
        vel[k] = make_float4(vx, vy, vz, im);
        velc[k] = make_float4(ux, uy, uz, 0.f);
    };
    int k = 0;
    for (int c = 0; c < h.n_c; c++)
        for (int t = 0; t < h.comps[c].n_particles; t++, k++) {
            const int type = h.comps[c].atom_types[t];
            put(k, h.states[c].positions[t], h.comps[c].prev_positions[t], type,
                1.f / h.ff->particle_parameters[type].mass);
        }
    const float im_sol = 1.f / h.ff->particle_parameters[LIMA_ATOMTYPE_SOL].mass;
    for (int si = 0; si < h.n_s; si++, k++) put(k, h.sols[si].pos, h.sols[si].pos_tsub1, LIMA_ATOMTYPE_SOL, im_sol);
    for (int i = d.n; i < d.n_pad; i++) {
        pos[i] = make_float4(0, 0, 0, host_int_as_float(0));
        vel[i] = posc[i] = velc[i] = make_float4(0, 0, 0, 0);
    }
    for (int i = 0; i < d.n_pad; i++) ident[i] = i < d.n ? i : 0xffffffffu;
    cudaMemcpyAsync(d.pos[cur], pos, sizeof(float4) * d.n_pad, cudaMemcpyHostToDevice, s);
    if (d.n_cp) cudaMemcpyAsync(d.pos_orig[cur], pos, sizeof(float4) * d.n_cp, cudaMemcpyHostToDevice, s);
    if (d.n_cp) cudaMemcpyAsync(d.posc_orig[cur], posc, sizeof(float4) * d.n_cp, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d.vel, vel, sizeof(float4) * d.n_pad, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d.posc, posc, sizeof(float4) * d.n_pad, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d.velc, velc, sizeof(float4) * d.n_pad, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d.orig_of_sorted, ident, sizeof(uint32_t) * d.n_pad, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d.sorted_of_orig, ident, sizeof(uint32_t) * d.n, cudaMemcpyHostToDevice, s);
    set_device_float(d.lambda, 1.f, s);
    set_device_float(d.lambda + 1, 1.f, s);
    cudaMemsetAsync(d.force, 0, sizeof(float4) * d.n_pad, s);
    cudaStreamSynchronize(s);   // the staging block is reused after this
    if (fallback.empty()) pinned_free(block);
}

void phys_rebuild(const PhysDev& d, int cur, cudaStream_t s) {
    const bool mixed = d.precision == LIMA_PRECISION_MIXED;
    launch_sort(d, d.pos[cur], s);
    launch_permute(d, cur, mixed, s);
    launch_build_list(d, d.pos_tmp[0], d.orig_tmp, nullptr, cur, mixed, s);
}

// The list of positions `pos` without moving any particle: the sort of the
// slots by cell (order), reference positions, then the build through order.
void phys_rebuild_inplace(const PhysDev& d, const float4* pos, cudaStream_t s) {
    launch_sort(d, pos, s);
    launch_set_xref(d, pos, s);
    launch_build_list(d, pos, d.orig_of_sorted, d.order, -1, false, s);
}

void phys_prime(PhysDev&, int, cudaStream_t) {}

bool phys_fit_list(PhysDev& d, cudaStream_t s, std::vector<void*>& allocs) {
    int err = 0, need = 0;
    cudaMemcpyAsync(&err, d.err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&need, d.nl_need, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    if (!(err & ERR_BIT_PHYS_LIST_OVERFLOW) || need <= d.nl_cap) return false;
    const int cap = std::min(nl_round_cap(d.n), nl_round_cap(need * 5 / 4 + 32));
    uint32_t* nl = reinterpret_cast<uint32_t*>(dalloc<uint8_t>(allocs, (size_t)cap * d.n_pad * nl_entry_bytes(d), s));   // throws like the other allocations
    for (auto it = allocs.begin(); it != allocs.end(); ++it)
        if (*it == d.nl) {
            pool_free(d.nl, s);
            allocs.erase(it);
            break;
        }
    d.nl = nl;
    d.nl_cap = cap;
    const int zero = 0;
    const int keep = err & ~ERR_BIT_PHYS_LIST_OVERFLOW;
    cudaMemcpyAsync(d.err, &keep, sizeof(int), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d.nl_need, &zero, sizeof(int), cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    return true;
}

bool phys_rebuild_pending(const PhysDev& d, cudaStream_t s) {
    int h = 0;
    cudaMemcpyAsync(&h, d.need_rebuild, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return h != 0;
}

unsigned long long phys_device_rebuilds(const PhysDev& d, cudaStream_t s) {
    unsigned long long h = 0;
    cudaMemcpyAsync(&h, d.rebuild_count, sizeof(h), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return h;
}

namespace {
// ends a capture left open by a failed step of phys_capture_dynamic
void end_open_capture(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
    }
    cudaGetLastError();
}
}  // namespace

// The rebuild of pos[parity] as a graph the step kernel launches from the
// device (instantiated for device launch and uploaded), one per parity.
int phys_capture_rebuild(PhysDev& d, cudaStream_t s, std::string& msg) {
    for (int parity = 0; parity < 2; parity++) {
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            msg = "cannot capture the list rebuild";
            cudaGetLastError();
            return LIMA_ERR_CUDA;
        }
        phys_rebuild(d, parity, s);
        if (cudaStreamEndCapture(s, &g) != cudaSuccess || !g) {
            end_open_capture(s);
            msg = "cannot capture the list rebuild";
            return LIMA_ERR_CUDA;
        }
        const cudaError_t ie = cudaGraphInstantiate(&d.rebuild_exec[parity], g, cudaGraphInstantiateFlagDeviceLaunch);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess || cudaGraphUpload(d.rebuild_exec[parity], s) != cudaSuccess) {
            cudaGetLastError();
            msg = std::string("dynamic pair lists need device-launchable CUDA graphs: ") + cudaGetErrorString(ie);
            phys_free_rebuild(d);
            return LIMA_ERR_CUDA;
        }
    }
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : LIMA_ERR_CUDA;
}

void phys_free_rebuild(PhysDev& d) {
    for (auto& g : d.rebuild_exec) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

// The step graph of a dynamic list: the bonded and step kernels (and the
// `extra` kernels), with the rebuild of the next parity as the step kernel's
// tail launch, which runs after the whole graph.
int phys_capture_dynamic(const PhysDev& d, int cur, bool energy, cudaStream_t s, cudaGraphExec_t* out,
                         int (*extra)(void*, cudaStream_t), void* extra_ctx) {
    *out = nullptr;
    if (!d.rebuild_exec[cur ^ 1]) return -1;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    int k = phys_step_kernels(d, cur, s, energy, nullptr, true);
    if (extra) k += extra(extra_ctx, s);
    if (cudaStreamEndCapture(s, &g) != cudaSuccess || !g) {
        end_open_capture(s);
        return -1;
    }
    const cudaError_t ie = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return -1;
    }
    return k;
}

// The step of parity `cur` runs the step kernel in slot cur: it integrates
// with lambda[cur] and sets lambda[cur ^ 1] from its kinetic energy.
int phys_step_kernels(const PhysDev& d, int cur, cudaStream_t s, bool energy, cudaEvent_t* ev, bool tail) {
    if (ev) cudaEventRecord(ev[0], s);
    launch_bonded(d, cur, energy, s);
    if (ev) cudaEventRecord(ev[1], s);
    launch_step(d, cur, d.precision == LIMA_PRECISION_MIXED, energy, true, cur, tail ? d.rebuild_exec[cur ^ 1] : nullptr,
                s);
    if (ev) cudaEventRecord(ev[2], s);
    return 2;
}

void phys_energy_now(PhysDev& d, int cur, cudaStream_t s) {
    launch_bonded(d, cur, true, s);
    launch_step(d, cur, d.precision == LIMA_PRECISION_MIXED, true, false, kSlotEval, nullptr, s);
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
}  // namespace

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

uint32_t phys_read_list(const PhysDev& d, uint32_t* offsets, uint32_t* ids) {
    std::vector<uint32_t> cnt(d.n), orig(d.n), nl((size_t)d.nl_cap * d.n_pad);
    cudaMemcpy(cnt.data(), d.nl_cnt, sizeof(uint32_t) * d.n, cudaMemcpyDeviceToHost);
    cudaMemcpy(orig.data(), d.orig_of_sorted, sizeof(uint32_t) * d.n, cudaMemcpyDeviceToHost);
    if (d.nl16) {
        std::vector<uint16_t> n16(nl.size());
        cudaMemcpy(n16.data(), d.nl, sizeof(uint16_t) * n16.size(), cudaMemcpyDeviceToHost);
        std::copy(n16.begin(), n16.end(), nl.begin());
    } else {
        cudaMemcpy(nl.data(), d.nl, sizeof(uint32_t) * nl.size(), cudaMemcpyDeviceToHost);
    }
    std::vector<uint32_t> by_orig(d.n);
    for (int k = 0; k < d.n; k++) by_orig[orig[k]] = (uint32_t)k;
    uint32_t pos = 0;
    for (int o = 0; o < d.n; o++) {
        const uint32_t k = by_orig[o];
        offsets[o] = pos;
        if (ids) {
            std::vector<uint32_t> row(cnt[k]);
            for (uint32_t e = 0; e < cnt[k]; e++)
                row[e] = orig[nl[nl_word((uint32_t)d.n_pad, k, e)]];
            std::sort(row.begin(), row.end());
            std::copy(row.begin(), row.end(), ids + pos);
        }
        pos += cnt[k];
    }
    offsets[d.n] = pos;
    return pos;
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
