// One step of the reference's own physics on the device (compiled with
// -fmad=false; float operation order as the reference's device functions).
//
// The reference runs three kernels per step with a device sync between each
// (Engine::step, Quantom/Quantom/Engine.cu:400-451): compoundBridgeKernel
// (:1168-1223), compoundKernel (:880-1057) and solventForceKernel
// (:1070-1161).  Its compoundKernel uses one 64-thread block per compound for
// everything — bonded terms accumulated one thread at a time behind 64
// __syncthreads per term type, intra- and inter-compound LJ and ~3,000
// compound<-solvent pairs per particle — and its solventForceKernel one
// thread per solvent, so a 36-compound, 5,000-water box keeps a few of 148
// SMs busy.  Here every float sum keeps the reference's order, and:
//   k_bridge        one 32-thread block per bridge, as the reference;
//   k_partials      the LJ sums of each compound particle split over
//                   (source, compound) blocks: 256-neighbour chunks of the
//                   compound's solvent list, its own particles, each
//                   compound-list entry;
//   k_compound      bonded terms computed one thread per term into shared
//                   memory and summed per atom in term order (the order the
//                   reference's serialised loop produces), the LJ partials
//                   added in the reference's order, Stormer-Verlet, PBC;
//   k_solvent_compounds<W>, k_solvent_list<W>
//                   the solvent's two ordered loops (all compound particles,
//                   staged 16 compounds at a time; the solvent list, read
//                   column-major), run at the same time, with W = 1..16
//                   lanes per solvent each, the image chain replayed and
//                   partial terms added in order through warp shuffles;
//   k_solvent_integrate  the two sums added in the reference's order,
//                   Stormer-Verlet, PBC.
// The solvent kernels are independent of k_partials/k_compound (both read
// the current buffers and write the next ones); all run at once.
#include "refdev.cuh"
#include "refmath.cuh"

namespace lima {
using namespace refm;

namespace {

__device__ __forceinline__ void flag_nan(const RefDev& d, const F3& p) {
    if (p.x != p.x || p.y != p.y || p.z != p.z) atomicOr(d.err, ERR_BIT_NAN);
}

// Bonded forces of one entity with per-atom sums in term-index order and
// per-thread potE over terms t, t+NT, ... (Engine.cu:744-847).
template <int NT, int MAXB, int MAXA, int MAXD>
struct BondedScratch {
    F3 rb[MAXB][2];
    F3 ra[MAXA][3];
    F3 rd[MAXD][4];
};

template <int NT, int MAXB, int MAXA, int MAXD>
__device__ void bonded_entity(const F3* pos, int nb, const lima_pair_bond* bonds, int na,
                              const lima_angle_bond* angles, int nd, const lima_dihedral_bond* dihs,
                              BondedScratch<NT, MAXB, MAXA, MAXD>& sc, F3& force, float& potE) {
    const int t = threadIdx.x;
    for (int b = t; b < nb; b += NT) {
        const lima_pair_bond& pb = bonds[b];
        pairbond(pos[pb.atom_indexes[0]], pos[pb.atom_indexes[1]], pb.b0, pb.kb, sc.rb[b], potE);
    }
    __syncthreads();
    F3 acc = mk(0.f, 0.f, 0.f);
    for (int b = 0; b < nb; b++) {
        if ((int)bonds[b].atom_indexes[0] == t) acc = add(acc, sc.rb[b][0]);
        if ((int)bonds[b].atom_indexes[1] == t) acc = add(acc, sc.rb[b][1]);
    }
    force = add(force, acc);
    for (int a = t; a < na; a += NT) {
        const lima_angle_bond& ab = angles[a];
        anglebond(pos[ab.atom_indexes[0]], pos[ab.atom_indexes[1]], pos[ab.atom_indexes[2]], ab.theta_0, ab.k_theta,
                  sc.ra[a], potE);
    }
    __syncthreads();
    acc = mk(0.f, 0.f, 0.f);
    for (int a = 0; a < na; a++)
        for (int k = 0; k < 3; k++)
            if ((int)angles[a].atom_indexes[k] == t) acc = add(acc, sc.ra[a][k]);
    force = add(force, acc);
    for (int q = t; q < nd; q += NT) {
        const lima_dihedral_bond& db = dihs[q];
        dihedral(pos[db.atom_indexes[0]], pos[db.atom_indexes[1]], pos[db.atom_indexes[2]], pos[db.atom_indexes[3]],
                 db.phi_0, db.k_phi, db.n, sc.rd[q], potE);
    }
    __syncthreads();
    acc = mk(0.f, 0.f, 0.f);
    for (int q = 0; q < nd; q++)
        for (int k = 0; k < 4; k++)
            if ((int)dihs[q].atom_indexes[k] == t) acc = add(acc, sc.rd[q][k]);
    force = add(force, acc);
}

__global__ void __launch_bounds__(32) k_bridge(RefDev d, int cur) {
    __shared__ F3 pos[LIMA_MAX_PARTICLES_IN_BRIDGE];
    __shared__ BondedScratch<32, LIMA_MAX_SINGLEBONDS_IN_BRIDGE, LIMA_MAX_ANGLEBONDS_IN_BRIDGE,
                             LIMA_MAX_DIHEDRALBONDS_IN_BRIDGE> sc;
    const lima_compound_bridge_compact& br = d.bridges[blockIdx.x];
    const int t = threadIdx.x;
    const int n = br.n_particles;
    pos[t] = mk(0.f, 0.f, 0.f);
    if (t < n) pos[t] = mk4(d.cpos[cur][br.particle_refs[t].compound_id * kMaxCP + br.particle_refs[t].local_id_compound]);
    __syncthreads();
    F3 p0 = pos[0];
    if (t > 0) hyperpos(p0, pos[t], d.L, d.Lh);
    __syncthreads();
    F3 force = mk(0.f, 0.f, 0.f);
    float potE = 0.f;
    bonded_entity<32>(pos, br.n_singlebonds, br.singlebonds, br.n_anglebonds, br.anglebonds, br.n_dihedrals,
                      br.dihedrals, sc, force, potE);
    if (t < n) d.cbridge[br.particle_refs[t].compound_id * kMaxCP + br.particle_refs[t].local_id_compound] = to4(force);
}

// The LJ sums each compound particle receives, one block per (partial sum,
// compound), blockIdx.y the compound:
//   blockIdx.x <  n_chunks      compound <- solvent over one 256-entry chunk
//                               of the compound's solvent list
//                               (computeSolventToCompoundLJForces,
//                               Engine.cu:721-730, 965-973);
//   blockIdx.x == n_chunks      intramolecular LJ
//                               (computeIntramolecularLJForces, Engine.cu:678-700);
//   blockIdx.x == n_chunks+1+k  compound <- compound-list entry k
//                               (computerIntermolecularLJForces,
//                               Engine.cu:653-676, 939-958).
// Each is one of the reference's inner-loop sums for one particle, in its
// order; k_compound adds them to the particle's force in the reference's
// order, so the force is the reference's float sum.
__global__ void __launch_bounds__(64) k_partials(RefDev d, int cur) {
    __shared__ F3 buf[kCsChunk];
    __shared__ lima_particle_parameters opar[kMaxCP];
    const int c = blockIdx.y, t = threadIdx.x;
    const lima_compound& cp = d.comps[c];
    const int n = cp.n_particles;
    const F3 p0 = mk4(d.cpos[cur][c * kMaxCP]);
    if ((int)blockIdx.x < d.n_chunks) {
        const int cnt = d.cs_cnt[c];
        const int begin = blockIdx.x * kCsChunk;
        if (begin >= cnt) return;
        const int len_ = min(kCsChunk, cnt - begin);
        for (int q = t; q < len_; q += 64) {
            F3 v = mk4(d.spos[cur][d.cs_ids[(size_t)c * d.cs_cap + begin + q]]);
            hyperpos(p0, v, d.L, d.Lh);
            buf[q] = v;
        }
        __syncthreads();
        if (t >= n) return;
        F3 pt = mk4(d.cpos[cur][c * kMaxCP + t]);
        if (t > 0) hyperpos(p0, pt, d.L, d.Lh);
        const lima_particle_parameters a = d.pp[cp.atom_types[t]];
        const lima_particle_parameters sol = d.pp[LIMA_ATOMTYPE_SOL];
        const float sg = mix_sigma(a.sigma, sol.sigma), ep = eps_geo(a.epsilon, sol.epsilon);
        F3 acc = mk(0.f, 0.f, 0.f);
        for (int q = 0; q < len_; q++) acc = add(acc, lj_force(pt, buf[q], sg, ep));
        d.cs_partial[((size_t)c * d.n_chunks + blockIdx.x) * kMaxCP + t] = to4(acc);
        return;
    }
    const int k = (int)blockIdx.x - d.n_chunks;   // 0: intramolecular, 1 + e: list entry e
    if (k > (int)d.cc_cnt[c]) return;
    const int nb = k == 0 ? c : (int)d.cc_ids[c * kMaxCP + k - 1];
    const lima_compound& ncp = d.comps[nb];
    const int nn = ncp.n_particles;
    if (t < nn) {
        F3 v = mk4(d.cpos[cur][nb * kMaxCP + t]);
        // own particles move to particle 0's image except particle 0 itself;
        // every particle of another compound does
        if (k != 0 || t > 0) hyperpos(p0, v, d.L, d.Lh);
        buf[t] = v;
        opar[t] = d.pp[ncp.atom_types[t]];
    }
    __syncthreads();
    if (t >= n) return;
    F3 pt = mk4(d.cpos[cur][c * kMaxCP + t]);
    if (t > 0) hyperpos(p0, pt, d.L, d.Lh);
    const lima_particle_parameters a = d.pp[cp.atom_types[t]];
    // which particles of compound nb this particle ignores (LJ_Ignores::ignore, Bodies.cuh:191-197)
    unsigned long long msk = 0ull;
    {
        const lima_lj_ignores& ig = cp.lj_ignore_list[t];
        for (int q = 0; q < ig.n_ignores; q++)
            if (ig.compound_ids[q] == (uint8_t)nb) msk |= 1ull << ig.local_ids[q];
    }
    F3 acc = mk(0.f, 0.f, 0.f);
    if (k == 0) {
        for (int i = 0; i < nn; i++) {
            if (i == t || ((msk >> i) & 1ull)) continue;
            const lima_particle_parameters o = opar[i];
            acc = add(acc, lj_force(pt, buf[i], mix_sigma(a.sigma, o.sigma), eps_geo(a.epsilon, o.epsilon)));
        }
    } else {
        for (int j = 0; j < nn; j++) {
            if ((msk >> j) & 1ull) continue;
            const lima_particle_parameters o = opar[j];
            acc = add(acc, lj_force(pt, buf[j], mix_sigma(a.sigma, o.sigma), eps_arith(a.epsilon, o.epsilon)));
        }
    }
    d.cc_partial[((size_t)c * (1 + kMaxCP) + k) * kMaxCP + t] = to4(acc);
}

__global__ void __launch_bounds__(64) k_compound(RefDev d, int cur) {
    __shared__ F3 pos[kMaxCP];
    __shared__ BondedScratch<64, LIMA_MAX_PAIRBONDS, LIMA_MAX_ANGLEBONDS, LIMA_MAX_DIHEDRALS> sc;
    const int c = blockIdx.x, t = threadIdx.x;
    const lima_compound& cp = d.comps[c];
    const int n = cp.n_particles;
    pos[t] = t < n ? mk4(d.cpos[cur][c * kMaxCP + t]) : mk(0.f, 0.f, 0.f);
    F3 force = mk(0.f, 0.f, 0.f);
    if (t < n) {   // Compound::loadData takes the bridge forces and zeroes them (Bodies.cuh:437-438)
        force = mk4(d.cbridge[c * kMaxCP + t]);
        d.cbridge[c * kMaxCP + t] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    const F3 p0 = pos[0];
    if (t > 0 && t < n) hyperpos(p0, pos[t], d.L, d.Lh);
    __syncthreads();
    float potE = 0.f;
    // bonded terms: one thread per term, results in shared memory
    // (calcPairbondForces / calcAnglebondForces / calcDihedralbondForces)
    for (int b = t; b < cp.n_singlebonds; b += 64) {
        const lima_pair_bond& pb = cp.singlebonds[b];
        pairbond(pos[pb.atom_indexes[0]], pos[pb.atom_indexes[1]], pb.b0, pb.kb, sc.rb[b], potE);
    }
    for (int q = t; q < cp.n_anglebonds; q += 64) {
        const lima_angle_bond& ab = cp.anglebonds[q];
        anglebond(pos[ab.atom_indexes[0]], pos[ab.atom_indexes[1]], pos[ab.atom_indexes[2]], ab.theta_0, ab.k_theta,
                  sc.ra[q], potE);
    }
    for (int q = t; q < cp.n_dihedrals; q += 64) {
        const lima_dihedral_bond& db = cp.dihedrals[q];
        dihedral(pos[db.atom_indexes[0]], pos[db.atom_indexes[1]], pos[db.atom_indexes[2]], pos[db.atom_indexes[3]],
                 db.phi_0, db.k_phi, db.n, sc.rd[q], potE);
    }
    __syncthreads();
    // per-atom sums in the reference's order: the bonds in index order, then
    // the angles, then the dihedrals (Engine.cu:765-771, 799-806, 834-842)
    {
        F3 acc = mk(0.f, 0.f, 0.f);
        int kind = 0;
        for (uint32_t q = d.bt_off[c * 65 + t]; q < d.bt_off[c * 65 + t + 1]; q++) {
            const uint32_t code = d.bt_code[q];
            const int k = (int)(code >> 14), term = (int)((code >> 2) & 0x3ff), slot = (int)(code & 3);
            while (kind < k) {
                force = add(force, acc);
                acc = mk(0.f, 0.f, 0.f);
                kind++;
            }
            const F3 r = k == 0 ? sc.rb[term][slot] : (k == 1 ? sc.ra[term][slot] : sc.rd[term][slot]);
            acc = add(acc, r);
        }
        while (kind < 3) {
            force = add(force, acc);
            acc = mk(0.f, 0.f, 0.f);
            kind++;
        }
    }
    if (t < n) {
        // LJ in the reference's order: intramolecular, each compound-list
        // entry, then the compound <- solvent chunks (k_partials)
        const float4* part = d.cc_partial + (size_t)c * (1 + kMaxCP) * kMaxCP + t;
        force = add(force, mk4(part[0]));
        const int ncc = d.cc_cnt[c];
        for (int k = 1; k <= ncc; k++) force = add(force, mk4(part[(size_t)k * kMaxCP]));
        const int nch = (d.cs_cnt[c] + kCsChunk - 1) / kCsChunk;
        F3 acc = mk(0.f, 0.f, 0.f);
        for (int k = 0; k < nch; k++) acc = add(acc, mk4(d.cs_partial[((size_t)c * d.n_chunks + k) * kMaxCP + t]));
        force = add(force, acc);
        d.force_ljsol[c * kMaxCP + t] = to4(acc);
    }
    __syncthreads();
    // integratePosition (Engine.cu:981-984)
    if (t < n) {
        F3 prev = mk4(d.cprev[c * kMaxCP + t]);
        integrate(pos[t], prev, force, (double)d.pp[cp.atom_types[t]].mass, d.dt, *d.lambda, d.L, d.Lh);
        d.cprev[c * kMaxCP + t] = to4(prev);
        d.force_c[c * kMaxCP + t] = to4(force);
        if (len(force) > 2e12f) atomicOr(d.err, ERR_BIT_CRITICAL_FORCE);
    }
    __syncthreads();
    if (t == 0) apply_pbc(pos[0], d.L);   // Engine.cu:993-996
    __syncthreads();
    if (t < n) {
        F3 p = pos[t];
        if (t > 0) hyperpos(pos[0], p, d.L, d.Lh);
        flag_nan(d, p);
        d.cpos[cur ^ 1][c * kMaxCP + t] = to4(p);
    }
    d.potE[c * kMaxCP + t] = (double)potE;   // potE_buffer write for all 64 threads (Engine.cu:1009-1013)
}

constexpr int kSolBlock = 128;
constexpr int kStageCompounds = 16;
constexpr int kStageStride = kMaxCP + 1;   // lanes on different staged compounds read different banks

__device__ __forceinline__ F3 shfl3(unsigned mask, F3 v, int src, int width) {
    return mk(__shfl_sync(mask, v.x, src, width), __shfl_sync(mask, v.y, src, width), __shfl_sync(mask, v.z, src, width));
}

// applyHyperpos on one component, telling whether it moved
__device__ __forceinline__ bool hyperpos1_moved(float s, float& m, float L, float Lh) {
    const bool a = (s - m) > Lh;
    m += L * (float)a;
    const bool b = (s - m) < -Lh;
    m -= L * (float)b;
    return a || b;
}

// One component of the image chain over a block of nv neighbours, one per
// lane: m_q = hyperpos(s_q, m_{q-1}) from m_{-1} = m.  If no lane's
// neighbour moves the component, every m_q equals the value a lane got from
// its own neighbour (mine); else the block is replayed in order.  On return
// m is the block's last value and mine this lane's.
template <int W>
__device__ __forceinline__ void replay_component(unsigned gmask, bool moved, float s, int nv, int j, float& m,
                                                 float& mine, float L, float Lh) {
    if (!__any_sync(gmask, moved)) {
        m = mine;
        return;
    }
    for (int q = 0; q < nv; q++) {
        const float sq = __shfl_sync(gmask, s, q, W);
        const bool a = (sq - m) > Lh;
        m += L * (float)a;
        const bool b = (sq - m) < -Lh;
        m -= L * (float)b;
        if (q == j) mine = m;
    }
}

// solventForceKernel (Engine.cu:1070-1161) as three kernels: its two loops,
// run at the same time with W lanes per solvent each, then the sum of their
// results and the integration.  The reference's solvent loops are two
// ordered chains: over
// every compound (computeLJForces, Engine.cu:1099-1117; no list) the solvent
// moves to the image nearest the compound's particle 0 and adds that
// compound's LJ sum; over the solvent list (computeSolventToSolventLJForces,
// Engine.cu:706-720) it moves to each neighbour's image and adds the pair
// force.  Lane j takes compounds / neighbours j, j+W, ...; every lane replays
// the image chain (one hyperpos per compound; per block of W neighbours only
// when some neighbour of the block moves the image, the others leave it
// unchanged) and the lanes' terms are added in the reference's order through
// shuffles, so the result is the reference's float sum whatever W is.  The
// list loop's replay is frequent in small boxes (most solvents then have
// neighbours across a face), so its lane count is chosen separately.

// the loop over the compounds: the force summed over them -> sol_force
template <int W>
__global__ void __launch_bounds__(kSolBlock) k_solvent_compounds(RefDev d, int cur) {
    __shared__ float4 cbuf[kStageCompounds * kStageStride];   // x, y, z, sigma mixed with the solvent's
    __shared__ float cep[kStageCompounds * kStageStride];     // epsilon mixed with the solvent's
    __shared__ int cn[kStageCompounds];
    const int j = threadIdx.x % W;
    const int s = blockIdx.x * (kSolBlock / W) + threadIdx.x / W;
    const unsigned gmask = W == 32 ? 0xffffffffu : (((1u << W) - 1u) << ((threadIdx.x % 32) & ~(W - 1)));
    const bool active = s < d.n_s;
    F3 pos = active ? mk4(d.spos[cur][s]) : mk(0.f, 0.f, 0.f);
    const lima_particle_parameters sol = d.pp[LIMA_ATOMTYPE_SOL];
    F3 force = mk(0.f, 0.f, 0.f);
    // every compound particle, staged 16 compounds at a time
    for (int c0 = 0; c0 < d.n_c; c0 += kStageCompounds) {
        const int nst = min(kStageCompounds, d.n_c - c0);
        __syncthreads();
        for (int q = threadIdx.x; q < nst * kMaxCP; q += kSolBlock) {
            const int cc = q / kMaxCP, l = q % kMaxCP;
            const lima_compound& cp = d.comps[c0 + cc];
            if (l < cp.n_particles) {
                const float4 v = d.cpos[cur][(c0 + cc) * kMaxCP + l];
                const lima_particle_parameters o = d.pp[cp.atom_types[l]];
                cbuf[cc * kStageStride + l] = make_float4(v.x, v.y, v.z, mix_sigma(sol.sigma, o.sigma));
                cep[cc * kStageStride + l] = eps_arith(sol.epsilon, o.epsilon);
            }
            if (l == 0) cn[cc] = cp.n_particles;
        }
        __syncthreads();
        for (int b = 0; b < nst; b += W) {   // compounds b .. b+nv-1, compound b+j on lane j
            const int nv = min(W, nst - b);
            F3 mine = pos;
            for (int q = 0; q < nv; q++) {
                const float4 k0 = cbuf[(b + q) * kStageStride];
                hyperpos(mk(k0.x, k0.y, k0.z), pos, d.L, d.Lh);
                if (q == j) mine = pos;
            }
            F3 acc = mk(0.f, 0.f, 0.f);
            if (active && j < nv) {
                const float4* P = &cbuf[(b + j) * kStageStride];
                const float* EP = &cep[(b + j) * kStageStride];
                const int nn = cn[b + j];
                for (int i = 0; i < nn; i++) {
                    const float4 pi = P[i];
                    acc = add(acc, lj_force(mine, mk(pi.x, pi.y, pi.z), pi.w, EP[i]));
                }
            }
            if (W == 1) {
                force = add(force, acc);
            } else {
                for (int q = 0; q < nv; q++) force = add(force, shfl3(gmask, acc, q, W));
            }
        }
    }
    if (active && j == 0) d.sol_force[s] = to4(force);
}

// the loop over the solvent list (read column-major) -> sol_acc, sol_image.
// Its image chain starts where the loop over the compounds leaves it: the
// solvent moved to each compound's particle-0 image in compound order,
// recomputed here so that the two loops run at the same time.  U blocks of
// W neighbours are gathered before the chain walks them, so U gathers per
// lane are in flight at once.
template <int W, int U>
__global__ void __launch_bounds__(kSolBlock) k_solvent_list(RefDev d, int cur) {
    const int j = threadIdx.x % W;
    const int s = blockIdx.x * (blockDim.x / W) + threadIdx.x / W;
    const unsigned gmask = W == 32 ? 0xffffffffu : (((1u << W) - 1u) << ((threadIdx.x % 32) & ~(W - 1)));
    if (s >= d.n_s) return;   // a solvent's W lanes leave together
    const lima_particle_parameters sol = d.pp[LIMA_ATOMTYPE_SOL];
    F3 pos = mk4(d.spos[cur][s]);
    for (int c = 0; c < d.n_c; c++) hyperpos(mk4(__ldg(&d.cpos[cur][c * kMaxCP])), pos, d.L, d.Lh);
    {
        F3 acc = mk(0.f, 0.f, 0.f);
        const int cnt = d.ss_cnt[s];
        const float sg = sol.sigma, ep = sol.epsilon;
        for (int k0 = 0; k0 < cnt; k0 += W * U) {
            F3 nbs[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int k = k0 + u * W + j;
                nbs[u] = k < cnt ? mk4(__ldg(&d.spos[cur][__ldg(&d.ss_ids[(size_t)k * d.n_s + s])])) : pos;
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int base = k0 + u * W;
                if (base >= cnt) break;   // uniform over the solvent's lanes
                // a lane past the list's end stands at the current image, which no step moves
                const F3 nb = base + j < cnt ? nbs[u] : pos;
                if (W == 1) {
                    hyperpos(nb, pos, d.L, d.Lh);
                    acc = add(acc, lj_force(pos, nb, sg, ep));
                    continue;
                }
                const int nv = min(W, cnt - base);
                // each component's image chain is independent: replay only a
                // component that some neighbour of this block moves
                F3 mine = pos;
                const bool mx = hyperpos1_moved(nb.x, mine.x, d.L, d.Lh);
                const bool my = hyperpos1_moved(nb.y, mine.y, d.L, d.Lh);
                const bool mz = hyperpos1_moved(nb.z, mine.z, d.L, d.Lh);
                replay_component<W>(gmask, mx, nb.x, nv, j, pos.x, mine.x, d.L, d.Lh);
                replay_component<W>(gmask, my, nb.y, nv, j, pos.y, mine.y, d.L, d.Lh);
                replay_component<W>(gmask, mz, nb.z, nv, j, pos.z, mine.z, d.L, d.Lh);
                F3 f = mk(0.f, 0.f, 0.f);
                if (j < nv) f = lj_force(mine, nb, sg, ep);
                for (int q = 0; q < nv; q++) acc = add(acc, shfl3(gmask, f, q, W));
            }
        }
        if (j == 0) {   // every lane holds the same state
            d.sol_acc[s] = to4(acc);
            d.sol_image[s] = to4(pos);
        }
    }
}

// the solvent's force (the sum over the compounds, then the list loop's
// sum, as the reference adds them), integratePosition and applyPBC
__global__ void k_solvent_integrate(RefDev d, int cur) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.n_s) return;
    const lima_particle_parameters sol = d.pp[LIMA_ATOMTYPE_SOL];
    F3 force = d.n_c > 0 ? mk4(d.sol_force[s]) : mk(0.f, 0.f, 0.f);
    force = add(force, mk4(d.sol_acc[s]));
    F3 pos = mk4(d.sol_image[s]);
    F3 prev = mk4(d.sprev[cur][s]);
    integrate(pos, prev, force, (double)sol.mass, d.dt, *d.lambda, d.L, d.Lh);
    apply_pbc(pos, d.L);
    flag_nan(d, pos);
    d.spos[cur ^ 1][s] = to4(pos);
    d.sprev[cur ^ 1][s] = to4(prev);
    d.force_s[s] = to4(force);
}

template <int W>
void launch_solvent_compounds(const RefDev& d, int cur, cudaStream_t s) {
    constexpr int per_block = kSolBlock / W;
    k_solvent_compounds<W><<<(d.n_s + per_block - 1) / per_block, kSolBlock, 0, s>>>(d, cur);
}

template <int W>
void launch_solvent_list(const RefDev& d, int cur, cudaStream_t s) {
    constexpr int U = W == 1 ? 8 : (W <= 4 ? 4 : 2);
    const int per_block = d.sol_list_block / W;
    k_solvent_list<W, U><<<(d.n_s + per_block - 1) / per_block, d.sol_list_block, 0, s>>>(d, cur);
}

int launch_solvent_compounds_kernel(const RefDev& d, int cur, cudaStream_t s) {
    if (d.n_c == 0) return 0;
    switch (d.sol_lanes) {
        case 16: launch_solvent_compounds<16>(d, cur, s); break;
        case 8: launch_solvent_compounds<8>(d, cur, s); break;
        case 4: launch_solvent_compounds<4>(d, cur, s); break;
        case 2: launch_solvent_compounds<2>(d, cur, s); break;
        default: launch_solvent_compounds<1>(d, cur, s); break;
    }
    return 1;
}

int launch_solvent_list_kernel(const RefDev& d, int cur, cudaStream_t s) {
    switch (d.sol_list_lanes) {
        case 16: launch_solvent_list<16>(d, cur, s); break;
        case 8: launch_solvent_list<8>(d, cur, s); break;
        case 4: launch_solvent_list<4>(d, cur, s); break;
        case 2: launch_solvent_list<2>(d, cur, s); break;
        default: launch_solvent_list<1>(d, cur, s); break;
    }
    return 1;
}

int launch_solvent_integrate(const RefDev& d, int cur, cudaStream_t s) {
    k_solvent_integrate<<<(d.n_s + 255) / 256, 256, 0, s>>>(d, cur);
    return 1;
}

// Engine::getBoxTemperature's KE term (LIMAENG::calcKineticEnergy,
// Engine.cuh:32-45): positions two steps apart, central-difference speed.
__global__ void k_ref_ke(RefDev d, int cur) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n_cp = d.n_c * kMaxCP;
    double ke = 0.0;
    if (i < n_cp) {
        const int c = i / kMaxCP, l = i % kMaxCP;
        const lima_compound& cp = d.comps[c];
        if (l < cp.n_particles) {
            F3 a = mk4(d.cpos[cur][i]), b = mk4(d.csnap[i]);
            hyperpos(a, b, d.L, d.Lh);
            float vel = (float)((double)(len(sub(a, b)) * 0.5f) / d.dt);
            ke = (double)(float)(0.5 * (double)d.pp[cp.atom_types[l]].mass * vel * vel);
        }
    } else if (i < n_cp + d.n_s) {
        const int s = i - n_cp;
        F3 a = mk4(d.spos[cur][s]), b = mk4(d.ssnap[s]);
        hyperpos(a, b, d.L, d.Lh);
        float vel = (float)((double)(len(sub(a, b)) * 0.5f) / d.dt);
        ke = (double)(float)(0.5 * (double)d.pp[LIMA_ATOMTYPE_SOL].mass * vel * vel);
    }
    for (int o = 16; o > 0; o >>= 1) ke += __shfl_down_sync(0xffffffffu, ke, o);
    if ((threadIdx.x & 31) == 0 && ke != 0.0) atomicAdd(d.ke_accum, ke);
}

// Engine::handleBoxtemp (Engine.cu:362-393): lambda = clamp(T0/T, 0.9, 1.1).
__global__ void k_ref_lambda(RefDev d, int n_particles, float t_target, int apply) {
    double avg = *d.ke_accum / (double)n_particles;
    float temp = (float)(avg * 2.0 / (3.0 * 8.3145));
    temp = temp == 0.f ? 1.f : temp;
    float sc = t_target / temp;
    sc = fminf(sc, 1.1f);
    sc = fmaxf(sc, 0.9f);
    if (apply) *d.lambda = sc;
    *d.ke_accum = (double)temp;   // keep the temperature for readback
}

__global__ void k_snapshot(RefDev d, int cur) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.n_c * kMaxCP) d.csnap[i] = d.cpos[cur][i];
    if (i < d.n_s) d.ssnap[i] = d.spos[cur][i];
}

}  // namespace

// ev (nullable): events recorded before the bridges, after them, after the
// compound kernels and after the solvent kernel (the kernels then run one
// after another).  Without ev and with fk the solvent kernel runs on
// fk->side beside the bridge and compound kernels, joined before return.
// Returns kernels launched.
int ref_step_kernels(const RefDev& d, int cur, cudaStream_t s, cudaEvent_t* ev, const StepFork* fk) {
    int launched = 0;
    const bool forked = !ev && fk && fk->side && fk->side2 && d.n_s > 0;
    if (forked) {
        // side2: the loop over the compounds; side: the list loop, then the
        // sum of the two and the integration
        cudaEventRecord(fk->fork, s);
        cudaStreamWaitEvent(fk->side, fk->fork, 0);
        cudaStreamWaitEvent(fk->side2, fk->fork, 0);
        launched += launch_solvent_compounds_kernel(d, cur, fk->side2);
        cudaEventRecord(fk->join2, fk->side2);
        launched += launch_solvent_list_kernel(d, cur, fk->side);
        cudaStreamWaitEvent(fk->side, fk->join2, 0);
        launched += launch_solvent_integrate(d, cur, fk->side);
        cudaEventRecord(fk->join, fk->side);
    }
    if (ev) cudaEventRecord(ev[0], s);
    if (d.n_b > 0) {
        k_bridge<<<d.n_b, 32, 0, s>>>(d, cur);
        launched++;
    }
    if (ev) cudaEventRecord(ev[1], s);
    if (d.n_c > 0) {
        k_partials<<<dim3(d.n_chunks + 1 + kMaxCP, d.n_c), 64, 0, s>>>(d, cur);
        k_compound<<<d.n_c, 64, 0, s>>>(d, cur);
        launched += 2;
    }
    if (ev) cudaEventRecord(ev[2], s);
    if (forked) {
        cudaStreamWaitEvent(s, fk->join, 0);
    } else if (d.n_s > 0) {
        launched += launch_solvent_compounds_kernel(d, cur, s);
        launched += launch_solvent_list_kernel(d, cur, s);
        launched += launch_solvent_integrate(d, cur, s);
    }
    if (ev) cudaEventRecord(ev[3], s);
    return launched;
}

void ref_thermostat_snapshot(const RefDev& d, int cur, cudaStream_t s) {
    const int n = max(d.n_c * kMaxCP, d.n_s);
    if (n > 0) k_snapshot<<<(n + 255) / 256, 256, 0, s>>>(d, cur);
}

// n_particles: Simulation::total_particles (compound particles present + solvents)
void ref_thermostat_update(const RefDev& d, int cur, int n_particles, float t_target, bool apply, cudaStream_t s) {
    cudaMemsetAsync(d.ke_accum, 0, sizeof(double), s);
    const int n = d.n_c * kMaxCP + d.n_s;
    if (n > 0) k_ref_ke<<<(n + 255) / 256, 256, 0, s>>>(d, cur);
    k_ref_lambda<<<1, 1, 0, s>>>(d, n_particles, t_target, apply ? 1 : 0);
}

__global__ void k_set_float(float* p, float v) { *p = v; }

void set_device_float(float* p, float v, cudaStream_t s) { k_set_float<<<1, 1, 0, s>>>(p, v); }

}  // namespace lima
