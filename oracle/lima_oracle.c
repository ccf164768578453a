/*
 * lima_oracle.c — CPU oracle for the LIMA_MD per-step path.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load the library built from this file
 * (oracle/liblima_oracle.so); the product path never calls it and has no CPU
 * fallback.
 *
 * Two parts:
 *
 *  A. "reference semantics": a plain-C restatement of the reference's own
 *     algorithm — Engine::updateNeighborLists / cullDistantNeighbors /
 *     neighborWithinCutoff (Quantom/Quantom/Engine.cu:146-287) and one
 *     Engine::step (Engine.cu:400-451) = compoundBridgeKernel (:1168-1223),
 *     compoundKernel (:880-1057), solventForceKernel (:1070-1161) with their
 *     device functions (:461-869).  FP32 with the reference's operation order
 *     (build with -ffp-contract=off).  Pinned against the reference compiled
 *     from its own sources (oracle/_ref, tests/test_oracle_pin.py) and against
 *     committed fixtures from it (tests/golden/).
 *
 *  B. "physics semantics": FP64 evaluation of the same model's conservative
 *     functional forms (Lorentz-Berthelot LJ with cutoff and optional
 *     potential switch, harmonic bond/angle, periodic dihedral), energies and
 *     virial, and a velocity-Verlet step with a Berendsen thermostat — the
 *     accuracy reference for the FP32 and mixed-precision GPU paths.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/lima_abi.h"

#define MAXP LIMA_MAX_COMPOUND_PARTICLES

/* ======================================================================= */
/* A. Reference semantics                                                   */
/* ======================================================================= */

typedef lima_float3 f3;

static f3 v3(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
static f3 add3(f3 a, f3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static f3 sub3(f3 a, f3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
/* Float3::operator*(const double) (QuantomTypes.cuh:39): product in double, stored as float */
static f3 muld(f3 a, double s) { return v3((float)(a.x * s), (float)(a.y * s), (float)(a.z * s)); }
static float len3(f3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }        /* :60 */
static float len2(f3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }                /* :61 */
static float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }         /* :90 */
static f3 cross3(f3 a, f3 b) {                                                       /* :89 */
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static f3 norm3(f3 a) {                                                              /* :50-55 */
    float l = len3(a);
    if (l != 0.f) return muld(a, 1.f / l);
    return v3(0.f, 0.f, 0.f);
}
/* Float3::getAngle (QuantomTypes.cuh:74-83) */
static float get_angle(f3 a, f3 b) {
    float val = dot3(a, b) / (len3(a) * len3(b));
    val = val > 1.f ? 1.f : val;
    val = val < -1.f ? -1.f : val;
    return acosf(val);
}
static float comp(const f3* a, int d) { return d == 0 ? a->x : (d == 1 ? a->y : a->z); }
static float* compp(f3* a, int d) { return d == 0 ? &a->x : (d == 1 ? &a->y : &a->z); }

/* LIMAENG::applyHyperpos (Engine.cuh:24-30); the second test sees the first update */
static void hyperpos(const f3* stat, f3* mov, float L, float Lh) {
    for (int d = 0; d < 3; d++) {
        *compp(mov, d) += L * (float)((comp(stat, d) - comp(mov, d)) > Lh);
        *compp(mov, d) -= L * (float)((comp(stat, d) - comp(mov, d)) < -Lh);
    }
}
/* applyPBC (Engine.cu:461-466) */
static void apply_pbc(f3* p, float L) {
    for (int d = 0; d < 3; d++) {
        *compp(p, d) += L * (float)(comp(p, d) < 0);
        *compp(p, d) -= L * (float)(comp(p, d) > L);
    }
}
/* Engine::neighborWithinCutoff (Engine.cu:146-151) */
static int within(const f3* a, const f3* b, float C, float offset, float L, float Lh) {
    f3 bb = *b;
    hyperpos(a, &bb, L, Lh);
    float dist = len3(sub3(*a, bb));
    return dist < (C + offset);
}

/* calcLJForce (Engine.cu:475-522), force on p0 */
static f3 lj_force(f3 p0, f3 p1, float sigma, float epsilon) {
    f3 d = sub3(p1, p0);
    float d2 = len2(d);
    float s = sigma * sigma / d2;
    s = s * s * s;
    float fs = 24.f * epsilon * s / d2 * (1.f - 2.f * s);
    return muld(d, fs);
}
static float mix_arith_eps(float a, float b) { return (float)((double)(a + b) * 0.5); }   /* Engine.cu:645,670 */
static float mix_geo_eps(float a, float b) { return sqrtf(a * b); }                         /* Engine.cu:691,726 */
static float mix_sigma(float a, float b) { return (a + b) * 0.5f; }

/* calcPairbondForces (Engine.cu:525-548) */
static void pairbond(f3 a, f3 b, const lima_pair_bond* pb, f3* res, float* potE) {
    f3 diff = sub3(a, b);
    double error = (double)(len3(diff) - pb->b0);
    *potE = (float)((double)*potE + 0.5 * (double)pb->kb * (error * error));
    diff = norm3(diff);
    double fs = (double)(-pb->kb) * error;
    res[0] = muld(diff, fs);
    res[1] = muld(muld(diff, fs), -1.0);
}
/* calcAnglebondForces (Engine.cu:552-578) */
static void anglebond(f3 l, f3 m, f3 r, const lima_angle_bond* ab, f3* res, float* potE) {
    f3 v1 = sub3(l, m), v2 = sub3(r, m);
    f3 n1 = cross3(v1, v2), n2 = cross3(v2, v1);
    f3 in1 = norm3(cross3(v1, n2)), in2 = norm3(cross3(v2, n1));
    double angle = (double)get_angle(v1, v2);
    double error = angle - (double)ab->theta_0;
    *potE = (float)((double)*potE + 0.5 * (double)ab->k_theta * error * error * 0.5);
    double fs = (double)ab->k_theta * error;
    res[0] = muld(in1, fs);
    res[2] = muld(in2, fs);
    res[1] = muld(add3(res[0], res[2]), -1.0);
}
/* calcDihedralbondForces (Engine.cu:580-637); potE is assigned, not added */
static void dihedral(f3 l, f3 lm, f3 rm, f3 r, const lima_dihedral_bond* db, f3* res, float* potE) {
    f3 n1 = norm3(cross3(sub3(l, lm), sub3(rm, lm)));
    f3 n2 = norm3(cross3(sub3(lm, rm), sub3(r, rm)));
    float torsion = get_angle(n1, n2);
    if (len3(sub3(add3(l, n1), r)) < len3(sub3(sub3(l, n1), r))) {
        n2.x *= -1.f; n2.y *= -1.f; n2.z *= -1.f;
    } else {
        n1.x *= -1.f; n1.y *= -1.f; n1.z *= -1.f;
    }
    float arg = (float)db->n * torsion - db->phi_0;
    float fs = db->k_phi * sinf(arg);
    *potE = db->k_phi * (1.f - cosf(arg));
    res[0] = muld(n1, (double)fs);
    res[3] = muld(n2, (double)fs);
    res[1] = muld(muld(add3(res[0], res[3]), -1.0), 0.5);
    res[2] = muld(muld(add3(res[0], res[3]), -1.0), 0.5);
}
/* integratePosition (Engine.cu:849-869) */
static void integrate(f3* pos, f3* prev, f3 force, double mass, double dt, float lambda, float L, float Lh) {
    f3 temp = *pos;
    hyperpos(pos, prev, L, Lh);
    double mts = dt / mass * dt;
    *pos = add3(sub3(muld(*pos, 2.0), *prev), muld(force, mts));
    *prev = temp;
    f3 delta = sub3(*pos, *prev);
    *pos = add3(*prev, muld(delta, (double)lambda));
}
/* LJ_Ignores::ignore (Bodies.cuh:191-197) */
static int lj_ignored(const lima_lj_ignores* ig, int local, int cid) {
    for (int i = 0; i < ig->n_ignores; i++)
        if (ig->local_ids[i] == (uint8_t)local && ig->compound_ids[i] == (uint8_t)cid) return 1;
    return 0;
}

/* Bonded sums of one entity (compound or bridge) as in
   computePairbondForces/AnglebondForces/DihedralForces<T> (Engine.cu:744-847):
   contributions accumulate per atom in term-index order; thread t's potE
   collects terms t, t+nthreads, ... */
static void bonded_sums(const f3* pos, int nthreads, int nb, const lima_pair_bond* bonds, int na,
                        const lima_angle_bond* angles, int nd, const lima_dihedral_bond* dihs, f3* force,
                        float* potE) {
    f3 util[MAXP];
    f3 res[4];
    for (int t = 0; t < nthreads; t++) util[t] = v3(0, 0, 0);
    for (int b = 0; b < nb; b++) {
        const lima_pair_bond* pb = &bonds[b];
        pairbond(pos[pb->atom_indexes[0]], pos[pb->atom_indexes[1]], pb, res, &potE[b % nthreads]);
        util[pb->atom_indexes[0]] = add3(util[pb->atom_indexes[0]], res[0]);
        util[pb->atom_indexes[1]] = add3(util[pb->atom_indexes[1]], res[1]);
    }
    for (int t = 0; t < nthreads; t++) { force[t] = add3(force[t], util[t]); util[t] = v3(0, 0, 0); }
    for (int b = 0; b < na; b++) {
        const lima_angle_bond* ab = &angles[b];
        anglebond(pos[ab->atom_indexes[0]], pos[ab->atom_indexes[1]], pos[ab->atom_indexes[2]], ab, res,
                  &potE[b % nthreads]);
        for (int k = 0; k < 3; k++) util[ab->atom_indexes[k]] = add3(util[ab->atom_indexes[k]], res[k]);
    }
    for (int t = 0; t < nthreads; t++) { force[t] = add3(force[t], util[t]); util[t] = v3(0, 0, 0); }
    for (int b = 0; b < nd; b++) {
        const lima_dihedral_bond* db = &dihs[b];
        dihedral(pos[db->atom_indexes[0]], pos[db->atom_indexes[1]], pos[db->atom_indexes[2]],
                 pos[db->atom_indexes[3]], db, res, &potE[b % nthreads]);
        for (int k = 0; k < 4; k++) util[db->atom_indexes[k]] = add3(util[db->atom_indexes[k]], res[k]);
    }
    for (int t = 0; t < nthreads; t++) force[t] = add3(force[t], util[t]);
}

/*
 * Neighbour lists after one reference update (Engine.cu:155-287), as sets.
 * prev_cc[n_c*n_c] (nullable): 1 where the previous compound-compound list
 * holds the pair.  Outputs: fixed-capacity id arrays in ascending order plus
 * counts.  Returns 0, or -1 when a list exceeds its capacity.
 */
int orc_ref_nlist(float L, float C, int n_c, const lima_compound* comps, const lima_compound_state* states, int n_s,
                  const lima_solvent* sols, const uint8_t* prev_cc, int* cc_ids, int* cc_cnt, int cs_cap,
                  int* cs_ids, int* cs_cnt, int ss_cap, int* ss_ids, int* ss_cnt, int sc_cap, int* sc_ids,
                  int* sc_cnt) {
    const float Lh = L / 2.f;
    int rc = 0;
    f3* key = (f3*)malloc(sizeof(f3) * (n_c > 0 ? n_c : 1));
    for (int c = 0; c < n_c; c++) key[c] = states[c].positions[comps[c].key_particle_index];
    for (int c = 0; c < n_c; c++) cc_cnt[c] = 0;
    for (int s = 0; s < n_s; s++) { ss_cnt[s] = 0; sc_cnt[s] = 0; }
    /* compound-compound: cull (Engine.cu:162-174) keeps a previous pair
       within C + ((r_i + r_j) + C); add (:241-252) takes pairs within
       C + ((r_i + r_i) + C) — the reference reads id_self's sphere twice. */
    for (int i = 0; i < n_c; i++) {
        const float ri = comps[i].confining_particle_sphere;
        for (int j = i + 1; j < n_c; j++) {
            const float rj = comps[j].confining_particle_sphere;
            int keep = prev_cc && prev_cc[i * n_c + j] && within(&key[i], &key[j], C, ri + rj + C, L, Lh);
            int add = within(&key[i], &key[j], C, ri + ri + C, L, Lh);
            if (keep || add) {
                if (cc_cnt[i] >= LIMA_MAX_COMPOUND_PARTICLES || cc_cnt[j] >= LIMA_MAX_COMPOUND_PARTICLES) { rc = -1; continue; }
                cc_ids[i * MAXP + cc_cnt[i]++] = j;
                cc_ids[j * MAXP + cc_cnt[j]++] = i;
            }
        }
    }
    /* list order: ascending (entries from lower ids were appended first) */
    for (int c = 0; c < n_c; c++) {
        int* a = &cc_ids[c * MAXP];
        for (int x = 1; x < cc_cnt[c]; x++) {
            int v = a[x], y = x - 1;
            while (y >= 0 && a[y] > v) { a[y + 1] = a[y]; y--; }
            a[y + 1] = v;
        }
    }
    /* compound-solvent (Engine.cu:177-187, 229-238) */
    for (int c = 0; c < n_c; c++) {
        const float r = comps[c].confining_particle_sphere;
        cs_cnt[c] = 0;
        for (int s = 0; s < n_s; s++) {
            if (within(&key[c], &sols[s].pos, C, r + C, L, Lh)) {
                if (cs_cnt[c] >= cs_cap || sc_cnt[s] >= sc_cap) { rc = -1; continue; }
                cs_ids[(size_t)c * cs_cap + cs_cnt[c]++] = s;
                sc_ids[(size_t)s * sc_cap + sc_cnt[s]++] = c;
            }
        }
    }
    /* solvent-solvent (Engine.cu:191-205, 256-275): the pair is tested from
       the lower id, with the same float expression as the add loop. */
    for (int i = 0; i < n_s && ss_cap > 0; i++) {   /* ss_cap == 0: caller uses orc_ref_nlist_ss_cells */
        for (int j = i + 1; j < n_s; j++) {
            if (within(&sols[i].pos, &sols[j].pos, C, C, L, Lh)) {
                if (ss_cnt[i] >= ss_cap || ss_cnt[j] >= ss_cap) { rc = -1; continue; }
                ss_ids[(size_t)i * ss_cap + ss_cnt[i]++] = j;
                ss_ids[(size_t)j * ss_cap + ss_cnt[j]++] = i;
            }
        }
    }
    free(key);
    return rc;
}

/*
 * Same solvent-solvent list with a cell grid (O(N)), for large boxes.  The
 * pair test is the identical float expression; ids come out ascending.
 */
/* periodic image in [0, L) of a coordinate, for cell assignment only */
static float wrapf(float x, float L) { return x - L * floorf(x / L); }

int orc_ref_nlist_ss_cells(float L, float C, int n_s, const lima_solvent* sols, int ss_cap, int* ss_ids,
                           int* ss_cnt) {
    const float Lh = L / 2.f;
    const float radius = C + C;
    int m = (int)floorf(L / (radius * 1.0001f));
    if (m < 3) m = 1;
    const float cell = L / (float)m;
    int* head = (int*)malloc(sizeof(int) * m * m * m);
    int* next = (int*)malloc(sizeof(int) * (n_s > 0 ? n_s : 1));
    for (int k = 0; k < m * m * m; k++) head[k] = -1;
    for (int s = n_s - 1; s >= 0; s--) {
        int ix = (int)(wrapf(sols[s].pos.x, L) / cell), iy = (int)(wrapf(sols[s].pos.y, L) / cell),
            iz = (int)(wrapf(sols[s].pos.z, L) / cell);
        ix = ix < 0 ? 0 : (ix >= m ? m - 1 : ix);
        iy = iy < 0 ? 0 : (iy >= m ? m - 1 : iy);
        iz = iz < 0 ? 0 : (iz >= m ? m - 1 : iz);
        int k = (ix * m + iy) * m + iz;
        next[s] = head[k];
        head[k] = s;
    }
    int rc = 0;
    int* tmp = (int*)malloc(sizeof(int) * (ss_cap + 1));
    for (int i = 0; i < n_s; i++) {
        int cnt = 0;
        int ix = (int)(wrapf(sols[i].pos.x, L) / cell), iy = (int)(wrapf(sols[i].pos.y, L) / cell),
            iz = (int)(wrapf(sols[i].pos.z, L) / cell);
        ix = ix < 0 ? 0 : (ix >= m ? m - 1 : ix);
        iy = iy < 0 ? 0 : (iy >= m ? m - 1 : iy);
        iz = iz < 0 ? 0 : (iz >= m ? m - 1 : iz);
        int span = m >= 3 ? 1 : 0;
        for (int dx = -span; dx <= span; dx++)
            for (int dy = -span; dy <= span; dy++)
                for (int dz = -span; dz <= span; dz++) {
                    int k = (((ix + dx + m) % m) * m + ((iy + dy + m) % m)) * m + ((iz + dz + m) % m);
                    for (int j = head[k]; j >= 0; j = next[j]) {
                        if (j == i) continue;
                        const lima_solvent* lo = &sols[i < j ? i : j];
                        const lima_solvent* hi = &sols[i < j ? j : i];
                        if (within(&lo->pos, &hi->pos, C, C, L, Lh)) {
                            if (cnt >= ss_cap) { rc = -1; continue; }
                            tmp[cnt++] = j;
                        }
                    }
                }
        for (int x = 1; x < cnt; x++) {
            int v = tmp[x], y = x - 1;
            while (y >= 0 && tmp[y] > v) { tmp[y + 1] = tmp[y]; y--; }
            tmp[y + 1] = v;
        }
        memcpy(&ss_ids[(size_t)i * ss_cap], tmp, sizeof(int) * cnt);
        ss_cnt[i] = cnt;
    }
    free(tmp);
    free(head);
    free(next);
    return rc;
}

/*
 * One reference step.  comps/states/sols are updated in place the way the
 * kernels update the Box (states := compound_state_array_next, solvents :=
 * solvents_next, Compound::prev_positions and ::forces).  Lists as produced
 * by orc_ref_nlist (list order = iteration order).  Outputs: the total force
 * each particle was integrated with and the per-particle potE the kernels
 * log (potE_buffer layout: c*64+t, then n_c*64+s).
 */
int orc_ref_step(float L, float C, double dt, float lambda, const lima_forcefield* ff, int n_c, lima_compound* comps,
                 lima_compound_state* states, int n_s, lima_solvent* sols, int n_b,
                 const lima_compound_bridge_compact* bridges, const int* cc_ids, const int* cc_cnt, int cs_cap,
                 const int* cs_ids, const int* cs_cnt, int ss_cap, const int* ss_ids, const int* ss_cnt,
                 float* force_c, float* force_s, double* potE) {
    (void)C;
    const float Lh = L / 2.f;
    const lima_particle_parameters* pp = ff->particle_parameters;
    const float sig_sol = pp[LIMA_ATOMTYPE_SOL].sigma, eps_sol = pp[LIMA_ATOMTYPE_SOL].epsilon;

    /* --- compoundBridgeKernel (Engine.cu:1168-1223), bridges in order --- */
    for (int b = 0; b < n_b; b++) {
        const lima_compound_bridge_compact* br = &bridges[b];
        f3 pos[LIMA_MAX_PARTICLES_IN_BRIDGE], force[LIMA_MAX_PARTICLES_IN_BRIDGE];
        float pe[LIMA_MAX_PARTICLES_IN_BRIDGE];
        for (int t = 0; t < LIMA_MAX_PARTICLES_IN_BRIDGE; t++) {
            pos[t] = v3(0, 0, 0);
            force[t] = v3(0, 0, 0);
            pe[t] = 0.f;
        }
        for (int t = 0; t < br->n_particles; t++)
            pos[t] = states[br->particle_refs[t].compound_id].positions[br->particle_refs[t].local_id_compound];
        for (int t = 1; t < LIMA_MAX_PARTICLES_IN_BRIDGE; t++) hyperpos(&pos[0], &pos[t], L, Lh);
        bonded_sums(pos, LIMA_MAX_PARTICLES_IN_BRIDGE, br->n_singlebonds, br->singlebonds, br->n_anglebonds,
                    br->anglebonds, br->n_dihedrals, br->dihedrals, force, pe);
        for (int t = 0; t < br->n_particles; t++)
            comps[br->particle_refs[t].compound_id].forces[br->particle_refs[t].local_id_compound] = force[t];
    }

    /* compoundKernel reads compound_state_array (current); keep a copy so
       the per-compound updates below read pre-step positions. */
    lima_compound_state* cur = (lima_compound_state*)malloc(sizeof(lima_compound_state) * (n_c > 0 ? n_c : 1));
    if (n_c > 0) memcpy(cur, states, sizeof(lima_compound_state) * (size_t)n_c);
    lima_solvent* scur = (lima_solvent*)malloc(sizeof(lima_solvent) * (n_s > 0 ? n_s : 1));
    if (n_s > 0) memcpy(scur, sols, sizeof(lima_solvent) * (size_t)n_s);

    /* --- compoundKernel (Engine.cu:880-1057) --- */
    for (int c = 0; c < n_c; c++) {
        lima_compound* cp = &comps[c];
        const int n = cp->n_particles;
        f3 pos[MAXP], force[MAXP];
        float pe[MAXP];
        f3* buf = (f3*)malloc(sizeof(f3) * (cs_cnt[c] > MAXP ? cs_cnt[c] : MAXP));
        for (int t = 0; t < MAXP; t++) {
            pos[t] = t < n ? cur[c].positions[t] : v3(0, 0, 0);
            force[t] = t < n ? cp->forces[t] : v3(0, 0, 0);
            pe[t] = 0.f;
        }
        for (int t = 0; t < n; t++) cp->forces[t] = v3(0, 0, 0);     /* Compound::loadData, Bodies.cuh:438 */
        for (int t = 1; t < n; t++) hyperpos(&pos[0], &pos[t], L, Lh);
        bonded_sums(pos, MAXP, cp->n_singlebonds, cp->singlebonds, cp->n_anglebonds, cp->anglebonds,
                    cp->n_dihedrals, cp->dihedrals, force, pe);
        /* computeIntramolecularLJForces (Engine.cu:678-700) */
        for (int t = 0; t < n; t++) {
            f3 acc = v3(0, 0, 0);
            const lima_particle_parameters* a = &pp[cp->atom_types[t]];
            for (int i = 0; i < n; i++) {
                if (i == t || lj_ignored(&cp->lj_ignore_list[t], i, c)) continue;
                const lima_particle_parameters* o = &pp[cp->atom_types[i]];
                acc = add3(acc, lj_force(pos[t], pos[i], mix_sigma(a->sigma, o->sigma), mix_geo_eps(a->epsilon, o->epsilon)));
            }
            force[t] = add3(force[t], acc);
        }
        /* inter-compound LJ over the compound list (Engine.cu:939-958) */
        for (int k = 0; k < cc_cnt[c]; k++) {
            const int nb = cc_ids[c * MAXP + k];
            const int nn = cur[nb].n_particles;
            for (int j = 0; j < nn; j++) {
                buf[j] = cur[nb].positions[j];
                hyperpos(&pos[0], &buf[j], L, Lh);
            }
            for (int t = 0; t < n; t++) {
                f3 acc = v3(0, 0, 0);
                const lima_particle_parameters* a = &pp[cp->atom_types[t]];
                for (int j = 0; j < nn; j++) {
                    if (lj_ignored(&cp->lj_ignore_list[t], j, nb)) continue;
                    const lima_particle_parameters* o = &pp[comps[nb].atom_types[j]];
                    acc = add3(acc, lj_force(pos[t], buf[j], mix_sigma(a->sigma, o->sigma), mix_arith_eps(a->epsilon, o->epsilon)));
                }
                force[t] = add3(force[t], acc);
            }
        }
        /* compound <- solvent LJ over the compound's solvent list (Engine.cu:965-973) */
        const int ncs = cs_cnt[c];
        for (int k = 0; k < ncs; k++) {
            buf[k] = scur[cs_ids[(size_t)c * cs_cap + k]].pos;
            hyperpos(&pos[0], &buf[k], L, Lh);
        }
        for (int t = 0; t < n; t++) {
            f3 acc = v3(0, 0, 0);
            const lima_particle_parameters* a = &pp[cp->atom_types[t]];
            const float sg = mix_sigma(a->sigma, sig_sol), ep = mix_geo_eps(a->epsilon, eps_sol);
            for (int k = 0; k < ncs; k++) acc = add3(acc, lj_force(pos[t], buf[k], sg, ep));
            force[t] = add3(force[t], acc);
        }
        free(buf);
        /* integratePosition + prev_positions write-back (Engine.cu:981-984) */
        for (int t = 0; t < n; t++) {
            integrate(&pos[t], &cp->prev_positions[t], force[t], (double)pp[cp->atom_types[t]].mass, dt, lambda, L, Lh);
            if (force_c) {
                force_c[(c * MAXP + t) * 3 + 0] = force[t].x;
                force_c[(c * MAXP + t) * 3 + 1] = force[t].y;
                force_c[(c * MAXP + t) * 3 + 2] = force[t].z;
            }
        }
        /* PBC on particle 0 then every particle follows it (Engine.cu:993-996) */
        apply_pbc(&pos[0], L);
        for (int t = 1; t < n; t++) hyperpos(&pos[0], &pos[t], L, Lh);
        for (int t = 0; t < n; t++) states[c].positions[t] = pos[t];
        if (potE)
            for (int t = 0; t < MAXP; t++) potE[c * MAXP + t] = (double)pe[t];
    }

    /* --- solventForceKernel (Engine.cu:1070-1161) --- */
    const double m_sol = (double)pp[LIMA_ATOMTYPE_SOL].mass;
    for (int s = 0; s < n_s; s++) {
        f3 pos = scur[s].pos, prev = scur[s].pos_tsub1;
        f3 force = v3(0, 0, 0);
        for (int c = 0; c < n_c; c++) {
            const int nn = cur[c].n_particles;
            hyperpos(&cur[c].positions[0], &pos, L, Lh);
            f3 acc = v3(0, 0, 0);
            for (int i = 0; i < nn; i++) {
                const lima_particle_parameters* o = &pp[comps[c].atom_types[i]];
                acc = add3(acc, lj_force(pos, cur[c].positions[i], mix_sigma(sig_sol, o->sigma), mix_arith_eps(eps_sol, o->epsilon)));
            }
            force = add3(force, acc);
        }
        f3 acc = v3(0, 0, 0);
        for (int k = 0; k < ss_cnt[s]; k++) {
            f3 nbp = scur[ss_ids[(size_t)s * ss_cap + k]].pos;
            hyperpos(&nbp, &pos, L, Lh);
            acc = add3(acc, lj_force(pos, nbp, sig_sol, eps_sol));
        }
        force = add3(force, acc);
        integrate(&pos, &prev, force, m_sol, dt, lambda, L, Lh);
        apply_pbc(&pos, L);
        sols[s].pos = pos;
        sols[s].pos_tsub1 = prev;
        if (force_s) {
            force_s[s * 3 + 0] = force.x;
            force_s[s * 3 + 1] = force.y;
            force_s[s * 3 + 2] = force.z;
        }
        if (potE) potE[n_c * MAXP + s] = 0.0;   /* solvent potE_sum is never added to (Engine.cu:1078,1141) */
    }
    free(cur);
    free(scur);
    return 0;
}

/* ======================================================================= */
/* B. Physics semantics, FP64                                               */
/* ======================================================================= */

typedef struct {
    int n;                    /* particles */
    double box;
    double rc, r_on;          /* cutoff, switch start (r_on >= rc: shifted potential) */
    const double* sigma;      /* per particle */
    const double* epsilon;    /* per particle */
    const int* excl_off;      /* CSR exclusions per particle (both directions) */
    const int* excl_ids;
    int n_bonds; const int* bond_idx; const double* bond_r0; const double* bond_k;
    int n_angles; const int* angle_idx; const double* angle_t0; const double* angle_k;
    int n_dih; const int* dih_idx; const double* dih_phi0; const double* dih_k; const int* dih_n;
} orc_phys_sys;

static double mimg(double d, double L) { return d - L * nearbyint(d / L); }

static int excluded(const orc_phys_sys* S, int i, int j) {
    for (int k = S->excl_off[i]; k < S->excl_off[i + 1]; k++)
        if (S->excl_ids[k] == j) return 1;
    return 0;
}

/* LJ pair: energy and f such that F_j = f * r_vec (r_vec = x_j - x_i). */
static void lj_pair64(const orc_phys_sys* S, double r2, double sig, double eps, double* e, double* f_over_r) {
    const double rc = S->rc, ron = S->r_on;
    double sr2 = sig * sig / r2, sr6 = sr2 * sr2 * sr2;
    double v = 4.0 * eps * (sr6 * sr6 - sr6);
    double dvdr_over_r = -24.0 * eps * (2.0 * sr6 * sr6 - sr6) / r2;   /* (dV/dr)/r */
    if (ron < rc) {
        double rc2 = rc * rc, ron2 = ron * ron;
        if (r2 > ron2) {
            /* C2 switch in r^2: S = t^3 (10 - 15 t + 6 t^2), t = (rc^2 - r^2) / (rc^2 - r_on^2);
               S, S' and S'' are continuous at r_on (t = 1) and r_c (t = 0) */
            double D = rc2 - ron2;
            double t = r2 < rc2 ? (rc2 - r2) / D : 0.0;
            double sw = t * t * t * (10.0 + t * (-15.0 + 6.0 * t));
            double dsw_over_r = -60.0 * t * t * (1.0 - t) * (1.0 - t) / D;   /* (dS/dr)/r = 2 dS/d(r^2) */
            dvdr_over_r = dvdr_over_r * sw + v * dsw_over_r;
            v *= sw;
        }
    } else {
        double src2 = sig * sig / (rc * rc), src6 = src2 * src2 * src2;
        v -= 4.0 * eps * (src6 * src6 - src6);
    }
    *e = v;
    *f_over_r = dvdr_over_r;   /* F_j = -dV/dr * r_hat = -(dV/dr)/r * r_vec ... sign handled by caller */
}

/*
 * Forces (n*3), energies[0..4] = E_LJ, E_bond, E_angle, E_dihedral, virial
 * (sum over interactions of r_ij . F_j).  Positions n*3 (any image).
 */
int orc_phys_forces(const orc_phys_sys* S, const double* x, double* F, double* energies) {
    const int n = S->n;
    const double L = S->box;
    memset(F, 0, sizeof(double) * 3 * n);
    double e_lj = 0, e_b = 0, e_a = 0, e_d = 0, vir = 0;
    /* cell grid */
    int m = (int)floor(L / S->rc);
    if (m < 3) m = 1;
    const double cell = L / m;
    int* head = (int*)malloc(sizeof(int) * m * m * m);
    int* next = (int*)malloc(sizeof(int) * n);
    int* cidx = (int*)malloc(sizeof(int) * n);
    for (int k = 0; k < m * m * m; k++) head[k] = -1;
    for (int i = 0; i < n; i++) {
        int c[3];
        for (int d = 0; d < 3; d++) {
            double w = x[3 * i + d] - L * floor(x[3 * i + d] / L);
            c[d] = (int)(w / cell);
            if (c[d] >= m) c[d] = m - 1;
        }
        cidx[i] = (c[0] * m + c[1]) * m + c[2];
        next[i] = head[cidx[i]];
        head[cidx[i]] = i;
    }
    const double rc2 = S->rc * S->rc;
    for (int i = 0; i < n; i++) {
        int ci = cidx[i];
        int cx = ci / (m * m), cy = (ci / m) % m, cz = ci % m;
        int span = m >= 3 ? 1 : 0;
        for (int dx = -span; dx <= span; dx++)
            for (int dy = -span; dy <= span; dy++)
                for (int dz = -span; dz <= span; dz++) {
                    int k = (((cx + dx + m) % m) * m + ((cy + dy + m) % m)) * m + ((cz + dz + m) % m);
                    for (int j = head[k]; j >= 0; j = next[j]) {
                        if (j <= i) continue;
                        double r[3], r2 = 0;
                        for (int d = 0; d < 3; d++) {
                            r[d] = mimg(x[3 * j + d] - x[3 * i + d], L);
                            r2 += r[d] * r[d];
                        }
                        if (r2 >= rc2) continue;
                        if (excluded(S, i, j)) continue;
                        double sig = 0.5 * (S->sigma[i] + S->sigma[j]);
                        double eps = sqrt(S->epsilon[i] * S->epsilon[j]);
                        double e, dvdr_r;
                        lj_pair64(S, r2, sig, eps, &e, &dvdr_r);
                        e_lj += e;
                        for (int d = 0; d < 3; d++) {
                            double fj = -dvdr_r * r[d];
                            F[3 * j + d] += fj;
                            F[3 * i + d] -= fj;
                            vir += r[d] * fj;
                        }
                    }
                }
    }
    free(head);
    free(next);
    free(cidx);
    /* harmonic bonds: V = k/2 (r - r0)^2 */
    for (int b = 0; b < S->n_bonds; b++) {
        int i = S->bond_idx[2 * b], j = S->bond_idx[2 * b + 1];
        double r[3], rr = 0;
        for (int d = 0; d < 3; d++) { r[d] = mimg(x[3 * j + d] - x[3 * i + d], L); rr += r[d] * r[d]; }
        rr = sqrt(rr);
        double dr = rr - S->bond_r0[b];
        e_b += 0.5 * S->bond_k[b] * dr * dr;
        double f = -S->bond_k[b] * dr / rr;   /* F_j = f * r */
        for (int d = 0; d < 3; d++) {
            F[3 * j + d] += f * r[d];
            F[3 * i + d] -= f * r[d];
            vir += r[d] * f * r[d];
        }
    }
    /* harmonic angles: V = k/2 (theta - theta0)^2 */
    for (int a = 0; a < S->n_angles; a++) {
        int i = S->angle_idx[3 * a], j = S->angle_idx[3 * a + 1], k = S->angle_idx[3 * a + 2];
        double u[3], v[3], uu = 0, vv = 0, uv = 0;
        for (int d = 0; d < 3; d++) {
            u[d] = mimg(x[3 * i + d] - x[3 * j + d], L);
            v[d] = mimg(x[3 * k + d] - x[3 * j + d], L);
            uu += u[d] * u[d]; vv += v[d] * v[d]; uv += u[d] * v[d];
        }
        double nu = sqrt(uu), nv = sqrt(vv);
        double c = uv / (nu * nv);
        if (c > 1) c = 1;
        if (c < -1) c = -1;
        double th = acos(c);
        double dth = th - S->angle_t0[a];
        e_a += 0.5 * S->angle_k[a] * dth * dth;
        double s = sqrt(1.0 - c * c);
        if (s < 1e-12) s = 1e-12;
        double dVdth = S->angle_k[a] * dth;
        /* dtheta/du = -(v/(|u||v|) - c u/|u|^2) / sin(theta) */
        double fi[3], fk[3];
        for (int d = 0; d < 3; d++) {
            double dcdu = v[d] / (nu * nv) - c * u[d] / uu;
            double dcdv = u[d] / (nu * nv) - c * v[d] / vv;
            fi[d] = dVdth * dcdu / s;   /* -dV/du = -dV/dth * dth/dc * dc/du, dth/dc = -1/s */
            fk[d] = dVdth * dcdv / s;
            F[3 * i + d] += fi[d];
            F[3 * k + d] += fk[d];
            F[3 * j + d] -= fi[d] + fk[d];
            vir += u[d] * fi[d] + v[d] * fk[d];
        }
    }
    /* periodic dihedrals: V = k (1 + cos(n phi - phi0)), IUPAC phi */
    for (int q = 0; q < S->n_dih; q++) {
        int i = S->dih_idx[4 * q], j = S->dih_idx[4 * q + 1], k = S->dih_idx[4 * q + 2], l = S->dih_idx[4 * q + 3];
        double b1[3], b2[3], b3[3];
        for (int d = 0; d < 3; d++) {
            b1[d] = mimg(x[3 * j + d] - x[3 * i + d], L);
            b2[d] = mimg(x[3 * k + d] - x[3 * j + d], L);
            b3[d] = mimg(x[3 * l + d] - x[3 * k + d], L);
        }
        double m1[3] = {b1[1] * b2[2] - b1[2] * b2[1], b1[2] * b2[0] - b1[0] * b2[2], b1[0] * b2[1] - b1[1] * b2[0]};
        double m2[3] = {b2[1] * b3[2] - b2[2] * b3[1], b2[2] * b3[0] - b2[0] * b3[2], b2[0] * b3[1] - b2[1] * b3[0]};
        double m1m1 = 0, m2m2 = 0, b2b2 = 0, m1m2 = 0, b1b2 = 0, b3b2 = 0, xx = 0;
        for (int d = 0; d < 3; d++) {
            m1m1 += m1[d] * m1[d]; m2m2 += m2[d] * m2[d]; b2b2 += b2[d] * b2[d];
            m1m2 += m1[d] * m2[d]; b1b2 += b1[d] * b2[d]; b3b2 += b3[d] * b2[d];
        }
        double nb2 = sqrt(b2b2);
        /* phi = atan2( |b2| b1 . m2, m1 . m2 ) */
        for (int d = 0; d < 3; d++) xx += b1[d] * m2[d];
        double phi = atan2(nb2 * xx, m1m2);
        double nn = (double)S->dih_n[q];
        e_d += S->dih_k[q] * (1.0 + cos(nn * phi - S->dih_phi0[q]));
        double dVdphi = -S->dih_k[q] * nn * sin(nn * phi - S->dih_phi0[q]);
        /* Bekker / Blondel-Karplus gradient */
        double fi[3], fl[3], fj[3], fk[3];
        for (int d = 0; d < 3; d++) {
            fi[d] = -dVdphi * (-nb2 / m1m1) * m1[d];
            fl[d] = -dVdphi * (nb2 / m2m2) * m2[d];
        }
        double p = b1b2 / b2b2, r_ = b3b2 / b2b2;
        for (int d = 0; d < 3; d++) {
            fj[d] = -fi[d] - p * fi[d] + r_ * fl[d];
            fk[d] = -fl[d] + p * fi[d] - r_ * fl[d];
            F[3 * i + d] += fi[d];
            F[3 * j + d] += fj[d];
            F[3 * k + d] += fk[d];
            F[3 * l + d] += fl[d];
        }
        /* virial with atom i as origin: sum (x_a - x_i) . F_a */
        for (int d = 0; d < 3; d++)
            vir += b1[d] * fj[d] + (b1[d] + b2[d]) * fk[d] + (b1[d] + b2[d] + b3[d]) * fl[d];
    }
    energies[0] = e_lj;
    energies[1] = e_b;
    energies[2] = e_a;
    energies[3] = e_d;
    energies[4] = vir;
    return 0;
}

/*
 * n_steps of the GPU path's physics integrator in FP64 (velocity Verlet
 * written as a kick-drift loop over half-step velocities):
 *   v_n      = v_{n-1/2} + F_n/m dt/2            (KE_n, T_n from v_n)
 *   v_{n+1/2}= lambda_n v_n + F_n/m dt/2,  lambda_n = Berendsen(T_{n-1}), lambda_0 = 1
 *   x_{n+1}  = x_n + v_{n+1/2} dt
 * x, v_half (n*3) updated in place; F must hold F(x) on entry and holds
 * F(x_final) on exit.  out_energies[step*8 + k] (nullable) gets LIMA_E_* of
 * every step n (energies at x_n, KE from v_n).
 */
int orc_phys_run(const orc_phys_sys* S, const double* mass, double dt, int n_steps, int thermostat, double t0,
                 double tau, double* x, double* v, double* F, double* t_prev_io, double* out_energies) {
    const int n = S->n;
    double en[5];
    double t_prev = t_prev_io ? *t_prev_io : -1.0;
    orc_phys_forces(S, x, F, en);
    const double R = 8.314462618;
    for (int step = 0; step < n_steps; step++) {
        double ke = 0;
        for (int i = 0; i < n; i++)
            for (int d = 0; d < 3; d++) {
                double vn = v[3 * i + d] + F[3 * i + d] / mass[i] * dt * 0.5;
                ke += 0.5 * mass[i] * vn * vn;
            }
        double temp = 2.0 * ke / (3.0 * n * R);
        double lambda = 1.0;
        if (thermostat == LIMA_THERMOSTAT_BERENDSEN && t_prev > 0)
            lambda = sqrt(1.0 + dt / tau * (t0 / t_prev - 1.0));
        if (out_energies) {
            double* o = &out_energies[step * LIMA_E_COUNT];
            o[LIMA_E_LJ] = en[0]; o[LIMA_E_BOND] = en[1]; o[LIMA_E_ANGLE] = en[2]; o[LIMA_E_DIHEDRAL] = en[3];
            o[LIMA_E_KINETIC] = ke; o[LIMA_E_VIRIAL] = en[4]; o[LIMA_E_TEMPERATURE] = temp;
            o[LIMA_E_TOTAL] = en[0] + en[1] + en[2] + en[3] + ke;
        }
        for (int i = 0; i < n; i++)
            for (int d = 0; d < 3; d++) {
                double vn = v[3 * i + d] + F[3 * i + d] / mass[i] * dt * 0.5;
                v[3 * i + d] = lambda * vn + F[3 * i + d] / mass[i] * dt * 0.5;
                x[3 * i + d] += v[3 * i + d] * dt;
            }
        t_prev = temp;
        orc_phys_forces(S, x, F, en);
    }
    if (t_prev_io) *t_prev_io = t_prev;
    return 0;
}

/*
 * Trajectory loss of the physics semantics (the definition the GPU adjoint
 * differentiates, include/lima_abi.h lima_loss):
 *   loss = (1/T) sum_{n=1..T} [ w_e U(x_n)/N + w_r sum_b (h_b(x_n) - target_b)^2 ]
 *   h_b(x) = (1/N) sum over non-excluded pairs i<j of B(r_ij/dr - b - 1/2),
 * B the quadratic B-spline (support |u| < 3/2), dr = r_max / n_bins.
 */
static double bspline2(double u) {
    u = fabs(u);
    if (u < 0.5) return 0.75 - u * u;
    if (u < 1.5) return 0.5 * (1.5 - u) * (1.5 - u);
    return 0.0;
}

int orc_phys_rdf(const orc_phys_sys* S, const double* x, int n_bins, double r_max, double* h) {
    const int n = S->n;
    const double L = S->box, dr = r_max / n_bins, sup = r_max + dr, sup2 = sup * sup;
    memset(h, 0, sizeof(double) * n_bins);
    int m = (int)floor(L / sup);
    if (m < 3) m = 1;
    const double cell = L / m;
    int* head = (int*)malloc(sizeof(int) * m * m * m);
    int* next = (int*)malloc(sizeof(int) * n);
    int* cidx = (int*)malloc(sizeof(int) * n);
    for (int k = 0; k < m * m * m; k++) head[k] = -1;
    for (int i = 0; i < n; i++) {
        int c[3];
        for (int d = 0; d < 3; d++) {
            double w = x[3 * i + d] - L * floor(x[3 * i + d] / L);
            c[d] = (int)(w / cell);
            if (c[d] >= m) c[d] = m - 1;
        }
        cidx[i] = (c[0] * m + c[1]) * m + c[2];
        next[i] = head[cidx[i]];
        head[cidx[i]] = i;
    }
    for (int i = 0; i < n; i++) {
        const int ci = cidx[i];
        const int cx = ci / (m * m), cy = (ci / m) % m, cz = ci % m;
        const int span = m >= 3 ? 1 : 0;
        for (int dx = -span; dx <= span; dx++)
            for (int dy = -span; dy <= span; dy++)
                for (int dz = -span; dz <= span; dz++) {
                    const int k = (((cx + dx + m) % m) * m + ((cy + dy + m) % m)) * m + ((cz + dz + m) % m);
                    for (int j = head[k]; j >= 0; j = next[j]) {
                        if (j <= i) continue;
                        double r2 = 0;
                        for (int d = 0; d < 3; d++) {
                            const double q = mimg(x[3 * j + d] - x[3 * i + d], L);
                            r2 += q * q;
                        }
                        if (r2 >= sup2 || excluded(S, i, j)) continue;
                        const double u = sqrt(r2) / dr;
                        const int b0 = (int)floor(u - 0.5) - 1;
                        for (int b = b0; b <= b0 + 3; b++)
                            if (b >= 0 && b < n_bins) h[b] += bspline2(u - b - 0.5);
                    }
                }
    }
    for (int b = 0; b < n_bins; b++) h[b] /= n;
    free(head);
    free(next);
    free(cidx);
    return 0;
}

/* NVE velocity Verlet (half-step velocities v) from x for n_steps; x and v
   are advanced in place; per_step (nullable) receives l(x_n), n = 1..T. */
double orc_phys_loss(const orc_phys_sys* S, const double* mass, double dt, int n_steps, double* x, double* v,
                     int n_bins, double r_max, double w_e, double w_r, const double* target, double* per_step) {
    const int n = S->n;
    double* F = (double*)malloc(sizeof(double) * 3 * n);
    double* h = (double*)malloc(sizeof(double) * n_bins);
    double en[5], total = 0.0;
    orc_phys_forces(S, x, F, en);
    for (int step = 0; step < n_steps; step++) {
        for (int i = 0; i < n; i++)
            for (int d = 0; d < 3; d++) {
                v[3 * i + d] += F[3 * i + d] / mass[i] * dt;
                x[3 * i + d] += v[3 * i + d] * dt;
            }
        orc_phys_forces(S, x, F, en);
        orc_phys_rdf(S, x, n_bins, r_max, h);
        double r = 0.0;
        for (int b = 0; b < n_bins; b++) {
            const double c = h[b] - (target ? target[b] : 0.0);
            r += c * c;
        }
        const double l = w_e * (en[0] + en[1] + en[2] + en[3]) / n + w_r * r;
        if (per_step) per_step[step] = l;
        total += l;
    }
    free(F);
    free(h);
    return total / n_steps;
}

long orc_sizeof(int which) {
    switch (which) {
        case 0: return (long)sizeof(lima_compound);
        case 1: return (long)sizeof(lima_compound_state);
        case 2: return (long)sizeof(lima_solvent);
        case 3: return (long)sizeof(lima_compound_bridge_compact);
        case 4: return (long)sizeof(lima_forcefield);
        case 5: return (long)sizeof(orc_phys_sys);
        default: return -1;
    }
}

/* ======================================================================= */
/* C. Headless rasterizer: restatement of Rasterizer.cu:150-251 (types,    */
/*    colours, radii, normalisation), the depth sort (Rasterizer.cu:254-  */
/*    293, here stable: equal depths keep slot order) and the display's    */
/*    back-to-front triangle-fan discs (DisplayV2.cpp:13-51) as an image.  */
/* ======================================================================= */

enum { RAS_NONE = 0, RAS_O = 1, RAS_C = 2, RAS_P = 3, RAS_N = 4, RAS_H = 5, RAS_SOL = 6 };

static void ras_color(int t, int* c) {                                  /* Rasterizer.cu:168-189 */
    static const int tab[7][3] = {{0xF2, 0xE5, 0xD9}, {0xE0, 0x20, 0x20}, {0x30, 0x10, 0x90}, {0xFC, 0xF7, 0x5E},
                                  {0x2E, 0x8B, 0x57}, {0xF1, 0xF1, 0xF1}, {0x03, 0xa9, 0xf4}};
    for (int q = 0; q < 3; q++) c[q] = (t >= 0 && t < 7) ? tab[t][q] : 0;
}

static float ras_radius(int t) {                                        /* Rasterizer.cu:191-213 */
    switch (t) {
        case RAS_H: return 0.04f;
        case RAS_C: return 0.1f;
        case RAS_N: return 0.1f;
        case RAS_O: return 0.12f;
        case RAS_SOL: return 0.08f;
        case RAS_P: return 0.15f;
        default: return 1.f;
    }
}

/* balls of n slots (positions n*3, kind = ATOM_TYPE per slot) sorted by pos.y */
int orc_render_balls(int n, const float* pos, const unsigned char* kind, float L, lima_render_ball* out) {
    lima_render_ball* tmp = (lima_render_ball*)malloc(sizeof(lima_render_ball) * (size_t)(n > 0 ? n : 1));
    lima_render_ball* src = (lima_render_ball*)malloc(sizeof(lima_render_ball) * (size_t)(n > 0 ? n : 1));
    if (!tmp || !src) return -1;
    for (int i = 0; i < n; i++) {
        const int t = kind[i];
        const float x = t == RAS_NONE ? 0.f : pos[3 * i], y = t == RAS_NONE ? 0.f : pos[3 * i + 1],
                    z = t == RAS_NONE ? 0.f : pos[3 * i + 2];
        lima_render_ball b;
        memset(&b, 0, sizeof b);
        int c[3];
        ras_color(t, c);
        const float rad = ras_radius(t) / (1.f + y * 0.001f);
        b.radius = 0.25f * rad;
        const double dl = (double)L;
        b.pos.x = (float)(((double)x / dl - 0.5) * 1.8);
        b.pos.y = (float)(((double)y / dl - 0.5) * 1.8);
        b.pos.z = (float)(((double)z / dl - 0.5) * 1.8);
        for (int q = 0; q < 3; q++) b.color[q] = c[q];
        b.disable = t == RAS_NONE;
        src[i] = b;
    }
    /* bottom-up merge sort by pos.y that takes the right run's element on a
       tie, as the reference's merge (Rasterizer.cu:254-271): equal depths end
       up in descending slot order */
    for (int w = 1; w < n; w *= 2) {
        for (int lo = 0; lo < n; lo += 2 * w) {
            int mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
            int a = lo, b = mid, k = lo;
            while (a < mid && b < hi) tmp[k++] = (src[a].pos.y < src[b].pos.y) ? src[a++] : src[b++];
            while (a < mid) tmp[k++] = src[a++];
            while (b < hi) tmp[k++] = src[b++];
        }
        lima_render_ball* sw = src;
        src = tmp;
        tmp = sw;
    }
    memcpy(out, src, sizeof(lima_render_ball) * (size_t)n);
    free(tmp);
    free(src);
    return 0;
}

static float ras_ndc_x(int px, int w) { return (float)(2 * px + 1) / (float)w + -1.f; }
static float ras_ndc_y(int py, int h) { return 1.f + -((float)(2 * py + 1) / (float)h); }

/* the sorted balls drawn back to front as shaded discs into w*h RGB */
int orc_render_image(const lima_render_ball* balls, int n, int w, int h, unsigned char* rgb) {
    int* win = (int*)malloc(sizeof(int) * (size_t)w * h);
    if (!win) return -1;
    for (size_t p = 0; p < (size_t)w * h; p++) win[p] = -1;
    for (int k = n - 1; k >= 0; k--) {
        const lima_render_ball b = balls[k];
        if (b.disable) continue;
        const float hw = 0.5f * (float)w, hh = 0.5f * (float)h;
        int x0 = (int)floorf((b.pos.x - b.radius + 1.f) * hw) - 1, x1 = (int)ceilf((b.pos.x + b.radius + 1.f) * hw) + 1;
        int y0 = (int)floorf((1.f - b.pos.z - b.radius) * hh) - 1, y1 = (int)ceilf((1.f - b.pos.z + b.radius) * hh) + 1;
        if (x0 < 0) x0 = 0;
        if (y0 < 0) y0 = 0;
        if (x1 > w - 1) x1 = w - 1;
        if (y1 > h - 1) y1 = h - 1;
        for (int py = y0; py <= y1; py++)
            for (int px = x0; px <= x1; px++) {
                const float dx = ras_ndc_x(px, w) + -b.pos.x, dy = ras_ndc_y(py, h) + -b.pos.z;
                if (dx * dx + dy * dy <= b.radius * b.radius) win[(size_t)py * w + px] = k;
            }
    }
    for (size_t p = 0; p < (size_t)w * h; p++) {
        unsigned char* o = rgb + 3 * p;
        if (win[p] < 0) {
            o[0] = o[1] = o[2] = 0;
            continue;
        }
        const lima_render_ball b = balls[win[p]];
        const float dy = ras_ndc_y((int)(p / (size_t)w), h) + -b.pos.z;
        const float light = 0.5f + 0.5f * (dy / b.radius);
        for (int q = 0; q < 3; q++) o[q] = (unsigned char)(int)floorf((float)b.color[q] * light);
    }
    free(win);
    return 0;
}
