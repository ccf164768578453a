"""ctypes front end of the CPU oracles.  TEST INFRASTRUCTURE: imported only by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.

* ``RefEngine`` — the reference's own Engine.cu built for the host
  (oracle/_ref/libref_lima.so, see oracle/build_ref.sh).
* ``ref_nlist`` / ``ref_step`` — the C restatement of the reference step path
  (oracle/lima_oracle.c, part A).
* ``PhysSystem`` / ``phys_forces`` / ``phys_run`` — FP64 physics oracle
  (oracle/lima_oracle.c, part B) over a flattened topology.
"""
from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np

from quantom_b200 import layout as L

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liblima_oracle.so"
REF_LIB = HERE / "_ref" / "libref_lima.so"
MAXP = L.MAX_COMPOUND_PARTICLES

_orc = None
_ref = None


def _p(a):
    return None if a is None else a.ctypes.data


def oracle_lib():
    global _orc
    if _orc is None:
        if not ORACLE_LIB.exists():
            raise RuntimeError(f"{ORACLE_LIB} missing: run `make -C oracle`")
        lib = ctypes.CDLL(str(ORACLE_LIB))
        vp, i, f, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
        lib.orc_ref_nlist.restype = i
        lib.orc_ref_nlist.argtypes = [f, f, i, vp, vp, i, vp, vp, vp, vp, i, vp, vp, i, vp, vp, i, vp, vp]
        lib.orc_ref_nlist_ss_cells.restype = i
        lib.orc_ref_nlist_ss_cells.argtypes = [f, f, i, vp, i, vp, vp]
        lib.orc_ref_step.restype = i
        lib.orc_ref_step.argtypes = [f, f, d, f, vp, i, vp, vp, i, vp, i, vp, vp, vp, i, vp, vp, i, vp, vp, vp, vp, vp]
        lib.orc_phys_forces.restype = i
        lib.orc_phys_forces.argtypes = [vp, vp, vp, vp]
        lib.orc_phys_run.restype = i
        lib.orc_phys_run.argtypes = [vp, vp, d, i, i, d, d, vp, vp, vp, vp, vp]
        lib.orc_phys_rdf.restype = i
        lib.orc_phys_rdf.argtypes = [vp, vp, i, d, vp]
        lib.orc_phys_loss.restype = d
        lib.orc_phys_loss.argtypes = [vp, vp, d, i, vp, vp, i, d, d, d, vp, vp]
        lib.orc_sizeof.restype = ctypes.c_long
        lib.orc_sizeof.argtypes = [i]
        _orc = lib
    return _orc


def ref_available() -> bool:
    return REF_LIB.exists()


def ref_lib():
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise RuntimeError(f"{REF_LIB} missing: run `bash oracle/build_ref.sh` where the reference sources exist")
        lib = ctypes.CDLL(str(REF_LIB))
        vp, i, f, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
        lib.ref_layout.restype = ctypes.c_long
        lib.ref_layout.argtypes = [i]
        lib.ref_create.restype = vp
        lib.ref_create.argtypes = [f, f, d, i]
        lib.ref_destroy.argtypes = [vp]
        lib.ref_last_error.restype = ctypes.c_char_p
        lib.ref_last_error.argtypes = [vp]
        lib.ref_set_threads.argtypes = [vp, i]
        lib.ref_load.restype = i
        lib.ref_load.argtypes = [vp, vp, i, vp, vp, i, vp, i, vp]
        lib.ref_update_nlists.restype = i
        lib.ref_update_nlists.argtypes = [vp]
        lib.ref_get_nlist_csr.restype = i
        lib.ref_get_nlist_csr.argtypes = [vp, i, vp, vp]
        lib.ref_set_nlist_csr.restype = i
        lib.ref_set_nlist_csr.argtypes = [vp, i, vp, vp]
        lib.ref_step.restype = i
        lib.ref_step.argtypes = [vp, i, f]
        lib.ref_get_state.restype = i
        lib.ref_get_state.argtypes = [vp, vp, vp, vp]
        lib.ref_get_forces.restype = i
        lib.ref_get_forces.argtypes = [vp, vp, vp]
        lib.ref_get_potE.restype = i
        lib.ref_get_potE.argtypes = [vp, vp]
        lib.ref_get_log.restype = i
        lib.ref_get_log.argtypes = [vp, vp, vp, vp, vp]
        lib.ref_get_step.restype = i
        lib.ref_get_step.argtypes = [vp]
        lib.ref_render.restype = i
        lib.ref_render.argtypes = [vp, vp]
        _ref = lib
    return _ref


def ref_cutoff_of(system) -> float:
    """The reference's CUTOFF constant for a workload whose physics cutoff is
    r_c: its lists use radius 2*CUTOFF (Engine.cu:198,264)."""
    return np.float32(system.spec.cutoff) / np.float32(2.0)


# ------------------------------------------------------------------------
class RefEngine:
    """The reference engine (host build) loaded with a System."""

    def __init__(self, system, n_threads: int = 1, cutoff: float | None = None):
        self.lib = ref_lib()
        self.system = system
        C = ref_cutoff_of(system) if cutoff is None else cutoff
        self.h = self.lib.ref_create(system.spec.box_len, C, system.spec.dt, n_threads)
        br = system.bridges if len(system.bridges) else None
        rc = self.lib.ref_load(self.h, _p(system.forcefield), system.n_compounds,
                               _p(system.compounds) if system.n_compounds else None,
                               _p(system.states) if system.n_compounds else None, system.n_solvents,
                               _p(system.solvents), len(system.bridges), _p(br))
        self._check(rc)

    def _check(self, rc):
        if rc < 0:
            raise RuntimeError("reference oracle: " + self.lib.ref_last_error(self.h).decode())
        return rc

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_threads(self, n):
        self.lib.ref_set_threads(self.h, n)

    def update_nlists(self):
        self._check(self.lib.ref_update_nlists(self.h))

    def nlist(self, which):
        n = self.system.n_compounds if which < 2 else self.system.n_solvents
        off = np.zeros(n + 1, np.int32)
        tot = self.lib.ref_get_nlist_csr(self.h, which, _p(off), None)
        ids = np.zeros(max(tot, 1), np.int32)
        self.lib.ref_get_nlist_csr(self.h, which, _p(off), _p(ids))
        return off, ids[:tot]

    def set_nlist(self, which, off, ids):
        off = np.ascontiguousarray(off, np.int32)
        ids = np.ascontiguousarray(ids if len(ids) else np.zeros(1), np.int32)
        self._check(self.lib.ref_set_nlist_csr(self.h, which, _p(off), _p(ids)))

    def step(self, n=1, thermostat_scalar=1.0):
        return self._check(self.lib.ref_step(self.h, n, thermostat_scalar))

    def state(self):
        s = self.system
        comps = np.zeros(s.n_compounds, L.Compound)
        st = np.zeros(s.n_compounds, L.CompoundState)
        sol = np.zeros(s.n_solvents, L.Solvent)
        self.lib.ref_get_state(self.h, _p(comps) if s.n_compounds else None, _p(st) if s.n_compounds else None,
                               _p(sol))
        return comps, st, sol

    def forces(self):
        s = self.system
        fc = np.zeros((s.n_compounds, MAXP, 3), np.float32)
        fs = np.zeros((s.n_solvents, 3), np.float32)
        self.lib.ref_get_forces(self.h, _p(fc) if s.n_compounds else None, _p(fs))
        return fc, fs

    def log(self):
        """The reference's logging buffers of its last step (traj_buffer,
        potE_buffer, outdata, data_GAN), in its slot order."""
        s = self.system
        tpu = s.n_compounds * MAXP + s.n_solvents
        pe = np.zeros(tpu, np.float64)
        tr = np.zeros((tpu, 3), np.float32)
        od = np.zeros(10, np.float32)
        gan = np.zeros((max(s.n_compounds, 1), MAXP, 3, 3), np.float32)
        self._check(self.lib.ref_get_log(self.h, _p(pe), _p(tr), _p(od), _p(gan)))
        return {"potE": pe, "traj": tr, "logdata": od, "train": gan[: s.n_compounds]}

    def render(self):
        """The reference Rasterizer's RenderBall list of the current box
        (its three kernels and merge sort, Rasterizer.cu:12-293)."""
        from quantom_b200 import layout as L
        s = self.system
        out = np.zeros(s.n_compounds * MAXP + s.n_solvents, L.RenderBall)
        self._check(self.lib.ref_render(self.h, _p(out)))
        return out

    def potE(self):
        s = self.system
        out = np.zeros(s.n_compounds * MAXP + s.n_solvents, np.float64)
        self._check(self.lib.ref_get_potE(self.h, _p(out)))
        return out


# ------------------------------------------------------------------------
def ref_nlist(system, prev_cc=None, cs_cap=6144, ss_cap=1024, sc_cap=64, cutoff=None, cells=False):
    """Reference-semantics lists after one update; dict of CSR (offsets, ids)."""
    lib = oracle_lib()
    s = system
    C = ref_cutoff_of(s) if cutoff is None else cutoff
    nc, ns = s.n_compounds, s.n_solvents
    cc_ids = np.zeros(max(nc, 1) * MAXP, np.int32)
    cc_cnt = np.zeros(max(nc, 1), np.int32)
    cs_ids = np.zeros(max(nc, 1) * cs_cap, np.int32)
    cs_cnt = np.zeros(max(nc, 1), np.int32)
    ss_ids = np.zeros(max(ns, 1) * ss_cap, np.int32)
    ss_cnt = np.zeros(max(ns, 1), np.int32)
    sc_ids = np.zeros(max(ns, 1) * sc_cap, np.int32)
    sc_cnt = np.zeros(max(ns, 1), np.int32)
    pcc = None
    if prev_cc is not None and nc:
        pcc = np.zeros((nc, nc), np.uint8)
        off, ids = prev_cc
        for c in range(nc):
            pcc[c, ids[off[c]:off[c + 1]]] = 1
    rc = lib.orc_ref_nlist(s.spec.box_len, C, nc, _p(s.compounds) if nc else None, _p(s.states) if nc else None,
                           ns, _p(s.solvents), _p(pcc), _p(cc_ids), _p(cc_cnt), cs_cap, _p(cs_ids), _p(cs_cnt),
                           0 if cells else ss_cap, _p(ss_ids), _p(ss_cnt), sc_cap, _p(sc_ids), _p(sc_cnt))
    if cells:
        rc2 = lib.orc_ref_nlist_ss_cells(s.spec.box_len, C, ns, _p(s.solvents), ss_cap, _p(ss_ids), _p(ss_cnt))
        rc = rc if rc2 == 0 else rc2
    if rc != 0:
        raise RuntimeError("oracle neighbour list overflow")

    def csr(ids, cnt, cap, n):
        off = np.zeros(n + 1, np.int64)
        off[1:] = np.cumsum(cnt[:n])
        flat = np.concatenate([ids[i * cap: i * cap + cnt[i]] for i in range(n)]) if n else np.zeros(0, np.int32)
        return off, flat.astype(np.int64)

    return {0: csr(cc_ids, cc_cnt, MAXP, nc), 1: csr(cs_ids, cs_cnt, cs_cap, nc),
            2: csr(sc_ids, sc_cnt, sc_cap, ns), 3: csr(ss_ids, ss_cnt, ss_cap, ns)}


def ref_step(system, lists, lam=1.0, cutoff=None):
    """One reference step with the given lists; returns (new System, forces_c,
    forces_s, potE)."""
    lib = oracle_lib()
    s = system.copy()
    C = ref_cutoff_of(s) if cutoff is None else cutoff
    nc, ns = s.n_compounds, s.n_solvents

    def fixed(which, cap, n):
        off, ids = lists[which]
        arr = np.zeros(max(n, 1) * cap, np.int32)
        cnt = np.zeros(max(n, 1), np.int32)
        for i in range(n):
            k = off[i + 1] - off[i]
            arr[i * cap: i * cap + k] = ids[off[i]:off[i + 1]]
            cnt[i] = k
        return arr, cnt

    cs_cap = max(1, int(max(np.diff(lists[1][0]).max(initial=0), 1)))
    ss_cap = max(1, int(max(np.diff(lists[3][0]).max(initial=0), 1)))
    cc_ids, cc_cnt = fixed(0, MAXP, nc)
    cs_ids, cs_cnt = fixed(1, cs_cap, nc)
    ss_ids, ss_cnt = fixed(3, ss_cap, ns)
    fc = np.zeros((max(nc, 1), MAXP, 3), np.float32)
    fs = np.zeros((max(ns, 1), 3), np.float32)
    pe = np.zeros(nc * MAXP + ns, np.float64)
    br = s.bridges if len(s.bridges) else None
    lib.orc_ref_step(s.spec.box_len, C, s.spec.dt, lam, _p(s.forcefield), nc, _p(s.compounds) if nc else None,
                     _p(s.states) if nc else None, ns, _p(s.solvents), len(s.bridges), _p(br), _p(cc_ids),
                     _p(cc_cnt), cs_cap, _p(cs_ids), _p(cs_cnt), ss_cap, _p(ss_ids), _p(ss_cnt), _p(fc), _p(fs),
                     _p(pe))
    return s, fc[:nc], fs[:ns], pe


# ------------------------------------------------------------------------
class _PhysSys(ctypes.Structure):
    vp = ctypes.c_void_p
    _fields_ = [("n", ctypes.c_int), ("box", ctypes.c_double), ("rc", ctypes.c_double), ("r_on", ctypes.c_double),
                ("sigma", vp), ("epsilon", vp), ("excl_off", vp), ("excl_ids", vp),
                ("n_bonds", ctypes.c_int), ("bond_idx", vp), ("bond_r0", vp), ("bond_k", vp),
                ("n_angles", ctypes.c_int), ("angle_idx", vp), ("angle_t0", vp), ("angle_k", vp),
                ("n_dih", ctypes.c_int), ("dih_idx", vp), ("dih_phi0", vp), ("dih_k", vp), ("dih_n", vp)]


class PhysSystem:
    """Flattened topology of a System: particle order = compound particles
    (compound by compound) then solvents; bonded terms and exclusions in
    global particle ids."""

    def __init__(self, system, rc=None, r_on=None):
        s = system
        ff = s.forcefield["particle_parameters"][0]
        nc = s.n_compounds
        npart = s.compounds["n_particles"].astype(np.int64) if nc else np.zeros(0, np.int64)
        base = np.concatenate([[0], np.cumsum(npart)]) if nc else np.zeros(1, np.int64)
        self.compound_base = base
        ncp = int(base[-1])
        n = ncp + s.n_solvents
        self.n = n
        self.n_compound_particles = ncp
        types = np.zeros(n, np.int64)
        x = np.zeros((n, 3))
        xprev = np.zeros((n, 3))
        for c in range(nc):
            k = int(npart[c])
            types[base[c]:base[c] + k] = s.compounds[c]["atom_types"][:k]
            x[base[c]:base[c] + k] = s.states[c]["positions"][:k]
            xprev[base[c]:base[c] + k] = s.compounds[c]["prev_positions"][:k]
        x[ncp:] = s.solvents["pos"]
        xprev[ncp:] = s.solvents["pos_tsub1"]
        self.types = types
        self.x = x
        self.xprev = xprev
        self.mass = ff["mass"][types].astype(np.float64)
        self.sigma = ff["sigma"][types].astype(np.float64)
        self.epsilon = ff["epsilon"][types].astype(np.float64)
        self.n_types = int(types.max()) + 1 if n else 1
        self.type_sigma = ff["sigma"][: self.n_types].astype(np.float64)
        self.type_epsilon = ff["epsilon"][: self.n_types].astype(np.float64)
        self.box = float(s.spec.box_len)
        self.rc = float(s.spec.cutoff if rc is None else rc)
        self.r_on = float(self.rc if r_on is None else r_on)
        # exclusions from LJ_Ignores
        excl = [[] for _ in range(n)]
        for c in range(nc):
            for t in range(int(npart[c])):
                ig = s.compounds[c]["lj_ignore_list"][t]
                for q in range(int(ig["n_ignores"])):
                    excl[base[c] + t].append(int(base[ig["compound_ids"][q]] + ig["local_ids"][q]))
        self.excl_off = np.zeros(n + 1, np.int32)
        self.excl_off[1:] = np.cumsum([len(e) for e in excl])
        self.excl_ids = np.array([j for e in excl for j in e] or [0], np.int32)
        bonds, angles, dihs = [], [], []
        for c in range(nc):
            cp = s.compounds[c]
            for b in cp["singlebonds"][: cp["n_singlebonds"]]:
                bonds.append((base[c] + b["atom_indexes"][0], base[c] + b["atom_indexes"][1], b["b0"], b["kb"]))
            for a in cp["anglebonds"][: cp["n_anglebonds"]]:
                ai = a["atom_indexes"]
                angles.append((base[c] + ai[0], base[c] + ai[1], base[c] + ai[2], a["theta_0"], a["k_theta"]))
            for dh in cp["dihedrals"][: cp["n_dihedrals"]]:
                di = dh["atom_indexes"]
                dihs.append((*(base[c] + di[k] for k in range(4)), dh["phi_0"], dh["k_phi"], dh["n"]))
        for br in s.bridges:
            g = [int(base[r["compound_id"]] + r["local_id_compound"]) for r in br["particle_refs"][: br["n_particles"]]]
            for b in br["singlebonds"][: br["n_singlebonds"]]:
                bonds.append((g[b["atom_indexes"][0]], g[b["atom_indexes"][1]], b["b0"], b["kb"]))
            for a in br["anglebonds"][: br["n_anglebonds"]]:
                ai = a["atom_indexes"]
                angles.append((g[ai[0]], g[ai[1]], g[ai[2]], a["theta_0"], a["k_theta"]))
            for dh in br["dihedrals"][: br["n_dihedrals"]]:
                di = dh["atom_indexes"]
                dihs.append((g[di[0]], g[di[1]], g[di[2]], g[di[3]], dh["phi_0"], dh["k_phi"], dh["n"]))
        self.bond_idx = np.array([b[:2] for b in bonds] or [(0, 0)], np.int32)
        self.bond_r0 = np.array([b[2] for b in bonds] or [0], np.float64)
        self.bond_k = np.array([b[3] for b in bonds] or [0], np.float64)
        self.n_bonds = len(bonds)
        self.angle_idx = np.array([a[:3] for a in angles] or [(0, 0, 0)], np.int32)
        self.angle_t0 = np.array([a[3] for a in angles] or [0], np.float64)
        self.angle_k = np.array([a[4] for a in angles] or [0], np.float64)
        self.n_angles = len(angles)
        self.dih_idx = np.array([d[:4] for d in dihs] or [(0, 0, 0, 0)], np.int32)
        self.dih_phi0 = np.array([d[4] for d in dihs] or [0], np.float64)
        self.dih_k = np.array([d[5] for d in dihs] or [0], np.float64)
        self.dih_n = np.array([d[6] for d in dihs] or [0], np.int32)
        self.n_dih = len(dihs)

    def _struct(self):
        st = _PhysSys()
        st.n, st.box, st.rc, st.r_on = self.n, self.box, self.rc, self.r_on
        for name in ("sigma", "epsilon", "excl_off", "excl_ids", "bond_idx", "bond_r0", "bond_k", "angle_idx",
                     "angle_t0", "angle_k", "dih_idx", "dih_phi0", "dih_k", "dih_n"):
            arr = np.ascontiguousarray(getattr(self, name))
            setattr(self, name, arr)
            setattr(st, name, arr.ctypes.data)
        st.n_bonds, st.n_angles, st.n_dih = self.n_bonds, self.n_angles, self.n_dih
        return st

    def velocities(self, dt):
        d = self.x - self.xprev
        d -= self.box * np.round(d / self.box)
        return d / dt

    def solvent_lj_on_compounds(self, x=None):
        """FP64 LJ force (same switched Lorentz-Berthelot form as orc_phys_forces)
        on every compound particle from the solvents alone: the reference's
        force_LJ_sol of a compound particle (Engine.cu:1034).  numpy, O(n_cp * n_s)."""
        x = np.asarray(self.x if x is None else x, np.float64)
        ncp = self.n_compound_particles
        F = np.zeros((ncp, 3))
        xs, sig_s, eps_s = x[ncp:], self.sigma[ncp:], self.epsilon[ncp:]
        rc2, ron2 = self.rc ** 2, self.r_on ** 2
        for i in range(ncp):
            r = xs - x[i]
            r -= self.box * np.round(r / self.box)
            r2 = (r * r).sum(1)
            m = r2 < rc2
            r, r2 = r[m], r2[m]
            sig = 0.5 * (self.sigma[i] + sig_s[m])
            eps = np.sqrt(self.epsilon[i] * eps_s[m])
            sr6 = (sig * sig / r2) ** 3
            v = 4 * eps * (sr6 * sr6 - sr6)
            dvdr_r = -24 * eps * (2 * sr6 * sr6 - sr6) / r2
            if self.r_on < self.rc:
                t = np.where(r2 > ron2, (rc2 - r2) / (rc2 - ron2), 1.0)
                sw = t ** 3 * (10 + t * (-15 + 6 * t))
                dsw_r = np.where(r2 > ron2, -60 * t * t * (1 - t) ** 2 / (rc2 - ron2), 0.0)
                dvdr_r = dvdr_r * sw + v * dsw_r
            F[i] = (dvdr_r[:, None] * r).sum(0)   # force on i = -dV/dr * (x_i - x_j)/r = dvdr_r * (x_j - x_i)
        return F

    def forces(self, x=None):
        x = np.ascontiguousarray(self.x if x is None else x, np.float64)
        F = np.zeros_like(x)
        en = np.zeros(5)
        st = self._struct()
        oracle_lib().orc_phys_forces(ctypes.byref(st), _p(x), _p(F), _p(en))
        return F, en

    # -- trajectory loss (the quantity lima_loss / lima_grad evaluate) ---------
    def term_types(self):
        """Bonded term types as lima_get_params orders them: per kind the
        distinct constant sets of the terms, (r0, k), (theta0, k), (phi0, k, n),
        in ascending order; returns [(type constants (n_types, 2|3), type of
        every term)] for bonds, angles, dihedrals."""
        out = []
        for keys, n in (((self.bond_r0, self.bond_k), self.n_bonds), ((self.angle_t0, self.angle_k), self.n_angles),
                        ((self.dih_phi0, self.dih_k, self.dih_n.astype(np.float64)), self.n_dih)):
            k = np.stack(keys, 1)[:n]
            if n == 0:
                out.append((np.zeros((0, k.shape[1])), np.zeros(0, np.int64)))
                continue
            u, inv = np.unique(k, axis=0, return_inverse=True)
            out.append((u, inv.reshape(-1)))
        return out

    def params(self):
        """theta in lima_get_params order: per-type sigma, per-type epsilon,
        bond / angle / dihedral scales (1 = as built), then (r0, k) per bond
        type, (theta0, k) per angle type, (phi0, k) per dihedral type."""
        tt = [u[:, :2].reshape(-1) for u, _ in self.term_types()]
        return np.concatenate([self.type_sigma, self.type_epsilon, [1.0, 1.0, 1.0], *tt])

    def with_params(self, theta):
        """A copy whose per-type LJ parameters and bonded constants follow
        theta: every term takes its type's r0 / theta0 / phi0 and the kind's
        scale times its type's k."""
        import copy
        theta = np.asarray(theta, np.float64)
        nt = self.n_types
        q = copy.copy(self)
        q.type_sigma = theta[:nt].copy()
        q.type_epsilon = theta[nt:2 * nt].copy()
        q.sigma = q.type_sigma[self.types]
        q.epsilon = q.type_epsilon[self.types]
        o = 2 * nt + 3
        for kind, ((u, inv), (c_name, k_name), n) in enumerate(zip(
                self.term_types(), (("bond_r0", "bond_k"), ("angle_t0", "angle_k"), ("dih_phi0", "dih_k")),
                (self.n_bonds, self.n_angles, self.n_dih))):
            tv = theta[o:o + 2 * len(u)].reshape(-1, 2)
            o += 2 * len(u)
            c = getattr(self, c_name).copy()
            k = getattr(self, k_name).copy()
            if n:
                c[:n] = tv[inv, 0]
                k[:n] = tv[inv, 1] * theta[2 * nt + kind]
            setattr(q, c_name, c)
            setattr(q, k_name, k)
        return q

    def rdf(self, n_bins, r_max, x=None):
        x = np.ascontiguousarray(self.x if x is None else x, np.float64)
        h = np.zeros(n_bins)
        st = self._struct()
        oracle_lib().orc_phys_rdf(ctypes.byref(st), _p(x), n_bins, r_max, _p(h))
        return h

    def loss(self, dt, n_steps, n_bins, r_max, w_energy, w_rdf, target=None, x=None, v=None):
        """FP64 loss over n_steps NVE steps from (x, v); returns (loss, per-step terms)."""
        x = np.ascontiguousarray((self.x if x is None else x).copy(), np.float64)
        v = np.ascontiguousarray((self.velocities(dt) if v is None else v).copy(), np.float64)
        per = np.zeros(n_steps)
        tg = np.ascontiguousarray(np.zeros(n_bins) if target is None else target, np.float64)
        st = self._struct()
        L = oracle_lib().orc_phys_loss(ctypes.byref(st), _p(np.ascontiguousarray(self.mass)), dt, n_steps, _p(x),
                                       _p(v), n_bins, r_max, w_energy, w_rdf, _p(tg), _p(per))
        return L, per

    def run(self, dt, n_steps, x=None, v=None, thermostat=0, t0=300.0, tau=1e-4, t_prev=-1.0):
        x = np.ascontiguousarray((self.x if x is None else x).copy(), np.float64)
        v = np.ascontiguousarray((self.velocities(dt) if v is None else v).copy(), np.float64)
        F = np.zeros_like(x)
        en = np.zeros((n_steps, 8))
        tp = ctypes.c_double(t_prev)
        st = self._struct()
        oracle_lib().orc_phys_run(ctypes.byref(st), _p(np.ascontiguousarray(self.mass)), dt, n_steps, thermostat,
                                  t0, tau, _p(x), _p(v), _p(F), ctypes.byref(tp), _p(en))
        return x, v, F, en


# ------------------------------------------------------------ rasterizer ---
def render_slots(system, comp_positions, sol_positions):
    """(positions n_slots*3 float32, ATOM_TYPE per slot) of a state in the
    reference's slot layout: compound c particle l at c*64 + l (empty slots
    NONE), solvents SOL after them."""
    from quantom_b200 import layout as L
    nc, ns = system.n_compounds, system.n_solvents
    pos = np.zeros((nc * 64 + ns, 3), np.float32)
    kind = np.zeros(nc * 64 + ns, np.uint8)
    for c in range(nc):
        k = int(system.compounds[c]["n_particles"])
        pos[c * 64: c * 64 + k] = comp_positions[c][:k]
        for l in range(k):
            t = int(system.compounds[c]["atom_color_types"][l])
            kind[c * 64 + l] = L.RENDER_TYPE_OF_COLOR[t] if t < 7 else 0
    pos[nc * 64:] = sol_positions
    kind[nc * 64:] = 6
    return pos, kind


def render_balls(pos, kind, box_len):
    """Oracle RenderBall list (lima_oracle.c part C), sorted by depth."""
    from quantom_b200 import layout as L
    lib = oracle_lib()
    n = len(kind)
    pos = np.ascontiguousarray(pos, np.float32)
    kind = np.ascontiguousarray(kind, np.uint8)
    out = np.zeros(n, L.RenderBall)
    lib.orc_render_balls.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p]
    if lib.orc_render_balls(n, _p(pos), _p(kind), float(box_len), _p(out)) != 0:
        raise MemoryError("orc_render_balls")
    return out


def render_image(balls, width, height):
    """Oracle image of sorted balls (lima_oracle.c part C), (h, w, 3) uint8."""
    lib = oracle_lib()
    balls = np.ascontiguousarray(balls)
    img = np.zeros((height, width, 3), np.uint8)
    lib.orc_render_image.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    if lib.orc_render_image(_p(balls), len(balls), int(width), int(height), _p(img)) != 0:
        raise MemoryError("orc_render_image")
    return img


# ------------------------------------------------------- reference input path --
REF_FFMAKER = HERE / "_ref" / "lima_ref_ffmaker"
REF_BOXDUMP = HERE / "_ref" / "lima_ref_boxdump"


def ref_input_available() -> bool:
    return REF_FFMAKER.exists() and REF_BOXDUMP.exists()


def ref_input_box(gro, top, prms):
    """The box the reference's own input path builds (LIMA_ForcefieldMaker,
    then ForceFieldMaker + CompoundBuilder + BoxBuilder as Environment.cpp:15-40
    does) from a conf.gro, topol.top and CHARMM parameter files, run in a
    temporary copy of the directory layout those programs expect.  Returns
    dict(forcefield, compounds, states, bridges, solvents) in the reference's
    dtypes.  The parameter files are given to the force-field maker in the
    order it reads them (par_all36_lipid, par_all36_na, par_all36m_prot)."""
    import shutil
    import subprocess
    import tempfile
    from quantom_b200 import layout as L
    names = ["par_all36_lipid.prm", "par_all36_na.prm", "par_all36m_prot.prm"]
    if [Path(p).name for p in prms] != names:
        raise ValueError(f"the reference's force-field maker reads exactly {names}")
    with tempfile.TemporaryDirectory() as tmp:
        t = Path(tmp)
        (t / "Simulation" / "Molecule").mkdir(parents=True)
        (t / "Simulation" / "Forcefield").mkdir(parents=True)
        (t / "a" / "b").mkdir(parents=True)
        shutil.copy(gro, t / "Simulation" / "Molecule" / "conf.gro")
        shutil.copy(top, t / "Simulation" / "Molecule" / "topol.top")
        for p in prms:
            shutil.copy(p, t / "Simulation" / "Forcefield" / Path(p).name)
        run = dict(cwd=t / "a" / "b", stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, check=True)
        subprocess.run([str(REF_FFMAKER)], **run)
        subprocess.run([str(REF_BOXDUMP), str(t / "box.bin")], **run)
        raw = (t / "box.bin").read_bytes()
    nc, nb, ns = np.frombuffer(raw[:12], np.int32)
    o = 12
    def take(dtype, n):
        nonlocal o
        a = np.frombuffer(raw[o:o + dtype.itemsize * n], dtype).copy()
        o += dtype.itemsize * n
        return a
    ff = take(L.ForceField, 1)
    comps = take(L.Compound, nc)
    states = take(L.CompoundState, nc)
    bridges = take(L.CompoundBridgeCompact, nb)
    sols = take(L.Solvent, ns)
    assert o == len(raw)
    return dict(forcefield=ff, compounds=comps, states=states, bridges=bridges, solvents=sols)
