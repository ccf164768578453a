"""Seeded synthetic systems in the reference LIMA_MD layout.

The workloads are the ones the benchmark names (no public dataset is
involved): single-site LJ solvent boxes and linear chains packed into
LIMA-style compounds of at most 64 particles, embedded in solvent.  Every
array is built in the reference's own struct layout (``layout.py``), the way
the reference's builders produce it:

* compounds as in ``CompoundBuilder`` (Quantom/Quantom/CompoundBuilder.cpp:7-48):
  per-compound bonded terms with compound-local atom indices, bonded LJ
  exclusions distributed to every pair of a bond/angle/dihedral
  (``distributeLJIgnores``, CompoundBuilder.cpp:307-318), key particle = the
  one nearest the centre of mass and confining sphere = the largest distance
  to it (``Compound::calcParticleSphere``, Bodies.cuh:407-423);
* terms spanning two compounds go to a ``CompoundBridgeCompact`` with
  bridge-local indices (``CompoundBridge::addBondParticles/localizeIDs``,
  Bodies.cuh:530-603);
* solvents as ``Solvent(pos, pos - v*dt)`` (``BoxBuilder::createSolvent``,
  BoxBuilder.cu:273-276), compounds likewise with ``prev_positions``.

Positions are uniform in the box conditioned on a 0.28 nm minimum separation
(hard-sphere Monte Carlo from a lattice, ``lima_builder_pack_spheres``);
velocities are Maxwell-Boltzmann with the centre-of-mass momentum removed.
"""
from __future__ import annotations

import ctypes
import math
from pathlib import Path
from dataclasses import dataclass, field

import numpy as np

from . import layout as L

R_GAS = 8.314462618  # J/(mol K)


@dataclass
class ChainSpec:
    n_chains: int
    chain_len: int
    bond_r0: float = 0.153            # nm
    bond_k: float = 2.5e8             # J/(mol nm^2)  (2.5e5 kJ/mol/nm^2)
    angle_theta0_deg: float = 111.0
    angle_k: float = 4.6e5            # J/(mol rad^2) (460 kJ/mol/rad^2)
    dihedral_n: int = 3
    dihedral_phi0: float = 0.0
    dihedral_k: float = 1.2e3         # J/mol        (1.2 kJ/mol)
    n_types: int = 4
    sigma_range: tuple = (0.25, 0.40)           # nm
    epsilon_range: tuple = (200.0, 1000.0)      # J/mol
    mass: float = 14.027e-3           # kg/mol (united-atom CH2)
    compound_size: int = 64           # particles per compound (the reference packs up to 64)


@dataclass
class SystemSpec:
    name: str
    box_len: float
    n_solvents: int
    cutoff: float = 1.2               # nm, physics cutoff (= 2 * reference CUTOFF)
    dt: float = 2e-6                  # ns
    temperature: float = 300.0
    min_sep: float = 0.28             # nm
    solvent_mass: float = 18e-3       # kg/mol
    solvent_sigma: float = 0.3166     # nm
    solvent_epsilon: float = 650.0    # J/mol
    chains: ChainSpec | None = None
    n_steps: int = 1000
    thermostat: str = "none"          # "none" | "berendsen"
    tau_t: float = 1e-4               # ns (0.1 ps)
    mc_sweeps: int = 30


@dataclass
class System:
    spec: SystemSpec
    seed: int
    forcefield: np.ndarray                 # ForceField, shape (1,)
    compounds: np.ndarray                  # Compound, (n_compounds,)
    states: np.ndarray                     # CompoundState, (n_compounds,)
    solvents: np.ndarray                   # Solvent, (n_solvents,)
    bridges: np.ndarray                    # CompoundBridgeCompact, (n_bridges,)
    info: dict = field(default_factory=dict)

    def with_state(self, states, prev_positions, solvents) -> "System":
        """The same topology with positions and previous positions from a
        readback (Engine.compound_states / Engine.solvents)."""
        import copy
        s = copy.copy(self)
        s.compounds = self.compounds.copy()
        s.states = self.states.copy()
        s.solvents = np.array(solvents, copy=True)
        for c in range(self.n_compounds):
            s.states[c]["positions"] = states[c]["positions"]
            s.compounds[c]["prev_positions"] = prev_positions[c]
        return s

    @property
    def n_compounds(self) -> int:
        return len(self.compounds)

    @property
    def n_solvents(self) -> int:
        return len(self.solvents)

    @property
    def n_particles(self) -> int:
        return int(self.compounds["n_particles"].sum()) + len(self.solvents)

    def copy(self) -> "System":
        return System(self.spec, self.seed, self.forcefield.copy(), self.compounds.copy(), self.states.copy(),
                      self.solvents.copy(), self.bridges.copy(), dict(self.info))


# Workloads of the benchmark (sizes, boxes and parameter distributions) and
# small variants of the same shape for CPU-sized parity tests.
CONFIGS = {
    "lj_solvent_4096": SystemSpec("lj_solvent_4096", 5.0, 4096, n_steps=1000),
    "solvated_chains_32k": SystemSpec("solvated_chains_32k", 10.0, 31000, chains=ChainSpec(16, 64), n_steps=5000,
                                      thermostat="berendsen"),
    "lj_solvent_8192": SystemSpec("lj_solvent_8192", 6.3, 8192, n_steps=200),
    "solvated_chains_258k": SystemSpec("solvated_chains_258k", 20.0, 250000, chains=ChainSpec(64, 128),
                                       n_steps=10000, mc_sweeps=12),
    # small cases, same densities and parameter distributions
    "tiny_solvent": SystemSpec("tiny_solvent", 3.0, 880),
    "tiny_chains": SystemSpec("tiny_chains", 4.0, 1900, chains=ChainSpec(2, 24)),
    "small_chains": SystemSpec("small_chains", 5.0, 3800, chains=ChainSpec(4, 40)),
    "small_bridged": SystemSpec("small_bridged", 5.0, 3700, chains=ChainSpec(2, 96)),
}


def _lib_builder(lib_path=None):
    """`lima_builder_pack_spheres` from the product library, or from the
    library at `lib_path` (the same builder.cpp compiled on its own for the
    host, so that a caller timing a CPU implementation builds identical inputs
    without loading any CUDA code)."""
    if lib_path is not None:
        lib = ctypes.CDLL(str(lib_path))
    else:
        from .engine import load_library
        lib = load_library()
    fn = lib.lima_builder_pack_spheres
    fn.restype = ctypes.c_long
    fn.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                   ctypes.c_ulonglong, ctypes.c_int, ctypes.c_void_p]
    return fn


def _grow_chain(rng, n, spec: ChainSpec, box, placed, min_sep, sig, placed_sig, max_tries=200):
    """Self-avoiding chain with fixed bond length and bond angle and a uniform
    random dihedral; non-bonded beads (|i-j| >= 4, and beads of earlier
    chains) stay at least max(min_sep, 0.95 sigma_ij) apart under the
    minimum image (sig: per-bead sigma of this chain)."""
    theta = math.radians(spec.angle_theta0_deg)
    b = spec.bond_r0
    for _attempt in range(1000):
        pts = np.zeros((n, 3))
        pts[0] = rng.uniform(0, box, 3)
        ok = True
        for i in range(1, n):
            for _t in range(max_tries):
                if i == 1:
                    v = rng.normal(size=3)
                    cand = pts[0] + b * v / np.linalg.norm(v)
                elif i == 2:
                    u = pts[0] - pts[1]
                    u /= np.linalg.norm(u)
                    w = rng.normal(size=3)
                    w -= w.dot(u) * u
                    w /= np.linalg.norm(w)
                    cand = pts[1] + b * (math.cos(theta) * u + math.sin(theta) * w)
                else:
                    # natural extension reference frame placement
                    a_, b_, c_ = pts[i - 3], pts[i - 2], pts[i - 1]
                    bc = c_ - b_
                    bc /= np.linalg.norm(bc)
                    nrm = np.cross(b_ - a_, bc)
                    nrm /= np.linalg.norm(nrm)
                    m = np.cross(nrm, bc)
                    phi = rng.uniform(0, 2 * math.pi)
                    d_loc = np.array([-b * math.cos(theta), b * math.sin(theta) * math.cos(phi),
                                      b * math.sin(theta) * math.sin(phi)])
                    cand = c_ + d_loc[0] * bc + d_loc[1] * m + d_loc[2] * nrm
                others = [pts[: max(0, i - 3)]]
                osig = [sig[: max(0, i - 3)]]
                if placed is not None and len(placed):
                    others.append(placed)
                    osig.append(placed_sig)
                oth = np.concatenate(others)
                if len(oth):
                    d = oth - cand
                    d -= box * np.round(d / box)
                    lim = np.maximum(min_sep, 0.95 * 0.5 * (np.concatenate(osig) + sig[i]))
                    if np.any(np.einsum("ij,ij->i", d, d) < lim * lim):
                        continue
                pts[i] = cand
                break
            else:
                ok = False
                break
        if ok:
            return pts
    raise RuntimeError("chain growth failed")


def _sphere(pos32: np.ndarray):
    """Key particle (nearest the centre of mass) and confining radius, in
    float32 as Compound::calcParticleSphere (Bodies.cuh:407-423) does."""
    n = len(pos32)
    com = np.zeros(3, np.float32)
    inv = np.float32(1.0) / np.float32(n)
    for i in range(n):
        com = (com + (pos32[i].astype(np.float64) * float(inv)).astype(np.float32)).astype(np.float32)
    d = np.sqrt(((pos32 - com) ** 2).sum(axis=1, dtype=np.float32)).astype(np.float32)
    return int(np.argmin(d)), float(d.max())


def _mb_velocities(rng, masses, temperature):
    v = rng.normal(size=(len(masses), 3)) * np.sqrt(R_GAS * temperature / masses)[:, None]
    p = (v * masses[:, None]).sum(axis=0)
    v -= p / masses.sum()
    return v


def make_system(name_or_spec, seed: int = 2024, packer_lib=None) -> System:
    """The seeded system `name_or_spec`.  packer_lib (optional): path of a
    host build of builder.cpp to pack the solvents with instead of the
    product library (bit-identical output)."""
    spec = CONFIGS[name_or_spec] if isinstance(name_or_spec, str) else name_or_spec
    rng = np.random.default_rng(seed)
    box = spec.box_len

    # ---- force field (type 0 = solvent) --------------------------------
    ff = np.zeros(1, L.ForceField)
    pp = ff["particle_parameters"][0]
    pp["mass"][:] = -1
    pp["sigma"][:] = -1
    pp["epsilon"][:] = -1
    pp[0] = (spec.solvent_mass, spec.solvent_sigma, spec.solvent_epsilon)
    cs = spec.chains
    if cs is not None:
        sig = rng.uniform(*cs.sigma_range, cs.n_types)
        eps = rng.uniform(*cs.epsilon_range, cs.n_types)
        for t in range(cs.n_types):
            pp[1 + t] = (cs.mass, sig[t], eps[t])

    # ---- chains --------------------------------------------------------
    # Rejection distance between two particles: the workload's 0.28 nm, or
    # 0.95 of the pair's Lorentz-Berthelot sigma where that is larger (chain
    # types go up to sigma 0.40 nm; a contact at 0.28 nm would start the
    # dynamics with ~1e7 J/(mol nm) forces).
    chain_pts = []
    chain_types = []
    placed = np.zeros((0, 3))
    placed_sig = np.zeros(0)
    sig_of = pp["sigma"].astype(np.float64)
    if cs is not None:
        for _c in range(cs.n_chains):
            types = rng.integers(1, 1 + cs.n_types, cs.chain_len)
            # the reference keeps every compound particle at the image nearest
            # its particle 0 (Engine.cu:996), which needs the box to exceed
            # twice a compound's extent (Constants.cuh:35): regrow otherwise
            for _try in range(200):
                pts = _grow_chain(rng, cs.chain_len, cs, box, placed, spec.min_sep, sig_of[types], placed_sig)
                ext = max(np.linalg.norm(pts[k:k + cs.compound_size] - pts[k], axis=1).max()
                          for k in range(0, cs.chain_len, cs.compound_size))
                if ext < 0.45 * box:
                    break
            else:
                raise RuntimeError("could not grow a chain that fits the reference's compound convention")
            chain_pts.append(pts)
            chain_types.append(types)
            placed = np.concatenate([placed, pts])
            placed_sig = np.concatenate([placed_sig, sig_of[types]])
    fixed = np.mod(placed, box) if len(placed) else np.zeros((0, 3))
    fixed_rmin = np.maximum(spec.min_sep, 0.95 * 0.5 * (placed_sig + spec.solvent_sigma))

    # ---- solvents --------------------------------------------------------
    out = np.zeros((spec.n_solvents, 3))
    pack = _lib_builder(packer_lib)
    fixed_c = np.ascontiguousarray(fixed, dtype=np.float64)
    fixed_r = np.ascontiguousarray(fixed_rmin if len(fixed_rmin) else np.zeros(1), dtype=np.float64)
    acc = pack(box, spec.min_sep, fixed_c.ctypes.data, fixed_r.ctypes.data, len(fixed_c), spec.n_solvents,
               int(rng.integers(0, 2**63)), spec.mc_sweeps, out.ctypes.data)
    if acc < 0:
        raise RuntimeError("solvent packing failed")

    # ---- velocities ------------------------------------------------------
    n_chain_atoms = sum(len(p) for p in chain_pts)
    masses = np.concatenate([np.full(n_chain_atoms, cs.mass if cs else 0.0),
                             np.full(spec.n_solvents, spec.solvent_mass)])
    vel = _mb_velocities(rng, masses, spec.temperature)
    v_chain, v_sol = vel[:n_chain_atoms], vel[n_chain_atoms:]

    solvents = np.zeros(spec.n_solvents, L.Solvent)
    solvents["pos"] = out.astype(np.float32)
    solvents["pos_tsub1"] = (out - v_sol * spec.dt).astype(np.float32)

    # ---- compounds and bridges -------------------------------------------
    compounds, states, bridges = _pack_chains(chain_pts, chain_types, v_chain, cs, spec, box)
    info = {"mc_accepted": int(acc), "n_chain_atoms": n_chain_atoms}
    return System(spec, seed, ff, compounds, states, solvents, bridges, info)


def _pack_chains(chain_pts, chain_types, v_chain, cs, spec, box):
    if cs is None or not chain_pts:
        return (np.zeros(0, L.Compound), np.zeros(0, L.CompoundState), np.zeros(0, L.CompoundBridgeCompact))
    per = cs.compound_size
    comp_list, state_list, bridge_list = [], [], []
    vofs = 0
    for pts, types in zip(chain_pts, chain_types):
        n = len(pts)
        v = v_chain[vofs: vofs + n]
        vofs += n
        n_comp = (n + per - 1) // per
        base_cid = len(comp_list)
        # atom a -> (compound id, local id)
        cid = base_cid + np.arange(n) // per
        lid = np.arange(n) % per
        comps = np.zeros(n_comp, L.Compound)
        sts = np.zeros(n_comp, L.CompoundState)
        for k in range(n_comp):
            a0, a1 = k * per, min(n, (k + 1) * per)
            seg = pts[a0:a1].copy()
            # particle 0 of the compound inside the box, the rest unwrapped next to it
            shift = np.floor(seg[0] / box) * box
            seg -= shift
            seg32 = seg.astype(np.float32)
            c = comps[k]
            c["n_particles"] = a1 - a0
            c["prev_positions"][: a1 - a0] = (seg - v[a0:a1] * spec.dt).astype(np.float32)
            c["atom_types"][: a1 - a0] = types[a0:a1]
            c["atom_color_types"][: a1 - a0] = types[a0:a1]
            c["particle_global_ids"][: a1 - a0] = np.arange(a0, a1)
            key, rad = _sphere(seg32)
            c["key_particle_index"] = key
            c["confining_particle_sphere"] = rad
            c["center_of_mass"] = seg32.mean(axis=0)
            sts[k]["positions"][: a1 - a0] = seg32
            sts[k]["n_particles"] = a1 - a0
        # bonded terms (topology order: bonds, angles, dihedrals)
        terms = ([("bond", (i, i + 1)) for i in range(n - 1)] +
                 [("angle", (i, i + 1, i + 2)) for i in range(n - 2)] +
                 [("dihedral", (i, i + 1, i + 2, i + 3)) for i in range(n - 3)])
        bridges = {}   # one CompoundBridge per pair of compounds (CompoundBridgeBundle::addBridge)
        for kind, atoms in terms:
            cids = {int(cid[a]) for a in atoms}
            # bonded LJ exclusions (distributeLJIgnores)
            for a in atoms:
                for b_ in atoms:
                    if a == b_:
                        continue
                    ig = comps[cid[a] - base_cid]["lj_ignore_list"][lid[a]]
                    nig = int(ig["n_ignores"])
                    if any(ig["local_ids"][q] == lid[b_] and ig["compound_ids"][q] == cid[b_] for q in range(nig)):
                        continue
                    if nig >= L.LJ_IGNORES_MAX:
                        raise RuntimeError("too many LJ ignores")
                    ig["local_ids"][nig] = lid[b_]
                    ig["compound_ids"][nig] = cid[b_]
                    ig["n_ignores"] = nig + 1
            if len(cids) == 1:
                c = comps[cid[atoms[0]] - base_cid]
                loc = [int(lid[a]) for a in atoms]
                if kind == "bond":
                    i = int(c["n_singlebonds"]); c["n_singlebonds"] = i + 1
                    c["singlebonds"][i] = (cs.bond_r0, cs.bond_k, loc)
                elif kind == "angle":
                    i = int(c["n_anglebonds"]); c["n_anglebonds"] = i + 1
                    c["anglebonds"][i] = (math.radians(cs.angle_theta0_deg), cs.angle_k, loc)
                else:
                    i = int(c["n_dihedrals"]); c["n_dihedrals"] = i + 1
                    c["dihedrals"][i] = (cs.dihedral_phi0, cs.dihedral_k, cs.dihedral_n, loc)
            else:
                if len(cids) > 2:
                    raise RuntimeError("term spans more than two compounds")
                key = tuple(sorted(cids))
                bridge = bridges.setdefault(key, {"refs": [], "types": [], "bonds": [], "angles": [], "dihedrals": []})
                loc = []
                for a in atoms:
                    ref = (int(cid[a]), int(lid[a]))
                    if ref not in bridge["refs"]:
                        bridge["refs"].append(ref)
                        bridge["types"].append(int(types[a]))
                    loc.append(bridge["refs"].index(ref))
                bridge[{"bond": "bonds", "angle": "angles", "dihedral": "dihedrals"}[kind]].append(loc)
        for key in sorted(bridges):
            bridge = bridges[key]
            br = np.zeros(1, L.CompoundBridgeCompact)[0]
            if len(bridge["refs"]) > L.MAX_PARTICLES_IN_BRIDGE:
                raise RuntimeError("too many particles in bridge")
            br["n_particles"] = len(bridge["refs"])
            for i, (c_, l_) in enumerate(bridge["refs"]):
                br["particle_refs"][i] = (c_, l_)
                br["atom_types"][i] = bridge["types"][i]
            br["n_singlebonds"] = len(bridge["bonds"])
            for i, loc in enumerate(bridge["bonds"]):
                br["singlebonds"][i] = (cs.bond_r0, cs.bond_k, loc)
            br["n_anglebonds"] = len(bridge["angles"])
            for i, loc in enumerate(bridge["angles"]):
                br["anglebonds"][i] = (math.radians(cs.angle_theta0_deg), cs.angle_k, loc)
            br["n_dihedrals"] = len(bridge["dihedrals"])
            for i, loc in enumerate(bridge["dihedrals"]):
                br["dihedrals"][i] = (cs.dihedral_phi0, cs.dihedral_k, cs.dihedral_n, loc)
            bridge_list.append(br)
        comp_list.extend(list(comps))
        state_list.extend(list(sts))
    if len(comp_list) > L.MAX_COMPOUNDS:
        raise RuntimeError("more compounds than the reference layout holds")
    def pack(items, dt):   # zero-initialised so padding bytes are deterministic
        out = np.zeros(len(items), dt)
        for i, it in enumerate(items):
            out[i] = it
        return out

    return pack(comp_list, L.Compound), pack(state_list, L.CompoundState), pack(bridge_list, L.CompoundBridgeCompact)


# --------------------------------------------------------- real topology ---
class TopologyOptions(ctypes.Structure):
    """lima_topology_options (include/lima_abi.h)."""
    _fields_ = [("box_len", ctypes.c_float), ("min_residue_id", ctypes.c_int), ("max_residue_id", ctypes.c_int),
                ("ignore_hydrogens", ctypes.c_int), ("solvate", ctypes.c_int), ("dt", ctypes.c_double),
                ("temperature", ctypes.c_double), ("seed", ctypes.c_uint64)]


def topology_options(**kw) -> TopologyOptions:
    lib = _lib_topology()
    o = TopologyOptions()
    lib.lima_topology_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _lib_topology():
    from .engine import load_library
    lib = load_library()
    vp = ctypes.c_void_p
    lib.lima_topology_default_options.argtypes = [vp]
    lib.lima_topology_default_options.restype = None
    lib.lima_topology_build.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                                        vp, ctypes.POINTER(vp)]
    lib.lima_topology_build.restype = ctypes.c_int
    lib.lima_topology_error.argtypes = [vp]
    lib.lima_topology_error.restype = ctypes.c_char_p
    lib.lima_topology_sizes.argtypes = [vp, vp, vp, vp, vp]
    lib.lima_topology_export.argtypes = [vp, vp, vp, vp, vp, vp]
    lib.lima_topology_destroy.argtypes = [vp]
    lib.lima_topology_destroy.restype = None
    return lib


def from_topology(gro, top, prms, options: TopologyOptions | None = None, name: str = "topology",
                  cutoff: float = 1.4) -> System:
    """A box from a GROMACS conf.gro + topol.top and CHARMM parameter files
    through lima_topology_build (the reference's force-field maker, compound
    builder and box builder in one native pass).  cutoff is the physics cutoff
    r_c; the reference semantics use r_c / 2 as their CUTOFF (the demo's 0.7 nm
    for the default 1.4)."""
    lib = _lib_topology()
    opt = options if options is not None else topology_options()
    arr = (ctypes.c_char_p * len(prms))(*[str(p).encode() for p in prms])
    h = ctypes.c_void_p()
    st = lib.lima_topology_build(str(gro).encode(), str(top).encode(), arr, len(prms), ctypes.byref(opt),
                                 ctypes.byref(h))
    try:
        if st != 0:
            raise RuntimeError(f"lima_topology_build status {st}: {lib.lima_topology_error(h).decode()}")
        nc, nb, nt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ns = ctypes.c_uint32()
        lib.lima_topology_sizes(h, ctypes.byref(nc), ctypes.byref(nb), ctypes.byref(ns), ctypes.byref(nt))
        ff = np.zeros(1, L.ForceField)
        comps = np.zeros(nc.value, L.Compound)
        states = np.zeros(nc.value, L.CompoundState)
        bridges = np.zeros(nb.value, L.CompoundBridgeCompact)
        sols = np.zeros(ns.value, L.Solvent)
        ptr = lambda a: a.ctypes.data if a.size else None
        st = lib.lima_topology_export(h, ptr(ff), ptr(comps), ptr(states), ptr(bridges), ptr(sols))
        if st != 0:
            raise RuntimeError(f"lima_topology_export status {st}")
    finally:
        lib.lima_topology_destroy(h)
    spec = SystemSpec(name, float(opt.box_len), int(ns.value), cutoff=cutoff, dt=float(opt.dt),
                      temperature=float(opt.temperature))
    return System(spec, int(opt.seed), ff, comps, states, sols, bridges,
                  {"n_atom_types": nt.value, "n_compound_particles": int(comps["n_particles"].sum())})


SIXLZM_FIXTURE = Path(__file__).resolve().parents[1] / "tests" / "golden" / "golden_6lzm.npz"


def load_6lzm(path=None) -> System:
    """The reference's 6LZM demo box (T4 lysozyme heavy atoms in 36 compounds
    and 35 bridges, 5,000 single-site waters, 7 nm box), as its own input path
    built it (tests/golden/make_6lzm.py); the native builder reproduces it from
    the same files.  Settings of the reference's run: CUTOFF 0.7 nm (physics
    cutoff 1.4), dt 0.1 fs (Constants.cuh:35,52; Simulation.cuh:152)."""
    d = np.load(SIXLZM_FIXTURE if path is None else path)
    spec = SystemSpec("6lzm", 7.0, int(len(d["solvents"])), cutoff=1.4, dt=1e-7, temperature=313.0)
    return System(spec, 0, d["forcefield"].copy(), d["compounds"].copy(), d["states"].copy(), d["solvents"].copy(),
                  d["bridges"].copy(), {"n_compound_particles": int(d["compounds"]["n_particles"].sum())})
