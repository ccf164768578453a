"""Python host side of the B200 LIMA_MD step engine, over the C-ABI.

Mirrors the reference's driver-facing interface (Quantom/Quantom/Engine.cuh:
109-208, Environment.cpp:100-122): build an ``Engine`` for a box, call
``deviceMaster()`` / ``hostMaster()`` (or ``step(n)``) and read back
positions, forces, energies and neighbour lists.  Every call goes through
``liblima_b200.so``; there is no CPU fallback — constructing an Engine without
the built library or without a CUDA device raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

from . import layout as L

_LIB = None
# the library: LIMA_B200_LIB if set (e.g. a build variant), else the in-tree build
LIB_PATH = Path(os.environ.get("LIMA_B200_LIB") or Path(__file__).resolve().parent / "liblima_b200.so")

OK, ERR_ARGUMENT, ERR_CUDA, ERR_CAPACITY, ERR_STATE, ERR_NUMERIC, ERR_UNSUPPORTED = range(7)
SEMANTICS_REFERENCE, SEMANTICS_PHYSICS = 0, 1
PRECISION_FP32, PRECISION_MIXED = 0, 1
THERMOSTAT_NONE, THERMOSTAT_REFERENCE, THERMOSTAT_BERENDSEN = 0, 1, 2
NL_COMPOUND_COMPOUND, NL_COMPOUND_SOLVENT, NL_SOLVENT_COMPOUND, NL_SOLVENT_SOLVENT, NL_PAIR = 0, 1, 2, 3, 4
E_LJ, E_BOND, E_ANGLE, E_DIHEDRAL, E_KINETIC, E_VIRIAL, E_TEMPERATURE, E_TOTAL = range(8)
E_COUNT = 8
PROF_NAMES = ("total", "nlist", "bonded", "pair", "compound")
PROF_COUNT = len(PROF_NAMES)


class LimaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"lima status {status}: {message}")
        self.status = status


class LossSpec(ctypes.Structure):
    """lima_loss_spec (include/lima_abi.h)."""
    _fields_ = [("n_steps", ctypes.c_int), ("checkpoint_every", ctypes.c_int), ("n_bins", ctypes.c_int),
                ("r_max", ctypes.c_float), ("w_energy", ctypes.c_double), ("w_rdf", ctypes.c_double),
                ("rdf_target", ctypes.c_void_p)]


LOG_TRAJ, LOG_POTE, LOG_TRAIN = 1, 2, 4
LOG_DATA_FLOATS = 10


class LogParams(ctypes.Structure):
    """lima_log_params (include/lima_abi.h)."""
    _fields_ = [("every", ctypes.c_int), ("ring_frames", ctypes.c_int), ("flags", ctypes.c_int)]


class Params(ctypes.Structure):
    """lima_params (include/lima_abi.h)."""
    _fields_ = [("box_len", ctypes.c_float), ("cutoff", ctypes.c_float), ("ref_cutoff", ctypes.c_float),
                ("skin", ctypes.c_float), ("switch_on", ctypes.c_float), ("dt", ctypes.c_double),
                ("nlist_period", ctypes.c_int), ("semantics", ctypes.c_int), ("precision", ctypes.c_int),
                ("thermostat", ctypes.c_int), ("t_target", ctypes.c_double), ("tau_t", ctypes.c_double),
                ("thermostat_period", ctypes.c_int), ("energy_period", ctypes.c_int),
                ("solvent_list_capacity", ctypes.c_int), ("compound_list_capacity", ctypes.c_int),
                ("device", ctypes.c_int), ("stream", ctypes.c_void_p)]


def load_library():
    """Loads the in-tree liblima_b200.so (built by quantom_b200.build)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m quantom_b200.build`")
    lib = ctypes.CDLL(str(LIB_PATH))
    vp, i, u32, f, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_float, ctypes.c_double
    sigs = {
        "lima_default_params": (None, [vp]),
        "lima_create": (i, [vp, ctypes.POINTER(vp)]),
        "lima_destroy": (None, [vp]),
        "lima_last_error": (ctypes.c_char_p, [vp]),
        "lima_set_forcefield": (i, [vp, vp]),
        "lima_load_compounds": (i, [vp, vp, vp, i]),
        "lima_load_bridges": (i, [vp, vp, i]),
        "lima_load_solvents": (i, [vp, vp, u32]),
        "lima_finish_box": (i, [vp]),
        "lima_step": (i, [vp, i]),
        "lima_synchronize": (i, [vp]),
        "lima_get_compound_states": (i, [vp, vp, vp]),
        "lima_get_solvents": (i, [vp, vp]),
        "lima_get_positions": (i, [vp, vp, vp]),
        "lima_set_state": (i, [vp, vp, vp, vp]),
        "lima_get_forces": (i, [vp, vp, vp]),
        "lima_get_energies": (i, [vp, vp, vp]),
        "lima_compute_energies": (i, [vp]),
        "lima_build_nlist": (i, [vp]),
        "lima_get_nlist": (i, [vp, i, vp, vp, ctypes.POINTER(u32)]),
        "lima_set_nlist": (i, [vp, i, vp, vp]),
        "lima_set_thermostat_scalar": (i, [vp, f]),
        "lima_get_step": (i, [vp, ctypes.POINTER(ctypes.c_uint64)]),
        "lima_get_last_step_ms": (i, [vp, ctypes.POINTER(f)]),
        "lima_profile_steps": (i, [vp, i, vp]),
        "lima_get_rebuild_count": (i, [vp, ctypes.POINTER(ctypes.c_uint64)]),
        "lima_get_param_count": (i, [vp, ctypes.POINTER(i)]),
        "lima_get_param_layout": (i, [vp, vp]),
        "lima_get_bonded_types": (i, [vp, i, ctypes.POINTER(i), vp]),
        "lima_get_params": (i, [vp, vp]),
        "lima_set_params": (i, [vp, vp]),
        "lima_loss": (i, [vp, vp, ctypes.POINTER(d)]),
        "lima_grad": (i, [vp, vp, ctypes.POINTER(d), vp]),
        "lima_rdf": (i, [vp, i, f, vp]),
        "lima_get_kernel_launches": (i, [vp, ctypes.POINTER(ctypes.c_uint64)]),
        "lima_log_start": (i, [vp, vp]),
        "lima_log_stop": (i, [vp]),
        "lima_log_count": (i, [vp, ctypes.POINTER(ctypes.c_uint64)]),
        "lima_log_read": (i, [vp, ctypes.c_uint64, ctypes.c_uint64, vp, vp, vp, vp, vp, vp]),
        "lima_log_write": (i, [vp, ctypes.c_char_p]),
        "lima_render": (i, [vp, vp]),
        "lima_render_image": (i, [vp, i, i, vp]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def default_params(**kw) -> Params:
    lib = load_library()
    p = Params()
    lib.lima_default_params(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _ptr(a):
    return None if a is None else a.ctypes.data


class Engine:
    """Engine(Simulation*, ForceField) (Engine.cu:9-38) for a System."""

    def __init__(self, system, params: Params | None = None, **kw):
        self.lib = load_library()
        self.system = system
        if params is None:
            spec = system.spec
            params = default_params(box_len=spec.box_len, cutoff=spec.cutoff, dt=spec.dt)
        for k, v in kw.items():
            setattr(params, k, v)
        self.params = params
        h = ctypes.c_void_p()
        st = self.lib.lima_create(ctypes.byref(params), ctypes.byref(h))
        if st != OK:
            raise LimaError(st, "lima_create failed")
        self.h = h
        try:
            self._check(self.lib.lima_set_forcefield(self.h, _ptr(system.forcefield)))
            if system.n_compounds:
                self._check(self.lib.lima_load_compounds(self.h, _ptr(system.compounds), _ptr(system.states),
                                                         system.n_compounds))
            if len(system.bridges):
                self._check(self.lib.lima_load_bridges(self.h, _ptr(system.bridges), len(system.bridges)))
            self._check(self.lib.lima_load_solvents(self.h, _ptr(system.solvents), system.n_solvents))
            self._check(self.lib.lima_finish_box(self.h))
        except Exception:
            self.close()
            raise

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.lima_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        if st != OK:
            msg = self.lib.lima_last_error(self.h)
            raise LimaError(st, msg.decode() if msg else "")

    # -- reference driver interface ----------------------------------------
    def deviceMaster(self):
        """One step of forces + integration (Engine::deviceMaster, Engine.cu:44-47)."""
        self._check(self.lib.lima_step(self.h, 1))

    def hostMaster(self):
        """The reference's per-step host work (lists, thermostat) runs on the
        device inside lima_step; this only surfaces device-side errors."""
        self._check(self.lib.lima_synchronize(self.h))

    def step(self, n: int = 1):
        self._check(self.lib.lima_step(self.h, int(n)))

    def synchronize(self):
        self._check(self.lib.lima_synchronize(self.h))

    @property
    def current_step(self) -> int:
        v = ctypes.c_uint64()
        self._check(self.lib.lima_get_step(self.h, ctypes.byref(v)))
        return int(v.value)

    def last_step_ms(self) -> float:
        v = ctypes.c_float()
        self._check(self.lib.lima_get_last_step_ms(self.h, ctypes.byref(v)))
        return float(v.value)

    def profile_steps(self, n: int) -> dict:
        """Mean device ms per step of each kernel group over n steps
        (CUDA events on the engine's stream; Engine::timings)."""
        out = np.zeros(PROF_COUNT, np.float32)
        self._check(self.lib.lima_profile_steps(self.h, int(n), _ptr(out)))
        return {name: float(out[k]) for k, name in enumerate(PROF_NAMES)}

    def kernel_launches(self) -> int:
        v = ctypes.c_uint64()
        self._check(self.lib.lima_get_kernel_launches(self.h, ctypes.byref(v)))
        return int(v.value)

    # -- parameters, trajectory loss and its gradient (physics semantics) -----
    def param_count(self) -> int:
        n = ctypes.c_int()
        self._check(self.lib.lima_get_param_count(self.h, ctypes.byref(n)))
        return int(n.value)

    def param_layout(self) -> dict:
        """Entry counts of theta: n_types, n_bond_types, n_angle_types, n_dihedral_types."""
        c = np.zeros(4, np.int32)
        self._check(self.lib.lima_get_param_layout(self.h, _ptr(c)))
        return dict(zip(("n_types", "n_bond_types", "n_angle_types", "n_dihedral_types"), (int(x) for x in c)))

    def param_names(self) -> list:
        """A name for every entry of theta, in order."""
        lay = self.param_layout()
        nt = lay["n_types"]
        names = [f"sigma[{t}]" for t in range(nt)] + [f"epsilon[{t}]" for t in range(nt)]
        names += ["s_bond", "s_angle", "s_dihedral"]
        for kind, c in (("bond", "r0"), ("angle", "theta0"), ("dihedral", "phi0")):
            for q in range(lay[f"n_{kind}_types"]):
                names += [f"{kind}[{q}].{c}", f"{kind}[{q}].k"]
        return names

    def bonded_types(self, kind: int) -> np.ndarray:
        """Type of every term of a kind (0 bond, 1 angle, 2 dihedral), in load order."""
        n = ctypes.c_int()
        self._check(self.lib.lima_get_bonded_types(self.h, int(kind), ctypes.byref(n), None))
        out = np.zeros(n.value, np.int32)
        self._check(self.lib.lima_get_bonded_types(self.h, int(kind), ctypes.byref(n), _ptr(out)))
        return out

    def get_params(self) -> np.ndarray:
        """theta = [sigma per type, epsilon per type, bond / angle / dihedral scales,
        (r0, k) per bond type, (theta0, k) per angle type, (phi0, k) per dihedral type]
        (lima_get_params)."""
        th = np.zeros(self.param_count(), np.float64)
        self._check(self.lib.lima_get_params(self.h, _ptr(th)))
        return th

    def set_params(self, theta):
        th = np.ascontiguousarray(theta, np.float64)
        if th.shape != (self.param_count(),):
            raise ValueError(f"expected {self.param_count()} parameters")
        self._check(self.lib.lima_set_params(self.h, _ptr(th)))

    @staticmethod
    def loss_spec(n_steps, checkpoint_every, n_bins, r_max, w_energy, w_rdf, target=None):
        tg = None if target is None else np.ascontiguousarray(target, np.float64)
        spec = LossSpec(int(n_steps), int(checkpoint_every), int(n_bins), float(r_max), float(w_energy),
                        float(w_rdf), tg.ctypes.data if tg is not None else None)
        return spec, tg

    def loss(self, n_steps, checkpoint_every, n_bins, r_max, w_energy, w_rdf, target=None) -> float:
        spec, keep = self.loss_spec(n_steps, checkpoint_every, n_bins, r_max, w_energy, w_rdf, target)
        out = ctypes.c_double()
        self._check(self.lib.lima_loss(self.h, ctypes.byref(spec), ctypes.byref(out)))
        del keep
        return float(out.value)

    def grad(self, n_steps, checkpoint_every, n_bins, r_max, w_energy, w_rdf, target=None):
        """(loss, d loss / d theta) by the adjoint of the unrolled steps."""
        spec, keep = self.loss_spec(n_steps, checkpoint_every, n_bins, r_max, w_energy, w_rdf, target)
        out = ctypes.c_double()
        g = np.zeros(self.param_count(), np.float64)
        self._check(self.lib.lima_grad(self.h, ctypes.byref(spec), ctypes.byref(out), _ptr(g)))
        del keep
        return float(out.value), g

    def rdf(self, n_bins, r_max) -> np.ndarray:
        h = np.zeros(int(n_bins), np.float64)
        self._check(self.lib.lima_rdf(self.h, int(n_bins), float(r_max), _ptr(h)))
        return h

    def rebuild_count(self) -> int:
        """Physics semantics: pair-list builds since creation."""
        v = ctypes.c_uint64()
        self._check(self.lib.lima_get_rebuild_count(self.h, ctypes.byref(v)))
        return int(v.value)

    # -- frame log ---------------------------------------------------------
    def log_start(self, every: int, ring_frames: int = 64, flags: int = LOG_TRAJ | LOG_POTE | LOG_TRAIN):
        """Record the state of every `every`-th step: the reference's logging
        buffers (traj, potE, data_GAN, outdata) and per-step energies."""
        lp = LogParams(int(every), int(ring_frames), int(flags))
        self._check(self.lib.lima_log_start(self.h, ctypes.byref(lp)))
        self._log_flags = int(flags)

    def log_stop(self):
        self._check(self.lib.lima_log_stop(self.h))

    def log_count(self) -> int:
        v = ctypes.c_uint64()
        self._check(self.lib.lima_log_count(self.h, ctypes.byref(v)))
        return int(v.value)

    def log_read(self, first: int = 0, count: int | None = None) -> dict:
        """Frames [first, first+count) as arrays in the reference's indexing:
        traj (F, n_c*64 + n_s, 3), potE (F, n_c*64 + n_s), train
        (F, n_c, 64, 3, 3), energies (F, E_COUNT), logdata (F, 10), steps (F,)."""
        total = self.log_count()
        count = total - first if count is None else int(count)
        nc, ns = self.system.n_compounds, self.system.n_solvents
        slots = nc * L.MAX_COMPOUND_PARTICLES + ns
        flags = getattr(self, "_log_flags", 0)
        out = {"steps": np.zeros(count, np.uint64), "energies": np.zeros((count, E_COUNT), np.float64),
               "logdata": np.zeros((count, LOG_DATA_FLOATS), np.float32)}
        if flags & LOG_TRAJ:
            out["traj"] = np.zeros((count, slots, 3), np.float32)
        if flags & LOG_POTE:
            out["potE"] = np.zeros((count, slots), np.float64)
        if flags & LOG_TRAIN and nc:
            out["train"] = np.zeros((count, nc, L.MAX_COMPOUND_PARTICLES, 3, 3), np.float32)
        self._check(self.lib.lima_log_read(self.h, int(first), count, _ptr(out["steps"]), _ptr(out["energies"]),
                                           _ptr(out.get("traj")), _ptr(out.get("potE")), _ptr(out.get("train")),
                                           _ptr(out["logdata"])))
        return out

    def log_write(self, directory) -> None:
        """The recorded frames as the reference's output files (logdata.bin,
        energy.bin, temperature.bin, sim_traindata.bin, traj.bin, potE.bin)."""
        self._check(self.lib.lima_log_write(self.h, str(directory).encode()))

    # -- headless rasterizer -------------------------------------------------
    def render(self) -> np.ndarray:
        """RenderBall per particle slot of the current state, sorted by depth
        (Rasterizer::render, Rasterizer.cu:12-27)."""
        n = self.system.n_compounds * L.MAX_COMPOUND_PARTICLES + self.system.n_solvents
        balls = np.zeros(n, L.RenderBall)
        self._check(self.lib.lima_render(self.h, _ptr(balls)))
        return balls

    def render_image(self, width: int = 1080, height: int = 1080) -> np.ndarray:
        """The picture the reference's display draws of render(): (height,
        width, 3) uint8, row 0 at the top."""
        img = np.zeros((int(height), int(width), 3), np.uint8)
        self._check(self.lib.lima_render_image(self.h, int(width), int(height), _ptr(img)))
        return img

    # -- state ---------------------------------------------------------------
    def compound_states(self):
        n = self.system.n_compounds
        st = np.zeros(n, L.CompoundState)
        prev = np.zeros((n, L.MAX_COMPOUND_PARTICLES, 3), np.float32)
        if n:
            self._check(self.lib.lima_get_compound_states(self.h, _ptr(st), _ptr(prev)))
        return st, prev

    def solvents(self):
        s = np.zeros(self.system.n_solvents, L.Solvent)
        if len(s):
            self._check(self.lib.lima_get_solvents(self.h, _ptr(s)))
        return s

    def positions(self):
        """Flat float32 positions: compound slots (n_compounds, 64, 3), empty
        slots zero, and solvents (n_solvents, 3) (lima_get_positions)."""
        c = np.zeros((self.system.n_compounds, 64, 3), np.float32)
        s = np.zeros((self.system.n_solvents, 3), np.float32)
        self._check(self.lib.lima_get_positions(self.h, _ptr(c) if c.size else None, _ptr(s) if s.size else None))
        return c, s

    def set_state(self, states, prev_positions, solvents):
        self._check(self.lib.lima_set_state(self.h, _ptr(states), _ptr(prev_positions), _ptr(solvents)))

    def forces(self):
        nc = self.system.n_compounds
        fc = np.zeros((nc, L.MAX_COMPOUND_PARTICLES, 3), np.float32)
        fs = np.zeros((self.system.n_solvents, 3), np.float32)
        self._check(self.lib.lima_get_forces(self.h, _ptr(fc) if nc else None, _ptr(fs)))
        return fc, fs

    def energies(self, per_particle: bool = False):
        tot = np.zeros(E_COUNT, np.float64)
        pp = None
        if per_particle:
            pp = np.zeros(self.system.n_compounds * L.MAX_COMPOUND_PARTICLES + self.system.n_solvents, np.float64)
        self._check(self.lib.lima_get_energies(self.h, _ptr(tot), _ptr(pp)))
        return (tot, pp) if per_particle else tot

    def compute_energies(self):
        self._check(self.lib.lima_compute_energies(self.h))
        return self.energies()

    def set_thermostat_scalar(self, s: float):
        self._check(self.lib.lima_set_thermostat_scalar(self.h, float(s)))

    # -- neighbour lists -------------------------------------------------------
    def build_nlist(self):
        self._check(self.lib.lima_build_nlist(self.h))

    def nlist(self, which: int):
        """CSR (offsets, ids) of a neighbour list; NL_PAIR (physics): the Verlet
        list of every particle, compound particles first, then solvents."""
        if which == NL_PAIR:
            n = self.system.n_particles
        else:
            n = self.system.n_compounds if which in (NL_COMPOUND_COMPOUND, NL_COMPOUND_SOLVENT) else self.system.n_solvents
        off = np.zeros(n + 1, np.uint32)
        tot = ctypes.c_uint32()
        self._check(self.lib.lima_get_nlist(self.h, which, _ptr(off), None, ctypes.byref(tot)))
        ids = np.zeros(max(1, tot.value), np.uint32)
        self._check(self.lib.lima_get_nlist(self.h, which, _ptr(off), _ptr(ids), ctypes.byref(tot)))
        return off, ids[: tot.value]

    def set_nlist(self, which: int, offsets, ids):
        offsets = np.ascontiguousarray(offsets, np.uint32)
        ids = np.ascontiguousarray(ids if len(ids) else np.zeros(1), np.uint32)
        self._check(self.lib.lima_set_nlist(self.h, which, _ptr(offsets), _ptr(ids)))


def save_ppm(path, img: np.ndarray) -> None:
    """Writes an (h, w, 3) uint8 image as binary PPM."""
    h, w, _ = img.shape
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (w, h))
        f.write(np.ascontiguousarray(img, np.uint8).tobytes())


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def lib_built() -> bool:
    return LIB_PATH.exists()


os.environ.setdefault("LIMA_B200_LIB", str(LIB_PATH))
