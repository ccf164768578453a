"""GPU physics semantics against the FP64 oracle (oracle/lima_oracle.c part B).

The physics path evaluates the conservative forces of the same model
(Lorentz-Berthelot LJ with a 1.2 nm cutoff and a potential switch from 1.0 nm,
harmonic bonds and angles, periodic dihedrals) in FP32 (plain) or FP32 with
compensated sums and FP64 reductions (mixed).  Stated errors: forces within
5e-5 relative RMS of FP64 (FP32 positions in a 10 nm box quantise distances
at ~1e-6 nm), energies within 1e-5 relative, trajectories within 1e-5 nm
over 20 steps.
"""
import functools

import numpy as np
import pytest

from conftest import make_named, relrms
from oracle import pyoracle as po
from quantom_b200 import systems as S

pytestmark = pytest.mark.gpu


def _params(E, s, **kw):
    p = E.default_params(box_len=s.spec.box_len, cutoff=s.spec.cutoff, dt=s.spec.dt, semantics=E.SEMANTICS_PHYSICS,
                         skin=0.1, switch_on=1.0, nlist_period=10)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _flat(s, fc, fs):
    parts = [fc[c, : s.compounds[c]["n_particles"]] for c in range(s.n_compounds)]
    return np.concatenate(parts + [fs]) if parts else fs


def _positions(E, eng, s):
    st, _ = eng.compound_states()
    sol = eng.solvents()
    parts = [st[c]["positions"][: s.compounds[c]["n_particles"]] for c in range(s.n_compounds)]
    return np.concatenate(parts + [sol["pos"]]) if parts else sol["pos"]


@functools.lru_cache(maxsize=2)
def _system_and_fp64_forces(name, seed, raw=False):
    """The FP64 oracle at the positions the engine holds.  Plain FP32: the
    loader wraps every coordinate into [0, L) and rounds it to FP32 (compound
    particles of bridged chains start outside the box), which moves the forces
    of the raw input by up to 3.9e-4 relative RMS; the bar is on the
    evaluation, not on that rounding.  Mixed precision (raw=True) keeps the
    rounding residual in its low words, so its state is the input itself."""
    s = make_named(name, seed)
    ps = po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0)
    F64, en64 = ps.forces() if raw else ps.forces(_wrapped_f32(s).astype(np.float64))
    return s, F64, en64


# solvated_chains_258k: 64 chains of 128 particles (two compounds and a bridge
# each) in 250,000 solvents, beyond the reference's 65,535-solvent layout
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["tiny_chains", "small_bridged", "lj_solvent_4096", "solvated_chains_32k",
                                  "solvated_chains_258k", "6lzm", "small_bridged_dry"])
def test_forces_and_energies_match_fp64(gpu, name, precision):
    E = gpu
    s, F64, en64 = _system_and_fp64_forces(name, 7, raw=precision == E.PRECISION_MIXED)
    with E.Engine(s, _params(E, s, precision=precision)) as eng:
        tot = eng.compute_energies()
        fc, fs = eng.forces()
    F = _flat(s, fc, fs)
    # solvated_chains_258k: FP32 coordinates in a 20 nm box round at 1.9e-6 nm
    # inside the FP32 arithmetic too (minimum images, differences): 5e-5.
    # *_dry (no solvent): the forces are the stiff bonds' (k 2.5e8 J/(mol nm^2)),
    # whose FP32 bond vectors at ~5 nm from the origin carry 2.4e-7 nm of
    # rounding, ~60 J/(mol nm) against bond forces of ~1e6: measured 7.6e-5
    tol = 5e-5 if name == "solvated_chains_258k" else (1e-4 if name.endswith("_dry") else 1e-5)
    err = relrms(F, F64)
    assert err < tol, err
    scale = abs(en64[0]) + abs(en64[3])
    assert abs(tot[E.E_LJ] - en64[0]) < 1e-5 * scale
    for k, q in ((E.E_BOND, 1), (E.E_ANGLE, 2), (E.E_DIHEDRAL, 3)):
        assert abs(tot[k] - en64[q]) < 1e-5 * scale
    # the virial of a box with no solvent is a sum of large intra-chain pair terms
    # that mostly cancel (and takes the FP32 face-crossing pairs above): 3e-4 there
    assert abs(tot[E.E_VIRIAL] - en64[4]) < (3e-4 if name.endswith("_dry") else 1e-5) * abs(en64[4])


@pytest.mark.parametrize("name", ["tiny_chains", "small_bridged", "lj_solvent_4096"])
@pytest.mark.parametrize("precision", [0, 1])
def test_trajectory_matches_fp64(gpu, name, precision):
    E = gpu
    s = S.make_system(name, seed=7)
    ps = po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0)
    x64, _, _, _ = ps.run(s.spec.dt, 20)
    with E.Engine(s, _params(E, s, precision=precision)) as eng:
        eng.step(20)
        x = _positions(E, eng, s)
    d = x - x64
    d -= s.spec.box_len * np.round(d / s.spec.box_len)
    assert np.abs(d).max() < 1e-5


def test_energy_step_matches_oracle_run(gpu):
    """Energies evaluated inside lima_step (energy_period) equal the oracle's
    energies along the same velocity-Verlet trajectory."""
    E = gpu
    s = S.make_system("tiny_chains", seed=3)
    ps = po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0)
    _, _, _, en = ps.run(s.spec.dt, 11)
    with E.Engine(s, _params(E, s, precision=1, energy_period=10)) as eng:
        eng.step(11)          # energies of step 10 (before its kick-drift)
        tot = eng.energies()
    ref = en[10]
    assert abs(tot[E.E_TOTAL] - ref[E.E_TOTAL]) < 1e-5 * abs(ref[E.E_KINETIC])
    assert abs(tot[E.E_KINETIC] - ref[E.E_KINETIC]) < 1e-6 * ref[E.E_KINETIC]


def test_berendsen_drives_temperature(gpu):
    E = gpu
    s = S.make_system("lj_solvent_4096", seed=5)
    with E.Engine(s, _params(E, s, thermostat=E.THERMOSTAT_BERENDSEN, t_target=250.0, tau_t=1e-4)) as eng:
        eng.step(600)
        T = eng.energies()[E.E_TEMPERATURE]
    assert abs(T - 250.0) < 15.0


def test_stale_list_is_reported(gpu):
    E = gpu
    s = S.make_system("tiny_solvent", seed=5)
    with E.Engine(s, _params(E, s, skin=0.002, nlist_period=1000)) as eng:
        eng.step(50)
        with pytest.raises(E.LimaError) as ei:
            eng.synchronize()
    assert "stale" in str(ei.value)


def test_deterministic_across_runs(gpu):
    E = gpu
    s = S.make_system("small_bridged", seed=9)
    out = []
    for _ in range(2):
        with E.Engine(s, _params(E, s)) as eng:
            eng.step(25)
            out.append(_positions(E, eng, s))
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("precision", [0, 1])
def test_deterministic_with_berendsen_and_rebuilds(gpu, precision):
    """The Berendsen scalar comes from the FP64 kinetic energy, summed per
    block in a fixed order and over the blocks in block order: two runs with
    the thermostat on and on-demand list rebuilds give bit-identical states
    and energies."""
    E = gpu
    s = S.make_system("small_chains", seed=11)
    out, en = [], []
    for _ in range(2):
        with E.Engine(s, _params(E, s, precision=precision, nlist_period=0, skin=0.05,
                                  thermostat=E.THERMOSTAT_BERENDSEN, t_target=250.0, tau_t=1e-4)) as eng:
            eng.step(300)
            assert eng.rebuild_count() >= 2
            out.append(_positions(E, eng, s))
            en.append(eng.compute_energies())
    assert np.array_equal(out[0], out[1])
    assert np.array_equal(en[0], en[1])


@pytest.mark.parametrize("precision", [0, 1])
def test_dynamic_list_trajectory_matches_fp64(gpu, precision):
    """nlist_period 0: rebuilds decided and launched on the device (the step
    kernel's tail launch of the rebuild graph) leave the trajectory on the
    FP64 oracle's."""
    E = gpu
    s = S.make_system("small_chains", seed=3)
    ps = po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0)
    x64, _, _, _ = ps.run(s.spec.dt, 20)
    with E.Engine(s, _params(E, s, precision=precision, nlist_period=0)) as eng:
        eng.step(20)
        x = _positions(E, eng, s)
        assert eng.rebuild_count() >= 1
    d = x - x64
    d -= s.spec.box_len * np.round(d / s.spec.box_len)
    assert np.abs(d).max() < 1e-5


def test_dynamic_list_stays_valid_over_a_long_run(gpu):
    """Small skin, 3000 steps: the list is rebuilt on demand (never a stale
    error), and the forces at the final positions still match FP64."""
    E = gpu
    s = S.make_system("small_bridged", seed=4)
    with E.Engine(s, _params(E, s, nlist_period=0, skin=0.04, thermostat=E.THERMOSTAT_BERENDSEN,
                              t_target=300.0, tau_t=1e-4)) as eng:
        eng.step(3000)
        eng.synchronize()
        n_rb = eng.rebuild_count()
        st, prev = eng.compound_states()
        sol = eng.solvents()
        eng.compute_energies()
        F = _flat(s, *eng.forces())
        launches = eng.kernel_launches()
    assert 10 < n_rb < 3000
    assert launches >= 2 * 3000   # the bonded and the step kernel per step, plus the rebuilds
    s2 = S.System(s.spec, s.seed, s.forcefield, s.compounds.copy(), st, sol, s.bridges)
    for c in range(s.n_compounds):
        s2.compounds[c]["prev_positions"] = prev[c]
    F64, _ = po.PhysSystem(s2, rc=s.spec.cutoff, r_on=1.0).forces()
    assert relrms(F, F64) < 5e-5


def test_compute_energies_reports_its_own_kinetic_energy(gpu):
    """lima_compute_energies after steps: the kinetic energy and temperature
    are those of the evaluated state, not of the step before it (the last
    step's pending FP64 sums are folded first)."""
    E = gpu
    s = S.make_system("tiny_chains", seed=8)
    with E.Engine(s, _params(E, s, nlist_period=0)) as eng:
        eng.step(7)
        a = eng.compute_energies()
        b = eng.compute_energies()
    for q in (E.E_KINETIC, E.E_TEMPERATURE, E.E_TOTAL, E.E_LJ):
        assert abs(a[q] - b[q]) <= 1e-9 * abs(b[q]), q


def _wrapped_f32(s):
    """Positions as the physics loader stores them: wrapped into [0, L) in
    double, then rounded to FP32, compound particles first, then solvents."""
    parts = [s.states[c]["positions"][: s.compounds[c]["n_particles"]] for c in range(s.n_compounds)]
    x = np.concatenate(parts + [s.solvents["pos"]]).astype(np.float64) if parts else s.solvents["pos"].astype(np.float64)
    L = s.spec.box_len
    w = np.mod(x, L).astype(np.float32)
    w[w >= np.float32(L)] = 0.0
    return w


@pytest.mark.parametrize("name", ["tiny_chains", "small_bridged", "lj_solvent_4096"])
def test_verlet_list_matches_brute_force(gpu, name):
    """The Verlet list of a fresh engine against every pair of the loaded
    positions: all pairs closer than r_list (outside a 1e-5 rounding band)
    are listed, none farther, no particle twice or itself, and no bonded
    exclusion (LJ_Ignores)."""
    E = gpu
    s = make_named(name, 2)
    skin = 0.1
    with E.Engine(s, _params(E, s, skin=skin)) as eng:
        off, ids = eng.nlist(E.NL_PAIR)
    off = off.astype(np.int64)
    ids = ids.astype(np.int64)
    x = _wrapped_f32(s).astype(np.float64)
    n = len(x)
    L = s.spec.box_len
    rl2 = (s.spec.cutoff + skin) ** 2
    ps = po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0)
    excl = {(i, int(j)) for i in range(n) for j in ps.excl_ids[ps.excl_off[i]:ps.excl_off[i + 1]]}
    for i in range(n):
        row = ids[off[i]:off[i + 1]]
        assert len(np.unique(row)) == len(row) and i not in row
        d = x - x[i]
        d -= L * np.round(d / L)
        r2 = (d * d).sum(1)
        must = set(np.nonzero(r2 < rl2 * (1 - 1e-5))[0].tolist()) - {i}
        may = set(np.nonzero(r2 < rl2 * (1 + 1e-5))[0].tolist()) - {i}
        must -= {j for j in must if (i, j) in excl}
        got = set(row.tolist())
        assert must <= got, (i, sorted(must - got)[:5])
        assert got <= may, (i, sorted(got - may)[:5])
        assert not any((i, j) in excl for j in got)
