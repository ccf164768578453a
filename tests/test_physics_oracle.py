"""Self-consistency of the FP64 physics oracle (CPU): forces are minus the
gradient of its energy (central differences), momentum is conserved, the
switched LJ is continuous at both ends of the switch, and a velocity-Verlet
run conserves energy on a small time step."""
import numpy as np
import pytest

from oracle import pyoracle as po
from quantom_b200 import systems as S


@pytest.fixture(scope="module")
def chains():
    s = S.make_system("tiny_chains", seed=13)
    # perturb the ideal chain geometry so bonded terms carry force
    rng = np.random.default_rng(1)
    for c in range(s.n_compounds):
        n = s.compounds[c]["n_particles"]
        s.states[c]["positions"][:n] += rng.normal(0, 0.01, (n, 3)).astype(np.float32)
    return po.PhysSystem(s, rc=1.2, r_on=1.0)


def _energy(ps, x):
    _, en = ps.forces(x)
    return en[:4].sum()


def test_forces_are_minus_energy_gradient(chains):
    ps = chains
    F, _ = ps.forces()
    rng = np.random.default_rng(2)
    picks = list(rng.choice(ps.n_compound_particles, 6, replace=False)) + list(rng.choice(ps.n, 6, replace=False))
    h = 1e-6
    for i in picks:
        for d in range(3):
            xp = ps.x.copy(); xp[i, d] += h
            xm = ps.x.copy(); xm[i, d] -= h
            fd = -(_energy(ps, xp) - _energy(ps, xm)) / (2 * h)
            assert abs(fd - F[i, d]) <= 2e-5 * max(1.0, abs(F[i, d])) + 1e-4 * np.abs(F[i]).max()


def test_momentum_conserved(chains):
    F, _ = chains.forces()
    assert np.abs(F.sum(axis=0)).max() < 1e-6 * np.abs(F).max() * np.sqrt(len(F))


def test_switch_is_continuous():
    s = S.make_system("tiny_solvent", seed=2)
    ps = po.PhysSystem(s, rc=1.2, r_on=1.0)
    # two particles along x at distances straddling r_on and rc
    ps.n = 2
    ps.sigma = ps.sigma[:2].copy(); ps.epsilon = ps.epsilon[:2].copy()
    ps.excl_off = np.zeros(3, np.int32)
    for r0 in (1.0, 1.2):
        e, f = [], []
        for r in (r0 - 1e-7, r0 + 1e-7):
            x = np.array([[0.5, 0.5, 0.5], [0.5 + r, 0.5, 0.5]])
            F, en = ps.forces(x)
            e.append(en[0])
            f.append(F[1, 0])
        # a jump would be O(1); continuity leaves slope * 2e-7
        assert abs(e[0] - e[1]) <= 2.5e-7 * max(abs(f[0]), abs(f[1])) + 1e-9
        assert abs(f[0] - f[1]) < 1e-3
        # C2: the force's slope is continuous too (a C1 switch jumps by V(r) S''(r), ~1e2 here)
        h = 1e-5   # smooth: the one-sided slopes differ by ~F'' * 1.5 h
        fx = []
        for r in (r0 - 2 * h, r0 - h, r0 + h, r0 + 2 * h):
            x = np.array([[0.5, 0.5, 0.5], [0.5 + r, 0.5, 0.5]])
            fx.append(ps.forces(x)[0][1, 0])
        left, right = (fx[1] - fx[0]) / h, (fx[3] - fx[2]) / h
        assert abs(left - right) < 1.0


def test_velocity_verlet_conserves_energy_small_dt():
    s = S.make_system("tiny_solvent", seed=5)
    ps = po.PhysSystem(s, rc=1.2, r_on=1.0)
    # relax first so the start is not dominated by contact pairs
    x, v, _, _ = ps.run(1e-6, 200, thermostat=2, t0=300.0, tau=2e-5)
    _, _, _, en = ps.run(2e-7, 200, x=x, v=v)
    tot = en[:, 7]
    assert (tot.max() - tot.min()) / abs(en[0, 4]) < 2e-4


def test_wrapping_input_positions_to_fp32_moves_the_forces():
    """The physics loader wraps input positions into [0, L) and rounds them to
    FP32; for positions outside the box that moves them by up to half a float
    spacing.  The FP64 forces at the moved positions differ from those at the
    raw positions by 3.9e-4 relative RMS in a stiff box without solvent
    (small_bridged_dry, 28 of 192 particles outside [0, L)) and stay within
    the 5e-5 force bar with solvent (small_bridged)."""
    from conftest import make_named, relrms
    out = {}
    for name in ("small_bridged_dry", "small_bridged"):
        s = make_named(name, 7)
        ps = po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0)
        F, _ = ps.forces()
        L = ps.box
        xw = np.fmod(ps.x, L)
        xw[xw < 0] += L
        x32 = xw.astype(np.float32).astype(np.float64)
        x32[x32 >= L] = 0.0
        out[name] = relrms(ps.forces(x32)[0], F)
    assert 1e-4 < out["small_bridged_dry"] < 1e-3
    assert out["small_bridged"] < 5e-5


def test_lj_matches_the_reference_where_the_forms_coincide():
    """Pins the oracle's LJ to the reference's calcLJForce (Engine.cu:475-522)
    where the two functional forms coincide: one particle type (Lorentz-
    Berthelot and the reference's arithmetic/geometric mixing agree), no
    switch, and the physics cutoff equal to the reference's solvent list
    radius 2 CUTOFF, inside which the reference sums the full LJ force.  The
    reference's own step code (oracle/_ref) gives the forces of one step;
    FP32 against FP64."""
    if not po.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    s = S.make_system("lj_solvent_4096", seed=21)
    ref = po.RefEngine(s)
    ref.update_nlists()
    ref.step(1)
    _, fs_ref = ref.forces()
    ref.close()
    rc = 2.0 * float(po.ref_cutoff_of(s))            # the reference's solvent-solvent list radius
    F64, _ = po.PhysSystem(s, rc=rc, r_on=rc).forces()
    err = np.sqrt(((fs_ref.astype(np.float64) - F64) ** 2).sum() / (F64 ** 2).sum())
    assert err < 1e-5, err
