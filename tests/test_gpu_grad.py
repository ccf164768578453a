"""GPU trajectory loss and its adjoint gradient (lima_loss / lima_grad).

The loss (include/lima_abi.h) averages w_e U/N + w_r sum_b (h_b - target_b)^2
over the states after steps 1..T of NVE velocity Verlet.  The GPU computes it
in FP32 with FP64 reductions; the oracle (oracle/lima_oracle.c
orc_phys_loss) restates it in FP64.  The gradient with respect to the per-type
sigma / epsilon, the bonded scales and the bonded type constants comes from
the hand-written adjoint and
is checked against central finite differences of the FP64 oracle loss
(relative step 1e-4), on a box whose bonds, angles and dihedrals come in two
types each, so that every type's constants (r0 | theta0 | phi0 and k) are
differentiated.  Stated bars: loss within 1e-5 relative of FP64,
gradient within 1e-3 relative of the FP64 finite differences on every
parameter whose derivative is not negligible (theta_k dL/dtheta_k above 1e-6
of the largest); measured on B200: every one of the 25 entries within 1e-4.
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from quantom_b200 import systems as S

pytestmark = pytest.mark.gpu

NB = 50
RMAX = 1.2 * NB / (NB + 1)   # support r_max + dr ends at the 1.2 nm cutoff


def _params(E, s, **kw):
    p = E.default_params(box_len=s.spec.box_len, cutoff=s.spec.cutoff, dt=s.spec.dt, semantics=E.SEMANTICS_PHYSICS,
                         skin=0.2, switch_on=1.0, nlist_period=0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _relaxed(E, name, seed, steps=400, edit=None):
    s = S.make_system(name, seed=seed)
    if edit is not None:
        edit(s)
    p = _params(E, s, thermostat=E.THERMOSTAT_BERENDSEN, t_target=300.0, tau_t=1e-4)
    with E.Engine(s, p) as eng:
        eng.step(steps)
        st, prev = eng.compound_states()
        sol = eng.solvents()
    return s.with_state(st, prev, sol)


def _target(ps):
    # a target the box is not at: the occupancy of the same box shrunk by 3 %
    x = ps.x * 0.97
    return ps.rdf(NB, RMAX, x) * 1.0


@pytest.mark.parametrize("name", ["tiny_chains", "lj_solvent_4096"])
def test_rdf_matches_oracle(gpu, name):
    E = gpu
    s = _relaxed(E, name, 3)
    with E.Engine(s, _params(E, s)) as eng:
        h = eng.rdf(NB, RMAX)
    h64 = po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0).rdf(NB, RMAX)
    assert h64.sum() > 10
    assert np.abs(h - h64).max() < 1e-5 * h64.max()


def test_loss_matches_oracle(gpu):
    E = gpu
    s = _relaxed(E, "tiny_chains", 4)
    ps = po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0)
    tg = _target(ps)
    L64, _ = ps.loss(s.spec.dt, 30, NB, RMAX, 1.0, 1e3, tg)
    with E.Engine(s, _params(E, s)) as eng:
        L = eng.loss(30, 10, NB, RMAX, 1.0, 1e3, tg)
    assert abs(L - L64) < 1e-5 * abs(L64)


def _two_types_per_kind(s):
    """Gives every other bonded term of the box a second constant set, so
    each kind has two types: bonds (r0 x 1.06, k x 0.7), angles (theta0 -
    0.12 rad, k x 1.3), dihedrals (phi0 0.4 rad, k x 2, n 2)."""
    for c in s.compounds:
        for q in range(0, int(c["n_singlebonds"]), 2):
            c["singlebonds"][q]["b0"] *= 1.06
            c["singlebonds"][q]["kb"] *= 0.7
        for q in range(1, int(c["n_anglebonds"]), 2):
            c["anglebonds"][q]["theta_0"] -= 0.12
            c["anglebonds"][q]["k_theta"] *= 1.3
        for q in range(1, int(c["n_dihedrals"]), 2):
            c["dihedrals"][q]["phi_0"] = 0.4
            c["dihedrals"][q]["k_phi"] *= 2.0
            c["dihedrals"][q]["n"] = 2


def _fd_one(args):
    ps, th64, k, h, dt, T, tg = args
    e = np.zeros(len(th64))
    e[k] = h
    lp, _ = ps.with_params(th64 + e).loss(dt, T, NB, RMAX, 1.0, 1e3, tg)
    lm, _ = ps.with_params(th64 - e).loss(dt, T, NB, RMAX, 1.0, 1e3, tg)
    return (lp - lm) / (2 * h)


def test_grad_matches_fp64_finite_differences(gpu):
    """Every entry of theta: per-type sigma and epsilon, the three bonded
    scales and (r0 | theta0 | phi0, k) of two types per bonded kind."""
    import multiprocessing as mp
    import os
    from concurrent.futures import ProcessPoolExecutor
    E = gpu
    s = _relaxed(E, "tiny_chains", 5, edit=_two_types_per_kind)
    ps = po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0)
    tg = _target(ps)
    T, dt = 30, s.spec.dt
    with E.Engine(s, _params(E, s)) as eng:
        theta = eng.get_params()
        names = eng.param_names()
        lay = eng.param_layout()
        types = [eng.bonded_types(k) for k in range(3)]
        L, g = eng.grad(T, 10, NB, RMAX, 1.0, 1e3, tg)
    th64 = ps.params()
    assert (lay["n_bond_types"], lay["n_angle_types"], lay["n_dihedral_types"]) == (2, 2, 2)
    assert all(np.array_equal(t, inv) for t, (_, inv) in zip(types, ps.term_types()))
    assert len(theta) == len(th64) == len(names) and np.allclose(theta, th64, rtol=1e-6)
    steps = [1e-4 * abs(v) if v != 0.0 else 1e-4 for v in th64]
    jobs = [(ps, th64, k, steps[k], dt, T, tg) for k in range(len(theta))]
    with ProcessPoolExecutor(min(8, os.cpu_count() or 1), mp_context=mp.get_context("spawn")) as ex:
        fd = np.array(list(ex.map(_fd_one, jobs)))
    # not negligible: theta_k dL/dtheta_k above 1e-6 of the largest (1 rad for a zero phase);
    # on this box every entry is (the smallest, a dihedral phase, is 4e-5 of sigma_0's)
    sens = np.abs(fd) * np.where(th64 != 0.0, np.abs(th64), 1.0)
    big = sens > 1e-6 * sens.max()
    bonded = np.arange(len(theta)) >= 2 * lay["n_types"] + 3
    assert big[bonded].all() and big.sum() >= len(theta) - 2
    rel = np.abs(g - fd)[big] / np.abs(fd)[big]
    assert rel.max() < 1e-3, dict(zip(np.array(names)[big], rel))


def test_checkpoint_interval_does_not_change_the_gradient(gpu):
    """C only moves the re-sorts of the unroll (the list is also rebuilt in
    place every 10 steps inside a segment), which changes FP32 summation
    order: loss and gradient agree to rounding."""
    E = gpu
    s = _relaxed(E, "small_bridged", 6)
    tg = _target(po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0))
    out = []
    with E.Engine(s, _params(E, s)) as eng:
        for c in (1, 7, 40):
            out.append(eng.grad(40, c, NB, RMAX, 1.0, 1e3, tg))
    for L, g in out[1:]:
        assert abs(L - out[0][0]) <= 1e-7 * abs(out[0][0])
        assert np.abs(g - out[0][1]).max() <= 1e-4 * np.abs(out[0][1]).max()


def test_grad_leaves_the_state_unchanged(gpu):
    E = gpu
    s = _relaxed(E, "small_chains", 7)
    with E.Engine(s, _params(E, s)) as eng:
        st0, _ = eng.compound_states()
        eng.grad(20, 5, NB, RMAX, 1.0, 0.0)
        st1, _ = eng.compound_states()
        eng.step(10)
        a, _ = eng.compound_states()
    with E.Engine(s, _params(E, s)) as eng:
        eng.step(10)
        b, _ = eng.compound_states()
    assert np.array_equal(st0["positions"], st1["positions"])
    assert np.abs(a["positions"] - b["positions"]).max() < 1e-5


def test_autograd_function_returns_the_adjoint_gradient(gpu):
    torch = pytest.importorskip("torch")
    from quantom_b200.grad import trajectory_loss
    E = gpu
    s = _relaxed(E, "tiny_chains", 8)
    tg = _target(po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0))
    spec = dict(n_steps=20, checkpoint_every=5, n_bins=NB, r_max=RMAX, w_energy=1.0, w_rdf=1e3, target=tg)
    with E.Engine(s, _params(E, s)) as eng:
        theta = torch.tensor(eng.get_params(), dtype=torch.float64, requires_grad=True)
        loss = trajectory_loss(theta, eng, **spec)
        loss.backward()
        L, g = eng.grad(**spec)
    assert abs(loss.item() - L) <= 1e-12 * abs(L)
    assert np.allclose(theta.grad.numpy(), g, rtol=1e-6)


def test_grad_config4_chain_topology_matches_fp64_finite_differences(gpu):
    """The chain topology of the 258k box (64 chains x 128 particles, two
    compounds and one bridge each, 4 chain types) in 16,000 solvents at the
    same density (9 nm box, 24,192 particles): every entry of theta, chain-type
    sigma included, against FP64 central differences over a 20-step unroll
    with checkpoints every 10."""
    import multiprocessing as mp
    import os
    from concurrent.futures import ProcessPoolExecutor
    E = gpu
    spec = S.SystemSpec("chains_64x128_in_16k", 9.0, 16000, chains=S.ChainSpec(64, 128), mc_sweeps=12)
    s0 = S.make_system(spec, seed=7)
    assert s0.n_compounds == 128 and len(s0.bridges) == 64
    p = _params(E, s0, thermostat=E.THERMOSTAT_BERENDSEN, t_target=300.0, tau_t=1e-4)
    with E.Engine(s0, p) as eng:
        eng.step(400)
        st, prev = eng.compound_states()
        s = s0.with_state(st, prev, eng.solvents())
    ps = po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0)
    tg = _target(ps)
    T, dt = 20, s.spec.dt
    with E.Engine(s, _params(E, s)) as eng:
        names = eng.param_names()
        nt = eng.param_layout()["n_types"]
        _, g = eng.grad(T, 10, NB, RMAX, 1.0, 1e3, tg)
    th64 = ps.params()
    steps = [1e-4 * abs(v) if v != 0.0 else 1e-4 for v in th64]
    jobs = [(ps, th64, k, steps[k], dt, T, tg) for k in range(len(th64))]
    with ProcessPoolExecutor(min(16, os.cpu_count() or 1), mp_context=mp.get_context("spawn")) as ex:
        fd = np.array(list(ex.map(_fd_one, jobs)))
    sens = np.abs(fd) * np.where(th64 != 0.0, np.abs(th64), 1.0)
    big = sens > 1e-6 * sens.max()
    assert big[1:nt].all()                      # the chain types' sigma
    rel = np.abs(g - fd)[big] / np.abs(fd)[big]
    assert rel.max() < 1e-3, dict(zip(np.array(names)[big], rel))
