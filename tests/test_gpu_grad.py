"""GPU trajectory loss and its adjoint gradient (lima_loss / lima_grad).

The loss (include/lima_abi.h) averages w_e U/N + w_r sum_b (h_b - target_b)^2
over the states after steps 1..T of NVE velocity Verlet.  The GPU computes it
in FP32 with FP64 reductions; the oracle (oracle/lima_oracle.c
orc_phys_loss) restates it in FP64.  The gradient with respect to the per-type
sigma / epsilon and the bonded scales comes from the hand-written adjoint and
is checked against central finite differences of the FP64 oracle loss
(relative step 1e-4).  Stated bars: loss within 1e-5 relative of FP64,
gradient within 1e-3 relative of the FP64 finite differences on every
parameter whose derivative is not negligible (> 1e-3 of the largest).
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


def _relaxed(E, name, seed, steps=400):
    s = S.make_system(name, seed=seed)
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


def test_grad_matches_fp64_finite_differences(gpu):
    E = gpu
    s = _relaxed(E, "tiny_chains", 5)
    ps = po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0)
    tg = _target(ps)
    T, dt = 30, s.spec.dt
    with E.Engine(s, _params(E, s)) as eng:
        theta = eng.get_params()
        L, g = eng.grad(T, 10, NB, RMAX, 1.0, 1e3, tg)
    th64 = ps.params()
    assert np.allclose(theta, th64, rtol=1e-6)
    fd = np.zeros_like(g)
    for k in range(len(theta)):
        h = 1e-4 * abs(th64[k])
        lp, _ = ps.with_params(th64 + h * np.eye(len(theta))[k]).loss(dt, T, NB, RMAX, 1.0, 1e3, tg)
        lm, _ = ps.with_params(th64 - h * np.eye(len(theta))[k]).loss(dt, T, NB, RMAX, 1.0, 1e3, tg)
        fd[k] = (lp - lm) / (2 * h)
    big = np.abs(fd) > 1e-3 * np.abs(fd).max()
    assert big.sum() >= 4
    rel = np.abs(g - fd)[big] / np.abs(fd)[big]
    assert rel.max() < 1e-3, (rel, g, fd)


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
