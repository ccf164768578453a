"""GPU parity of the reference-semantics step path (through the C-ABI).

Compared with the reference itself (golden fixtures made from the reference's
own Engine.cu, tests/golden/) and with the CPU oracle (oracle/lima_oracle.c,
pinned bit-exactly to the reference) on seeded workloads up to the full
32,024-particle solvated-chain box.  Bars, as the benchmark states them:
neighbour lists bit-exact (identical sorted sets; the order after a build
from empty lists is the reference's too), forces within 1e-5 relative RMS,
per-particle potE within 1e-6 relative.
"""
import numpy as np
import pytest

from conftest import compound_mask, golden_lists, load_golden, make_named, relrms, sorted_csr
from oracle import pyoracle as po
from quantom_b200 import systems as S

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5
POTE_TOL = 1e-6


def _engine(E, system, **kw):
    p = E.default_params(box_len=system.spec.box_len, cutoff=system.spec.cutoff, dt=system.spec.dt)
    for k, v in kw.items():
        setattr(p, k, v)
    return E.Engine(system, p)


def _lists_equal(a, b):
    return np.array_equal(np.asarray(a[0], np.int64), np.asarray(b[0], np.int64)) and \
        np.array_equal(np.asarray(a[1], np.int64), np.asarray(b[1], np.int64))


def _check_step(system, eng, fc_ref, fs_ref, pe_ref, st_ref, prev_ref, sol_ref, pos_tol=1e-5):
    m = compound_mask(system)
    fc, fs = eng.forces()
    _, pe = eng.energies(per_particle=True)
    st, prev = eng.compound_states()
    sol = eng.solvents()
    if system.n_compounds:
        assert relrms(fc[m], fc_ref[m]) < FORCE_TOL
        ref = pe_ref[: system.n_compounds * 64]
        assert np.abs(pe[: system.n_compounds * 64] - ref).max() <= POTE_TOL * max(np.abs(ref).max(), 1e-30)
        assert np.abs(st["positions"][m] - st_ref["positions"][m]).max() < pos_tol
        assert np.abs(prev[m] - prev_ref[m]).max() < pos_tol
    if system.n_solvents:
        assert relrms(fs, fs_ref) < FORCE_TOL
        assert np.abs(sol["pos"] - sol_ref["pos"]).max() < pos_tol
        assert np.abs(sol["pos_tsub1"] - sol_ref["pos_tsub1"]).max() < pos_tol


@pytest.mark.parametrize("name", ["golden_chain", "golden_bridge", "golden_solvent"])
def test_matches_reference_fixtures(gpu, name):
    E = gpu
    system, z = load_golden(name)
    ref_lists = golden_lists(z)
    with _engine(E, system) as eng:
        for w in range(4):
            assert _lists_equal(eng.nlist(w), ref_lists[w]), f"list kind {w}"
        eng.step(1)
        _check_step(system, eng, z["step1_fc"], z["step1_fs"], z["step1_potE"], z["step1_states"], z["step1_prev"],
                    z["step1_solvents"])
        # one step with thermostat scalar 1.02, then two plain steps
        eng.set_thermostat_scalar(1.02)
        eng.step(3)
        st, _ = eng.compound_states()
        sol = eng.solvents()
        m = compound_mask(system)
        if system.n_compounds:
            assert np.abs(st["positions"][m] - z["step4_states"]["positions"][m]).max() < 1e-5
        assert np.abs(sol["pos"] - z["step4_solvents"]["pos"]).max() < 1e-5


# 6lzm: the reference's own demo box (T4 lysozyme, 36 compounds, 35 bridges,
# 5,000 waters) as its input path built it (tests/golden/golden_6lzm.npz);
# *_dry: compounds (and bridges) with no solvent
@pytest.mark.parametrize("name", ["tiny_chains", "small_bridged", "lj_solvent_4096", "lj_solvent_8192",
                                  "solvated_chains_32k", "6lzm", "tiny_chains_dry", "small_bridged_dry"])
def test_one_step_matches_oracle(gpu, name):
    E = gpu
    s = make_named(name, 7)
    lists = po.ref_nlist(s, ss_cap=1024, cells=True)
    new, fc_o, fs_o, pe_o = po.ref_step(s, lists)
    with _engine(E, s) as eng:
        for w in range(4):
            assert _lists_equal(eng.nlist(w), lists[w]), f"list kind {w}"
        eng.step(1)
        _check_step(s, eng, fc_o, fs_o, pe_o, new.states, new.compounds["prev_positions"], new.solvents)


_ORACLE_STEP = {}


def _oracle_step(name):
    if name not in _ORACLE_STEP:
        s = S.load_6lzm() if name == "6lzm" else S.make_system(name, seed=7)
        lists = po.ref_nlist(s, ss_cap=1024, cells=True)
        _ORACLE_STEP[name] = (s, po.ref_step(s, lists))
    return _ORACLE_STEP[name]


# The solvent kernels split each solvent's two ordered loops (compounds,
# solvent list) over 1-16 lanes each; the image chain is replayed and the
# lanes' terms added in order, so the solvent path stays the oracle's (and
# the reference's) float arithmetic.
@pytest.mark.parametrize("lanes", [(1, 1), (1, 16), (2, 8), (4, 4), (8, 2), (16, 1), (16, 16)])
@pytest.mark.parametrize("name", ["small_bridged", "lj_solvent_4096", "6lzm"])
def test_solvent_path_bit_identical_at_every_lane_count(gpu, name, lanes, monkeypatch):
    E = gpu
    monkeypatch.setenv("LIMA_SOLVENT_LANES", str(lanes[0]))
    monkeypatch.setenv("LIMA_SOLVENT_LIST_LANES", str(lanes[1]))
    s, (new, fc_o, fs_o, pe_o) = _oracle_step(name)
    with _engine(E, s) as eng:
        eng.step(1)
        fc, fs = eng.forces()
        sol = eng.solvents()
        st, _ = eng.compound_states()
    np.testing.assert_array_equal(fs, fs_o)
    np.testing.assert_array_equal(sol["pos"], new.solvents["pos"])
    np.testing.assert_array_equal(sol["pos_tsub1"], new.solvents["pos_tsub1"])
    if s.n_compounds:
        m = compound_mask(s)
        assert relrms(fc[m], fc_o[m]) < FORCE_TOL
        assert np.abs(st["positions"][m] - new.states["positions"][m]).max() < 1e-5


@pytest.mark.parametrize("semantics", ["reference", "physics"])
def test_flat_positions_are_the_struct_positions(gpu, semantics):
    """lima_get_positions returns the positions lima_get_compound_states and
    lima_get_solvents return, flattened, with empty compound slots zero."""
    E = gpu
    s = S.make_system("small_bridged", seed=5)
    kw = {} if semantics == "reference" else dict(semantics=E.SEMANTICS_PHYSICS, skin=0.1, switch_on=1.0)
    with _engine(E, s, **kw) as eng:
        eng.step(3)
        cxyz, sxyz = eng.positions()
        st, _ = eng.compound_states()
        sol = eng.solvents()
    for c in range(s.n_compounds):
        k = s.compounds[c]["n_particles"]
        np.testing.assert_array_equal(cxyz[c, :k], st[c]["positions"][:k])
        assert not cxyz[c, k:].any()
    np.testing.assert_array_equal(sxyz, sol["pos"])


def test_multistep_with_list_rebuilds_matches_oracle(gpu):
    E = gpu
    s = S.make_system("small_bridged", seed=3)
    n_steps, period = 30, 10
    o = s
    for k in range(n_steps):
        if k % period == 0:
            lists = po.ref_nlist(o, ss_cap=1024, cells=True)
        o, _, _, _ = po.ref_step(o, lists)
    with _engine(E, s, nlist_period=period) as eng:
        eng.step(n_steps)
        assert eng.current_step == n_steps
        st, _ = eng.compound_states()
        sol = eng.solvents()
    m = compound_mask(s)
    assert np.abs(st["positions"][m] - o.states["positions"][m]).max() < 1e-4
    d = sol["pos"] - o.solvents["pos"]
    d -= s.spec.box_len * np.round(d / s.spec.box_len)
    assert np.abs(d).max() < 1e-4


def test_compound_list_history_via_set_nlist(gpu):
    """The reference keeps a compound pair listed before if it is within
    C+((r_i+r_j)+C) but adds new pairs only within C+((r_i+r_i)+C)
    (Engine.cu:168, 243-246); lima_set_nlist installs that history."""
    E = gpu
    s = S.make_system("tiny_chains", seed=4)
    C = float(po.ref_cutoff_of(s))
    s.compounds["confining_particle_sphere"][0] = 0.3
    s.compounds["confining_particle_sphere"][1] = 0.9
    k0 = s.states[0]["positions"][s.compounds[0]["key_particle_index"]].astype(np.float64)
    k1 = s.states[1]["positions"][s.compounds[1]["key_particle_index"]].astype(np.float64)
    shift = (k0 + np.array([C + (0.3 + 0.3 + C) + 0.25, 0, 0]) - k1).astype(np.float32)
    s.states[1]["positions"][: s.compounds[1]["n_particles"]] += shift
    s.compounds[1]["prev_positions"][: s.compounds[1]["n_particles"]] += shift
    with _engine(E, s) as eng:
        off, ids = eng.nlist(E.NL_COMPOUND_COMPOUND)
        assert len(ids) == 0                                    # not within the add radius
        eng.set_nlist(E.NL_COMPOUND_COMPOUND, [0, 1, 2], [1, 0])
        eng.build_nlist()
        off, ids = eng.nlist(E.NL_COMPOUND_COMPOUND)
        expect = po.ref_nlist(s, prev_cc=(np.array([0, 1, 2]), np.array([1, 0])))[0]
        assert _lists_equal((off, ids), expect) and len(ids) == 2


def test_lists_set_in_reference_order_give_reference_forces(gpu):
    """Lists handed over in the reference's own (history-dependent) order are
    used as given: the step reproduces the reference on them."""
    if not po.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    E = gpu
    s = S.make_system("tiny_chains", seed=8)
    ref = po.RefEngine(s)
    ref.update_nlists()
    with _engine(E, s) as eng:
        for w in (0, 1, 3):
            off, ids = ref.nlist(w)
            eng.set_nlist(w, off, ids)
        ref.step(1, 1.0)
        eng.step(1)
        fcr, fsr = ref.forces()
        fc, fs = eng.forces()
    m = compound_mask(s)
    assert relrms(fc[m], fcr[m]) < FORCE_TOL
    assert relrms(fs, fsr) < FORCE_TOL
    ref.close()


def test_list_overflow_is_a_status_not_an_exit(gpu):
    E = gpu
    s = S.make_system("tiny_solvent", seed=2)
    with pytest.raises(E.LimaError) as ei:
        _engine(E, s, solvent_list_capacity=64)
    assert ei.value.status == E.ERR_CAPACITY


def test_reference_thermostat_temperature(gpu):
    """Engine::getBoxTemperature (Engine.cu:314-359): every 40 steps T from
    positions two steps apart; lambda = clamp(T0/T, 0.9, 1.1) for one step."""
    E = gpu
    s = S.make_system("tiny_chains", seed=6)
    with _engine(E, s, thermostat=E.THERMOSTAT_REFERENCE, t_target=310.0) as eng:
        eng.step(38)
        st38, _ = eng.compound_states()
        sol38 = eng.solvents()
        eng.step(2)
        st40, _ = eng.compound_states()
        sol40 = eng.solvents()
        tot = eng.energies()
    L = s.spec.box_len
    ff = s.forcefield["particle_parameters"][0]
    ke, n = 0.0, 0
    for c in range(s.n_compounds):
        for t in range(s.compounds[c]["n_particles"]):
            d = st40[c]["positions"][t].astype(np.float64) - st38[c]["positions"][t]
            d -= L * np.round(d / L)
            v = np.linalg.norm(d) * 0.5 / s.spec.dt
            ke += 0.5 * ff["mass"][s.compounds[c]["atom_types"][t]] * v * v
            n += 1
    d = sol40["pos"].astype(np.float64) - sol38["pos"]
    d -= L * np.round(d / L)
    v = np.linalg.norm(d, axis=1) * 0.5 / s.spec.dt
    ke += (0.5 * ff["mass"][0] * v * v).sum()
    n += len(v)
    T = ke / n * 2 / (3 * 8.3145)
    assert abs(tot[E.E_TEMPERATURE] - T) < 1e-3 * T


def test_invalid_box_is_rejected(gpu):
    E = gpu
    s = S.make_system("tiny_solvent", seed=2)
    s.solvents["pos"][3] = (np.nan, 0.0, 0.0)
    with pytest.raises(E.LimaError) as ei:
        _engine(E, s)
    assert ei.value.status == E.ERR_ARGUMENT


def test_reference_thermostat_schedule_matches_the_reference(gpu):
    """100 steps with the reference thermostat against the reference's own step
    code (oracle/_ref) driven by the reference's rule (Engine::hostMaster and
    handleBoxtemp, Engine.cu:45-75, 362-393): after every 40th step the
    temperature from the positions two steps apart (getBoxTemperature,
    Engine.cu:314-359), lambda = clamp(310 / T, 0.9, 1.1) for the next step
    only, none before step 20.  Two thermostat events (steps 40 and 80)."""
    if not po.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    E = gpu
    s = S.make_system("tiny_chains", seed=6)
    L = s.spec.box_len
    ff = s.forcefield["particle_parameters"][0]
    mass = np.concatenate([ff["mass"][s.compounds[c]["atom_types"][: s.compounds[c]["n_particles"]]]
                           for c in range(s.n_compounds)] + [np.full(s.n_solvents, ff["mass"][0])]).astype(np.float64)

    def flat(state):
        _, st, sol = state
        parts = [st[c]["positions"][: s.compounds[c]["n_particles"]] for c in range(s.n_compounds)]
        return np.concatenate(parts + [sol["pos"]]).astype(np.float64)

    ref = po.RefEngine(s)
    ref.update_nlists()
    lam, lams, snap = 1.0, [], {}
    for k in range(1, 101):
        ref.step(1, lam)
        lam = 1.0
        if k % 40 == 38:
            snap[k] = flat(ref.state())
        if k % 40 == 0:
            d = flat(ref.state()) - snap[k - 2]
            d -= L * np.round(d / L)
            v = np.linalg.norm(d, axis=1) * 0.5 / s.spec.dt
            T = (0.5 * mass * v * v).mean() * 2.0 / (3.0 * 8.3145)
            lam = float(np.float32(min(max(310.0 / T, 0.9), 1.1))) if k > 20 else 1.0
            lams.append(lam)
    _, st_r, sol_r = ref.state()
    ref.close()
    assert any(abs(x - 1.0) > 1e-3 for x in lams)   # the thermostat acted
    with _engine(E, s, thermostat=E.THERMOSTAT_REFERENCE, t_target=310.0) as eng:
        eng.step(100)
        st, _ = eng.compound_states()
        sol = eng.solvents()
    m = compound_mask(s)
    dc = st["positions"][m].astype(np.float64) - st_r["positions"][m]
    dc -= L * np.round(dc / L)
    ds = sol["pos"].astype(np.float64) - sol_r["pos"]
    ds -= L * np.round(ds / L)
    assert np.abs(dc).max() < 1e-4 and np.abs(ds).max() < 1e-4
