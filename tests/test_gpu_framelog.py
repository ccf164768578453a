"""Frame log (lima_log_*): the reference's logging buffers
(traj_buffer, potE_buffer, data_GAN, outdata: Engine.cu:1007-1047,
1136-1145), their offload and the post-run energy analysis and output files
(Environment.cpp:124-166, Analyzer.cu:33-207).

Physics semantics: checked against a second engine stepped to the same steps
(positions bit-identical, FP64 energies to 1e-9 relative), the FP64 oracle
(LJ force from solvents on compound particles within 5e-5 relative RMS, the
stated FP32 force error), the per-particle energies summing to the FP64
totals, and the files read back in the reference's layouts.  Reference
semantics: checked frame by frame against the reference's own buffers.
"""
import numpy as np
import pytest

from conftest import relrms
from oracle import pyoracle as po
from quantom_b200 import systems as S

pytestmark = pytest.mark.gpu

EVERY, STEPS = 5, 40


def _params(E, s, **kw):
    p = E.default_params(box_len=s.spec.box_len, cutoff=s.spec.cutoff, dt=s.spec.dt, semantics=E.SEMANTICS_PHYSICS,
                         skin=0.1, switch_on=1.0, nlist_period=0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _slots(E, eng, s):
    """Positions of the current state in the reference slot layout."""
    st, _ = eng.compound_states()
    out = np.zeros((s.n_compounds * 64 + s.n_solvents, 3), np.float32)
    for c in range(s.n_compounds):
        k = s.compounds[c]["n_particles"]
        out[c * 64: c * 64 + k] = st[c]["positions"][:k]
    out[s.n_compounds * 64:] = eng.solvents()["pos"]
    return out


@pytest.fixture(scope="module", params=["tiny_chains", "small_bridged"])
def logged(request, gpu):
    E = gpu
    s = S.make_system(request.param, seed=5)
    with E.Engine(s, _params(E, s)) as eng:
        eng.log_start(EVERY, ring_frames=3)      # the ring wraps twice
        eng.step(STEPS)
        frames = eng.log_read()
        # a second engine at the same steps, energy steps where the first one logged
        ref_pos, ref_e = [], []
        with E.Engine(s, _params(E, s, energy_period=EVERY)) as ref:
            for k in range(STEPS // EVERY):
                ref_pos.append(_slots(E, ref, s))
                ref_e.append(ref.compute_energies())
                ref.step(EVERY)
        yield E, s, eng, frames, np.array(ref_pos), np.array(ref_e)


def test_frames_are_the_logged_steps(logged):
    E, s, eng, fr, ref_pos, _ = logged
    assert fr["steps"].tolist() == list(range(0, STEPS, EVERY))
    assert eng.log_count() == STEPS // EVERY
    # positions the forces of each logged step were evaluated at
    np.testing.assert_array_equal(fr["traj"], ref_pos)


def test_frame_energies_match_the_step(logged):
    E, s, eng, fr, _, ref_e = logged
    e = fr["energies"]
    for q in (E.E_LJ, E.E_BOND, E.E_ANGLE, E.E_DIHEDRAL, E.E_KINETIC, E.E_TOTAL, E.E_TEMPERATURE):
        np.testing.assert_allclose(e[:, q], ref_e[:, q], rtol=1e-9, atol=1e-9 * np.abs(ref_e[:, E.E_TOTAL]).max())


def test_per_particle_energies_sum_to_the_totals(logged):
    E, s, eng, fr, _, _ = logged
    e = fr["energies"]
    pot = e[:, E.E_LJ] + e[:, E.E_BOND] + e[:, E.E_ANGLE] + e[:, E.E_DIHEDRAL]
    scale = np.abs(e[:, E.E_LJ]) + np.abs(e[:, E.E_DIHEDRAL])
    np.testing.assert_array_less(np.abs(fr["potE"].sum(1) - pot), 1e-5 * scale)
    # empty compound slots stay zero
    for c in range(s.n_compounds):
        k = s.compounds[c]["n_particles"]
        assert not fr["potE"][:, c * 64 + k: (c + 1) * 64].any()


def test_train_record_matches_fp64_solvent_forces(logged):
    E, s, eng, fr, _, _ = logged
    ps = po.PhysSystem(s, rc=s.spec.cutoff, r_on=1.0)
    tr = fr["train"]
    assert tr.shape == (len(fr["steps"]), s.n_compounds, 64, 3, 3)
    for f in (0, len(fr["steps"]) - 1):
        x = np.concatenate([fr["traj"][f, c * 64: c * 64 + s.compounds[c]["n_particles"]]
                            for c in range(s.n_compounds)] + [fr["traj"][f, s.n_compounds * 64:]])
        F64 = ps.solvent_lj_on_compounds(x.astype(np.float64))
        got = np.concatenate([tr[f, c, : s.compounds[c]["n_particles"], 1] for c in range(s.n_compounds)])
        pos = np.concatenate([tr[f, c, : s.compounds[c]["n_particles"], 0] for c in range(s.n_compounds)])
        assert relrms(got, F64) < 5e-5
        np.testing.assert_array_equal(pos, x[: len(pos)])
    for c in range(s.n_compounds):
        k = s.compounds[c]["n_particles"]
        assert (tr[:, c, k:, 0] == -1.0).all() and not tr[:, c, k:, 1:].any()
        assert not tr[:, c, :k, 2].any()


def test_logdata_line(logged):
    E, s, eng, fr, _, _ = logged
    ld = fr["logdata"]
    np.testing.assert_allclose(ld[:, 2], fr["potE"][:, 0].astype(np.float32), rtol=1e-6)
    assert np.isfinite(ld).all() and (ld[:, 0] > 0).all() and (ld[:, 3] > 0).all() and not ld[:, 4:].any()
    m = s.forcefield["particle_parameters"][0]["mass"][s.compounds[0]["atom_types"][0]]
    np.testing.assert_allclose(ld[:, 1], 0.5 * m * ld[:, 0] ** 2, rtol=1e-5)


def test_files_in_reference_layout(logged, tmp_path):
    E, s, eng, fr, _, _ = logged
    eng.log_write(tmp_path)
    nf, nc, ns = len(fr["steps"]), s.n_compounds, s.n_solvents
    n = s.n_particles
    ld = np.fromfile(tmp_path / "logdata.bin", np.float32).reshape(nf, 10)
    np.testing.assert_array_equal(ld, fr["logdata"])
    en = np.fromfile(tmp_path / "energy.bin", np.float32).reshape(nf, 3)
    e = fr["energies"]
    pot = e[:, E.E_LJ] + e[:, E.E_BOND] + e[:, E.E_ANGLE] + e[:, E.E_DIHEDRAL]
    np.testing.assert_allclose(en[:, 0], pot / n, rtol=1e-6)
    np.testing.assert_allclose(en[:, 1], e[:, E.E_KINETIC] / n, rtol=1e-6)
    np.testing.assert_allclose(en[:, 2], e[:, E.E_TOTAL] / n, rtol=1e-6)
    temp = np.fromfile(tmp_path / "temperature.bin", np.float32)
    np.testing.assert_allclose(temp, e[:, E.E_TEMPERATURE], rtol=1e-6)
    # sim_traindata.bin as LIMA_services reads it (main.cpp:269-300): per step, per
    # particle slot, FLOAT3_PER_ATOM = 3 float3 (position, LJ force)
    td = np.fromfile(tmp_path / "sim_traindata.bin", np.float32).reshape(nf, nc * 64, 3, 3)
    np.testing.assert_array_equal(td, fr["train"].reshape(nf, nc * 64, 3, 3))
    tj = np.fromfile(tmp_path / "traj.bin", np.float32).reshape(nf, nc * 64 + ns, 3)
    np.testing.assert_array_equal(tj, fr["traj"])
    pe = np.fromfile(tmp_path / "potE.bin", np.float64).reshape(nf, nc * 64 + ns)
    np.testing.assert_array_equal(pe, fr["potE"])


def test_stop_keeps_frames_and_stops_recording(gpu):
    E = gpu
    s = S.make_system("tiny_chains", seed=6)
    with E.Engine(s, _params(E, s, precision=E.PRECISION_MIXED)) as eng:
        eng.log_start(2, ring_frames=64, flags=E.LOG_TRAJ)
        eng.step(10)
        eng.log_stop()
        eng.step(10)
        fr = eng.log_read()
        assert fr["steps"].tolist() == [0, 2, 4, 6, 8]
        assert "potE" not in fr and "train" not in fr
        buf = np.zeros(s.n_compounds * 64 + s.n_solvents)   # potentials were not recorded
        assert eng.lib.lima_log_read(eng.h, 0, 1, None, None, None, buf.ctypes.data, None, None) == E.ERR_ARGUMENT


def test_energy_only_frames_and_reads_during_the_run(gpu):
    """A log of energies and the log line only (one block per frame) read part
    way through the run, which drains the device ring early, gives the same
    frames as a full log read once at the end: the frame kernels take their
    ring position from the device, inside the logged step's graph."""
    E = gpu
    s = S.make_system("tiny_chains", seed=8)
    with E.Engine(s, _params(E, s)) as eng:
        eng.log_start(1, ring_frames=4, flags=0)
        eng.step(6)                      # the ring wraps once; two frames wait in it
        first = eng.log_read()
        eng.step(7)
        assert eng.log_count() == 13
        late = eng.log_read(6)
    with E.Engine(s, _params(E, s)) as ref:
        ref.log_start(1, ring_frames=64, flags=E.LOG_TRAJ | E.LOG_POTE | E.LOG_TRAIN)
        ref.step(13)
        full = ref.log_read()
    assert first["steps"].tolist() == list(range(6)) and late["steps"].tolist() == list(range(6, 13))
    for key in ("energies", "logdata"):
        got = np.concatenate([first[key], late[key]])
        np.testing.assert_array_equal(got, full[key])
    assert "traj" not in first and "potE" not in first


def _analyze_energy(s, traj, potE, dt):
    """Analyzer::analyzeEnergy (Analyzer.cu:33-207) restated over frames of
    consecutive steps: per frame f (1 .. F-3) the particle's potE plus the
    kinetic energy of calcKineticEnergy (Engine.cuh:32-45) over frames f-1 and
    f+1 with the solvent mass, averaged over solvents and over compound
    particles, the two averages weighed by their counts."""
    L = s.spec.box_len
    mass = float(s.forcefield["particle_parameters"][0]["mass"][0])
    nc, ns = s.n_compounds, s.n_solvents
    live = np.concatenate([np.arange(c * 64, c * 64 + s.compounds[c]["n_particles"]) for c in range(nc)] +
                          [nc * 64 + np.arange(ns)]).astype(np.int64)
    is_sol = live >= nc * 64
    out = []
    for f in range(1, len(traj) - 2):
        a = traj[f + 1][live].astype(np.float64)
        b = traj[f - 1][live].astype(np.float64)
        d = a - b
        d -= L * np.round(d / L)
        vel = np.linalg.norm(d, axis=1) * 0.5 / dt
        ke = 0.5 * mass * vel * vel
        pe = potE[f][live]
        row = []
        for q in (pe, ke, pe + ke):
            avg_s = q[is_sol].mean() if ns else 0.0
            avg_c = q[~is_sol].mean() if (~is_sol).any() else 0.0
            row.append((avg_s * ns + avg_c * (~is_sol).sum()) / len(live))
        out.append(row)
    return np.array(out)


def test_reference_semantics_frames_match_the_reference(gpu, tmp_path):
    """A reference-semantics run logged every step against the reference's own
    logging buffers (oracle/_ref: traj_buffer, potE_buffer, outdata, data_GAN
    of its step code, Engine.cu:1007-1047, 1136-1145) over the same 12 steps;
    the frame ring (5 frames) wraps twice.  Positions within 1e-5 nm, potE
    within 1e-6 relative, the solvent LJ force on compound particles within
    1e-5 relative RMS, the outdata line within 1e-5 relative; energy.bin is
    the Analyzer's central-difference product of the reference's frames."""
    if not po.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    E = gpu
    s = S.make_system("tiny_chains", seed=4)
    n_steps = 12
    ref = po.RefEngine(s)
    ref.update_nlists()
    refl = []
    for _ in range(n_steps):
        ref.step(1)
        refl.append(ref.log())
    ref.close()
    p = E.default_params(box_len=s.spec.box_len, cutoff=s.spec.cutoff, dt=s.spec.dt)
    with E.Engine(s, p) as eng:
        eng.log_start(1, ring_frames=5, flags=E.LOG_TRAJ | E.LOG_POTE | E.LOG_TRAIN)
        eng.step(n_steps)
        fr = eng.log_read()
        eng.log_write(tmp_path)
    nc, ns = s.n_compounds, s.n_solvents
    assert fr["steps"].tolist() == list(range(n_steps))
    live = np.concatenate([np.arange(c * 64, c * 64 + s.compounds[c]["n_particles"]) for c in range(nc)] +
                          [nc * 64 + np.arange(ns)]).astype(np.int64)
    comp = live[live < nc * 64]
    for k in range(n_steps):
        r = refl[k]
        assert np.abs(fr["traj"][k][live] - r["traj"][live]).max() < 1e-5, k
        pe, pe_r = fr["potE"][k][: nc * 64], r["potE"][: nc * 64]
        assert np.abs(pe - pe_r).max() <= 1e-6 * np.abs(pe_r).max(), k
        assert not fr["potE"][k][nc * 64:].any()
        tr, tr_r = fr["train"][k], r["train"]
        assert np.abs(tr[:, :, 0].reshape(-1, 3)[comp] - tr_r[:, :, 0].reshape(-1, 3)[comp]).max() < 1e-5
        pad = np.setdiff1d(np.arange(nc * 64), comp)
        assert (tr[:, :, 0].reshape(-1, 3)[pad] == -1.0).all() and (tr_r[:, :, 0].reshape(-1, 3)[pad] == -1.0).all()
        assert relrms(tr[:, :, 1].reshape(-1, 3)[comp], tr_r[:, :, 1].reshape(-1, 3)[comp]) < 1e-5
        np.testing.assert_allclose(fr["logdata"][k][:4], r["logdata"][:4], rtol=1e-5)
    en = np.fromfile(tmp_path / "energy.bin", np.float32).reshape(-1, 3)
    want = _analyze_energy(s, np.array([r["traj"] for r in refl]), np.array([r["potE"] for r in refl]), s.spec.dt)
    assert en.shape == want.shape == (n_steps - 3, 3)
    np.testing.assert_allclose(en, want, rtol=1e-5)
    np.testing.assert_array_equal(np.fromfile(tmp_path / "logdata.bin", np.float32).reshape(n_steps, 10), fr["logdata"])
