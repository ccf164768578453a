"""Pinning the oracle (CPU).

The C restatement of the reference step path (oracle/lima_oracle.c, part A)
is checked against the reference itself:
  * the committed golden fixtures (tests/golden/*.npz, made by
    tests/golden/make_golden.py from the reference compiled for the host);
  * live, against oracle/_ref/libref_lima.so when it has been built here.
Bars: neighbour lists identical (sets and order), forces within 1e-5 relative
RMS, per-particle potE within 1e-6 relative, positions within 1e-5 nm (the
solvent path is bit-identical; compound forces differ by float regrouping of
the bonded sums, see oracle/ref_emu.cpp).
"""
import numpy as np
import pytest

from conftest import compound_mask, golden_lists, load_golden, make_named, relrms, sorted_csr
from oracle import pyoracle as po
from quantom_b200 import systems as S

GOLDEN = ["golden_chain", "golden_bridge", "golden_solvent"]
FORCE_TOL = 1e-5
POTE_TOL = 1e-6


def _lists_equal(a, b):
    return np.array_equal(np.asarray(a[0], np.int64), np.asarray(b[0], np.int64)) and \
        np.array_equal(np.asarray(a[1], np.int64), np.asarray(b[1], np.int64))


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_matches_reference_fixtures(name):
    system, z = load_golden(name)
    ref_lists = golden_lists(z)
    lists = po.ref_nlist(system, ss_cap=1024)
    for w in range(4):
        assert _lists_equal(lists[w], ref_lists[w]), f"list kind {w}"
    new, fc, fs, pe = po.ref_step(system, lists)
    m = compound_mask(system)
    if system.n_compounds:
        assert relrms(fc[m], z["step1_fc"][m]) < FORCE_TOL
        ref_pe = z["step1_potE"][: system.n_compounds * 64]
        assert np.abs(pe[: system.n_compounds * 64] - ref_pe).max() <= POTE_TOL * np.abs(ref_pe).max()
        assert np.abs(new.states["positions"][m] - z["step1_states"]["positions"][m]).max() < 1e-5
        assert np.abs(new.compounds["prev_positions"][m] - z["step1_prev"][m]).max() < 1e-5
    assert np.array_equal(fs, z["step1_fs"])                       # solvent path: bit-identical
    assert np.array_equal(new.solvents["pos"], z["step1_solvents"]["pos"])
    assert np.array_equal(new.solvents["pos_tsub1"], z["step1_solvents"]["pos_tsub1"])


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_multistep_matches_reference_fixtures(name):
    system, z = load_golden(name)
    lists = po.ref_nlist(system, ss_cap=1024)
    s = system
    for lam in (1.0, 1.02, 1.0, 1.0):
        s, _, _, _ = po.ref_step(s, lists, lam=lam)
    m = compound_mask(system)
    if system.n_compounds:
        assert np.abs(s.states["positions"][m] - z["step4_states"]["positions"][m]).max() < 1e-5
    assert np.abs(s.solvents["pos"] - z["step4_solvents"]["pos"]).max() < 1e-5


@pytest.mark.parametrize("name", ["tiny_solvent", "6lzm"])
def test_cell_list_solvent_lists_equal_all_pairs(name):
    # 6lzm: the reference's demo box, 18 of whose waters sit up to 0.01 nm
    # outside [0, box_len] as loaded; cells are assigned from the wrapped image
    s = S.load_6lzm() if name == "6lzm" else S.make_system(name, seed=9)
    a = po.ref_nlist(s, ss_cap=1024)
    b = po.ref_nlist(s, ss_cap=1024, cells=True)
    assert _lists_equal(a[3], b[3])


ref_needed = pytest.mark.skipif(not po.ref_available(), reason="reference build (oracle/_ref) not present")


@ref_needed
@pytest.mark.parametrize("name", ["tiny_chains", "small_bridged", "tiny_solvent", "6lzm", "small_bridged_dry"])
def test_oracle_matches_reference_live(name):
    s = make_named(name, 21)
    ref = po.RefEngine(s, n_threads=4)
    ref.update_nlists()
    lists = po.ref_nlist(s, ss_cap=1024)
    for w in range(4):
        assert _lists_equal(sorted_csr(*ref.nlist(w)), lists[w]), f"list kind {w}"
    ref.step(1, 1.0)
    fcr, fsr = ref.forces()
    _, fc, fs, pe = po.ref_step(s, lists)
    m = compound_mask(s)
    if s.n_compounds:
        assert relrms(fc[m], fcr[m]) < FORCE_TOL
        per = ref.potE()[: s.n_compounds * 64]
        assert np.abs(pe[: s.n_compounds * 64] - per).max() <= POTE_TOL * np.abs(per).max()
    assert np.array_equal(fs, fsr)
    ref.close()


@ref_needed
def test_compound_lists_keep_history_like_reference():
    """Engine.cu:168 culls a previous compound pair beyond C+((r_i+r_j)+C),
    while Engine.cu:243-246 adds only pairs within C+((r_i+r_i)+C): a pair in
    between survives only if it was listed before."""
    s = S.make_system("tiny_chains", seed=4)
    C = float(po.ref_cutoff_of(s))
    s.compounds["confining_particle_sphere"][0] = 0.3
    s.compounds["confining_particle_sphere"][1] = 0.9
    k0 = s.states[0]["positions"][s.compounds[0]["key_particle_index"]].astype(np.float64)
    k1 = s.states[1]["positions"][s.compounds[1]["key_particle_index"]].astype(np.float64)
    d_target = C + (0.3 + 0.3 + C) + 0.25          # beyond add, within keep (C + 1.2 + C)
    shift = k0 + np.array([d_target, 0, 0]) - k1
    s.states[1]["positions"][: s.compounds[1]["n_particles"]] += shift.astype(np.float32)
    s.compounds[1]["prev_positions"][: s.compounds[1]["n_particles"]] += shift.astype(np.float32)
    for prev_listed in (False, True):
        ref = po.RefEngine(s)
        prev = (np.array([0, 1, 2]), np.array([1, 0])) if prev_listed else None
        if prev_listed:
            ref.set_nlist(0, prev[0], prev[1])
        ref.update_nlists()
        got_ref = sorted_csr(*ref.nlist(0))
        got = po.ref_nlist(s, prev_cc=prev)[0]
        assert _lists_equal(got_ref, got)
        assert len(got[1]) == (2 if prev_listed else 0)
        ref.close()


def test_oracle_capacity_overflow_is_reported():
    s = S.make_system("tiny_solvent", seed=1)
    with pytest.raises(RuntimeError):
        po.ref_nlist(s, ss_cap=16)
