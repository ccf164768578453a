"""Seeded workload generators (CPU): sizes, separations, velocities and the
reference-layout topology they produce."""
import math

import numpy as np
import pytest

from quantom_b200 import systems as S


def _min_sep(pos, L):
    pos = np.asarray(pos, np.float64)
    best = np.inf
    for i in range(0, len(pos), 256):
        d = pos[i:i + 256, None, :] - pos[None, :, :]
        d -= L * np.round(d / L)
        r2 = (d ** 2).sum(-1)
        for k in range(min(256, len(pos) - i)):
            r2[k, i + k] = np.inf
        best = min(best, r2.min())
    return math.sqrt(best)


@pytest.mark.parametrize("name", ["tiny_solvent", "tiny_chains", "small_bridged"])
def test_generator_basics(name):
    s = S.make_system(name, seed=3)
    spec = S.CONFIGS[name]
    assert s.n_solvents == spec.n_solvents
    pos = [s.solvents["pos"]]
    for c in range(s.n_compounds):
        n = s.compounds[c]["n_particles"]
        pos.append(np.mod(s.states[c]["positions"][:n], spec.box_len))
    allpos = np.concatenate(pos)
    # chain beads closer than 0.28 are bonded neighbours only (1-2, 1-3)
    sol = s.solvents["pos"]
    assert _min_sep(sol, spec.box_len) >= spec.min_sep * (1 - 1e-5)
    assert ((sol >= 0) & (sol <= spec.box_len)).all()
    # Maxwell-Boltzmann velocities, no centre-of-mass drift
    v = s.solvents["pos"].astype(np.float64) - s.solvents["pos_tsub1"]
    v /= spec.dt
    T = (spec.solvent_mass * (v ** 2).sum(1)).mean() / (3 * S.R_GAS)
    assert abs(T - spec.temperature) < 0.15 * spec.temperature
    assert len(allpos) == s.n_particles


def test_generator_deterministic():
    a = S.make_system("tiny_chains", seed=11)
    b = S.make_system("tiny_chains", seed=11)
    assert np.array_equal(a.solvents, b.solvents)
    assert a.compounds.tobytes() == b.compounds.tobytes()
    assert a.bridges.tobytes() == b.bridges.tobytes()
    c = S.make_system("tiny_chains", seed=12)
    assert not np.array_equal(a.solvents["pos"], c.solvents["pos"])


def test_chain_topology_and_compound_convention():
    s = S.make_system("small_bridged", seed=5)
    cs = S.CONFIGS["small_bridged"].chains
    L = S.CONFIGS["small_bridged"].box_len
    # 2 chains of 96 -> compounds of 64 + 32 each, one bridge per chain
    assert s.n_compounds == 4 and len(s.bridges) == 2
    for c in range(s.n_compounds):
        cp = s.compounds[c]
        n = cp["n_particles"]
        pos = s.states[c]["positions"][:n].astype(np.float64)
        assert ((pos[0] >= 0) & (pos[0] < L)).all()                      # particle 0 in the box
        assert np.linalg.norm(pos - pos[0], axis=1).max() < 0.5 * L     # the rest next to it
        for b in cp["singlebonds"][: cp["n_singlebonds"]]:
            r = np.linalg.norm(pos[b["atom_indexes"][0]] - pos[b["atom_indexes"][1]])
            assert abs(r - cs.bond_r0) < 1e-5
        # bonded LJ exclusions: 1-2, 1-3, 1-4 (distributeLJIgnores)
        assert cp["lj_ignore_list"]["n_ignores"][:n].max() <= 6
        assert 0 <= cp["key_particle_index"] < n
    br = s.bridges[0]
    assert br["n_singlebonds"] == 1 and br["n_anglebonds"] == 2 and br["n_dihedrals"] == 3
    assert br["n_particles"] == 6
