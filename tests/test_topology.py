"""Real-topology input (lima_topology_*): the native builder against the box
the reference's own input path builds (LIMA_ForcefieldMaker, ForceFieldMaker,
CompoundBuilder, BoxBuilder; tests/golden/golden_6lzm.npz and, where the
reference tree is present, a live run of it), and its rules on a small system
written here."""
import ctypes
import os
from pathlib import Path

import numpy as np
import pytest

from oracle import pyoracle as po
from quantom_b200 import systems as S

# the reference tree: $LIMA_REF_ROOT, as the oracle build scripts read it
REF = Path(os.environ.get("LIMA_REF_ROOT", "/root/reference"))
DEMO = REF / "Demo"
PRMS = [DEMO / "CHARMM_FF" / n for n in ("par_all36_lipid.prm", "par_all36_na.prm", "par_all36m_prot.prm")]
GRO, TOP = DEMO / "6lzm" / "conf.gro", DEMO / "6lzm" / "topol.top"
have_demo = pytest.mark.skipif(not GRO.exists(), reason="the reference's demo files are not present")


def _same_terms(x, y):
    """Structured term arrays equal field by field (the padding after a
    dihedral's n is left uninitialised by the reference)."""
    return all(np.array_equal(x[f], y[f]) for f in x.dtype.names)


def _same_box(mine, ref):
    """Every field the reference sets, compared up to its counts (bit-exact)."""
    assert len(mine.compounds) == len(ref["compounds"])
    assert len(mine.bridges) == len(ref["bridges"]) and len(mine.solvents) == len(ref["solvents"])
    nt = mine.info["n_atom_types"]
    assert mine.forcefield["particle_parameters"][0][:nt].tobytes() == \
        ref["forcefield"]["particle_parameters"][0][:nt].tobytes()
    for a, b, sa, sb in zip(mine.compounds, ref["compounds"], mine.states, ref["states"]):
        n = int(a["n_particles"])
        assert n == b["n_particles"] and sa["n_particles"] == sb["n_particles"] == n
        for f in ("prev_positions", "atom_types", "atom_color_types", "particle_global_ids"):
            assert a[f][:n].tobytes() == b[f][:n].tobytes(), f
        assert sa["positions"][:n].tobytes() == sb["positions"][:n].tobytes()
        for f in ("center_of_mass", "key_particle_index", "confining_particle_sphere"):
            assert np.array_equal(a[f], b[f]), f
        for arr, cnt in (("singlebonds", "n_singlebonds"), ("anglebonds", "n_anglebonds"),
                         ("dihedrals", "n_dihedrals")):
            m = int(a[cnt])
            assert m == b[cnt] and _same_terms(a[arr][:m], b[arr][:m]), arr
        for i in range(n):
            x, y = a["lj_ignore_list"][i], b["lj_ignore_list"][i]
            k = int(x["n_ignores"])
            assert k == y["n_ignores"]
            assert x["local_ids"][:k].tobytes() == y["local_ids"][:k].tobytes()
            assert x["compound_ids"][:k].tobytes() == y["compound_ids"][:k].tobytes()
    for a, b in zip(mine.bridges, ref["bridges"]):
        n = int(a["n_particles"])
        assert n == b["n_particles"]
        assert a["particle_refs"][:n].tobytes() == b["particle_refs"][:n].tobytes()
        assert a["atom_types"][:n].tobytes() == b["atom_types"][:n].tobytes()
        for arr, cnt in (("singlebonds", "n_singlebonds"), ("anglebonds", "n_anglebonds"),
                         ("dihedrals", "n_dihedrals")):
            m = int(a[cnt])
            assert m == b[cnt] and _same_terms(a[arr][:m], b[arr][:m]), arr
    # positions bit-exact; previous positions come from random velocities in both
    assert mine.solvents["pos"].tobytes() == ref["solvents"]["pos"].tobytes()


@have_demo
def test_6lzm_matches_the_reference_box():
    mine = S.from_topology(GRO, TOP, PRMS)
    ref = np.load(Path(__file__).resolve().parent / "golden" / "golden_6lzm.npz")
    assert mine.info["n_compound_particles"] == 1293 and mine.info["n_atom_types"] == 19
    _same_box(mine, {k: ref[k] for k in ref.files})
    # solvent speeds as the reference's box builder draws them, sqrt(3 R 313 K / M); a
    # 0.1 fs displacement (6.6e-5 nm) of an FP32 position near 3.5 nm keeps ~0.2 % of it
    v = (mine.solvents["pos"].astype(np.float64) - mine.solvents["pos_tsub1"]) / 1e-7
    speed = np.sqrt((v ** 2).sum(1))
    np.testing.assert_allclose(speed, np.sqrt(3 * 8.3144 * 313 / (18.01528e-3)), rtol=1e-2)


@have_demo
@pytest.mark.skipif(not po.ref_input_available(), reason="the reference's input path is not built (make -C oracle ref)")
def test_fixture_is_the_live_reference_box():
    ref = po.ref_input_box(GRO, TOP, PRMS)
    fix = np.load(Path(__file__).resolve().parent / "golden" / "golden_6lzm.npz")
    mine = S.from_topology(GRO, TOP, PRMS)
    _same_box(mine, ref)
    assert ref["solvents"]["pos"].tobytes() == fix["solvents"]["pos"].tobytes()


def test_errors_are_reported():
    lib = S._lib_topology()
    h = ctypes.c_void_p()
    prm = (ctypes.c_char_p * 1)(b"/nonexistent.prm")
    st = lib.lima_topology_build(b"/nonexistent.gro", b"/nonexistent.top", prm, 1, None, ctypes.byref(h))
    assert st != 0 and b"cannot open" in lib.lima_topology_error(h)
    lib.lima_topology_destroy(h)
    assert lib.lima_topology_build(b"a", b"b", prm, 0, None, ctypes.byref(h)) != 0
    lib.lima_topology_destroy(h)


# ------------------------------------------------------------ small system --
PRM = """* minimal parameter file
ATOMS
MASS  -1  CT2  12.01100
MASS  -1  HA2   1.00800
MASS  -1  OT   15.99940

BONDS
CT2  CT2   222.500     1.5300
CT2  HA2   309.000     1.1110

ANGLES
CT2  CT2  CT2   58.350    113.60
HA2  CT2  CT2   26.500    110.10

DIHEDRALS
CT2  CT2  CT2  CT2     0.1500  1     0.00

NONBONDED nbxmod  5 atom cdiel
CT2    0.000000  -0.055000     2.175000
HA2    0.000000  -0.035000     1.340000
OT     0.000000  -0.152100     1.768200

END
"""


def _write_small(tmp, n_res=10, per_res=5, waters=()):
    """A linear chain of n_res residues of per_res carbons (one hydrogen on
    each residue's first carbon), bonded end to end, plus waters.  Conf atom
    names are the type names: the builder maps names onto non-bonded types by
    prefix, as the reference does."""
    atoms, lines = [], []
    serial = 0
    for r in range(n_res):
        for k in range(per_res):
            serial += 1
            x = 0.153 * (r * per_res + k)
            atoms.append((serial, "CT2", r + 1, "CT2", x))
            lines.append(f"{r + 1:5d}{'RES':<5s}{'CT2':>5s}{serial:5d}{x:8.3f}{1.000:8.3f}{1.000:8.3f}")
            if k == 0:
                serial += 1
                atoms.append((serial, "HA2", r + 1, "HA2", x))
                lines.append(f"{r + 1:5d}{'RES':<5s}{'HA2':>5s}{serial:5d}{x:8.3f}{1.100:8.3f}{1.000:8.3f}")
    carbons = [a[0] for a in atoms if a[1] == "CT2"]
    for w, (x, y, z) in enumerate(waters):
        serial += 1
        lines.append(f"{n_res + 1 + w:5d}{'SOL':<5s}{'OT':>5s}{serial:5d}{x:8.3f}{y:8.3f}{z:8.3f}")
    gro = tmp / "conf.gro"
    gro.write_text("small chain\n" + f"{len(lines)}\n" + "\n".join(lines) + "\n   5.00000   5.00000   5.00000\n")
    top = ["[ moleculetype ]", "Small 3", "", "[ atoms ]"]
    for (s, t, r, name, _) in atoms:
        top.append(f"{s:6d} {t:>6s} {r:6d} {'RES':>6s} {name:>6s} {s:6d} 0.0 12.011")
    top += ["", "[ bonds ]"]
    for a, b in zip(carbons, carbons[1:]):
        top.append(f"{a:5d} {b:5d} 1")
    for h in (a[0] for a in atoms if a[1] == "HA2"):
        top.append(f"{h - 1:5d} {h:5d} 1")
    top += ["", "[ angles ]"]
    for a, b, c in zip(carbons, carbons[1:], carbons[2:]):
        top.append(f"{a:5d} {b:5d} {c:5d} 5")
    top += ["", "[ dihedrals ]"]
    for a, b, c, d in zip(carbons, carbons[1:], carbons[2:], carbons[3:]):
        top.append(f"{a:5d} {b:5d} {c:5d} {d:5d} 9")
    top.append("")
    (tmp / "topol.top").write_text("\n".join(top) + "\n")
    (tmp / "small.prm").write_text(PRM)
    return tmp / "conf.gro", tmp / "topol.top", [tmp / "small.prm"]


def test_small_chain_packing_bridges_and_parameters(tmp_path):
    gro, top, prms = _write_small(tmp_path)
    s = S.from_topology(gro, top, prms, S.topology_options(box_len=5.0, solvate=0))
    # a residue opens a new compound once the current one holds more than 32 particles:
    # 7 residues x 5 heavy atoms, then 3 (hydrogens left out)
    assert list(s.compounds["n_particles"]) == [35, 15]
    assert len(s.bridges) == 1
    br = s.bridges[0]
    # the bridge holds the terms that span compounds 0 and 1: one bond, two angles, three dihedrals
    assert (br["n_singlebonds"], br["n_anglebonds"], br["n_dihedrals"]) == (1, 2, 3)
    c0, c1 = s.compounds
    assert (c0["n_singlebonds"], c1["n_singlebonds"]) == (34, 14)
    # CHARMM units as the reference converts them (ForcefieldMerger.h:64-94): kcal -> J with
    # 4184 (epsilon) and 4183 (force constants), Rmin/2 (A) x 2 / 10 as sigma (nm)
    b = c0["singlebonds"][0]
    assert b["b0"] == np.float32(np.float32(1.53) * np.float32(0.1))
    assert b["kb"] == np.float32(np.float32(222.5) * np.float32(4183) * np.float32(100))
    pp = s.forcefield["particle_parameters"][0]
    assert pp[1]["sigma"] == np.float32(0.435) and abs(pp[1]["epsilon"] - 0.055 * 4184) < 1e-3
    # LJ exclusions: every pair sharing a bond, angle or dihedral (1-2, 1-3, 1-4 along the chain)
    ig = c0["lj_ignore_list"][10]
    assert sorted(ig["local_ids"][: ig["n_ignores"]]) == [7, 8, 9, 11, 12, 13]
    # centred in the box: the mean of the compound centres at box_len / 2
    com = np.mean([c["prev_positions"][: c["n_particles"]].mean(0) for c in s.compounds], axis=0)
    np.testing.assert_allclose(com, 2.5, atol=1e-5)


def test_small_chain_solvent_room_rules(tmp_path):
    # waters: far from everything; 0.1 nm from a chain atom (dropped); 0.2 nm from the
    # first water (dropped); 0.3 nm from the first water (kept)
    gro, top, prms = _write_small(tmp_path, waters=[(3.0, 3.5, 3.5), (0.0, 1.1, 1.0), (3.0, 3.7, 3.5),
                                                   (3.0, 3.8, 3.5)])
    s = S.from_topology(gro, top, prms, S.topology_options(box_len=5.0))
    assert len(s.solvents) == 2
