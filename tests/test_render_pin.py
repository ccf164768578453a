"""Pinning the rasterizer restatement (CPU).

The oracle's RenderBall list (oracle/lima_oracle.c part C, which the GPU
rasterizer is checked against bit for bit) against the reference's own
Rasterizer run on the host: loadCompoundatomsKernel, loadSolventatomsKernel,
processAtomsKernel and mergeSortAPI (Rasterizer.cu:12-293) compiled from the
reference sources by oracle/build_ref.sh and launched by ref_emu.cpp's
ref_render on the same box.  Bar: every field of every ball identical, in
the same order, including the order of equal depths (a box whose solvents
sit on a lattice, so whole planes share one depth).
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from quantom_b200 import layout as L
from quantom_b200 import systems as S

pytestmark = pytest.mark.skipif(not po.ref_available(), reason="reference build (oracle/_ref) not present")

FIELDS = ("pos", "radius", "color", "disable")


def _same(a, b):
    assert len(a) == len(b)
    for f in FIELDS:
        x, y = a[f], b[f]
        if x.dtype.kind == "f":
            x, y = x.view(np.uint32), y.view(np.uint32)
        assert np.array_equal(x, y), f


def _lattice_box(side, box):
    """side^3 solvents on a cubic lattice: side^2 of them share each depth."""
    g = (np.arange(side, dtype=np.float32) + 0.5) * np.float32(box / side)
    p = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    sol = np.zeros(len(p), L.Solvent)
    sol["pos"] = p
    sol["pos_tsub1"] = p
    spec = S.SystemSpec("lattice", box, len(p), cutoff=1.2, dt=2e-6)
    ff = np.zeros(1, L.ForceField)
    ff["particle_parameters"][0][0] = (0.018, 0.3166, 650.0)
    return S.System(spec, 0, ff, np.zeros(0, L.Compound), np.zeros(0, L.CompoundState), sol,
                    np.zeros(0, L.CompoundBridgeCompact))


def _oracle_balls(s, ref):
    comps, states, sols = ref.state()
    pos, kind = po.render_slots(s, [states[c]["positions"] for c in range(s.n_compounds)], sols["pos"])
    return po.render_balls(pos, kind, s.spec.box_len)


@pytest.mark.parametrize("name,steps", [("tiny_chains", 0), ("tiny_chains", 3), ("small_bridged", 2),
                                        ("lattice", 0)])
def test_oracle_balls_match_reference_rasterizer(name, steps):
    s = _lattice_box(8, 4.0) if name == "lattice" else S.make_system(name, seed=11)
    ref = po.RefEngine(s, n_threads=4)
    if steps:
        ref.update_nlists()
        ref.step(steps)
    got = ref.render()
    _same(_oracle_balls(s, ref), got)
    if name == "lattice":
        y = got["pos"][:, 1]
        assert (np.diff(y) == 0).sum() > len(y) // 2      # ties are most of the list
    ref.close()
