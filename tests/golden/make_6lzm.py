"""Writes tests/golden/golden_6lzm.npz: the box the reference's own input path
builds for its 6LZM demo (T4 lysozyme conf.gro + topol.top, CHARMM36
parameter files; LIMA_ForcefieldMaker, then ForceFieldMaker + CompoundBuilder +
BoxBuilder as Environment.cpp:15-40 does), run from the reference's sources
compiled for the host (oracle/build_ref_input.sh).  The fixture lets GPU tests
and bench.py run the demo system where the reference tree is absent, and pins
the native builder (lima_topology_build) in tests/test_topology.py.

    python tests/golden/make_6lzm.py [reference root]
"""
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import pyoracle as po  # noqa: E402


def demo_paths(ref_root):
    d = Path(ref_root) / "Demo"
    prms = [d / "CHARMM_FF" / n for n in ("par_all36_lipid.prm", "par_all36_na.prm", "par_all36m_prot.prm")]
    return d / "6lzm" / "conf.gro", d / "6lzm" / "topol.top", prms


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LIMA_REF_ROOT", "/root/reference")
    gro, top, prms = demo_paths(ref_root)
    box = po.ref_input_box(gro, top, prms)
    # entries past each count are left uninitialised by the reference: zero them
    for b in box["bridges"]:
        for arr, cnt in (("singlebonds", "n_singlebonds"), ("anglebonds", "n_anglebonds"), ("dihedrals", "n_dihedrals")):
            b[arr][b[cnt]:] = 0
    out = Path(__file__).resolve().parent / "golden_6lzm.npz"
    np.savez_compressed(out, **box)
    print(out, {k: len(v) for k, v in box.items()})


if __name__ == "__main__":
    main()
