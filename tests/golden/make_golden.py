"""Generates the golden fixtures in this folder from the REFERENCE itself.

The reference LIMA_MD engine (Quantom/Quantom/Engine.cu and its headers) is
compiled for the host by oracle/build_ref.sh into oracle/_ref/libref_lima.so
and run through its own host neighbour-list code and its own three kernels
(emulated CUDA blocks, see oracle/ref_emu.cpp).  For each small seeded system
this script stores the inputs (reference-layout arrays) and the reference's
outputs:

* neighbour lists after Engine::updateNeighborLists from empty lists
  (all four kinds, CSR, list order as the reference leaves it);
* after one Engine::step: the force each particle was integrated with,
  the per-particle potE the kernels logged, the new compound states,
  Compound::prev_positions and solvents;
* after three more steps with a thermostat scalar of 1.02 on the first.

Run from the repository root where the reference sources exist:
    bash oracle/build_ref.sh && python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from quantom_b200 import systems as S  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

CASES = {
    "golden_chain": (S.SystemSpec("golden_chain", 3.0, 520, chains=S.ChainSpec(1, 20), mc_sweeps=20), 101),
    "golden_bridge": (S.SystemSpec("golden_bridge", 3.3, 660, chains=S.ChainSpec(1, 40, compound_size=16),
                                   mc_sweeps=20), 202),
    "golden_solvent": (S.SystemSpec("golden_solvent", 2.6, 560, mc_sweeps=20), 303),
}


def csr_pack(off, ids):
    return np.asarray(off, np.int32), np.asarray(ids, np.uint16)


def make(name):
    spec, seed = CASES[name]
    sysm = S.make_system(spec, seed=seed)
    ref = po.RefEngine(sysm, n_threads=1)
    ref.update_nlists()
    out = {
        "box_len": np.float32(spec.box_len), "cutoff": np.float32(spec.cutoff), "dt": np.float64(spec.dt),
        "forcefield": sysm.forcefield, "compounds": sysm.compounds, "states": sysm.states,
        "solvents": sysm.solvents, "bridges": sysm.bridges,
    }
    for w in range(4):
        off, ids = ref.nlist(w)
        out[f"nl{w}_off"], out[f"nl{w}_ids"] = csr_pack(off, ids)
    ref.step(1, 1.0)
    fc, fs = ref.forces()
    comps, st, sol = ref.state()
    out.update(step1_fc=fc, step1_fs=fs, step1_potE=ref.potE(), step1_states=st,
               step1_prev=comps["prev_positions"], step1_solvents=sol)
    ref.step(1, 1.02)
    ref.step(2, 1.0)
    comps, st, sol = ref.state()
    out.update(step4_states=st, step4_prev=comps["prev_positions"], step4_solvents=sol)
    ref.close()
    np.savez_compressed(Path(__file__).with_name(f"{name}.npz"), **out)
    print(name, sysm.n_compounds, sysm.n_solvents, len(sysm.bridges))


if __name__ == "__main__":
    if not po.ref_available():
        raise SystemExit("oracle/_ref/libref_lima.so missing: run bash oracle/build_ref.sh first")
    for n in CASES:
        make(n)
