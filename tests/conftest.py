"""Shared test set-up.

Markers: ``gpu`` — needs a CUDA device and the built liblima_b200.so; the
GPU tests call the product through its C-ABI and compare with the CPU oracle
(oracle/) and with fixtures of the reference itself (tests/golden/).
"""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and quantom_b200/liblima_b200.so")


def _cuda_device_present() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """A CUDA device must be present; the product library must then load —
    a missing library on a GPU machine is a failure, not a skip."""
    if not _cuda_device_present():
        pytest.skip("no CUDA device")
    from quantom_b200 import engine
    engine.load_library()
    return engine


def relrms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def compound_mask(system):
    m = np.zeros((system.n_compounds, 64), bool)
    for c in range(system.n_compounds):
        m[c, : system.compounds[c]["n_particles"]] = True
    return m


def load_golden(name):
    from quantom_b200 import systems as S
    z = np.load(GOLDEN / f"{name}.npz")
    spec = S.SystemSpec(name, float(z["box_len"]), len(z["solvents"]), cutoff=float(z["cutoff"]), dt=float(z["dt"]))
    system = S.System(spec, 0, z["forcefield"], z["compounds"], z["states"], z["solvents"], z["bridges"])
    return system, z


def golden_lists(z):
    return {w: (z[f"nl{w}_off"].astype(np.int64), z[f"nl{w}_ids"].astype(np.int64)) for w in range(4)}


def sorted_csr(off, ids):
    off = np.asarray(off, np.int64)
    ids = np.asarray(ids, np.int64)
    return off, np.concatenate([np.sort(ids[off[i]:off[i + 1]]) for i in range(len(off) - 1)]) if len(off) > 1 \
        else np.zeros(0, np.int64)


def make_named(name, seed):
    """A workload by name: "6lzm" (the reference's demo box), "<config>_dry"
    (that config with its solvents removed: compounds and bridges only), or a
    config of quantom_b200.systems."""
    import dataclasses
    from quantom_b200 import systems as S
    if name == "6lzm":
        return S.load_6lzm()
    if name.endswith("_dry"):
        spec = dataclasses.replace(S.CONFIGS[name[:-4]], name=name, n_solvents=0)
        return S.make_system(spec, seed=seed)
    return S.make_system(name, seed=seed)
