"""Layout compatibility and C-ABI surface (CPU only).

* the numpy views (quantom_b200/layout.py), the C-ABI structs
  (include/lima_abi.h, compiled into the oracle library) and the reference's
  own structs (Quantom/Quantom/Bodies.cuh etc., compiled into oracle/_ref)
  have identical sizes and field offsets;
* liblima_b200.so loads without a GPU and exports every function the header
  declares; without a device, lima_create fails with a status, not a crash.
"""
import ctypes
import re

import pytest

from conftest import ROOT
from quantom_b200 import layout as L


def test_numpy_layout_matches_c_abi():
    from oracle import pyoracle as po
    lib = po.oracle_lib()
    assert lib.orc_sizeof(0) == L.Compound.itemsize == 24036
    assert lib.orc_sizeof(1) == L.CompoundState.itemsize == 772
    assert lib.orc_sizeof(2) == L.Solvent.itemsize == 24
    assert lib.orc_sizeof(3) == L.CompoundBridgeCompact.itemsize == 2352
    assert lib.orc_sizeof(4) == L.ForceField.itemsize == 384


def test_numpy_layout_matches_reference_structs():
    from oracle import pyoracle as po
    if not po.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    lib = po.ref_lib()
    for which, (name, size) in L.REF_LAYOUT_IDS.items():
        assert lib.ref_layout(which) == size, name
    for which, (dt, field) in L.REF_OFFSET_IDS.items():
        assert lib.ref_layout(which) == dt.fields[field][1], field


def _declared_functions():
    text = (ROOT / "include" / "lima_abi.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:[\w\*]+\s+)+\**(lima_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from quantom_b200 import engine
    lib = engine.load_library()
    names = _declared_functions()
    assert "lima_step" in names and "lima_create" in names and len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_create_without_device_returns_status():
    from quantom_b200 import engine
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except Exception:
        pass
    lib = engine.load_library()
    p = engine.default_params()
    h = ctypes.c_void_p()
    st = lib.lima_create(ctypes.byref(p), ctypes.byref(h))
    assert st != engine.OK and not h.value


def test_default_params():
    from quantom_b200 import engine
    p = engine.default_params()
    assert p.semantics == engine.SEMANTICS_REFERENCE
    assert p.nlist_period == 200          # Constants.cuh:71
    assert p.thermostat_period == 40      # Constants.cuh:82
    assert abs(p.dt - 1e-7) < 1e-20       # Simulation.cuh:152
    assert abs(p.box_len - 7.0) < 1e-6    # Constants.cuh:35


def test_frame_log_entry_points_reject_a_null_context():
    from quantom_b200 import engine
    lib = engine.load_library()
    lp = engine.LogParams(1, 1, engine.LOG_TRAJ)
    n = ctypes.c_uint64()
    assert lib.lima_log_start(None, ctypes.byref(lp)) == engine.ERR_ARGUMENT
    assert lib.lima_log_stop(None) == engine.ERR_ARGUMENT
    assert lib.lima_log_count(None, ctypes.byref(n)) == engine.ERR_ARGUMENT
    assert lib.lima_log_read(None, 0, 0, None, None, None, None, None, None) == engine.ERR_ARGUMENT
    assert lib.lima_log_write(None, b".") == engine.ERR_ARGUMENT


def test_positions_entry_point_rejects_a_null_context():
    from quantom_b200 import engine
    lib = engine.load_library()
    assert lib.lima_get_positions(None, None, None) == engine.ERR_ARGUMENT
