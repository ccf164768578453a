"""GPU parity of lima_ss_nlist_noalloc, the allocation-free solvent-solvent
list build, against the CPU oracle's restatement of the reference's list
update (oracle/lima_oracle.c, pinned to the reference) and against the
context entry points (lima_build_nlist + lima_get_nlist(LIMA_NL_SOLVENT_SOLVENT))
on the same inputs.

Integer work, so the bar is the one of the other list tests: identical sorted
rows.  Two calls in a row on different boxes share the library's fixed device
scratch; the second must not see anything of the first.  The test owns every
device buffer (torch allocations); the entry point itself allocates nothing.
"""
import ctypes

import numpy as np
import pytest

from oracle import pyoracle as po
from quantom_b200 import layout as L
from quantom_b200 import systems as S

pytestmark = pytest.mark.gpu

MAX_SOLVENTS = 65536     # LIMA_NOALLOC_MAX_SOLVENTS
LIMA_OK, LIMA_ERR_CAPACITY = 0, 3


def _fn(E):
    lib = E.load_library()
    f = lib.lima_ss_nlist_noalloc
    vp = ctypes.c_void_p
    f.restype = ctypes.c_int
    f.argtypes = [vp, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, vp, vp, vp, vp,
                  ctypes.c_char_p, ctypes.c_size_t]
    return f


def _context_lists(E, system, cap):
    p = E.default_params(box_len=system.spec.box_len, cutoff=system.spec.cutoff, dt=system.spec.dt)
    p.solvent_list_capacity = cap
    with E.Engine(system, p) as eng:
        eng.build_nlist()
        off, ids = eng.nlist(E.NL_SOLVENT_SOLVENT)
    return off.astype(np.int64), ids.astype(np.int64)


def _noalloc(E, f, system, cap):
    import torch
    n = system.n_solvents
    sol = torch.from_numpy(np.ascontiguousarray(system.solvents).view(np.uint8).copy()).cuda()
    ids = torch.full((cap * n,), -1, dtype=torch.int32, device="cuda")
    cnt = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    ovf = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    err = ctypes.create_string_buffer(256)
    st = f(sol.data_ptr(), n, system.spec.box_len, system.spec.cutoff / 2.0, cap, ids.data_ptr(), cnt.data_ptr(),
           ovf.data_ptr(), torch.cuda.current_stream().cuda_stream, err, 256)
    assert st == LIMA_OK, err.value
    torch.cuda.synchronize()
    return ids.cpu().numpy().view(np.uint32).reshape(cap, n), cnt.cpu().numpy(), int(ovf.item())


def _same(ref, got, n):
    off, ref_ids = ref
    ids, cnt, ovf = got
    assert ovf == 0
    assert np.array_equal(cnt.astype(np.int64), np.diff(off))
    for i in range(n):
        assert np.array_equal(ids[: cnt[i], i].astype(np.int64), ref_ids[off[i]: off[i + 1]]), i


def _oracle_lists(system, cap, cutoff=None):
    lists = po.ref_nlist(system, ss_cap=cap, cells=True, cutoff=cutoff)
    return lists[3][0].astype(np.int64), lists[3][1].astype(np.int64)


def test_noalloc_matches_oracle_and_context_two_calls(gpu):
    E = gpu
    f = _fn(E)
    cap = 512
    first = S.make_system("solvated_chains_32k", seed=11)      # 31,000 solvents, 10 nm box
    second = S.make_system("lj_solvent_8192", seed=12)         # 8,192 solvents, 6.3 nm box
    got1 = _noalloc(E, f, first, cap)
    got2 = _noalloc(E, f, second, cap)
    _same(_oracle_lists(first, cap), got1, first.n_solvents)
    _same(_oracle_lists(second, cap), got2, second.n_solvents)
    _same(_context_lists(E, first, cap), got1, first.n_solvents)
    _same(_context_lists(E, second, cap), got2, second.n_solvents)


def _dilute_box(n, box, seed):
    """n solvents uniform in a cubic box (no minimum separation): a list test input."""
    rng = np.random.default_rng(seed)
    sol = np.zeros(n, L.Solvent)
    sol["pos"] = rng.uniform(0.0, box, (n, 3)).astype(np.float32)
    sol["pos_tsub1"] = sol["pos"]
    spec = S.SystemSpec("dilute", box, n, cutoff=0.5, dt=2e-6)
    ff = np.zeros(1, L.ForceField)
    ff["particle_parameters"][0][0] = (0.018, 0.3166, 650.0)
    return S.System(spec, seed, ff, np.zeros(0, L.Compound), np.zeros(0, L.CompoundState), sol,
                    np.zeros(0, L.CompoundBridgeCompact))


def test_noalloc_with_more_than_32_cells_per_side(gpu):
    """A 20 nm box with list radius 0.5 nm has 40 cells of >= 2 * cutoff per
    side; the build caps the grid at 32 (coarser cells, the same candidates
    or more), which must leave the sorted rows unchanged."""
    E = gpu
    f = _fn(E)
    system = _dilute_box(60000, 20.0, 3)
    cutoff = 0.25
    n = system.n_solvents
    import torch
    sol = torch.from_numpy(np.ascontiguousarray(system.solvents).view(np.uint8).copy()).cuda()
    cap = 64
    ids = torch.full((cap * n,), -1, dtype=torch.int32, device="cuda")
    cnt = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    ovf = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    err = ctypes.create_string_buffer(256)
    st = f(sol.data_ptr(), n, system.spec.box_len, cutoff, cap, ids.data_ptr(), cnt.data_ptr(), ovf.data_ptr(),
           torch.cuda.current_stream().cuda_stream, err, 256)
    assert st == LIMA_OK, err.value
    torch.cuda.synchronize()
    got = (ids.cpu().numpy().view(np.uint32).reshape(cap, n), cnt.cpu().numpy(), int(ovf.item()))
    ref = _oracle_lists(system, cap, cutoff=cutoff)
    assert np.diff(ref[0]).sum() > n   # the rows are not empty
    _same(ref, got, n)


def test_noalloc_overflow_and_limits(gpu):
    E = gpu
    f = _fn(E)
    system = S.make_system("lj_solvent_4096", seed=5)
    off, ref_ids = _context_lists(E, system, 512)
    ids, cnt, ovf = _noalloc(E, f, system, 32)
    full = np.diff(off)
    assert ovf != 0 and (full > 32).any()
    assert np.array_equal(cnt, np.minimum(full, 32))
    for i in range(system.n_solvents):
        row = ids[: cnt[i], i].astype(np.int64)
        assert np.all(np.diff(row) > 0)
        assert np.isin(row, ref_ids[off[i]: off[i + 1]]).all()
    # sizes beyond the stated maxima are rejected before any device work
    err = ctypes.create_string_buffer(256)
    dummy = ctypes.c_void_p(256)
    st = f(dummy, MAX_SOLVENTS + 1, 5.0, 0.6, 512, dummy, dummy, dummy, None, err, 256)
    assert st == LIMA_ERR_CAPACITY and b"maximum" in err.value
    st = f(dummy, 100, 5.0, 0.6, 4096, dummy, dummy, dummy, None, err, 256)
    assert st == LIMA_ERR_CAPACITY and b"capacity" in err.value
