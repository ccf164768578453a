"""The multi-GPU path is replicas only: one process per GPU, no data-path
collective; the ranks share a barrier around the timed region and the max
of their step times, and rank 0 alone prints the result.  That plumbing is
run here as world_size-2 gloo process groups on host processes."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, values):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, str(ROOT))
    import bench
    ws, r, local, pg = bench.dist_setup(None, backend="gloo", timeout_s=30)
    try:
        assert (ws, r, local) == (world, rank, rank) and pg is not None
        bench.barrier(pg)
        got = bench.max_over_ranks(values[rank], pg, torch.device("cpu"))
        assert got == max(values), (rank, got)
        bench.barrier(pg)
    finally:
        pg.destroy_process_group()


def test_max_over_ranks_and_barrier_with_two_gloo_ranks():
    mp.spawn(_rank_main, args=(2, _free_port(), [0.0712, 0.0735]), nprocs=2, join=True)


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT))
    import bench
    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        ws, rank, local, pg = bench.dist_setup(None, backend="gloo")
        assert (ws, rank, local, pg) == (1, 0, 0, None)
        assert bench.max_over_ranks(1.5, pg, torch.device("cpu")) == 1.5
    finally:
        os.environ.update(env)


def test_reference_arm_under_torchrun_prints_one_line_from_rank_0():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "1", "--workload", "lj_solvent_4096"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["value"] == d["value"]
