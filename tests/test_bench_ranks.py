"""The multi-rank plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1.
Each rank decodes its own replica (no collective on the data path); the
timing is the maximum over ranks, and the reference arm runs on rank 0
only."""
import os
import socket
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")
        ref = bench.run_reference(None, rank) if rank else "skipped"
        results[rank] = (got, ref)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_reference_arm_on_rank_zero_only():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        results = m.dict()
        mp.start_processes(_rank, args=(world, _free_port(), results), nprocs=world, join=True,
                           start_method="spawn")
        got = dict(results)
    assert got[0][0] == got[1][0] == 20.0
    assert got[1][1] is None  # rank 1 returns without running the CPU reference


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
