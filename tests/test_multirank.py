"""CPU, world size 2 over gloo: the multi-rank host logic of bench.py.

Multi-GPU runs are replicas (every rank its own seeded batch, no data-path
collective); the only cross-rank steps are the barrier and the max-over-ranks
time from which the whole-job rate is formed.  Two processes on 127.0.0.1
check exactly those steps, and that the reference arm runs on rank 0 only.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout
from types import SimpleNamespace

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_body(rank, ws, port):
    import numpy as np
    import torch.distributed as dist

    import bench
    from tblite_b200 import geometry

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        # every rank its own batch
        mols = geometry.water_clusters(4, seed=bench.rank_seed(rank))
        key = float(sum(float(np.sum(m.xyz)) for m in mols))
        keys = [None] * ws
        dist.all_gather_object(keys, key)
        assert len(set(keys)) == ws, keys
        # the slowest rank's time, on every rank, and the whole-job rate from it
        elapsed = [2.0, 3.0][rank]
        dist.barrier()
        slowest = bench.max_over_ranks(elapsed, ws, device="cpu")
        assert slowest == 3.0
        assert bench.job_rate(ws, 5, len(mols), slowest) == ws * 5 * len(mols) / 3.0
        # one rank: no collective, the value itself
        assert bench.max_over_ranks(elapsed, 1) == elapsed
    finally:
        dist.destroy_process_group()


def test_replica_ranks_gloo():
    mp = pytest.importorskip("torch.multiprocessing")
    mp.spawn(_rank_body, args=(2, _free_port()), nprocs=2, join=True)


def test_reference_arm_runs_on_rank_zero_only():
    import bench

    args = SimpleNamespace(count=4, steps=1, warmup=0)
    out = io.StringIO()
    with redirect_stdout(out):
        assert bench.run_reference(args, ws=2, rank=1) is None
    assert out.getvalue() == ""
