"""The replicas' host logic across ranks, on CPU with gloo and two processes: the job time is the slowest rank's
(max over ranks) and every replica gets its own scene of the same distribution. The reduction itself has no
cross-GPU exchange (each rank reduces its own problem), so this is the whole N > 1 path apart from the device work."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sys.path.insert(0, str(ROOT))
        import bench
        t = bench.max_over_ranks(1.5 + rank, world, "cpu")
        sys.path.insert(0, str(ROOT / "tests"))
        from conftest import load_package
        bls = load_package()
        spec = bench.replica_spec(bls.scenes.workload("sparse_1000x200k"), rank, world)
        out.put((rank, t, spec.seed, spec.npoints, spec.ncams))
    finally:
        torch.distributed.destroy_process_group()


def test_two_ranks_max_time_and_own_scenes():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [2.5, 2.5]                    # both ranks see the slowest rank's time
    assert got[0][2] != got[1][2]                                # their own seeds
    assert got[0][3:] == got[1][3:]                              # the same scene sizes


def test_one_rank_is_unchanged():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.25, 1, "cpu") == 3.25
    sentinel = object()
    assert bench.replica_spec(sentinel, 0, 1) is sentinel
