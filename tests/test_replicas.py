"""Host logic of the multi-GPU bench (replicas only) on CPU: two ranks over
gloo combine their timings and halo counts the way bench.py does on N GPUs
(the slowest rank's time, the halos of all ranks)."""

import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    w, r, _ = bench.dist_setup(backend="gloo")
    ms, halos = bench.combine_replicas(10.0 + 5.0 * r, 100 * (r + 1), w)
    e2e = bench.max_over_ranks(20.0 - r, w)
    bench.barrier(w)
    q.put((r, ms, halos, e2e))
    dist.destroy_process_group()


def test_two_replicas_over_gloo():
    pytest.importorskip("torch")
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, ms, halos, e2e in out:
        assert ms == 15.0  # the slower rank
        assert halos == 300  # 100 + 200
        assert e2e == 20.0


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.combine_replicas(12.5, 7, 1) == (12.5, 7)
    assert bench.max_over_ranks(3.0, 1) == 3.0
