"""The multi-rank plumbing of bench.py (replicas, max-over-ranks timing) with
two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from acoustics_b200 import dist
    r = dist.init_from_env(backend="gloo", timeout_s=60)
    # rank r did (r+1) * 1e9 cell-steps in (r+1) * 0.5 s
    thr = dist.weak_scaling_throughput((rank + 1) * 1e9, (rank + 1) * 0.5, r)
    mx = dist.max_over_ranks(float(rank), r)
    dist.barrier(r)
    q.put((rank, thr, mx, r.world))
    dist.shutdown(r)


def test_two_gloo_ranks_aggregate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(i, 2, port, q)) for i in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, thr, mx, world in res:
        assert world == 2
        assert thr == pytest.approx(3e9 / 1.0)     # (1e9 + 2e9) / slowest 1.0 s
        assert mx == 1.0


def test_single_rank_defaults():
    from acoustics_b200 import dist
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    r = dist.init_from_env()
    assert r.world == 1 and r.pg is None
    assert dist.weak_scaling_throughput(5.0, 2.0, r) == 2.5
