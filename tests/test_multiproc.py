"""Multi-process (replica) path on CPU: world size 2 over gloo.

The JW step shards over independent right-hand sides with no data-path
collective.  These tests check the sharding helpers, that the union of the
ranks' shard solves equals the unsharded solve (bit for bit, oracle `double`
path: each system is solved independently), and the max-over-ranks timing
reduction that bench.py uses."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pfsolve_b200 import replicas
from pfsolve_b200 import workloads as WL


def test_shard_covers_and_balances():
    for total in (0, 1, 7, 131072, 65537):
        for world in (1, 2, 3, 8):
            parts = [replicas.shard(total, r, world) for r in range(world)]
            assert parts[0][0] == 0
            assert sum(c for _, c in parts) == total
            for (s0, c0), (s1, _) in zip(parts, parts[1:]):
                assert s0 + c0 == s1
            assert max(c for _, c in parts) - min(c for _, c in parts) <= 1
    with pytest.raises(ValueError):
        replicas.shard(10, 2, 2)


def test_weighted_shards_of_uneven_timestep():
    ls, Ns, nsys = WL.config4_sizes()
    w = (nsys * Ns).astype(float)
    for world in (2, 4, 8):
        parts = replicas.shard_weighted(w, world)
        assert sorted(i for p in parts for i in p) == list(range(len(ls)))
        loads = [w[p].sum() for p in parts]
        assert max(loads) / (sum(loads) / world) <= 1.01


def test_job_throughput():
    assert replicas.job_throughput(1000, 2.0, 4) == pytest.approx(2e6)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        wl = WL.config3(B=64)
        M, B = wl.M, wl.nrhs
        start, count = replicas.shard(B, rank, world)
        case = O.Case(M=M, batch=count, upperBanded=2, jw_type=13)
        x = O.jw_step(case, wl.jw_bands, wl.rhs[start * M:(start + count) * M], "d")
        t = replicas.max_over_ranks(float(10 + rank))
        q.put((rank, start, x, t))
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_equal_unsharded_solve():
    from oracle import oracle as O
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    wl = WL.config3(B=64)
    whole = O.jw_step(O.Case(M=wl.M, batch=wl.nrhs, upperBanded=2, jw_type=13), wl.jw_bands, wl.rhs, "d")
    got = np.concatenate([r[2] for r in res])
    assert np.array_equal(got, whole)
    assert all(r[3] == 11.0 for r in res)  # max over ranks of 10 + rank
