"""Multi-rank host logic on CPU: world_size-2 gloo ranks shard a batch with no
data-path collective, solve their shards (the LAPACK oracle stands in for the
GPU here), and the gathered results equal the single-process solve; timing is
reduced with MAX over ranks, as bench.py does."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from sbg.sharding import shard_bounds, shard_uneven


def test_shard_bounds_cover_exactly():
    for total in (0, 1, 7, 262144):
        for world in (1, 2, 3, 8):
            got = [shard_bounds(total, world, r) for r in range(world)]
            assert sum(c for _, c in got) == total
            pos = 0
            for s, c in got:
                assert s == pos
                pos += c
            assert max(c for _, c in got) - min(c for _, c in got) <= 1


def test_shard_uneven_balances_cost():
    from sbg.workloads import uneven_sizes
    ns = uneven_sizes(20000, seed=3)
    parts = [shard_uneven(ns, 4, r) for r in range(4)]
    allidx = np.sort(np.concatenate(parts))
    assert np.array_equal(allidx, np.arange(len(ns)))
    cost = [float((ns[p].astype(float) ** 3).sum()) for p in parts]
    assert max(cost) / min(cost) < 1.05


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    sys.path[:0] = out["paths"]
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    import torch
    from oracle import oracle as O
    from sbg.sharding import shard_bounds
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    n, total = 16, 10
    H, S = O.gen_fixture_pairs(n, total, 42, "random")
    s0, c = shard_bounds(total, world, rank)
    W, U, info = O.hegv(H[s0:s0 + c], S[s0:s0 + c], n)
    gathered = [None] * world
    dist.all_gather_object(gathered, (s0, W.tolist(), info.tolist()))
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        Wfull, _, _ = O.hegv(H, S, n)
        Wg = np.concatenate([np.array(w) for _, w, _ in sorted(gathered)], axis=0)
        out["ok"] = bool(np.array_equal(Wg, Wfull)) and float(t.item()) == float(world)
    dist.destroy_process_group()


def test_gloo_two_ranks_shard_and_gather():
    import sys
    mgr = mp.Manager()
    out = mgr.dict()
    out["paths"] = [p for p in sys.path if p]
    port = _free_port()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    assert out.get("ok") is True
