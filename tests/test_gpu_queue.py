"""The uneven-n queue (sbg_queue_create / sbg_launch_queue) on the GPU.

Every pair of a shuffled mixed-n batch is checked against the LAPACK oracle with the same
gates as test_gpu_parity.py, and against the per-n solver bit for bit (the queue runs the
same kernels with the same schedules, only gathered into per-n buckets and replayed as one
CUDA graph).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import sbg
from sbg import workloads as wl
from test_gpu_parity import check

pytestmark = pytest.mark.gpu


def make_batch(oracle_mod, counts, seed=0):
    """Shuffled batch with counts[n] pairs of each n: (ns, per-pair flat A list, B list)."""
    ns = np.concatenate([np.full(c, n, dtype=np.int32) for n, c in counts.items()])
    rng = np.random.default_rng(seed)
    rng.shuffle(ns)
    mats = {n: oracle_mod.gen_fixture_pairs(n, c, seed + n, "random") for n, c in counts.items()}
    used = {n: 0 for n in counts}
    As, Bs = [], []
    for n in ns:
        k = used[int(n)]; used[int(n)] += 1
        As.append(np.asarray(mats[int(n)][0][k]).reshape(-1)); Bs.append(np.asarray(mats[int(n)][1][k]).reshape(-1))
    return ns, As, Bs


def launch(q, As, Bs, stream=None):
    A = torch.as_tensor(np.concatenate(As)).cuda()
    B = torch.as_tensor(np.concatenate(Bs)).cuda()
    W = torch.empty(q.vector_elements, dtype=torch.float64, device="cuda")
    X = torch.empty_like(A)
    info = torch.full((len(q),), -7, dtype=torch.int32, device="cuda")
    q.launch(A, B, W, X, info, stream)
    torch.cuda.synchronize()
    return A, B, W, X, info


def per_n(ns, n, As, Bs, W, X):
    pos = np.nonzero(ns == n)[0]
    Wl = sbg.unpack(W.cpu(), ns, square=False)
    Xl = sbg.unpack(X.cpu(), ns)
    A = np.stack([As[p] for p in pos]); B = np.stack([Bs[p] for p in pos])
    return pos, A, B, np.stack([Wl[p].numpy() for p in pos]), np.stack([Xl[p].numpy() for p in pos])


COUNTS = {12: 6, 24: 5, 32: 5, 54: 8, 96: 4, 128: 3, 5: 3, 77: 3, 130: 2}


def test_queue_matches_oracle_and_per_n_solver(oracle_mod):
    ns, As, Bs = make_batch(oracle_mod, COUNTS, seed=1)
    q = sbg.Queue(ns)
    assert [b["n"] for b in q.buckets()] == sorted(COUNTS, reverse=True)
    assert sum(b["count"] for b in q.buckets()) == len(ns)
    _, _, W, X, info = launch(q, As, Bs)
    info = info.cpu().numpy()
    for n in COUNTS:
        pos, A, B, Wq, Xq = per_n(ns, n, As, Bs, W, X)
        Wr, Xr, _ = oracle_mod.hegv(A, B, n, nthreads=8)
        check(A, B, Wq, Xq, info[pos], Wr, Xr, n)
        s = sbg.Solver(n)                            # the per-n solver gives the same bits
        dA = torch.as_tensor(A).cuda(); dB = torch.as_tensor(B).cuda()
        W1 = torch.empty((len(pos), n), dtype=torch.float64, device="cuda"); X1 = torch.empty_like(dA)
        i1 = torch.empty(len(pos), dtype=torch.int32, device="cuda")
        s.launch(dA, dB, W1, X1, i1)
        torch.cuda.synchronize()
        assert np.array_equal(W1.cpu().numpy(), Wq) and np.array_equal(X1.cpu().numpy(), Xq)


def test_queue_graph_reuse_and_rebuild(oracle_mod):
    ns, As, Bs = make_batch(oracle_mod, {16: 4, 54: 4, 100: 2}, seed=2)
    q = sbg.Queue(ns)
    A, B, W, X, info = launch(q, As, Bs)
    assert q.graph_builds == 1
    W0, X0 = W.clone(), X.clone()
    q.launch(A, B, W, X, info)                       # same buffers: the graph is replayed
    torch.cuda.synchronize()
    assert q.graph_builds == 1
    assert torch.equal(W, W0) and torch.equal(X, X0)
    X2 = torch.empty_like(X)
    q.launch(A, B, W, X2, info)                      # new output buffer: captured again
    torch.cuda.synchronize()
    assert q.graph_builds == 2
    assert torch.equal(X2, X0)
    s = torch.cuda.Stream()                          # any stream
    X3 = torch.empty_like(X)
    q.launch(A, B, W, X3, info, s)
    s.synchronize()
    assert torch.equal(X3, X0)


def test_queue_chunks_and_mixed_buckets(oracle_mod):
    ns, As, Bs = make_batch(oracle_mod, {20: 7, 54: 5, 96: 3}, seed=3)
    q = sbg.Queue(ns, precision="mixed", chunk_pairs=2)      # several chunks per bucket
    bk = {b["n"]: b for b in q.buckets()}
    assert all(b["chunk"] == 2 for b in bk.values())
    assert bk[20]["precision"] == "mixed" and bk[54]["precision"] == "mixed"
    assert bk[96]["precision"] == ("mixed" if 96 <= sbg.max_n("mixed") else "fp64")
    _, _, W, X, info = launch(q, As, Bs)
    info = info.cpu().numpy()
    for n in (20, 54, 96):
        pos, A, B, Wq, Xq = per_n(ns, n, As, Bs, W, X)
        Wr, Xr, _ = oracle_mod.hegv(A, B, n, nthreads=8)
        check(A, B, Wq, Xq, info[pos], Wr, Xr, n)


def test_queue_uneven_workload(oracle_mod):
    """The uneven spin-wave batch (n in {12, 24, 32, 54, 96, 128}, 10/20/20/30/15/5 %)."""
    ns, A, B = wl.uneven(200, seed=3)
    q = sbg.Queue(ns)
    A = A.cuda(); B = B.cuda()
    W = torch.empty(q.vector_elements, dtype=torch.float64, device="cuda")
    X = torch.empty_like(A)
    info = torch.empty(len(ns), dtype=torch.int32, device="cuda")
    q.launch(A, B, W, X, info)
    torch.cuda.synchronize()
    As = [t.numpy() for t in sbg.unpack(A.cpu(), ns)]
    Bs = [t.numpy() for t in sbg.unpack(B.cpu(), ns)]
    info = info.cpu().numpy()
    for n in sorted(set(ns.tolist())):
        pos, a, b, Wq, Xq = per_n(ns, n, As, Bs, W, X)
        Wr, Xr, _ = oracle_mod.hegv(a, b, n, nthreads=8)
        check(a, b, Wq, Xq, info[pos], Wr, Xr, n, relative=True)


def test_queue_info_lands_on_the_right_pair(oracle_mod):
    ns, As, Bs = make_batch(oracle_mod, {30: 4, 90: 3}, seed=4)
    bad = [i for i, n in enumerate(ns) if n == 90][1]
    Bm = Bs[bad].reshape(90, 90).T.copy()            # column-major -> [i, j]
    Bm -= 1e4 * np.eye(90)
    Bs = list(Bs); Bs[bad] = Bm.T.reshape(-1)
    q = sbg.Queue(ns)
    _, _, W, X, info = launch(q, As, Bs)
    info = info.cpu().numpy()
    assert info[bad] == 90 + 1
    assert (np.delete(info, bad) == 0).all()
    assert np.isnan(sbg.unpack(W.cpu(), ns, square=False)[bad].numpy()).all()


def test_queue_edges():
    q = sbg.Queue([])
    assert len(q) == 0 and q.buckets() == []
    e = torch.empty(0, dtype=torch.complex128, device="cuda")
    q.launch(e, e, torch.empty(0, dtype=torch.float64, device="cuda"), e.clone(),
             torch.empty(0, dtype=torch.int32, device="cuda"))
    with pytest.raises(sbg.SolverError):
        sbg.Queue([12, 0, 54])
    with pytest.raises(sbg.SolverError):
        sbg.Queue([12, sbg.max_n("fp64") + 1])
