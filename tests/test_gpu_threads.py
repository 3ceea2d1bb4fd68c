"""Host threads calling the library at the same time.

The reference's launchers set their shared-memory attribute through an unsynchronised static
(src/geneig_fixed.cu:481-487) and its autotune memo is an unguarded static map
(src/nvrtc/nvrtc_solver.cpp:647, 973-990); here those are std::call_once / mutex-guarded.  These
tests create solvers and launch from several threads at once (ctypes releases the GIL during the
calls), each thread on its own stream, and require the results to equal, bit for bit, a
sequential run of the same inputs.
"""
from __future__ import annotations

import threading

import numpy as np
import pytest
import torch

import sbg

pytestmark = pytest.mark.gpu

SIZES = [20, 54, 33, 96, 12, 54, 130, 7]


def solve_on_stream(n, A, B, stream):
    with torch.cuda.stream(stream):
        dA = torch.as_tensor(A).cuda(non_blocking=False)
        dB = torch.as_tensor(B).cuda(non_blocking=False)
        W = torch.empty((A.shape[0], n), dtype=torch.float64, device="cuda")
        X = torch.empty_like(dA)
        info = torch.empty(A.shape[0], dtype=torch.int32, device="cuda")
        s = sbg.Solver(n)
        s.launch(dA, dB, W, X, info, stream)
        stream.synchronize()
        out = (W.cpu().numpy(), X.cpu().numpy(), info.cpu().numpy())
        s.close()
    return out


def test_concurrent_create_and_launch(oracle_mod):
    inputs = [oracle_mod.gen_fixture_pairs(n, 6, 100 + i, "random") for i, n in enumerate(SIZES)]
    ref = [solve_on_stream(n, A, B, torch.cuda.Stream()) for n, (A, B) in zip(SIZES, inputs)]
    results = [None] * len(SIZES)
    errors = []
    start = threading.Barrier(len(SIZES))

    def worker(i):
        try:
            start.wait()
            results[i] = solve_on_stream(SIZES[i], *inputs[i], torch.cuda.Stream())
        except Exception as e:                       # noqa: BLE001 - reported below
            errors.append((i, repr(e)))

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(len(SIZES))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    for i, n in enumerate(SIZES):
        assert (results[i][2] == 0).all()
        assert np.array_equal(results[i][0], ref[i][0]) and np.array_equal(results[i][1], ref[i][1]), n


def test_concurrent_fixed_n54_launches(oracle_mod):
    inputs = [oracle_mod.gen_fixture_pairs(54, 16, 200 + i, "random") for i in range(4)]

    def run_fixed(A, B, stream):
        with torch.cuda.stream(stream):
            dA = torch.as_tensor(A).cuda(); dB = torch.as_tensor(B).cuda()
            W = torch.empty((A.shape[0], 54), dtype=torch.float64, device="cuda")
            X = torch.empty_like(dA)
            info = torch.empty(A.shape[0], dtype=torch.int32, device="cuda")
            sbg.geneig_full_n54_batched(dA, dB, W, X, info, stream)
            stream.synchronize()
            return W.cpu().numpy(), X.cpu().numpy()

    ref = [run_fixed(A, B, torch.cuda.Stream()) for A, B in inputs]
    results = [None] * len(inputs)
    start = threading.Barrier(len(inputs))

    def worker(i):
        start.wait()
        results[i] = run_fixed(*inputs[i], torch.cuda.Stream())

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(len(inputs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    for r, q in zip(results, ref):
        assert r is not None
        assert np.array_equal(r[0], q[0]) and np.array_equal(r[1], q[1])
