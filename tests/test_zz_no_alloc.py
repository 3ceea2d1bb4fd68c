"""The allocation-free entry point, sbg_geneig_full_noalloc_launch.

It exists for callers that must not have a library call cudaMalloc: frameworks
that own all device memory through their own pool, programs that pre-allocate a
fixed memory budget, and loops that cannot absorb the device-wide synchronisation
of cudaMalloc/cudaFree.  Its scratch is a fixed array compiled into the library.

These tests call it through the C ABI (ctypes) and compare it with the regular
entry point, sbg_solver_launch, on the same inputs, for two calls in a row (the
second call finds the first call's data still in the shared scratch), using the
tolerances of the other parity tests; check it against LAPACK zhegv directly at
every kernel family it routes to (register-row n <= 32, warp / column kernels
n <= 56, one CTA per pair for 85..160, clusters above 160); and check that a call
leaves the device's free memory unchanged.  The file is named so that pytest
collects it last; it also runs on its own in a fresh process.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import sbg
from sbg import _lib
from sbg import workloads as wl
from oracle import metrics as Mx

pytestmark = pytest.mark.gpu

TOL = 1e-12
REF_TOL = 1e-10
N = 54


def _noalloc(A, B, n):
    lib = _lib.load()
    batch = A.shape[0]
    W = torch.empty((batch, n), dtype=torch.float64, device="cuda")
    X = torch.empty_like(A)
    info = torch.full((batch,), -7, dtype=torch.int32, device="cuda")
    st = lib.sbg_geneig_full_noalloc_launch(n, ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(B.data_ptr()),
                                            ctypes.c_void_p(W.data_ptr()), ctypes.c_void_p(X.data_ptr()),
                                            ctypes.c_void_p(info.data_ptr()), batch,
                                            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, W, X, info


def _regular(A, B, n):
    s = sbg.Solver(n)
    batch = A.shape[0]
    W = torch.empty((batch, n), dtype=torch.float64, device="cuda")
    X = torch.empty_like(A)
    info = torch.full((batch,), -7, dtype=torch.int32, device="cuda")
    s.launch(A, B, W, X, info)
    return W, X, info


def _scratch_bytes():
    """SBG_NOALLOC_SCRATCH_BYTES as include/sbg/geneig.h defines it."""
    import os
    import re
    from conftest import REPO
    src = open(os.path.join(REPO, "include", "sbg", "geneig.h")).read()
    m = re.search(r"#define\s+SBG_NOALLOC_SCRATCH_BYTES\s+\((\d+)u\s*<<\s*(\d+)\)", src)
    return int(m.group(1)) << int(m.group(2))


def _max_pairs(n):
    lib = _lib.load()
    per = int(lib.sbg_workspace_bytes_per_pair(n, 0))
    p = (_scratch_bytes() - 7 * 256) // per
    while int(lib.sbg_workspace_bytes(n, 0, p + 1)) <= _scratch_bytes():
        p += 1
    return p


def test_noalloc_matches_regular_entry_point_two_calls():
    calls = [wl.bogoliubov(27, 200, seed=11), wl.qsweep(27, grid=64, start=4321, count=_max_pairs(N))]
    for A, B in calls:
        dA, dB = A.cuda(), B.cuda()
        st, W, X, info = _noalloc(dA, dB, N)
        assert st == 0, _lib.load().sbg_last_error().decode()
        Wr, Xr, infor = _regular(dA, dB, N)
        torch.cuda.synchronize()
        W, X, info = W.cpu().numpy(), X.cpu().numpy(), info.cpu().numpy()
        Wr, Xr, infor = Wr.cpu().numpy(), Xr.cpu().numpy(), infor.cpu().numpy()
        assert (info == 0).all() and (infor == 0).all()
        a, b = A.numpy(), B.numpy()
        assert Mx.eig_rel(W, Wr).max() <= TOL
        assert Mx.phase_err(b, X, Xr, Wr, N).max() < REF_TOL
        assert Mx.residual(a, b, X, W, N).max() <= TOL
        assert Mx.orth(b, X, N).max() <= TOL


def test_noalloc_rejects_batches_beyond_its_scratch():
    lib = _lib.load()
    too_many = _max_pairs(N) + 1
    A = torch.zeros((too_many, N * N), dtype=torch.complex128, device="cuda")
    st, _, _, _ = _noalloc(A, A, N)
    assert st == 1                                       # SBG_ERR_INVALID_VALUE
    msg = lib.sbg_last_error().decode()
    assert "scratch" in msg and str(_max_pairs(N)) in msg


@pytest.mark.parametrize("N", [6, 16, 27, 48, 96])
def test_noalloc_against_zhegv_every_kernel_family(N, oracle_mod):
    """n = 12, 32, 54, 96, 192 against LAPACK zhegv with the parity gates, two calls in a row
    with different pairs (the second finds the first's leftovers in the shared scratch)."""
    from test_gpu_parity import check
    n = 2 * N
    batch = min(48 if n <= 96 else 8, _max_pairs(n))
    for seed in (N, N + 1000):
        A, B = wl.bogoliubov(N, batch, seed=seed)
        st, W, X, info = _noalloc(A.cuda(), B.cuda(), n)
        assert st == 0, _lib.load().sbg_last_error().decode()
        torch.cuda.synchronize()
        a, b = A.numpy(), B.numpy()
        Wr, Xr, _ = oracle_mod.hegv(a, b, n, nthreads=8)
        check(a, b, W.cpu().numpy(), X.cpu().numpy(), info.cpu().numpy(), Wr, Xr, n, relative=True)


def test_noalloc_allocates_nothing():
    """After one warm-up call (which may load the module and look up the scratch address),
    further calls leave cudaMemGetInfo's free bytes exactly where they were."""
    A, B = wl.bogoliubov(27, 64, seed=3)
    dA, dB = A.cuda(), B.cuda()
    st, W, X, info = _noalloc(dA, dB, N)
    assert st == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        st = lib.sbg_geneig_full_noalloc_launch(N, ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()),
                                                ctypes.c_void_p(W.data_ptr()), ctypes.c_void_p(X.data_ptr()),
                                                ctypes.c_void_p(info.data_ptr()), 64, stream)
        assert st == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert (info.cpu().numpy() == 0).all()
