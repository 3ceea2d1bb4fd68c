"""GPU parity of the cluster (DSMEM) path for 84 < n <= 256 against the LAPACK oracle.

The same gates as test_gpu_parity.py: eigenvalues within 1e-12 of zhegv (norm-wise for
random-H pairs, relative for the spin-wave pairs), residual ||AX - BXW||/(||A|| ||X||)
<= 1e-12, max|X^H B X - I| <= 1e-12, clusters by subspace angle; plus the reference's
own gates (eig_rel_ref, S-phase < 1e-10) and its n96 / n128 fixtures.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import sbg
from sbg import workloads as wl
from oracle import metrics as Mx
from test_gpu_parity import REF_TOL, TOL, check, run

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", (96, 128))
@pytest.mark.parametrize("mode", ["random", "nearid"])
def test_reference_fixtures_big(n, mode, manifest, golden_W, golden_U0, oracle_mod):
    name = f"n{n}_b8_s42_{mode}"
    e = manifest[name]
    H, S = oracle_mod.gen_fixture_pairs(n, e["batch"], e["seed"], mode)
    W, X, info = run(n, H, S)
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=8)
    check(H, S, W, X, info, Wr, Xr, n)
    assert Mx.eig_rel_ref(W, golden_W[name]).max() < REF_TOL
    assert Mx.eig_rel_norm(W, golden_W[name]).max() <= TOL
    if name in golden_U0:
        assert Mx.phase_err(S[:1], X[:1], golden_U0[name][None], golden_W[name][:1], n).max() < REF_TOL


@pytest.mark.parametrize("n", [85, 97, 113, 129, 150, 161, 192, 200, 233, 256])
def test_big_sizes(n, oracle_mod):
    H, S = oracle_mod.gen_fixture_pairs(n, 3, 21, "random")
    W, X, info = run(n, H, S)
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=8)
    check(H, S, W, X, info, Wr, Xr, n)


@pytest.mark.parametrize("N", [48, 64, 96])
def test_big_bogoliubov(N, oracle_mod):
    A, B = wl.bogoliubov(N, 6, seed=N)
    A, B = A.numpy(), B.numpy()
    n = 2 * N
    W, X, info = run(n, A, B)
    Wr, Xr, _ = oracle_mod.hegv(A, B, n, nthreads=8)
    check(A, B, W, X, info, Wr, Xr, n, relative=True)


@pytest.mark.parametrize("N", [48, 96])
def test_big_near_goldstone(N, oracle_mod):
    """kappa(B) ~ 1e8 at n = 96 and 192: eigenvalues against each one's perturbation scale
    |l_i| kappa_i + ||C|| (see test_gpu_parity.test_near_goldstone_both_forms), backward
    error at the FP64 level of LAPACK's own."""
    n = 2 * N
    A, B = wl.bogoliubov(N, 4, seed=11, frac=1e-3, goldstone=1e-8)
    A, B = A.numpy(), B.numpy()
    Wr, Xr, _ = oracle_mod.hegv(A, B, n, nthreads=8)
    normB = np.linalg.norm(Mx.as_mats(B, n), ord=2, axis=(1, 2))
    cond = normB[:, None] * np.linalg.norm(Mx.as_mats(Xr, n), axis=1) ** 2
    assert cond.max() > 1e7
    scale = np.abs(Wr) * cond + np.abs(Wr).max(axis=1, keepdims=True)
    res_ref = float(Mx.residual(A, B, Xr, Wr, n).max())
    orth_ref = float(Mx.orth(B, Xr, n).max())
    W, X, info = run(n, A, B)
    assert (info == 0).all()
    assert (np.abs(W - Wr) / scale).max() < 1e-12
    assert Mx.residual(A, B, X, W, n).max() < max(1e-12, 4 * res_ref)
    assert Mx.orth(B, X, n).max() < max(1e-9, 4 * orth_ref)


def test_big_not_positive_definite_and_nan(oracle_mod):
    n = 96
    H, S = oracle_mod.gen_fixture_pairs(n, 5, 4, "random")
    Sm = Mx.as_mats(S.copy(), n).copy()
    Sm[1] -= 1e4 * np.eye(n)                       # fails at the first minor
    Sm[3, 70, 70] = -1.0                           # fails at a later minor
    Sbad = Mx.from_mats(Sm)
    H = H.copy()
    H[4, 9] = np.nan                               # NaN in A: the QL cannot converge
    W, X, info = run(n, H, Sbad)
    assert info[1] == n + 1
    assert n + 1 < info[3] <= 2 * n
    assert 1 <= info[4] <= n
    for p in (1, 3):
        assert np.isnan(W[p]).all() and np.isnan(X[p]).all()
    good = [0, 2]
    Wr, Xr, _ = oracle_mod.hegv(H[good], Sbad[good], n, nthreads=8)
    check(H[good], Sbad[good], W[good], X[good], info[good], Wr, Xr, n)


def test_big_log_overflow_falls_back(monkeypatch, oracle_mod):
    """A rotation log too small for the QL: every pair takes the warp QL with Z in the X buffer."""
    monkeypatch.setenv("SBG_QL_LOG_CAPACITY", "40")
    A, B = wl.bogoliubov(48, 5, seed=5)
    A, B = A.numpy(), B.numpy()
    W, X, info = run(96, A, B)
    Wr, Xr, _ = oracle_mod.hegv(A, B, 96, nthreads=8)
    check(A, B, W, X, info, Wr, Xr, 96, relative=True)


def test_big_chunked_and_deterministic(oracle_mod):
    n = 130
    H, S = oracle_mod.gen_fixture_pairs(n, 7, 3, "nearid")
    s = sbg.Solver(n, workspace_pairs=3)           # three internal chunks
    a = run(s, H, S)
    b = run(s, H, S)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=8)
    check(H, S, a[0], a[1], a[2], Wr, Xr, n)


def test_big_limits():
    assert sbg.max_n("fp64") == 256
    with pytest.raises(sbg.SolverError):
        sbg.Solver(257)
    mx = sbg.max_n("mixed")                  # the complex64 Householder's tile: 235 on B200
    assert 192 <= mx < 256
    with pytest.raises(sbg.SolverError):
        sbg.Solver(mx + 1, precision="mixed")


@pytest.mark.parametrize("n", [72, 96, 160, 192])
def test_big_scalar_reduction_schedule(n, oracle_mod):
    """The scalar triangular stages (schedule reduce_tc = 0: the CTA-per-pair kernels for n <= 84,
    above that the one-CTA and cluster kernels doing Cholesky, reduction and Householder together;
    the default above n = 56 is the blocked tensor-core Cholesky, reduction and L^{-H}) against
    zhegv, and equal to the default schedule's results to 1e-12."""
    H, S = oracle_mod.gen_fixture_pairs(n, 4, 29, "random")
    s = sbg.Solver(n)
    assert s.schedule["reduce_tc"] == 1
    W1, X1, info1 = run(s, H, S)
    s.schedule = dict(reduce_tc=0)
    W0, X0, info0 = run(s, H, S)
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=8)
    check(H, S, W0, X0, info0, Wr, Xr, n)
    check(H, S, W1, X1, info1, Wr, Xr, n)
    assert Mx.eig_rel_norm(W0, W1).max() <= 1e-12
