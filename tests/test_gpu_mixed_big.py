"""The mixed form above n = 63 (63 < n <= sbg.max_n("mixed")) against LAPACK zhegv, through the C ABI.

There the complex64 Householder runs one CTA per pair, the FP64 eigenpairs of its T and
Y = Q Z come from the FP64 kernels, and the Ogita-Aishima refinement works on the pair's
matrices in the workspace; pairs it cannot bring to the gates are solved again by the FP64
kernels (a per-pair selection that leaves every other pair untouched).  Gates as in
test_gpu_parity: eigenvalues within 1e-12 of zhegv, residual and B-orthonormality <= 1e-12,
clusters by subspace angle; near-Goldstone pairs against each eigenvalue's perturbation scale.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import sbg
from sbg import workloads as wl
from oracle import metrics as Mx
from test_gpu_parity import check, run

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [64, 65, 72, 84, 85, 96, 100, 128, 129, 160, 161, 192, 235])
def test_mixed_big_sizes(n, oracle_mod):
    """Both sides of every boundary the path crosses: the small-path reflector layout (n <= 84)
    and the cluster back-transform's (n > 84), partial and whole 32-wide refinement tiles, the
    inverse-iteration (85..128) and rotation-log (64..84, 129..) eigenvectors of T, the one-CTA
    (85..160) and cluster (161..) FP64 reductions, and the largest n."""
    if n > sbg.max_n("mixed"):
        pytest.skip(f"the mixed form covers n <= {sbg.max_n('mixed')}")
    H, S = oracle_mod.gen_fixture_pairs(n, 6 if n <= 160 else 3, 13, "random")
    W, X, info = run(n, H, S, "mixed")
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=8)
    check(H, S, W, X, info, Wr, Xr, n)


@pytest.mark.parametrize("N", [32, 48, 64])
def test_mixed_big_bogoliubov(N, oracle_mod):
    """Spin-wave pairs (A = diag(I, -I), Bogoliubov B) at n = 64, 96, 128: pure relative error."""
    n = 2 * N
    A, B = wl.bogoliubov(N, 24, seed=N, frac=1e-3)
    A, B = A.numpy(), B.numpy()
    W, X, info = run(n, A, B, "mixed")
    Wr, Xr, _ = oracle_mod.hegv(A, B, n, nthreads=8)
    check(A, B, W, X, info, Wr, Xr, n, relative=True)


@pytest.mark.parametrize("n", [64, 96, 128])
@pytest.mark.parametrize("mode", ["random", "nearid"])
def test_mixed_big_reference_fixtures(n, mode, manifest, golden_W, oracle_mod):
    name = f"n{n}_b8_s42_{mode}"
    if name not in manifest:
        pytest.skip(f"no fixture {name}")
    e = manifest[name]
    H, S = oracle_mod.gen_fixture_pairs(n, e["batch"], e["seed"], mode)
    W, X, info = run(n, H, S, "mixed")
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=8)
    check(H, S, W, X, info, Wr, Xr, n)
    assert Mx.eig_rel_norm(W, golden_W[name]).max() <= 1e-12


@pytest.mark.parametrize("n", [72, 96])
def test_mixed_big_redo_path(n, oracle_mod):
    """One refinement update is not enough from complex64 (the orthonormality stops near 1e-12),
    so with refine_steps = 1 the pairs go to the FP64 re-solve: the results pass the gates, and
    pairs the re-solve took equal the FP64 solver's bit for bit (same kernels, same inputs)."""
    N = n // 2
    A, B = wl.bogoliubov(N, 16, seed=5, frac=1e-3)
    A, B = A.numpy(), B.numpy()
    s = sbg.Solver(n, precision="mixed", refine_steps=1)
    W, X, info = run(s, A, B)
    Wr, Xr, _ = oracle_mod.hegv(A, B, n, nthreads=8)
    check(A, B, W, X, info, Wr, Xr, n, relative=True)
    W64, X64, _ = run(n, A, B, "fp64")
    same = [(W[p] == W64[p]).all() and (X[p] == X64[p]).all() for p in range(len(W))]
    assert sum(same) >= 1, "no pair went through the FP64 re-solve"
    assert s.refine_redo_pairs() == sum(same)            # the counter names exactly those pairs
    assert s.refine_redo_pairs(reset=True) == sum(same) and s.refine_redo_pairs() == 0
    assert sbg.Solver(n).refine_redo_pairs() == 0        # FP64 form: nothing to count


@pytest.mark.parametrize("N", [48, 96])
def test_mixed_big_near_goldstone(N, oracle_mod):
    """kappa(B) ~ 1e8 at n = 96 and 192 (config 5's sizes): C's norm is ~1e8 against O(1)
    eigenvalues, so complex64 resolves them only coarsely; the refinement against the FP64 C brings
    most pairs to the gates and hands the rest to the FP64 re-solve.  Gates as for the FP64 form:
    eigenvalues against |l_i| kappa_i + ||C||, residual and orthogonality within 4x of LAPACK's."""
    n = 2 * N
    A, B = wl.bogoliubov(N, 6 if N <= 48 else 3, seed=11, frac=1e-3, goldstone=1e-8)
    A, B = A.numpy(), B.numpy()
    Wr, Xr, _ = oracle_mod.hegv(A, B, n, nthreads=8)
    normB = np.linalg.norm(Mx.as_mats(B, n), ord=2, axis=(1, 2))
    cond = normB[:, None] * np.linalg.norm(Mx.as_mats(Xr, n), axis=1) ** 2
    assert cond.max() > 1e7
    scale = np.abs(Wr) * cond + np.abs(Wr).max(axis=1, keepdims=True)
    res_ref = float(Mx.residual(A, B, Xr, Wr, n).max())
    orth_ref = float(Mx.orth(B, Xr, n).max())
    W, X, info = run(n, A, B, "mixed")
    assert (info == 0).all()
    assert (np.abs(W - Wr) / scale).max() < 1e-12
    assert Mx.residual(A, B, X, W, n).max() < max(1e-12, 4 * res_ref)
    assert Mx.orth(B, X, n).max() < max(1e-9, 4 * orth_ref)


def test_mixed_big_failures_and_nan(oracle_mod):
    """The FP64 form's info codes and NaN outputs: B not positive definite (n + i), a NaN in A
    (the eigensolve cannot converge: 1..n, through the re-solve); the other pairs unharmed."""
    n = 96
    H, S = oracle_mod.gen_fixture_pairs(n, 5, 4, "random")
    Sm = Mx.as_mats(S.copy(), n).copy()
    Sm[1] -= 1e4 * np.eye(n)
    Sbad = Mx.from_mats(Sm)
    H = H.copy()
    H[4, 9] = np.nan
    W, X, info = run(n, H, Sbad, "mixed")
    W64, X64, info64 = run(n, H, Sbad, "fp64")
    assert info[1] == n + 1 and info64[1] == n + 1
    assert 1 <= info[4] <= n
    assert np.isnan(W[1]).all() and np.isnan(X[1]).all()
    good = [0, 2, 3]
    Wr, Xr, _ = oracle_mod.hegv(H[good], S[good], n, nthreads=8)
    check(H[good], S[good], W[good], X[good], info[good], Wr, Xr, n)


def test_mixed_big_chunks_and_determinism(oracle_mod):
    """Chunked launches (5-pair workspace) equal one-chunk launches bit for bit, run to run."""
    n = 72
    H, S = oracle_mod.gen_fixture_pairs(n, 13, 21, "nearid")
    a = run(sbg.Solver(n, precision="mixed", workspace_pairs=5), H, S)
    b = run(sbg.Solver(n, precision="mixed"), H, S)
    c = run(sbg.Solver(n, precision="mixed"), H, S)
    for x, y, z in zip(a, b, c):
        assert np.array_equal(x, y, equal_nan=True) and np.array_equal(y, z, equal_nan=True)
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=8)
    check(H, S, a[0], a[1], a[2], Wr, Xr, n)


def _tc_solver(n, **kw):
    s = sbg.Solver(n, precision="mixed", **kw)
    s.schedule = dict(reduce_tc=1)
    assert s.schedule["reduce_tc"] == 1
    return s


@pytest.mark.parametrize("n", [85, 96, 100, 128, 160, 161, 192, 235])
def test_mixed_big_tensor_core_reduction(n, oracle_mod):
    """The blocked Cholesky and reduction on the FP64 tensor cores (schedule reduce_tc = 1): whole
    and partial 32-blocks, one to eight block rows, against zhegv with the parity gates."""
    if n > sbg.max_n("mixed"):
        pytest.skip(f"the mixed form covers n <= {sbg.max_n('mixed')}")
    H, S = oracle_mod.gen_fixture_pairs(n, 6 if n <= 160 else 3, 17, "random")
    W, X, info = run(_tc_solver(n), H, S)
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=8)
    check(H, S, W, X, info, Wr, Xr, n)


@pytest.mark.parametrize("N", [48, 96])
def test_mixed_big_tensor_core_reduction_near_goldstone(N, oracle_mod):
    """kappa(B) ~ 1e8 through the blocked reduction (its diagonal blocks inverted explicitly): the
    same gates as the FP64 form's near-Goldstone tests."""
    n = 2 * N
    A, B = wl.bogoliubov(N, 6 if N <= 48 else 3, seed=23, frac=1e-3, goldstone=1e-8)
    A, B = A.numpy(), B.numpy()
    Wr, Xr, _ = oracle_mod.hegv(A, B, n, nthreads=8)
    normB = np.linalg.norm(Mx.as_mats(B, n), ord=2, axis=(1, 2))
    cond = normB[:, None] * np.linalg.norm(Mx.as_mats(Xr, n), axis=1) ** 2
    scale = np.abs(Wr) * cond + np.abs(Wr).max(axis=1, keepdims=True)
    res_ref = float(Mx.residual(A, B, Xr, Wr, n).max())
    orth_ref = float(Mx.orth(B, Xr, n).max())
    W, X, info = run(_tc_solver(n), A, B)
    assert (info == 0).all()
    assert (np.abs(W - Wr) / scale).max() < 1e-12
    assert Mx.residual(A, B, X, W, n).max() < max(1e-12, 4 * res_ref)
    assert Mx.orth(B, X, n).max() < max(1e-9, 4 * orth_ref)


@pytest.mark.parametrize("n", [96, 192])
def test_mixed_big_tensor_core_reduction_not_positive_definite(n, oracle_mod):
    """zpotrf's info through the blocked Cholesky: n + i for the first leading minor i that is not
    positive definite, in the first block and in a later one; NaN outputs for those pairs only."""
    H, S = oracle_mod.gen_fixture_pairs(n, 3, 4, "random")
    Sm = Mx.as_mats(S.copy(), n).copy()
    Sm[0] -= 1e4 * np.eye(n)                       # the first minor
    Sm[1, 70, 70] = -1.0                           # a minor in the third block
    W, X, info = run(_tc_solver(n), H, Mx.from_mats(Sm))
    W64, X64, info64 = run(n, H, Mx.from_mats(Sm), "fp64")
    assert info[0] == n + 1 and info64[0] == n + 1
    assert info[1] == info64[1] and n + 32 < info[1] <= n + 71
    assert np.isnan(W[:2]).all() and np.isnan(X[:2]).all()
    Wr, Xr, _ = oracle_mod.hegv(H[2:], S[2:], n, nthreads=8)
    check(H[2:], S[2:], W[2:], X[2:], info[2:], Wr, Xr, n)
