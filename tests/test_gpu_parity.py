"""GPU parity of the CUDA path against the LAPACK oracle, through the C ABI.

Gates (tolerances written here, as the reference's tests do):
  * reference gates (tests/test_full_batched_n54.cpp:44-46): eig_rel_ref < 1e-10,
    S-inner-product phase error < 1e-10 on non-degenerate columns (gap >= 1e-6);
  * the B200 build's own gates: eigenvalue error vs zhegv <= 1e-12, residual
    ||AX - BXW||/(||A|| ||X||) <= 1e-12 and max|X^H B X - I| <= 1e-12, with
    clusters compared by subspace angle.  The eigenvalue gate is the pure
    relative error |dl|/|l| for the spin-wave pairs (A = diag(I, -I) keeps every
    |l| >= 1/||B||), and the norm-wise one |dl|/max|l| for the reference's
    random-H pairs, whose eigenvalues can sit arbitrarily close to 0 where no
    two FP64 solvers agree to 1e-12 relative.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import sbg
from sbg import workloads as wl
from oracle import metrics as Mx

pytestmark = pytest.mark.gpu

REF_TOL = 1e-10
TOL = 1e-12


def run(solver_or_n, A, B, precision="fp64"):
    """Solves host pairs on the GPU through the C ABI; returns numpy (W, X, info)."""
    A = torch.as_tensor(np.ascontiguousarray(A)).cuda()
    B = torch.as_tensor(np.ascontiguousarray(B)).cuda()
    s = solver_or_n if isinstance(solver_or_n, sbg.Solver) else sbg.Solver(solver_or_n, precision=precision)
    n = s.n
    W = torch.empty((A.shape[0], n), dtype=torch.float64, device="cuda")
    X = torch.empty_like(A)
    info = torch.full((A.shape[0],), -7, dtype=torch.int32, device="cuda")
    s.launch(A, B, W, X, info)
    torch.cuda.synchronize()
    return W.cpu().numpy(), X.cpu().numpy(), info.cpu().numpy()


def check(A, B, W, X, info, Wr, Xr, n, *, tol=TOL, cluster_gap=1e-6, relative=False):
    A = np.asarray(A); B = np.asarray(B)
    assert (info == 0).all(), f"info {np.unique(info)}"
    s = Mx.summarize(A, B, W, X, Wr, Xr, n, degen_gap=cluster_gap)
    assert s["eig_rel_ref"] < REF_TOL and s["phase_err"] < REF_TOL, s
    assert s["eig_rel" if relative else "eig_rel_norm"] <= tol, s
    assert s["residual"] <= tol, s
    assert s["orth"] <= tol, s
    assert s["cluster_sin"] <= 1e-8, s
    return s


FIXTURE_NS = (16, 32, 48, 54, 64)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n", FIXTURE_NS)
@pytest.mark.parametrize("mode", ["random", "nearid"])
def test_reference_fixtures(n, mode, precision, manifest, golden_W, golden_U0, oracle_mod):
    if n > sbg.max_n(precision):
        pytest.skip(f"the {precision} form covers n <= {sbg.max_n(precision)}")
    name = f"n{n}_b8_s42_{mode}"
    e = manifest[name]
    H, S = oracle_mod.gen_fixture_pairs(n, e["batch"], e["seed"], mode)
    W, X, info = run(n, H, S, precision)
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=4)
    check(H, S, W, X, info, Wr, Xr, n)
    # against the fixture's own zhegvd eigenvalues and pair-0 eigenvectors
    assert Mx.eig_rel_ref(W, golden_W[name]).max() < REF_TOL
    assert Mx.eig_rel_norm(W, golden_W[name]).max() <= TOL
    if name in golden_U0:
        assert Mx.phase_err(S[:1], X[:1], golden_U0[name][None], golden_W[name][:1], n).max() < REF_TOL


def test_fixture_b32_slices_through_fixed_drop_in(manifest, golden_W, oracle_mod):
    """test_full_batched_n54.cpp:355-366: slices B = 1, 8, 32 of n54_b32_s123_random."""
    e = manifest["n54_b32_s123_random"]
    H, S = oracle_mod.gen_fixture_pairs(54, 32, 123, "random")
    Wg = golden_W["n54_b32_s123_random"]
    for b in (1, 8, 32):
        dA = torch.as_tensor(H[:b]).cuda(); dB = torch.as_tensor(S[:b]).cuda()
        W = torch.empty((b, 54), dtype=torch.float64, device="cuda")
        X = torch.empty_like(dA)
        info = torch.full((b,), -7, dtype=torch.int32, device="cuda")
        sbg.geneig_full_n54_batched(dA, dB, W, X, info)
        torch.cuda.synchronize()
        assert (info.cpu().numpy() == 0).all()
        assert Mx.eig_rel_ref(W.cpu().numpy(), Wg[:b]).max() < REF_TOL
        assert Mx.eig_rel_norm(W.cpu().numpy(), Wg[:b]).max() <= TOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_synthetic_1024_batch(precision, oracle_mod):
    """test_full_batched_n54.cpp:222-334: 1024 synthetic random pairs at n = 54."""
    import numpy.random as npr
    rng = npr.default_rng(0xC0FFEE)
    n, b = 54, 1024
    G = rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n))
    Hm = G + np.conj(np.swapaxes(G, 1, 2))
    K = rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n))
    Sm = K @ np.conj(np.swapaxes(K, 1, 2)) + n * np.eye(n)
    H, S = Mx.from_mats(Hm), Mx.from_mats(Sm)
    W, X, info = run(n, H, S, precision)
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=8)
    check(H, S, W, X, info, Wr, Xr, n)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bogoliubov_config(precision, oracle_mod):
    """The n = 54 Bogoliubov workload (lambda_min(B) = 1e-2 ||B||, A = diag(I, -I)), sampled."""
    A, B = wl.bogoliubov(27, 512, seed=0)
    A, B = A.numpy(), B.numpy()
    W, X, info = run(54, A, B, precision)
    Wr, Xr, _ = oracle_mod.hegv(A, B, 54, nthreads=8)
    check(A, B, W, X, info, Wr, Xr, 54, relative=True)
    # eigenvalues come in +-lambda pairs (the Bogoliubov spectrum is symmetric)
    assert np.abs(W + W[:, ::-1]).max() < 1e-10 * np.abs(W).max()


@pytest.mark.parametrize("N", [16, 27])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_qsweep_config(N, precision, oracle_mod):
    """q-sweep pairs (n = 32, 54), lambda_min(B) = 1e-3 ||B||, a strided sample of the 64^3 grid."""
    A, B = wl.qsweep(N, grid=64, start=12345, count=256)
    A, B = A.numpy(), B.numpy()
    n = 2 * N
    W, X, info = run(n, A, B, precision)
    Wr, Xr, _ = oracle_mod.hegv(A, B, n, nthreads=8)
    check(A, B, W, X, info, Wr, Xr, n, relative=True)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 9, 12, 17, 24, 31, 33, 40, 49, 57, 60, 63])
def test_mixed_form_sizes(n, oracle_mod):
    """The mixed form (complex64 Householder, FP64 refinement on the tensor cores) at every tile
    size of its refinement kernel (n padded to 8, 16, ..., 64) and both sides of each."""
    H, S = oracle_mod.gen_fixture_pairs(n, 6, 13, "random")
    W, X, info = run(n, H, S, "mixed")
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=4)
    check(H, S, W, X, info, Wr, Xr, n)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 12, 17, 24, 31, 33, 63, 65, 77, 83])
def test_sizes_and_odd_n(n, oracle_mod):
    H, S = oracle_mod.gen_fixture_pairs(n, 6, 11, "random")
    W, X, info = run(n, H, S)
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=4)
    check(H, S, W, X, info, Wr, Xr, n)


def test_batch_zero_and_chunking(oracle_mod):
    n = 20
    s = sbg.Solver(n, workspace_pairs=7)          # forces 7-pair internal chunks
    H, S = oracle_mod.gen_fixture_pairs(n, 30, 5, "nearid")
    W, X, info = run(s, H, S)
    Wr, Xr, _ = oracle_mod.hegv(H, S, n, nthreads=4)
    check(H, S, W, X, info, Wr, Xr, n)
    e = torch.empty((0, n * n), dtype=torch.complex128, device="cuda")
    s.launch(e, e, torch.empty((0, n), dtype=torch.float64, device="cuda"), e.clone(),
             torch.empty(0, dtype=torch.int32, device="cuda"))


def test_launch_chunked_multistream_matches_single(oracle_mod):
    n = 54
    H, S = oracle_mod.gen_fixture_pairs(n, 40, 9, "random")
    s = sbg.Solver(n)
    W1, X1, _ = run(s, H, S)
    dA = torch.as_tensor(H).cuda(); dB = torch.as_tensor(S).cuda()
    W = torch.empty((40, n), dtype=torch.float64, device="cuda"); X = torch.empty_like(dA)
    info = torch.empty(40, dtype=torch.int32, device="cuda")
    streams = [torch.cuda.Stream() for _ in range(3)]
    torch.cuda.synchronize()
    s.launch_chunked(dA, dB, W, X, info, 7, streams)
    torch.cuda.synchronize()
    assert (info.cpu().numpy() == 0).all()
    assert np.array_equal(W.cpu().numpy(), W1) and np.array_equal(X.cpu().numpy(), X1)


def test_deterministic_bitwise(oracle_mod):
    """Same inputs, same schedule -> bit-identical W and X (test_cache_n54.cpp:308-313)."""
    n = 54
    H, S = oracle_mod.gen_fixture_pairs(n, 16, 2, "random")
    s = sbg.Solver(n)
    a = run(s, H, S)
    b = run(s, H, S)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_not_positive_definite_flags_only_that_pair(oracle_mod):
    n = 32
    H, S = oracle_mod.gen_fixture_pairs(n, 5, 4, "random")
    Sbad = S.copy()
    Sm = Mx.as_mats(Sbad, n).copy()
    Sm[2] -= 1e4 * np.eye(n)                       # pair 2 indefinite: fails at the first minor
    Sm[3, 7, 7] = -1.0                             # pair 3 fails later (leading minor of order > 1)
    Sbad = Mx.from_mats(Sm)
    W, X, info = run(n, H, Sbad)
    assert info[2] == n + 1
    assert info[3] > n + 1 and info[3] <= 2 * n
    assert np.isnan(W[2]).all() and np.isnan(X[2]).all()
    good = [0, 1, 4]
    Wr, Xr, _ = oracle_mod.hegv(H[good], Sbad[good], n, nthreads=4)
    check(H[good], Sbad[good], W[good], X[good], info[good], Wr, Xr, n)


def test_nan_input_terminates_with_info(oracle_mod):
    n = 24
    H, S = oracle_mod.gen_fixture_pairs(n, 3, 8, "random")
    H = H.copy(); S = S.copy()
    H[0, 5] = np.nan                                 # NaN in A: the QL cannot converge
    S[1, 0] = np.nan                                 # NaN on B's diagonal: potrf fails at order 1
    W, X, info = run(n, H, S)
    assert 1 <= info[0] <= n
    assert info[1] == n + 1
    assert info[2] == 0


@pytest.mark.parametrize("N", [12, 16, 27])
def test_ql_log_overflow_falls_back(N, monkeypatch, oracle_mod):
    """A rotation log too small for the QL: every pair takes the in-kernel warp QL (n <= 32:
    the register-row apply kernel's fallback, Z in the X buffer; n = 54: the shared-memory one)."""
    monkeypatch.setenv("SBG_QL_LOG_CAPACITY", "40")
    n = 2 * N
    A, B = wl.bogoliubov(N, 64, seed=3)
    A, B = A.numpy(), B.numpy()
    Wr, Xr, _ = oracle_mod.hegv(A, B, n, nthreads=8)
    for prec in ("fp64", "mixed"):
        W, X, info = run(n, A, B, prec)
        check(A, B, W, X, info, Wr, Xr, n, relative=True)


def test_near_goldstone_both_forms(oracle_mod):
    """kappa(B) ~ 1e8 (a near-zero mode injected into B).  After the Cholesky-based
    reduction C = L^{-1} A L^{-H} has norm ~1e8 / ||B||, so every eigenvalue carries an
    absolute error ~ eps ||C|| in any FP64 method of this kind, LAPACK's included, and the
    near-null mode's own eigenvalue is conditioned at kappa(B) eps.  Agreement with zhegv is
    therefore checked against each eigenvalue's perturbation scale
    |l_i| kappa_i + ||C||, kappa_i = ||B|| ||x_i||^2 (x_i B-normalised), and the backward
    error (residual, B-orthogonality) is held at the FP64 level."""
    A, B = wl.bogoliubov(27, 64, seed=7, frac=1e-3, goldstone=1e-8)
    A, B = A.numpy(), B.numpy()
    Wr, Xr, _ = oracle_mod.hegv(A, B, 54, nthreads=8)
    normB = np.linalg.norm(Mx.as_mats(B, 54), ord=2, axis=(1, 2))
    cond = normB[:, None] * np.linalg.norm(Mx.as_mats(Xr, 54), axis=1) ** 2       # (batch, n)
    assert cond.max() > 1e7                                                         # the mode is there
    scale = np.abs(Wr) * cond + np.abs(Wr).max(axis=1, keepdims=True)
    res_ref = float(Mx.residual(A, B, Xr, Wr, 54).max())
    orth_ref = float(Mx.orth(B, Xr, 54).max())
    for prec in ("fp64", "mixed"):
        W, X, info = run(54, A, B, prec)
        assert (info == 0).all()
        s = Mx.summarize(A, B, W, X, Wr, Xr, 54)
        err = np.abs(W - Wr) / scale
        at = np.unravel_index(int(err.argmax()), err.shape)
        assert err.max() < 1e-12, (prec, float(err.max()), at, float(W[at]), float(Wr[at]), float(cond[at]), s)
        # zhegv's own residual on these pairs is ~1.7e-12 (the 1e-12 gate is out of reach at
        # kappa(B) ~ 1e8 for any FP64 Cholesky-based solver); hold ours to LAPACK's level
        assert s["residual"] < max(1e-12, 4.0 * res_ref), (prec, s, res_ref)
        assert s["orth"] < max(1e-9, 4.0 * orth_ref), (prec, s, orth_ref)       # zhegv: ~4e-9 here


@pytest.mark.parametrize("n", [12, 54, 96])
def test_solve_host_paths_match_device_launch(n):
    """sbg_solver_solve_host from pinned host buffers (B's lower triangle pulled by a kernel) and
    from pageable ones (whole matrices copied) equals the device launch bit for bit, with NaN in
    B's strict upper triangle (never read), and reports the bytes it moved."""
    N = n // 2
    batch = 300
    A, B = wl.bogoliubov(N, batch, seed=11, frac=1e-2)
    Bm = B.reshape(batch, n, n)                   # [b, j, i] = B(i, j)
    upper = torch.triu(torch.ones(n, n, dtype=torch.bool), diagonal=1).T   # i < j, in [j, i] indexing
    Bm[:, upper] = complex("nan+nanj")
    B = Bm.reshape(batch, n * n).contiguous()
    s = sbg.Solver(n)
    dW = torch.empty((batch, n), dtype=torch.float64, device="cuda")
    dX = torch.empty((batch, n * n), dtype=torch.complex128, device="cuda")
    dI = torch.empty(batch, dtype=torch.int32, device="cuda")
    s.launch(A.cuda(), B.cuda(), dW, dX, dI)
    torch.cuda.synchronize()
    assert (dI == 0).all() and torch.isfinite(dW).all()
    nn = n * n
    for pinned in (True, False):
        hA = A.clone().pin_memory() if pinned else A.clone()
        hB = B.clone().pin_memory() if pinned else B.clone()
        hW = torch.empty((batch, n), dtype=torch.float64)
        hX = torch.empty((batch, nn), dtype=torch.complex128)
        hI = torch.empty(batch, dtype=torch.int32)
        if pinned:
            hW, hX, hI = hW.pin_memory(), hX.pin_memory(), hI.pin_memory()
        s.solve_host(hA, hB, hW, hX, hI, chunk_size=64, num_streams=3)
        assert torch.equal(hW, dW.cpu()) and torch.equal(hX, dX.cpu()) and torch.equal(hI, dI.cpu()), pinned
        h2d, d2h = s.host_transfer_bytes()
        b_bytes = 8 * n * (n + 1) if pinned else 16 * nn
        assert h2d == (16 * nn + b_bytes) * batch, (pinned, h2d)
        assert d2h == (16 * nn + 8 * n + 4) * batch
    s.close()
