"""Spectra that stress the inverse-iteration eigenvectors (FP64, n <= 63), checked against zhegv
with the gates of test_gpu_parity.check (eigenvalues norm-wise to 1e-12, residual and
B-orthogonality to 1e-12, clusters of eigenvalues closer than 1e-6 compared by subspace angle):

* exact multiplicities larger than the kernel's cluster limit (A = diag(+-1), B = I: two
  eigenvalues of multiplicity n/2), which the kernel hands to its warp-QL fallback;
* exact multiplicity 3 (B diagonal, A diagonal with every value three times), which it
  orthogonalises within the cluster;
* T with exact zeros off the diagonal (block-diagonal C with identical blocks: equal eigenvalues
  whose vectors live in different blocks);
* pairs of eigenvalues 1e-12, 1e-9, 1e-7, 1e-4 and 1e-3 apart (relative to ||C||), on both
  sides of the kernel's cluster threshold (3e-4 ||T||).
Every other gap is kept >= 1e-2 so that no accidental near-degeneracy sits at the checker's own
1e-6 cluster threshold, where single eigenvectors are too ill-conditioned to compare.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import metrics as Mx
from test_gpu_parity import check, run

pytestmark = pytest.mark.gpu


def colmajor(M):
    return Mx.from_mats(np.asarray(M, np.complex128))


def random_unitary(rng, n):
    Z = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    Q, R = np.linalg.qr(Z)
    return Q * (np.diag(R) / np.abs(np.diag(R)))


def solve_and_check(oracle_mod, n, A, B):
    W, X, info = run(n, A, B)
    Wr, Xr, ir = oracle_mod.hegv(A, B, n, nthreads=8)
    assert (ir == 0).all()
    return check(A, B, W, X, info, Wr, Xr, n)


@pytest.mark.parametrize("n", [12, 32, 54, 63])
def test_large_exact_multiplicity(oracle_mod, n):
    batch = 8
    a = np.where(np.arange(n) < n // 2, 1.0, -1.0)
    A = colmajor(np.broadcast_to(np.diag(a), (batch, n, n)))
    B = colmajor(np.broadcast_to(np.eye(n), (batch, n, n)))
    solve_and_check(oracle_mod, n, A, B)


@pytest.mark.parametrize("n", [12, 33, 54, 63])
def test_exact_triples(oracle_mod, n):
    rng = np.random.default_rng(n)
    batch = 8
    m = (n + 2) // 3
    vals = np.repeat(np.cumsum(rng.uniform(0.05, 0.5, m)) - 2.0, 3)[:n]
    d = rng.uniform(0.5, 2.0, n)
    A = colmajor(np.broadcast_to(np.diag(vals * d), (batch, n, n)))        # A x = l B x: l = vals
    B = colmajor(np.broadcast_to(np.diag(d), (batch, n, n)))
    solve_and_check(oracle_mod, n, A, B)


@pytest.mark.parametrize("n", [16, 54, 62])
def test_identical_blocks(oracle_mod, n):
    rng = np.random.default_rng(100 + n)
    batch = 6
    h = n // 2
    Cs = []
    for _ in range(batch):
        G = rng.normal(size=(h, h)) + 1j * rng.normal(size=(h, h))
        C1 = G + G.conj().T
        C = np.zeros((n, n), np.complex128)
        C[:h, :h] = C1
        C[h:, h:] = C1
        Cs.append(C)
    A = colmajor(np.array(Cs))
    B = colmajor(np.broadcast_to(np.eye(n), (batch, n, n)))
    solve_and_check(oracle_mod, n, A, B)


@pytest.mark.parametrize("gap", [1e-12, 1e-9, 1e-7, 1e-4, 1e-3])
def test_close_pairs(oracle_mod, gap):
    rng = np.random.default_rng(int(-np.log10(gap)))
    n, batch = 54, 12
    Cs = []
    for _ in range(batch):
        lam = np.cumsum(rng.uniform(0.01, 0.05, n)) - 0.8
        for k in range(0, n - 1, 9):                  # several pairs at the given distance
            lam[k + 1] = lam[k] + gap
        Q = random_unitary(rng, n)
        C = (Q * lam) @ Q.conj().T
        Cs.append(0.5 * (C + C.conj().T))
    A = colmajor(np.array(Cs))
    B = colmajor(np.broadcast_to(np.eye(n), (batch, n, n)))
    solve_and_check(oracle_mod, n, A, B)
