"""CPU checker for the spin-wave q-sweep steps either side of the solve.

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and the bench's
accuracy / cpu_baseline legs may use this module; the product path never does.

Restates, in numpy, the two steps ``sbg_spinwave_*`` runs on the GPU:

* ``assemble``: A(q) = diag(I_N, -I_N) and B(q) = [[P, Q], [conj Q, conj P]] + field I,
  where per bond k = (i, j, a, b, c, d), in bond order,
  P_ij += a/2 e^{iq.d}, P_ji += conj(a/2 e^{iq.d}), Q_ij += b/2 e^{iq.d},
  Q_ji += b/2 e^{iq.d}, and then P_ii, P_jj -= c/2 (the on-site sums added after the
  bond terms, the field last).
* ``intensities``: I_m(q) = |sum_{i<N} e^{-iq.r_i} (x_m[i] + x_m[N+i])|^2 / (N |lambda_m|),
  NaN for a pair whose info != 0.

The reference has no implementation of either step (its intended caller assembles the
pairs itself, and that caller is not part of the reference tree), so this restates the
definition above rather than reference code; the N = 1 closed form
omega(q) = sqrt((Re(a e^{iq.d}) - c + field)^2 - |b|^2) pins the assembly's meaning
(tests/test_spinwave_oracle.py), and the solve between the two steps stays pinned
through LAPACK zhegv (oracle.hegv).  Arrays are column-major per pair, flat (nq, n*n).
"""
from __future__ import annotations

import numpy as np


def _phase(q: np.ndarray, d: np.ndarray) -> np.ndarray:
    th = q @ np.asarray(d, dtype=np.float64)
    return np.cos(th) + 1j * np.sin(th)


def assemble(n_sites: int, sites, coef, disp, q, field: float = 0.0):
    """(A, B), each (nq, n*n) complex128 column-major, n = 2 n_sites."""
    N = n_sites
    q = np.asarray(q, dtype=np.float64).reshape(-1, 3)
    sites = np.asarray(sites, dtype=np.int64).reshape(-1, 2)
    coef = np.asarray(coef, dtype=np.float64).reshape(-1, 5)
    disp = np.asarray(disp, dtype=np.float64).reshape(-1, 3)
    nq = q.shape[0]
    P = np.zeros((nq, N, N), np.complex128)
    Q = np.zeros((nq, N, N), np.complex128)
    onsite = np.zeros(N)
    for k in range(sites.shape[0]):
        i, j = int(sites[k, 0]), int(sites[k, 1])
        ph = _phase(q, disp[k])
        ta = complex(0.5 * coef[k, 0], 0.5 * coef[k, 1]) * ph
        tb = complex(0.5 * coef[k, 2], 0.5 * coef[k, 3]) * ph
        P[:, i, j] += ta
        P[:, j, i] += np.conj(ta)
        Q[:, i, j] += tb
        Q[:, j, i] += tb
    for k in range(sites.shape[0]):
        onsite[sites[k, 0]] -= 0.5 * coef[k, 4]
        onsite[sites[k, 1]] -= 0.5 * coef[k, 4]
    idx = np.arange(N)
    P[:, idx, idx] += onsite
    n = 2 * N
    B = np.empty((nq, n, n), np.complex128)
    B[:, :N, :N] = P
    B[:, :N, N:] = Q
    B[:, N:, :N] = np.conj(Q)
    B[:, N:, N:] = np.conj(P)
    di = np.arange(n)
    B[:, di, di] += field
    A = np.zeros((nq, n, n), np.complex128)
    A[:, di, di] = np.where(di < N, 1.0, -1.0)
    colmajor = lambda M: np.ascontiguousarray(np.swapaxes(M, 1, 2)).reshape(nq, n * n)
    return colmajor(A), colmajor(B)


def intensities(n_sites: int, pos, q, W, X, info=None):
    """(nq, n) intensities of the eigenpairs (W (nq, n), X (nq, n*n) column-major)."""
    N = n_sites
    n = 2 * N
    q = np.asarray(q, dtype=np.float64).reshape(-1, 3)
    nq = q.shape[0]
    r = np.zeros((N, 3)) if pos is None else np.asarray(pos, dtype=np.float64).reshape(N, 3)
    th = q @ r.T                                            # (nq, N)
    ph = np.cos(th) - 1j * np.sin(th)                       # e^{-iq.r}
    Xm = np.asarray(X).reshape(nq, n, n)                    # [p, m, i] = x_m[i] (column-major pairs)
    s = np.einsum("pi,pmi->pm", ph, Xm[:, :, :N] + Xm[:, :, N:])
    out = np.abs(s) ** 2 / (N * np.abs(np.asarray(W).reshape(nq, n)))
    if info is not None:
        out[np.asarray(info).reshape(nq) != 0] = np.nan
    return out


def single_site_omega(a: complex, b: complex, c: float, d, field: float, q) -> np.ndarray:
    """Closed-form |1/lambda| of the one-site cell with one bond (0, 0, a, b, c, d): the pair is
    A = diag(1, -1), B = [[p, t], [conj t, p]] with p = Re(a e^{iq.d}) - c + field and
    t = b e^{iq.d}, whose two eigenvalues are +-1/sqrt(p^2 - |t|^2)."""
    q = np.asarray(q, dtype=np.float64).reshape(-1, 3)
    ph = _phase(q, d)
    p = (a * ph).real - c + field
    return np.sqrt(p ** 2 - abs(b) ** 2)
