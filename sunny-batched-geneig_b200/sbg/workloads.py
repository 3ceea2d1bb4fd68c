"""Seeded synthetic workloads with the shapes and spectra of the spin-wave pairs.

There is no public dataset for this path (Sunny.jl's SW08 matrices are not
available), so these generators stand in for it.  All return (A, B) as
(batch, n*n) complex128 tensors, column-major per pair, n = 2N:

* ``bogoliubov``: P Hermitian, Q complex symmetric, entries complex normal with
  E|z|^2 = 1/N; B0 = [[P, Q], [conj(Q), conj(P)]] shifted by s I so that
  lambda_min(B) = frac * ||B||_2; A = diag(I_N, -I_N) (the paraunitary metric).
  ``goldstone`` additionally injects a near-zero mode on a random unit
  v = [u; conj(u)] / ||.||: B <- (I - v v^H) B (I - v v^H) + goldstone ||B||_2 v v^H.
* ``qsweep``: a spin-wave-like cell of N sites with 4 random bonds per site
  (J 3x3 normal, displacement d uniform in [-1, 1]^3); per q = 2 pi k / G on a
  G^3 grid, P(q) and Q(q) are Hermitian / complex-symmetric sums of the bond
  terms u^T J conj(u), u^T J u (u = (1, i, 0)/sqrt 2) times exp(i q.d), with the
  -J_zz/2 on-site terms; B0(q) in the Bogoliubov form, shifted to
  lambda_min = frac * ||B||_2.
* ``spinwave_cell``: the same cell as a bond table for ``sbg.SpinWave`` (sites, coefficients
  (Re a, Im a, Re b, Im b, J_zz), displacements) plus seeded site positions in [0, 1)^3; its
  B(q) = B0(q) + field I, with ``spinwave_field`` choosing the one field of the whole sweep
  that puts min_q lambda_min(B) at frac * max_q ||B||_2.
* ``uneven_sizes``: the n of each pair of the uneven batch (proportions over
  {12, 24, 32, 54, 96, 128}), shuffled with the given seed.
"""
from __future__ import annotations

import math

import numpy as np
import torch


def _cnormal(rng: np.random.Generator, shape, var: float) -> np.ndarray:
    s = math.sqrt(var / 2.0)
    return rng.normal(0.0, s, shape) + 1j * rng.normal(0.0, s, shape)


def metric_A(N: int, batch: int, device="cpu") -> torch.Tensor:
    n = 2 * N
    a = torch.zeros((n, n), dtype=torch.complex128, device=device)
    idx = torch.arange(n, device=device)
    a[idx, idx] = torch.where(idx < N, 1.0, -1.0).to(torch.complex128)
    return a.reshape(1, n * n).expand(batch, n * n).contiguous()


def _shift(B0: torch.Tensor, frac: float, evals: torch.Tensor) -> torch.Tensor:
    """B0 + s I with s chosen so lambda_min(B) = frac * lambda_max(B)."""
    lmin = evals[:, 0]
    lmax = evals[:, -1]
    s = (frac * lmax - lmin) / (1.0 - frac)
    n = B0.shape[-1]
    idx = torch.arange(n, device=B0.device)
    B = B0.clone()
    B[:, idx, idx] += s[:, None].to(B.dtype)
    return B


def _eigvalsh(M: torch.Tensor, eigvalsh=None) -> torch.Tensor:
    if eigvalsh is not None:
        return eigvalsh(M)
    if M.is_cuda:
        return torch.linalg.eigvalsh(M)
    return torch.from_numpy(np.linalg.eigvalsh(M.numpy()))


def _colmajor(M: torch.Tensor) -> torch.Tensor:
    b, n, _ = M.shape
    return M.transpose(-1, -2).contiguous().reshape(b, n * n)


def bogoliubov(N: int, batch: int, seed: int = 0, frac: float = 1e-2, goldstone: float | None = None,
               device="cpu", eigvalsh=None):
    rng = np.random.default_rng(seed)
    G = _cnormal(rng, (batch, N, N), 1.0 / N)
    H = _cnormal(rng, (batch, N, N), 1.0 / N)
    P = (G + np.conj(np.swapaxes(G, -1, -2))) / math.sqrt(2.0)
    Q = (H + np.swapaxes(H, -1, -2)) / math.sqrt(2.0)
    B0 = np.block([[P, Q], [np.conj(Q), np.conj(P)]])
    B0 = torch.from_numpy(B0).to(device)
    B = _shift(B0, frac, _eigvalsh(B0, eigvalsh))
    if goldstone is not None:
        B = _inject_goldstone(B, N, goldstone, rng, eigvalsh)
    return metric_A(N, batch, device), _colmajor(B)


def _inject_goldstone(B: torch.Tensor, N: int, level: float, rng: np.random.Generator, eigvalsh=None):
    batch = B.shape[0]
    u = _cnormal(rng, (batch, N), 1.0)
    v = np.concatenate([u, np.conj(u)], axis=1)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    v = torch.from_numpy(v).to(B.device)
    norm = _eigvalsh(B, eigvalsh)[:, -1]
    n = B.shape[-1]
    Pm = torch.eye(n, dtype=B.dtype, device=B.device)[None] - v[:, :, None] * v.conj()[:, None, :]
    Bp = Pm @ B @ Pm
    Bp = Bp + (level * norm)[:, None, None].to(B.dtype) * (v[:, :, None] * v.conj()[:, None, :])
    return 0.5 * (Bp + Bp.conj().transpose(-1, -2))


def qsweep_cell(N: int, seed: int):
    """Bond table of the synthetic cell: (i, j, a, b, c, d) per bond."""
    rng = np.random.default_rng(seed)
    u = np.array([1.0, 1.0j, 0.0]) / math.sqrt(2.0)
    bonds = []
    for i in range(N):
        for _ in range(4):
            j = int(rng.integers(N))
            J = rng.normal(0.0, 1.0, (3, 3))
            d = rng.uniform(-1.0, 1.0, 3)
            a = complex(u @ J @ np.conj(u))
            b = complex(u @ J @ u)
            c = float(J[2, 2])
            bonds.append((i, j, a, b, c, d))
    return bonds


def qsweep_points(grid: int, start: int = 0, count: int | None = None, device="cpu") -> torch.Tensor:
    total = grid ** 3
    count = total - start if count is None else count
    k = torch.arange(start, start + count, device=device, dtype=torch.int64)
    k1, k2, k3 = k // (grid * grid), (k // grid) % grid, k % grid
    return (2.0 * math.pi / grid) * torch.stack([k1, k2, k3], dim=1).to(torch.float64)


def qsweep_B0(N: int, q: torch.Tensor, seed: int = 0) -> torch.Tensor:
    """Unshifted Bogoliubov blocks B0(q), shape (len(q), 2N, 2N)."""
    dev = q.device
    nq = q.shape[0]
    P = torch.zeros((nq, N, N), dtype=torch.complex128, device=dev)
    Q = torch.zeros((nq, N, N), dtype=torch.complex128, device=dev)
    onsite = torch.zeros(N, dtype=torch.float64)
    for (i, j, a, b, c, d) in qsweep_cell(N, seed):
        ph = torch.exp(1j * (q @ torch.tensor(d, dtype=torch.float64, device=dev)))
        P[:, i, j] += 0.5 * a * ph
        P[:, j, i] += 0.5 * np.conj(a) * ph.conj()
        Q[:, i, j] += 0.5 * b * ph
        Q[:, j, i] += 0.5 * b * ph
        onsite[i] -= 0.5 * c
        onsite[j] -= 0.5 * c
    idx = torch.arange(N, device=dev)
    P[:, idx, idx] += onsite.to(dev).to(torch.complex128)
    P = 0.5 * (P + P.conj().transpose(-1, -2))
    Q = 0.5 * (Q + Q.transpose(-1, -2))
    top = torch.cat([P, Q], dim=2)
    bot = torch.cat([Q.conj(), P.conj()], dim=2)
    return torch.cat([top, bot], dim=1)


def qsweep(N: int, grid: int = 64, seed: int = 0, frac: float = 1e-3, start: int = 0, count: int | None = None,
           device="cpu", eigvalsh=None):
    q = qsweep_points(grid, start, count, device)
    B0 = qsweep_B0(N, q, seed)
    B = _shift(B0, frac, _eigvalsh(B0, eigvalsh))
    return metric_A(N, q.shape[0], device), _colmajor(B)


def spinwave_cell(N: int, seed: int = 0) -> dict:
    """The q-sweep cell of ``qsweep_cell`` as arrays for ``sbg.SpinWave``."""
    bonds = qsweep_cell(N, seed)
    sites = np.array([[i, j] for (i, j, a, b, c, d) in bonds], dtype=np.int32).reshape(-1, 2)
    coef = np.array([[a.real, a.imag, b.real, b.imag, c] for (i, j, a, b, c, d) in bonds],
                    dtype=np.float64).reshape(-1, 5)
    disp = np.array([d for (i, j, a, b, c, d) in bonds], dtype=np.float64).reshape(-1, 3)
    pos = np.random.default_rng(seed + 7919).uniform(0.0, 1.0, (N, 3))
    return dict(n_sites=N, sites=sites, coef=coef, disp=disp, pos=pos)


def spinwave_field(lmin: float, lmax: float, frac: float) -> float:
    """Field h with min_q lambda_min(B0 + h I) = frac * max_q lambda_max(B0 + h I), from the sweep's
    extreme eigenvalues of B0 (h = (frac lmax - lmin) / (1 - frac), as ``_shift`` per pair)."""
    return (frac * lmax - lmin) / (1.0 - frac)


UNEVEN_SIZES = (12, 24, 32, 54, 96, 128)
UNEVEN_WEIGHTS = (0.10, 0.20, 0.20, 0.30, 0.15, 0.05)


def uneven_sizes(total: int, seed: int = 3, sizes=UNEVEN_SIZES, weights=UNEVEN_WEIGHTS) -> np.ndarray:
    counts = [int(round(w * total)) for w in weights]
    counts[-1] = total - sum(counts[:-1])
    ns = np.concatenate([np.full(c, s, dtype=np.int32) for s, c in zip(sizes, counts)])
    rng = np.random.default_rng(seed)
    rng.shuffle(ns)
    return ns


def uneven(total: int, seed: int = 3, frac: float = 1e-3, sizes=UNEVEN_SIZES, weights=UNEVEN_WEIGHTS,
           device="cpu", eigvalsh=None):
    """The uneven batch: `total` Bogoliubov pairs (A = diag(I, -I), B shifted to
    lambda_min = frac ||B||) with n drawn from `sizes` in proportions `weights`, shuffled
    with `seed`.  Returns (ns, A_packed, B_packed) in the queue's packed layout: the pairs
    of each n are generated together (seed + n) and scattered to their batch positions."""
    ns = uneven_sizes(total, seed, sizes, weights)
    mo = np.concatenate([[0], np.cumsum(ns.astype(np.int64) ** 2)])
    A = torch.empty(int(mo[-1]), dtype=torch.complex128, device=device)
    B = torch.empty_like(A)
    for n in sorted(set(int(v) for v in ns)):
        pos = np.nonzero(ns == n)[0]
        An, Bn = bogoliubov(n // 2, len(pos), seed=seed + n, frac=frac, device=device, eigvalsh=eigvalsh)
        idx = torch.as_tensor((mo[pos][:, None] + np.arange(n * n)[None, :]).reshape(-1), device=device)
        A[idx] = An.reshape(-1).to(device)
        B[idx] = Bn.reshape(-1).to(device)
    return ns, A, B
