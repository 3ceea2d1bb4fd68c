"""CPU model of the step order of the one-pass FP64 Householder kernel (k_hetrd_l2 in
sunny-batched-geneig_b200/csrc/bigsolve.cu), restated in numpy.

The kernel applies step k-1's rank-2 update lazily. Warp 0 applies it to column k just before it
forms reflector k from that column. All warps apply it to columns k+1.. in the same pass that forms
the Hermitian matvec with reflector k. A step whose reflector is the identity (tau = 0) leaves
nothing pending. This model runs the same sequence, including the (pending update, matvec) flag
logic. On random and structured Hermitian matrices it checks:

* the tridiagonal T and the stored reflectors reproduce C (Q^H C Q = T);
* T's eigenvalues are C's.

The reflector itself follows LAPACK zlarfg as used by zhetd2 (lower), the same steps as the kernel.
"""
import numpy as np
import pytest


def onepass_hetrd(C):
    """(d, e, tau, V): T = tridiag(e, d, e), reflector k = V[k+1:, k] with V[k+1, k] = 1."""
    n = C.shape[0]
    A = np.tril(C).astype(complex)                    # only the lower triangle is stored
    d = np.zeros(n)
    e = np.zeros(n)
    tau = np.zeros(n, complex)
    vbuf = np.zeros((2, n), complex)                  # reflectors k and k-1, by absolute row
    wb = np.zeros(n, complex)
    upd = False                                       # step k-1's update is pending
    for k in range(n - 1):
        vb, vp = vbuf[k & 1], vbuf[(k + 1) & 1]
        if upd:                                       # warp 0: step k-1's update on column k
            for i in range(k, n):
                a = A[i, k] - vp[i] * np.conj(wb[k]) - wb[i] * np.conj(vp[k])
                A[i, k] = a.real if i == k else a
        x = A[k + 1:, k]
        s2 = float(np.sum(np.abs(x[1:]) ** 2))
        alpha = x[0]
        if s2 == 0.0 and alpha.imag == 0.0:
            tk, beta = 0.0, alpha.real
        else:
            nrm = np.sqrt(abs(alpha) ** 2 + s2)
            beta = -nrm if alpha.real >= 0 else nrm
            tk = complex((beta - alpha.real) / beta, -alpha.imag / beta)
            v = x / (alpha - beta)
            v[0] = 1.0
            vb[k + 1:] = v
            A[k + 1:, k] = v
        d[k], e[k], tau[k] = A[k, k].real, beta, tk
        mv = tk != 0
        if not upd and not mv:
            continue
        # all warps: one pass over columns k+1.. (pending update, then the matvec with v_k)
        rows = np.zeros(n, complex)
        cols = np.zeros(n, complex)
        for j in range(k + 1, n):
            for i in range(j, n):
                a = A[i, j]
                if upd:
                    a = a - vp[i] * np.conj(wb[j]) - wb[i] * np.conj(vp[j])
                    if i == j:
                        a = a.real
                    A[i, j] = a
                if mv:
                    if i == j:
                        rows[i] += a.real * vb[j]
                    else:
                        rows[i] += a * vb[j]
                        cols[j] += np.conj(a) * vb[i]
        if not mv:
            upd = False
            continue
        p = tk * (rows[k + 1:] + cols[k + 1:])
        dot = np.sum(np.conj(p) * vb[k + 1:])
        wb[k + 1:] = p - 0.5 * tk * dot * vb[k + 1:]
        upd = True
    a = A[n - 1, n - 1]
    if upd:                                           # step n-2's update of A(n-1, n-1)
        vl = vbuf[(n - 2) & 1]
        a = a - vl[n - 1] * np.conj(wb[n - 1]) - wb[n - 1] * np.conj(vl[n - 1])
    d[n - 1] = a.real
    return d, e, tau, A


def check(C, tol=1e-12):
    n = C.shape[0]
    d, e, tau, V = onepass_hetrd(C)
    T = np.diag(d) + np.diag(e[:-1], 1) + np.diag(e[:-1], -1)
    Q = np.eye(n, dtype=complex)
    for k in range(n - 1):
        if tau[k] != 0:
            v = np.zeros(n, complex)
            v[k + 1:] = V[k + 1:, k]
            Q = Q @ (np.eye(n) - tau[k] * np.outer(v, v.conj()))
    scale = max(np.abs(C).max(), 1.0)
    assert np.abs(Q.conj().T @ C @ Q - T).max() <= tol * n * scale
    ev = np.linalg.eigvalsh(C)
    assert np.abs(np.linalg.eigvalsh(T) - ev).max() <= tol * n * max(np.abs(ev).max(), 1.0)


@pytest.mark.parametrize("n", [2, 3, 8, 33, 70])
def test_random_hermitian(n):
    rng = np.random.default_rng(n)
    G = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    check(G + G.conj().T)


def test_identity_steps_with_and_without_a_pending_update():
    # block diagonal: the reflector of the last column of each block is the identity (tau = 0), once
    # right after a real update and once after another identity step
    rng = np.random.default_rng(7)
    blocks = []
    for m in (5, 1, 1, 6, 4):
        G = rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))
        blocks.append(G + G.conj().T)
    n = sum(b.shape[0] for b in blocks)
    C = np.zeros((n, n), complex)
    o = 0
    for b in blocks:
        m = b.shape[0]
        C[o:o + m, o:o + m] = b
        o += m
    d, e, tau, _ = onepass_hetrd(C)
    assert np.count_nonzero(tau[:-1] == 0) >= 4
    check(C)


def test_already_tridiagonal_with_complex_subdiagonal():
    # every x has one entry: tau != 0 only where that entry is complex (zlarfg makes beta real)
    n = 9
    rng = np.random.default_rng(3)
    sub = rng.standard_normal(n - 1) + 1j * rng.standard_normal(n - 1)
    sub[::3] = sub[::3].real
    C = np.diag(rng.standard_normal(n)).astype(complex) + np.diag(sub, -1) + np.diag(sub.conj(), 1)
    check(C)
