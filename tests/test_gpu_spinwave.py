"""GPU parity of the spin-wave q-sweep path (sbg_spinwave_*) against the CPU checker.

* assembly: B(q) from the bond table equals oracle/spinwave.assemble to rounding
  (|dB| <= 1e-14 max|B|; the two differ only in sincos and the order of the three products
  in q.d), A exactly, and B is exactly Hermitian with the Bogoliubov block structure;
* solve: sbg_spinwave_solve equals, bit for bit, sbg_solver_launch on the assembled pairs,
  and matches LAPACK zhegv on the checker's pairs under the gates of test_gpu_parity.py;
* intensities: the GPU contraction of given (W, X) equals the checker's to 1e-13 relative,
  and the end-to-end intensities match those of zhegv's eigenvectors (summed over clusters
  of eigenvalues closer than 1e-6, where single modes are not unique) to 1e-10 of the
  pair's largest intensity;
* the host-buffer path equals the device path bit for bit; chunking does not change results;
  failed pairs give NaN intensities; bad arguments give status codes.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import sbg
from sbg import workloads as wl
from oracle import metrics as Mx
from oracle import spinwave as SW

pytestmark = pytest.mark.gpu

TOL = 1e-12


def model(N, seed=0, field=None, frac=1e-3, q=None):
    cell = wl.spinwave_cell(N, seed)
    if field is None:
        _, B0 = SW.assemble(N, cell["sites"], cell["coef"], cell["disp"], q, field=0.0)
        ev = np.linalg.eigvalsh(Mx.as_mats(B0, 2 * N))
        field = wl.spinwave_field(ev[:, 0].min(), ev[:, -1].max(), frac)
    m = sbg.SpinWave(N, cell["sites"], cell["coef"], cell["disp"], cell["pos"], field=field)
    return m, cell, field


def qpoints(count, seed=0):
    q = np.random.default_rng(seed).uniform(-np.pi, np.pi, (count, 3))
    q[0] = 0.0
    return q


def cluster_sums(I, W, gap=1e-6):
    """Per pair, I_m |lambda_m| summed over each cluster of eigenvalues (singletons included)."""
    out = []
    for b in range(W.shape[0]):
        w = W[b]
        v = I[b] * np.abs(w)
        groups, lo = [], 0
        for i in range(1, len(w) + 1):
            if i == len(w) or abs(w[i] - w[i - 1]) >= gap * max(abs(w[i]), abs(w[i - 1]), 1.0):
                groups.append(v[lo:i].sum())
                lo = i
        out.append(groups)
    return out


@pytest.mark.parametrize("N", [1, 6, 27, 48])
def test_assembly_matches_checker(N):
    q = qpoints(40, N)
    m, cell, field = model(N, q=q)
    A, B = m.assemble(torch.as_tensor(q).cuda())
    torch.cuda.synchronize()
    Ar, Br = SW.assemble(N, cell["sites"], cell["coef"], cell["disp"], q, field=field)
    Ag, Bg = A.cpu().numpy(), B.cpu().numpy()
    assert np.array_equal(Ag, Ar)
    assert np.abs(Bg - Br).max() <= 1e-14 * np.abs(Br).max()
    n = 2 * N
    M = Mx.as_mats(Bg, n)
    assert np.array_equal(M, np.conj(np.swapaxes(M, 1, 2)))
    assert np.array_equal(M[:, N:, N:], np.conj(M[:, :N, :N]))
    assert np.array_equal(M[:, N:, :N], np.conj(M[:, :N, N:]))
    # B only (A skipped) gives the same B
    _, B2 = m.assemble(torch.as_tensor(q).cuda(), A=False)
    torch.cuda.synchronize()
    assert torch.equal(B2, B)
    m.close()


def test_single_site_closed_form():
    a, b, c, d, h = 0.3 + 0.4j, 0.2 - 0.1j, -1.5, [0.3, -0.2, 0.7], 0.5
    q = qpoints(256, 9)
    m = sbg.SpinWave(1, [[0, 0]], [[a.real, a.imag, b.real, b.imag, c]], [d], None, field=h)
    s = sbg.Solver(2)
    dq = torch.as_tensor(q).cuda()
    W = torch.empty((256, 2), dtype=torch.float64, device="cuda")
    info = torch.empty(256, dtype=torch.int32, device="cuda")
    m.solve(s, dq, W, info)
    torch.cuda.synchronize()
    om = SW.single_site_omega(a, b, c, d, h, q)
    assert (info.cpu().numpy() == 0).all()
    assert np.abs(np.abs(1.0 / W.cpu().numpy()) - om[:, None]).max() <= 1e-13 * om.max()


@pytest.mark.parametrize("N", [6, 27, 48])
def test_solve_matches_solver_and_lapack(oracle_mod, N):
    n = 2 * N
    q = qpoints(48, 100 + N)
    m, cell, field = model(N, q=q)
    s = sbg.Solver(n)
    dq = torch.as_tensor(q).cuda()
    W = torch.empty((48, n), dtype=torch.float64, device="cuda")
    X = torch.empty((48, n * n), dtype=torch.complex128, device="cuda")
    I = torch.empty((48, n), dtype=torch.float64, device="cuda")
    info = torch.full((48,), -3, dtype=torch.int32, device="cuda")
    m.solve(s, dq, W, info, X=X, I=I)
    A, B = m.assemble(dq)
    W2 = torch.empty_like(W); X2 = torch.empty_like(X); info2 = torch.empty_like(info)
    s.launch(A, B, W2, X2, info2)
    torch.cuda.synchronize()
    assert torch.equal(W, W2) and torch.equal(X, X2) and torch.equal(info, info2)
    Ar, Br = SW.assemble(N, cell["sites"], cell["coef"], cell["disp"], q, field=field)
    Wr, Xr, ir = oracle_mod.hegv(Ar, Br, n)
    assert (ir == 0).all()
    Wg, Xg, ig = W.cpu().numpy(), X.cpu().numpy(), info.cpu().numpy()
    assert (ig == 0).all()
    sm = Mx.summarize(Ar, Br, Wg, Xg, Wr, Xr, n)
    assert sm["eig_rel"] <= TOL and sm["residual"] <= TOL and sm["orth"] <= TOL, sm
    assert sm["cluster_sin"] <= 1e-8, sm
    # intensities: the GPU contraction of (W, X) vs the checker's on the same (W, X)
    Ig = I.cpu().numpy()
    Ic = SW.intensities(N, cell["pos"], q, Wg, Xg)
    assert np.abs(Ig - Ic).max() <= 1e-13 * np.abs(Ic).max()
    # the standalone contraction gives the same
    I3 = m.intensities(dq, W, X, info)
    torch.cuda.synchronize()
    assert torch.equal(I3, I)
    # end to end vs zhegv's eigenvectors, cluster sums
    Ir = SW.intensities(N, cell["pos"], q, Wr, Xr)
    for b, (g, r) in enumerate(zip(cluster_sums(Ig, Wg), cluster_sums(Ir, Wr))):
        g, r = np.array(g), np.array(r)
        assert g.shape == r.shape
        assert np.abs(g - r).max() <= 1e-10 * np.abs(r).max(), b
    m.close(); s.close()


def test_host_path_and_chunking_bitwise():
    N, n, nq = 27, 54, 333
    q = qpoints(nq, 7)
    m, cell, field = model(N, q=q)
    s_big = sbg.Solver(n)
    s_small = sbg.Solver(n, workspace_pairs=100)          # 4 chunks of at most 100 pairs
    dq = torch.as_tensor(q).cuda()
    outs = []
    for s in (s_big, s_small):
        W = torch.empty((nq, n), dtype=torch.float64, device="cuda")
        I = torch.empty((nq, n), dtype=torch.float64, device="cuda")
        info = torch.empty(nq, dtype=torch.int32, device="cuda")
        m.solve(s, dq, W, info, I=I)
        torch.cuda.synchronize()
        outs.append((W.cpu(), I.cpu(), info.cpu()))
    assert all(torch.equal(a, b) for a, b in zip(*outs))
    hq = torch.as_tensor(q).pin_memory()
    hW = torch.empty((nq, n), dtype=torch.float64).pin_memory()
    hI = torch.empty((nq, n), dtype=torch.float64).pin_memory()
    hX = torch.empty((nq, n * n), dtype=torch.complex128).pin_memory()
    hinfo = torch.empty(nq, dtype=torch.int32).pin_memory()
    m.solve_host(s_small, hq, hW, hinfo, X=hX, I=hI, chunk_size=64, num_streams=3)
    assert torch.equal(hW, outs[0][0]) and torch.equal(hI, outs[0][1]) and torch.equal(hinfo, outs[0][2])
    dX = torch.empty((nq, n * n), dtype=torch.complex128, device="cuda")
    dW = torch.empty((nq, n), dtype=torch.float64, device="cuda")
    dinfo = torch.empty(nq, dtype=torch.int32, device="cuda")
    m.solve(s_big, dq, dW, dinfo, X=dX)
    torch.cuda.synchronize()
    assert torch.equal(hX, dX.cpu())
    m.close(); s_big.close(); s_small.close()


def test_failed_pairs_give_nan_intensities():
    N, n = 6, 12
    q = qpoints(16, 3)
    m, cell, _ = model(N, field=-50.0)                    # B indefinite at every q: Cholesky fails
    s = sbg.Solver(n)
    dq = torch.as_tensor(q).cuda()
    W = torch.empty((16, n), dtype=torch.float64, device="cuda")
    I = torch.empty((16, n), dtype=torch.float64, device="cuda")
    info = torch.zeros(16, dtype=torch.int32, device="cuda")
    m.solve(s, dq, W, info, I=I)
    torch.cuda.synchronize()
    assert (info.cpu().numpy() > 0).all()
    assert torch.isnan(I).all() and torch.isnan(W).all()
    m.close(); s.close()


def test_argument_errors():
    cell = wl.spinwave_cell(4, 0)
    with pytest.raises(sbg.SolverError):
        sbg.SpinWave(4, np.array([[0, 9]]), cell["coef"][:1], cell["disp"][:1])      # site out of range
    with pytest.raises(sbg.SolverError):
        sbg.SpinWave(0, cell["sites"], cell["coef"], cell["disp"])
    m = sbg.SpinWave(4, cell["sites"], cell["coef"], cell["disp"], field=10.0)
    s = sbg.Solver(10)                                    # order 10 != 2 x 4
    dq = torch.zeros((2, 3), dtype=torch.float64, device="cuda")
    W = torch.empty((2, 8), dtype=torch.float64, device="cuda")
    info = torch.empty(2, dtype=torch.int32, device="cuda")
    with pytest.raises(sbg.SolverError):
        m.solve(s, dq, W, info)
    # zero q-points is a no-op
    m.solve(sbg.Solver(8), dq[:0], W[:0], info[:0])
    m.close(); s.close()
