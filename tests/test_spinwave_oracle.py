"""The spin-wave checker (oracle/spinwave.py) on the CPU: its assembly against the closed form
of a one-site cell and against the torch q-sweep generator, and properties of its intensity
contraction.  No GPU."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import spinwave as SW
from sbg import workloads as wl


@pytest.fixture(scope="module")
def oracle_lib(oracle_mod):
    return oracle_mod


def test_single_site_closed_form(oracle_lib):
    """One site, one bond onto itself: |1/lambda| = sqrt((Re(a e^{iqd}) - c + h)^2 - |b|^2)."""
    rng = np.random.default_rng(5)
    a, b, c, d, h = 0.3 + 0.4j, 0.2 - 0.1j, -1.5, [0.3, -0.2, 0.7], 0.5
    q = rng.uniform(-np.pi, np.pi, (64, 3))
    A, B = SW.assemble(1, [[0, 0]], [[a.real, a.imag, b.real, b.imag, c]], [d], q, field=h)
    W, X, info = oracle_lib.hegv(A, B, 2)
    assert (info == 0).all()
    om = SW.single_site_omega(a, b, c, d, h, q)
    assert np.abs(np.abs(1.0 / W) - om[:, None]).max() <= 1e-13 * om.max()
    assert (W[:, 0] < 0).all() and (W[:, 1] > 0).all()          # one +omega and one -omega mode


@pytest.mark.parametrize("N", [6, 27])
def test_assembly_matches_qsweep_generator(N):
    """The bond-table assembly equals the torch q-sweep generator's B0(q) + field I (the same
    cell, an independent code path) to rounding."""
    cell = wl.spinwave_cell(N, 0)
    q = wl.qsweep_points(8, 0, 48).numpy()
    field = 2.25
    A, B = SW.assemble(N, cell["sites"], cell["coef"], cell["disp"], q, field=field)
    n = 2 * N
    B0 = wl.qsweep_B0(N, torch.from_numpy(q), 0).numpy() + field * np.eye(n)
    Bt = np.ascontiguousarray(np.swapaxes(B0, 1, 2)).reshape(-1, n * n)
    assert np.abs(B - Bt).max() <= 4e-16 * np.abs(Bt).max() * 4
    Am = A.reshape(-1, n, n)
    assert np.array_equal(Am[0], np.diag(np.where(np.arange(n) < N, 1.0, -1.0)).astype(np.complex128))


def test_assembly_is_exactly_hermitian_and_bogoliubov():
    cell = wl.spinwave_cell(9, 3)
    q = np.random.default_rng(1).uniform(-4, 4, (16, 3))
    _, B = SW.assemble(9, cell["sites"], cell["coef"], cell["disp"], q, field=0.0)
    n, N = 18, 9
    M = B.reshape(-1, n, n).transpose(0, 2, 1)
    assert np.array_equal(M, np.conj(np.swapaxes(M, 1, 2)))
    assert np.array_equal(M[:, N:, N:], np.conj(M[:, :N, :N]))
    assert np.array_equal(M[:, N:, :N], np.conj(M[:, :N, N:]))
    assert np.array_equal(M[:, :N, N:], np.swapaxes(M[:, :N, N:], 1, 2))      # Q symmetric


def test_intensities_are_phase_invariant_and_nan_on_failure(oracle_lib):
    cell = wl.spinwave_cell(6, 1)
    q = np.random.default_rng(2).uniform(-3, 3, (8, 3))
    A, B = SW.assemble(6, cell["sites"], cell["coef"], cell["disp"], q, field=0.0)
    ev = np.linalg.eigvalsh(B.reshape(-1, 12, 12).transpose(0, 2, 1))
    field = wl.spinwave_field(ev[:, 0].min(), ev[:, -1].max(), 1e-2)
    A, B = SW.assemble(6, cell["sites"], cell["coef"], cell["disp"], q, field=field)
    W, X, info = oracle_lib.hegv(A, B, 12)
    assert (info == 0).all()
    I0 = SW.intensities(6, cell["pos"], q, W, X)
    phase = np.exp(1j * np.random.default_rng(3).uniform(0, 2 * np.pi, (8, 12)))
    Xp = (X.reshape(8, 12, 12) * phase[:, :, None]).reshape(8, 144)
    assert np.allclose(SW.intensities(6, cell["pos"], q, W, Xp), I0, rtol=1e-13, atol=0)
    assert (I0 >= 0).all() and np.isfinite(I0).all()
    bad = np.zeros(8, np.int32); bad[3] = 7
    I1 = SW.intensities(6, cell["pos"], q, W, X, bad)
    assert np.isnan(I1[3]).all() and np.array_equal(np.delete(I1, 3, 0), np.delete(I0, 3, 0))


def test_field_puts_the_sweep_minimum_at_frac():
    lmin, lmax, frac = -3.0, 5.0, 1e-3
    h = wl.spinwave_field(lmin, lmax, frac)
    assert abs((lmin + h) - frac * (lmax + h)) <= 1e-15 * (lmax + h)
