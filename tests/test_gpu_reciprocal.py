"""The inverse iteration's reciprocal (Newton-Raphson from the hardware estimate, two steps)
against the correctly rounded 1.0 / u, through the C ABI's device self-test.

The factorization of T - lam I keeps |u| >= eps ||T|| (normal numbers), so the probes span
normal magnitudes 2^-1000 .. 2^1000 of both signs.  The bound checked is the one the
factorization relies on: at most one unit in the last place from 1.0 / u (two Newton steps from a
~2^-23 estimate leave ~2^-92 before rounding); exact equality is reported, not required.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from sbg import _lib

pytestmark = pytest.mark.gpu


def _ulps(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return np.abs(ia - ib)


def test_reciprocal_within_one_ulp_of_division():
    rng = np.random.default_rng(2024)
    count = 1 << 22
    mant = rng.uniform(1.0, 2.0, count)
    expo = rng.integers(-1000, 1000, count)
    sign = np.where(rng.random(count) < 0.5, -1.0, 1.0)
    u = sign * np.ldexp(mant, expo)
    # exact powers of two, mantissas next to 1 and 2, and moderate values of the eigenvalue scale
    edge = np.concatenate([np.ldexp(1.0, np.arange(-1000, 1000)), np.nextafter(np.ldexp(1.0, np.arange(-990, 990, 7)), 0),
                           np.nextafter(np.ldexp(2.0, np.arange(-990, 990, 7)), 4), np.linspace(-3.0, 3.0, 6001)])
    edge = edge[edge != 0.0]
    u = np.concatenate([u, edge, -edge])
    du = torch.as_tensor(u).cuda()
    dr = torch.empty_like(du)
    lib = _lib.load()
    st = lib.sbg_selftest_reciprocal(ctypes.c_void_p(du.data_ptr()), ctypes.c_void_p(dr.data_ptr()), du.numel(),
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, lib.sbg_last_error().decode()
    r = dr.cpu().numpy()
    want = 1.0 / u
    assert np.isfinite(r).all()
    assert (np.sign(r) == np.sign(want)).all()
    ulp = _ulps(np.abs(r), np.abs(want))
    assert ulp.max() <= 1, (u[ulp.argmax()], r[ulp.argmax()], want[ulp.argmax()])
    print(f"recip_nr equal to 1.0/u on {np.mean(ulp == 0):.6%} of {u.size} probes, max {ulp.max()} ulp")
