"""Every launch schedule the autotuner can choose, checked against the LAPACK oracle.

The reference validates an autotuned block size only against its own suggested configuration
(src/nvrtc/nvrtc_solver.cpp:735-740).  Here every candidate of the sweep -- pairs per CTA of the
warp-per-pair Cholesky / Householder kernels (the reference's batches per block), exact-n versus
generic column kernels, one or two lanes per column and one or two reflectors per pass in the
back-transform, the QL chain's CTA size -- is set through sbg_solver_set_schedule and its results are compared with zhegv under the
parity gates, and so is the schedule the autotuner picks at n = 32 and 54.
"""
from __future__ import annotations

import itertools

import numpy as np
import pytest

import sbg
from sbg import workloads as wl
from test_gpu_parity import check, run

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pairs_and_oracle(oracle_mod):
    out = {}
    for N in (16, 27):
        A, B = wl.bogoliubov(N, 96, seed=100 + N, frac=1e-3)
        A, B = A.numpy(), B.numpy()
        Wr, Xr, _ = oracle_mod.hegv(A, B, 2 * N, nthreads=8)
        out[2 * N] = (A, B, Wr, Xr)
    return out


@pytest.mark.parametrize("n", [32, 54])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_candidate_schedule_passes_the_gates(n, precision, pairs_and_oracle):
    A, B, Wr, Xr = pairs_and_oracle[n]
    s = sbg.Solver(n, precision=precision)
    base = s.schedule
    seen = 0
    for pw, ex, gl, qp, ct in itertools.product((1, 2, 4), (0, 1), (1, 2), (1, 2), (64, 128, 256)):
        s.schedule = dict(base, pairs_per_cta=pw, col_exact=ex, back_lanes=gl, back_qpass=qp, chain_threads=ct)
        assert s.schedule["pairs_per_cta"] == pw and s.batches_per_block == pw
        W, X, info = run(s, A, B)
        check(A, B, W, X, info, Wr, Xr, n, relative=True)
        seen += 1
    assert seen == 72
    s.close()


def test_schedule_values_are_checked():
    s = sbg.Solver(54)
    for bad in (dict(pairs_per_cta=3), dict(back_lanes=4), dict(hetrd_threads=96), dict(chain_threads=100),
                dict(back_qpass=3)):
        with pytest.raises(sbg.SolverError):
            s.schedule = bad
    s.close()


@pytest.mark.parametrize("n", [32, 54])
def test_autotuned_schedule_against_oracle(n, pairs_and_oracle, capfd):
    """The sweep's winner (measured on this GPU, cache disabled) passes the gates; whether it
    differs from the built-in schedule is reported."""
    A, B, Wr, Xr = pairs_and_oracle[n]
    builtin = sbg.Solver(n).schedule
    s = sbg.Solver(n, tuning="autotune", cache="none")
    assert s.was_autotuned and s.autotune_sweep_ran
    tuned = s.schedule
    W, X, info = run(s, A, B)
    check(A, B, W, X, info, Wr, Xr, n, relative=True)
    diff = {k: (builtin[k], tuned[k]) for k in builtin if builtin[k] != tuned[k]}
    print(f"n={n}: built-in {builtin}; autotuned {tuned}; differs in {diff or 'nothing'}")
    s.close()
