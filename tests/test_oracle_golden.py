"""Pins the oracle: the restated fixture generator and LAPACK against the
reference's golden fixtures (tests/data/*.bin of the reference, distilled into
tests/golden/ by tests/golden/make_golden.py)."""
from __future__ import annotations

import hashlib
import os

import numpy as np
import pytest

from oracle import metrics as Mx


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_manifest_covers_reference_fixtures(manifest):
    names = set(manifest)
    for n in (16, 32, 48, 54, 64, 96):
        for mode in ("random", "nearid"):
            assert f"n{n}_b8_s42_{mode}" in names
    assert {"n128_b8_s42_random", "n128_b8_s42_nearid", "n54_b32_s123_random"} <= names


def test_generator_regenerates_fixture_inputs_bit_exactly(manifest, oracle_mod):
    for name, e in manifest.items():
        H, S = oracle_mod.gen_fixture_pairs(e["n"], e["batch"], e["seed"], e["s_mode"])
        assert _sha(H) == e["sha256_H"], name
        assert _sha(S) == e["sha256_S"], name


@pytest.mark.parametrize("dc", [False, True], ids=["zhegv", "zhegvd"])
def test_lapack_matches_fixture_eigenpairs(manifest, golden_W, golden_U0, oracle_mod, dc):
    for name, e in manifest.items():
        n = e["n"]
        if n > 96:
            continue
        H, S = oracle_mod.gen_fixture_pairs(n, e["batch"], e["seed"], e["s_mode"])
        W, U, info = oracle_mod.hegv(H, S, n, nthreads=4, divide_and_conquer=dc)
        assert (info == 0).all()
        # the reference's own gate is 1e-10 (tests/test_full_n54.cpp:46-48); the oracle is far inside it
        assert Mx.eig_rel_ref(W, golden_W[name]).max() < 1e-13, name
        assert Mx.residual(H, S, U, W, n).max() < 1e-14
        assert Mx.orth(S, U, n).max() < 1e-13
        if name in golden_U0:
            ph = Mx.phase_err(S[:1], U[:1], golden_U0[name][None], golden_W[name][:1], n)
            assert ph.max() < 1e-12, name


def test_reference_generator_binary_when_built(oracle_mod, manifest, tmp_path):
    if not os.path.exists(oracle_mod.REF_GENERATOR):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    import subprocess
    out = tmp_path / "n32.bin"
    subprocess.run([oracle_mod.REF_GENERATOR, "--n", "32", "--batch", "8", "--seed", "42", "--out", str(out),
                    "--s-mode", "near-identity"], check=True, capture_output=True)
    fx = oracle_mod.read_geig(str(out))
    e = manifest["n32_b8_s42_nearid"]
    assert _sha(fx["H"]) == e["sha256_H"] and _sha(fx["S"]) == e["sha256_S"]


def test_stage_oracles_are_consistent(oracle_mod):
    """potrf -> hegst -> heev -> trsm (the reference's stage order) equals zhegv."""
    n = 24
    H, S = oracle_mod.gen_fixture_pairs(n, 4, 7, "random")
    W, U, _ = oracle_mod.hegv(H, S, n)
    Ws, Us, info = oracle_mod.staged_full(H, S, n)
    assert (info == 0).all()
    assert Mx.eig_rel(Ws, W).max() < 1e-13
    assert Mx.phase_err(S, Us, U, W, n).max() < 1e-12
    M, L, info = oracle_mod.reduce(H, S, n)
    Wf, Uf, info = oracle_mod.finish(L, M, n)
    assert Mx.eig_rel(Wf, W).max() < 1e-13
    Wv, V, _ = oracle_mod.reduce_eig(H, S, n)
    assert Mx.eig_rel(Wv, W).max() < 1e-13
    L2, info = oracle_mod.potrf(S, n)
    assert np.abs(L2 - L).max() == 0.0


def test_geig_roundtrip(tmp_path, oracle_mod):
    n = 8
    H, S = oracle_mod.gen_fixture_pairs(n, 2, 1, "random")
    W, U, _ = oracle_mod.hegv(H, S, n)
    p = tmp_path / "x.bin"
    oracle_mod.write_geig(str(p), n, 1, H, S, W, U)
    fx = oracle_mod.read_geig(str(p))
    assert np.array_equal(fx["H"], H) and np.array_equal(fx["W"], W) and np.array_equal(fx["U"], U)


def test_metrics_detect_planted_errors(oracle_mod):
    """A mistake planted in the oracle's output is caught by every metric."""
    n = 16
    H, S = oracle_mod.gen_fixture_pairs(n, 2, 3, "random")
    W, U, _ = oracle_mod.hegv(H, S, n)
    W2 = W.copy(); W2[0, 3] *= 1 + 1e-9
    assert Mx.eig_rel(W2, W).max() > 1e-10
    U2 = U.copy(); U2[1, 5 * n:6 * n] *= 1.0 + 1e-6
    assert Mx.orth(S, U2, n).max() > 1e-7
    assert Mx.residual(H, S, U2, W, n).max() < 1e-6  # scaling a vector keeps it an eigenvector
    U3 = U.copy(); U3[0, 2 * n:3 * n], U3[0, 3 * n:4 * n] = U[0, 3 * n:4 * n].copy(), U[0, 2 * n:3 * n].copy()
    assert Mx.phase_err(S, U3, U, W, n).max() > 0.5
