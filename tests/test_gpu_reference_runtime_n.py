"""The reference's own runtime-n solver tests, compiled unchanged against this library's drop-in
header include/sbg/compat/nvrtc/nvrtc_solver.hpp.

This file runs two of them:

* tests/test_nvrtc_n54.cpp: NvrtcGeneigSolver(54, 0) on the 8-pair random fixture.
* tests/test_nvrtc_multiN.cpp: the same for N in {16, 32, 48, 54, 64, 96, 128}, random and
  near-identity fixtures.

Both come from the reference and read tests/data/n<N>_b8_s42_<kind>.bin relative to the working
directory. They check eigenvalues (relative error < 1e-10) and eigenvector phases (< 1e-10 for
non-degenerate eigenvalues) against the fixture's zhegvd output, and exit 0 only when every case
passes. oracle/Makefile's `nvrtc-drivers` target builds them. The fixtures are regenerated by the
reference's own generator (oracle/_ref/lapack_reference) and checked against the SHA-256 of the
reference's fixtures before use.
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, REPO

pytestmark = pytest.mark.gpu

REF_BIN = os.path.join(REPO, "oracle", "_ref")
SIZES = (16, 32, 48, 54, 64, 96, 128)
KINDS = (("random", "random"), ("nearid", "near-identity"))


def _need(path):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.relpath(path, REPO)} not built (oracle/Makefile `ref` and `nvrtc-drivers` targets "
                    "need the reference tree at build time)")


@pytest.fixture(scope="module")
def data_dir(tmp_path_factory):
    gen = os.path.join(REF_BIN, "lapack_reference")
    _need(gen)
    root = tmp_path_factory.mktemp("refruntime")
    os.makedirs(root / "tests" / "data")
    manifest = json.load(open(os.path.join(GOLDEN, "manifest.json")))
    from oracle import oracle as O
    for n in SIZES:
        for tag, mode in KINDS:
            name = f"n{n}_b8_s42_{tag}"
            out = root / "tests" / "data" / f"{name}.bin"
            subprocess.run([gen, "--n", str(n), "--batch", "8", "--seed", "42", "--s-mode", mode, "--out", str(out)],
                           check=True, capture_output=True, timeout=300)
            fx = O.read_geig(str(out))
            assert hashlib.sha256(np.ascontiguousarray(fx["H"]).tobytes()).hexdigest() == manifest[name]["sha256_H"]
            assert hashlib.sha256(np.ascontiguousarray(fx["S"]).tobytes()).hexdigest() == manifest[name]["sha256_S"]
    return root


@pytest.mark.parametrize("test", ["test_nvrtc_n54", "test_nvrtc_multiN"])
def test_reference_runtime_n_test_passes(test, data_dir, tmp_path):
    exe = os.path.join(REF_BIN, test)
    _need(exe)
    env = dict(os.environ, SUNNY_GENEIG_CACHE_DIR=str(tmp_path))
    r = subprocess.run([exe], cwd=data_dir, capture_output=True, text=True, timeout=600, env=env)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-4000:]
    assert "FAIL" not in out, out[-4000:]
    if test == "test_nvrtc_n54":
        assert "SUMMARY: 8/8 passed" in out, out[-2000:]
    else:
        # every size runs: the solver reports the shared memory its kernels take, within the device limit
        assert "SKIP" not in out, out[-4000:]
        assert "OVERALL: 14/14" in out, out[-2000:]
