"""The reference's own C++ test drivers, compiled unchanged against this library.

tests/test_full_batched_n54.cpp, test_full_n54.cpp, test_chol_n54.cpp, test_reduce_n54.cpp and
test_reduce_eig_n54.cpp of the reference declare the fixed n = 54 entry points themselves
(e.g. test_full_batched_n54.cpp:28-37), read tests/data/*.bin relative to the working directory,
check the GPU results against the fixture's zhegvd output or their own LAPACKE calls with their
own gates (1e-12 zpotrf, 1e-11 zhegst, 1e-10 zheev / zhegv and S-phase), and exit 0 only when
every matrix passes.  oracle/Makefile's `drivers` target compiles them from the reference tree
and links them against libsbg_geneig.so in place of the reference's cuSolverDx build: passing
them is the drop-in's proof for a C/C++ caller.  The fixtures they read are regenerated here by
the reference's own generator (oracle/_ref/lapack_reference, built by the same Makefile) and
checked against the SHA-256 of the reference's fixtures before use.
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, REPO

pytestmark = pytest.mark.gpu

REF_BIN = os.path.join(REPO, "oracle", "_ref")
DRIVERS = ("test_full_batched_n54", "test_full_n54", "test_chol_n54", "test_reduce_n54", "test_reduce_eig_n54")
FIXTURES = (("n54_b8_s42_random", 54, 8, 42, "random"), ("n54_b8_s42_nearid", 54, 8, 42, "near-identity"),
            ("n54_b32_s123_random", 54, 32, 123, "random"))


def _need(path):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.relpath(path, REPO)} not built (oracle/Makefile `ref` and `drivers` targets need "
                    "the reference tree at build time)")


@pytest.fixture(scope="module")
def data_dir(tmp_path_factory):
    """A working directory holding tests/data/<fixture>.bin for the three fixtures the drivers read."""
    gen = os.path.join(REF_BIN, "lapack_reference")
    _need(gen)
    root = tmp_path_factory.mktemp("refdrivers")
    os.makedirs(root / "tests" / "data")
    manifest = json.load(open(os.path.join(GOLDEN, "manifest.json")))
    from oracle import oracle as O
    for name, n, b, seed, mode in FIXTURES:
        out = root / "tests" / "data" / f"{name}.bin"
        subprocess.run([gen, "--n", str(n), "--batch", str(b), "--seed", str(seed), "--s-mode", mode,
                        "--out", str(out)], check=True, capture_output=True, timeout=300)
        fx = O.read_geig(str(out))
        H, S = fx["H"], fx["S"]
        assert hashlib.sha256(np.ascontiguousarray(H).tobytes()).hexdigest() == manifest[name]["sha256_H"]
        assert hashlib.sha256(np.ascontiguousarray(S).tobytes()).hexdigest() == manifest[name]["sha256_S"]
    return root


@pytest.mark.parametrize("driver", DRIVERS)
def test_reference_driver_passes_against_this_library(driver, data_dir):
    exe = os.path.join(REF_BIN, driver)
    _need(exe)
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
    r = subprocess.run([exe], cwd=data_dir, capture_output=True, text=True, timeout=600, env=env)
    out = r.stdout + r.stderr
    with open(os.path.join(str(data_dir), f"{driver}.log"), "w") as f:
        f.write(out)
    assert r.returncode == 0, out[-4000:]
    assert "FAIL" not in out.replace("SOME FAILED", ""), out[-4000:]
    if driver == "test_full_batched_n54":
        assert "ALL PASSED" in out
        # the driver's own timing of the reference's CPU loop (one LAPACKE_zhegv per pair, one thread)
        m = re.search(r"LAPACK zhegv host\s*=\s*([0-9.]+) s\s*\(([0-9.]+) matrices/sec\)", out)
        assert m and float(m.group(2)) > 0, out[-2000:]
