"""Distils the reference's GEIG v1 fixtures into the compact golden vectors kept here.

Run in a checkout that has the reference tree (its location from --ref, else the
SBG_REFERENCE_DIR environment variable, else oracle.reference_dir()'s default):

    python tests/golden/make_golden.py [--ref DIR]

Sources:
  * tests/data/n{16,32,48,54,64,96}_b8_s42_{random,nearid}.bin of the reference
    (written by its tests/lapack_reference.cpp with LAPACKE_zhegvd);
  * the three blobs the reference lists as missing (.MISSING_LARGE_BLOBS):
    n128_b8_s42_{random,nearid} and n54_b32_s123_random, regenerated by the
    reference's own lapack_reference program built under oracle/_ref/.
Outputs (committed):
  manifest.json   per fixture: n, batch, seed, s_mode, SHA-256 of the H and S
                  blocks (so the inputs can be regenerated bit-exactly by the
                  oracle's restated generator and checked), source
  golden_W.npz    the fixture eigenvalues W (batch, n) per fixture
  golden_U0.npz   the eigenvectors U of pair 0 for fixtures with n <= 54
"""
from __future__ import annotations

import argparse
import glob
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import oracle as O  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=O.reference_dir())
    args = ap.parse_args()
    files = sorted(glob.glob(os.path.join(args.ref, "tests", "data", "*.bin")))
    entries = {}
    W_all = {}
    U0 = {}

    def add(name, fx, mode, source):
        entries[name] = dict(n=fx["n"], batch=fx["batch"], seed=fx["seed"], s_mode=mode,
                             sha256_H=sha(fx["H"]), sha256_S=sha(fx["S"]), source=source)
        W_all[name] = fx["W"]
        if fx["n"] <= 54:
            U0[name] = fx["U"][0]

    for path in files:
        name = os.path.basename(path)[:-4]
        mode = "nearid" if name.endswith("nearid") else "random"
        add(name, O.read_geig(path), mode, "reference tests/data")
    O.build()
    gen = O.REF_GENERATOR
    if not os.path.exists(gen):
        raise SystemExit("oracle/_ref/lapack_reference is missing (make -C oracle ref)")
    with tempfile.TemporaryDirectory() as td:
        for n, b, seed, mode in ((128, 8, 42, "random"), (128, 8, 42, "nearid"), (54, 32, 123, "random")):
            name = f"n{n}_b{b}_s{seed}_{mode}"
            out = os.path.join(td, name + ".bin")
            cmd = [gen, "--n", str(n), "--batch", str(b), "--seed", str(seed), "--out", out]
            if mode == "nearid":
                cmd += ["--s-mode", "near-identity"]
            subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
            add(name, O.read_geig(out), mode, "reference lapack_reference (missing blob)")
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(entries, f, indent=1, sort_keys=True)
    np.savez(os.path.join(HERE, "golden_W.npz"), **W_all)
    np.savez(os.path.join(HERE, "golden_U0.npz"), **U0)
    print(f"wrote {len(entries)} fixtures")


if __name__ == "__main__":
    main()
