"""The C-ABI library loads and exports every entry point include/sbg/geneig.h
declares (no compute calls: this runs without a GPU)."""
from __future__ import annotations

import ctypes
import os
import re

from conftest import REPO

HEADER = os.path.join(REPO, "include", "sbg", "geneig.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"^\s*#.*$", "", src, flags=re.M)           # preprocessor lines
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", src)
    return sorted(set(n for n in names if n not in ("if", "while", "sizeof")))


def test_header_declares_the_reference_drop_in():
    names = set(declared_functions())
    for n in ("geneig_full_n54_batched_launch", "geneig_full_n54_batched_block_dim_x",
              "geneig_full_n54_batched_shared_mem_bytes", "chol_n54_launch", "geneig_reduce_n54_launch",
              "geneig_reduce_eig_n54_launch", "geneig_full_n54_launch", "geneig_finish_n54_launch",
              "sbg_solver_create", "sbg_solver_launch", "sbg_solver_launch_chunked", "sbg_solver_destroy"):
        assert n in names, n


def test_library_exports_every_declared_symbol():
    import sbg
    from sbg import _lib
    lib = sbg.load()
    for name in declared_functions():
        assert hasattr(lib, name), f"missing export {name}"
    assert set(declared_functions()) == set(_lib.SIGNATURES), \
        set(declared_functions()) ^ set(_lib.SIGNATURES)


def test_library_links_no_oracle():
    from sbg import _lib
    data = open(_lib.LIB_PATH, "rb").read()
    assert b"sbo_hegv_batch" not in data and b"LAPACKE_" not in data


def test_status_strings_without_gpu():
    import sbg
    lib = sbg.load()
    assert lib.sbg_status_string(0) == b"ok"
    assert lib.sbg_status_string(5).startswith(b"workspace")
