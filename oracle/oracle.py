"""CPU checker for the batched Hermitian-definite generalized eigensolve.

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and the bench's
cpu_baseline / reference leg may use this module; the product path never does.

ctypes front end of ``libsbg_oracle.so`` (geneig_oracle.cpp): the reference's
fixture generator restated (tests/lapack_reference.cpp:86-150), LAPACK zhegv /
zhegvd per pair (tests/test_full_batched_n54.cpp:238-256,
tests/lapack_reference.cpp:186-194) and the per-stage LAPACK twins used by the
reference's staged tests.  All arrays are numpy, column-major per pair, pairs
contiguous: a batch of n x n complex matrices has shape (batch, n, n) in
"column-major" meaning ``M[b].T`` is the row-major view (we store M[b][j][i]).
To keep the layout obvious every function takes and returns flat
``complex128`` arrays of shape (batch, n*n) in column-major order.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsbg_oracle.so")
REF_GENERATOR = os.path.join(HERE, "_ref", "lapack_reference")

GEIG_MAGIC = 0x47454947
GEIG_VERSION = 1

_lib = None


def reference_dir() -> str:
    """Where the reference tree is read from when it is present (build time only): the
    SBG_REFERENCE_DIR environment variable, else the default the Makefile also uses."""
    return os.environ.get("SBG_REFERENCE_DIR", "/root/reference")


REF_DRIVERS = ("test_full_batched_n54", "test_full_n54", "test_chol_n54", "test_reduce_n54",
               "test_reduce_eig_n54")


def build(quiet: bool = True) -> None:
    """Compile libsbg_oracle.so and, when the reference tree is present, _ref/: the reference's
    fixture generator, its own n = 54 test drivers and its runtime-n solver tests (the latter
    through include/sbg/compat/nvrtc/nvrtc_solver.hpp), linked against libsbg_geneig.so (which
    must be built first)."""
    targets = ["all"]
    ref = reference_dir()
    if os.path.isdir(os.path.join(ref, "tests")):
        targets.append("ref")
        lib_so = os.path.join(os.path.dirname(HERE), "sunny-batched-geneig_b200", "sbg", "libsbg_geneig.so")
        if os.path.exists(lib_so):
            targets += ["drivers", "nvrtc-drivers"]
    subprocess.run(["make", "-C", HERE, f"SBG_REFERENCE_DIR={ref}", *targets], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        I = ctypes.c_int
        L.sbo_gen_fixture_pairs.argtypes = [I, I, I, I, P, P]
        L.sbo_hegv_batch.argtypes = [I, I, P, P, P, P, P, I, I]
        L.sbo_hegv_values_batch.argtypes = [I, I, P, P, P, P, I]
        L.sbo_potrf_batch.argtypes = [I, I, P, P, P, I]
        L.sbo_reduce_batch.argtypes = [I, I, P, P, P, P, P, I]
        L.sbo_reduce_eig_batch.argtypes = [I, I, P, P, P, P, P, I]
        L.sbo_finish_batch.argtypes = [I, I, P, P, P, P, P, I]
        L.sbo_staged_full_batch.argtypes = [I, I, P, P, P, P, P, I]
        L.sbo_heev_values_batch.argtypes = [I, I, P, P, P, I]
        L.sbo_hardware_threads.restype = I
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex128)


def host_threads() -> int:
    return max(1, int(lib().sbo_hardware_threads()))


# --------------------------------------------------------------------------- generators

def gen_fixture_pairs(n: int, batch: int, seed: int, s_mode: str = "random"):
    """Inputs of a reference GEIG v1 fixture (bit-identical to lapack_reference)."""
    H = np.empty((batch, n * n), np.complex128)
    S = np.empty((batch, n * n), np.complex128)
    mode = {"random": 0, "nearid": 1, "near-identity": 1}[s_mode]
    lib().sbo_gen_fixture_pairs(n, batch, seed, mode, _p(H), _p(S))
    return H, S


# --------------------------------------------------------------------------- solves

def hegv(H, S, n: int, nthreads: int = 1, divide_and_conquer: bool = False):
    """LAPACK zhegv (or zhegvd) per pair -> (W (batch,n), U (batch,n*n), info (batch,))."""
    H = _c128(H).reshape(-1, n * n)
    S = _c128(S).reshape(-1, n * n)
    b = H.shape[0]
    W = np.empty((b, n), np.float64)
    U = np.empty((b, n * n), np.complex128)
    info = np.empty(b, np.int32)
    lib().sbo_hegv_batch(n, b, _p(H), _p(S), _p(W), _p(U), _p(info), int(divide_and_conquer), nthreads)
    return W, U, info


def hegv_values(H, S, n: int, nthreads: int = 1):
    H = _c128(H).reshape(-1, n * n)
    S = _c128(S).reshape(-1, n * n)
    b = H.shape[0]
    W = np.empty((b, n), np.float64)
    info = np.empty(b, np.int32)
    lib().sbo_hegv_values_batch(n, b, _p(H), _p(S), _p(W), _p(info), nthreads)
    return W, info


def potrf(S, n: int, nthreads: int = 1):
    S = _c128(S).reshape(-1, n * n)
    b = S.shape[0]
    L = np.empty_like(S)
    info = np.empty(b, np.int32)
    lib().sbo_potrf_batch(n, b, _p(S), _p(L), _p(info), nthreads)
    return L, info


def reduce(H, S, n: int, nthreads: int = 1):
    """(M lower with strict upper zeroed, L lower with strict upper zeroed, info)."""
    H = _c128(H).reshape(-1, n * n)
    S = _c128(S).reshape(-1, n * n)
    b = H.shape[0]
    M = np.empty_like(H)
    L = np.empty_like(H)
    info = np.empty(b, np.int32)
    lib().sbo_reduce_batch(n, b, _p(H), _p(S), _p(M), _p(L), _p(info), nthreads)
    return M, L, info


def reduce_eig(H, S, n: int, nthreads: int = 1):
    H = _c128(H).reshape(-1, n * n)
    S = _c128(S).reshape(-1, n * n)
    b = H.shape[0]
    W = np.empty((b, n), np.float64)
    V = np.empty_like(H)
    info = np.empty(b, np.int32)
    lib().sbo_reduce_eig_batch(n, b, _p(H), _p(S), _p(W), _p(V), _p(info), nthreads)
    return W, V, info


def finish(L, M, n: int, nthreads: int = 1):
    L = _c128(L).reshape(-1, n * n)
    M = _c128(M).reshape(-1, n * n)
    b = L.shape[0]
    W = np.empty((b, n), np.float64)
    U = np.empty_like(L)
    info = np.empty(b, np.int32)
    lib().sbo_finish_batch(n, b, _p(L), _p(M), _p(W), _p(U), _p(info), nthreads)
    return W, U, info


def staged_full(H, S, n: int, nthreads: int = 1):
    H = _c128(H).reshape(-1, n * n)
    S = _c128(S).reshape(-1, n * n)
    b = H.shape[0]
    W = np.empty((b, n), np.float64)
    U = np.empty_like(H)
    info = np.empty(b, np.int32)
    lib().sbo_staged_full_batch(n, b, _p(H), _p(S), _p(W), _p(U), _p(info), nthreads)
    return W, U, info


def heev_values(M, n: int, nthreads: int = 1):
    M = _c128(M).reshape(-1, n * n)
    b = M.shape[0]
    W = np.empty((b, n), np.float64)
    info = np.empty(b, np.int32)
    lib().sbo_heev_values_batch(n, b, _p(M), _p(W), _p(info), nthreads)
    return W, info


# --------------------------------------------------------------------------- GEIG v1 files

def read_geig(path: str):
    """GEIG v1 (tests/lapack_reference.cpp:257-284): header 6 x int32 then H, S, W, U."""
    with open(path, "rb") as f:
        hdr = f.read(24)
        magic, version, n, b, seed, _ = struct.unpack("<6i", hdr)
        if magic != GEIG_MAGIC:
            raise ValueError(f"bad magic 0x{magic:08x}")
        if version != GEIG_VERSION:
            raise ValueError(f"unsupported version {version}")
        mat = n * n
        H = np.frombuffer(f.read(16 * mat * b), np.complex128).reshape(b, mat).copy()
        S = np.frombuffer(f.read(16 * mat * b), np.complex128).reshape(b, mat).copy()
        W = np.frombuffer(f.read(8 * n * b), np.float64).reshape(b, n).copy()
        U = np.frombuffer(f.read(16 * mat * b), np.complex128).reshape(b, mat).copy()
        if U.shape[0] != b:
            raise ValueError("short read")
    return dict(n=n, batch=b, seed=seed, H=H, S=S, W=W, U=U)


def write_geig(path: str, n: int, seed: int, H, S, W, U) -> None:
    b = H.shape[0]
    with open(path, "wb") as f:
        f.write(struct.pack("<6i", GEIG_MAGIC, GEIG_VERSION, n, b, seed, 0))
        for a, dt in ((H, np.complex128), (S, np.complex128), (W, np.float64), (U, np.complex128)):
            f.write(np.ascontiguousarray(a, dt).tobytes())
