"""ctypes binding of libsbg_geneig.so (the C ABI in include/sbg/geneig.h).

The library is the only compute path: nothing here falls back to a CPU or
library eigensolver.  Loading fails loudly if the shared object is missing.
"""
from __future__ import annotations

import ctypes
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsbg_geneig.so")

P = ctypes.c_void_p
I = ctypes.c_int
U = ctypes.c_uint
SZ = ctypes.c_size_t
LL = ctypes.c_longlong
D = ctypes.c_double

# Every exported symbol with (restype, argtypes); the CPU tests check this list
# against include/sbg/geneig.h.
SIGNATURES = {
    "sbg_status_string": (ctypes.c_char_p, [I]),
    "sbg_last_error": (ctypes.c_char_p, []),
    "geneig_full_n54_batched_launch": (None, [P, P, P, P, P, I, P]),
    "geneig_full_n54_batched_block_dim_x": (U, []),
    "geneig_full_n54_batched_shared_mem_bytes": (U, []),
    "chol_n54_launch": (None, [P, P, P, P]),
    "chol_n54_block_dim_x": (U, []),
    "chol_n54_shared_mem_bytes": (U, []),
    "geneig_reduce_n54_launch": (None, [P, P, P, P, P]),
    "geneig_reduce_n54_block_dim_x": (U, []),
    "geneig_reduce_n54_shared_mem_bytes": (U, []),
    "geneig_reduce_eig_n54_launch": (None, [P, P, P, P, P, P]),
    "geneig_reduce_eig_n54_block_dim_x": (U, []),
    "geneig_reduce_eig_n54_shared_mem_bytes": (U, []),
    "geneig_reduce_eig_n54_chol_smem_bytes": (U, []),
    "geneig_reduce_eig_n54_heev_smem_bytes": (U, []),
    "geneig_reduce_eig_n54_heev_workspace": (U, []),
    "geneig_full_n54_launch": (None, [P, P, P, P, P, P]),
    "geneig_full_n54_block_dim_x": (U, []),
    "geneig_full_n54_shared_mem_bytes": (U, []),
    "geneig_finish_n54_launch": (None, [P, P, P, P, P, I, P]),
    "geneig_finish_n54_block_dim_x": (U, []),
    "geneig_finish_n54_shared_mem_bytes": (U, []),
    "sbg_solver_options_init": (None, [P]),
    "sbg_solver_create": (I, [I, I, P, P]),
    "sbg_solver_destroy": (I, [P]),
    "sbg_solver_launch": (I, [P, P, P, P, P, P, I, P]),
    "sbg_solver_launch_chunked": (I, [P, P, P, P, P, P, I, I, I, P]),
    "sbg_solver_reserve": (I, [P, I, I]),
    "sbg_solver_solve_host": (I, [P, P, P, P, P, P, I, I, I]),
    "sbg_solver_host_transfer_bytes": (I, [P, P, P]),
    "sbg_solver_enable_stage_timing": (I, [P, I]),
    "sbg_solver_refine_redo_pairs": (I, [P, P, I]),
    "sbg_solver_read_stage_times": (I, [P, P, P]),
    "sbg_workspace_bytes_per_pair": (SZ, [I, I]),
    "sbg_workspace_bytes": (SZ, [I, I, I]),
    "sbg_selftest_reciprocal": (I, [P, P, I, P]),
    "sbg_selftest_fp64_fma": (I, [P, I, I, P]),
    "sbg_solver_schedule": (I, [P, P]),
    "sbg_solver_set_schedule": (I, [P, P]),
    "sbg_solver_matrix_size": (I, [P]),
    "sbg_solver_batches_per_block": (I, [P]),
    "sbg_solver_block_dim_x": (I, [P]),
    "sbg_solver_shared_mem_bytes": (U, [P]),
    "sbg_solver_was_autotuned": (I, [P]),
    "sbg_solver_autotune_sweep_ran": (I, [P]),
    "sbg_solver_cache_layer_used": (ctypes.c_char_p, [P]),
    "sbg_solver_precision": (I, [P]),
    "sbg_max_n": (I, [I]),
    "sbg_tuning_table_path": (I, [I, ctypes.c_char_p, SZ]),
    "sbg_tuning_forget_in_process": (I, []),
    "sbg_geneig_full_noalloc_launch": (I, [I, P, P, P, P, P, I, P]),
    "sbg_queue_create": (I, [P, I, I, P, P]),
    "sbg_queue_destroy": (I, [P]),
    "sbg_launch_queue": (I, [P, P, P, P, P, P, P]),
    "sbg_queue_size": (I, [P]),
    "sbg_queue_matrix_elements": (LL, [P]),
    "sbg_queue_vector_elements": (LL, [P]),
    "sbg_queue_buckets": (I, [P]),
    "sbg_queue_bucket": (I, [P, I, P, P, P, P, P]),
    "sbg_queue_graph_builds": (I, [P]),
    "sbg_spinwave_create": (I, [I, I, P, P, P, P, D, I, P]),
    "sbg_spinwave_destroy": (I, [P]),
    "sbg_spinwave_matrix_size": (I, [P]),
    "sbg_spinwave_assemble": (I, [P, P, I, P, P, P]),
    "sbg_spinwave_intensities": (I, [P, P, I, P, P, P, P, P]),
    "sbg_spinwave_solve": (I, [P, P, P, I, P, P, P, P, P]),
    "sbg_spinwave_solve_host": (I, [P, P, P, I, P, P, P, P, I, I]),
}


class SolverOptions(ctypes.Structure):
    _fields_ = [
        ("batches_per_block", I),
        ("force_block_dim_x", I),
        ("tuning_mode", I),
        ("cache_mode", I),
        ("precision", I),
        ("refine_steps", I),
        ("workspace_pairs", I),
    ]


_lib = None


def load():
    """Loads the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it first (python sunny-batched-geneig_b200/build.py)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
