"""B200 batched complex Hermitian-definite generalized eigensolver, A x = lambda B x.

Python host side over the C ABI (include/sbg/geneig.h).  Device buffers are
torch CUDA tensors, laid out as the reference's launchers expect
(src/geneig_fixed.cu:474-492, src/nvrtc/nvrtc_solver.hpp:112-120):
pairs contiguous, each n x n matrix column-major with leading dimension n.  The
Python functions take and return flat per-pair tensors of shape (batch, n*n)
(complex128) in that column-major order; ``to_colmajor`` / ``from_colmajor``
convert from / to (batch, n, n) row-indexed tensors.

    solver = sbg.Solver(54, precision="fp64")          # NvrtcGeneigSolver(54, 0)
    solver.launch(dA, dB, dW, dX, dinfo)               # ::launch(...)
    W, X, info = sbg.solve(A, B)                        # host or device inputs
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import SolverOptions, load

__all__ = [
    "Solver", "SolverError", "Queue", "SpinWave", "pack_pairs", "unpack", "solve", "to_colmajor", "from_colmajor", "max_n",
    "geneig_full_n54_batched", "chol_n54", "reduce_n54", "reduce_eig_n54", "full_n54", "finish_n54",
    "PRECISIONS", "fixed_n54_introspection", "tuning_table_path", "tuning_forget_in_process",
]

PRECISIONS = {"fp64": 0, "mixed": 1}
_TUNING = {"suggested": 0, "autotune": 1}
_CACHE = {"auto": 0, "no_disk": 1, "none": 2}


class SolverError(RuntimeError):
    def __init__(self, status: int, where: str):
        lib = load()
        msg = lib.sbg_last_error().decode() or lib.sbg_status_string(status).decode()
        super().__init__(f"{where}: {lib.sbg_status_string(status).decode()} ({msg})")
        self.status = status


def _check(status: int, where: str) -> None:
    if status != 0:
        raise SolverError(status, where)


def _ptr(t):
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def to_colmajor(M: torch.Tensor) -> torch.Tensor:
    """(batch, n, n) with [b, i, j] = M(i, j)  ->  (batch, n*n) column-major."""
    b, n, _ = M.shape
    return M.transpose(-1, -2).contiguous().reshape(b, n * n)


def from_colmajor(M: torch.Tensor, n: int) -> torch.Tensor:
    return M.reshape(-1, n, n).transpose(-1, -2)


def max_n(precision: str = "fp64") -> int:
    return int(load().sbg_max_n(PRECISIONS[precision]))


def _check_pair_buffers(n, A, B, W, X, info):
    for name, t, dt in (("A", A, torch.complex128), ("B", B, torch.complex128), ("W", W, torch.float64),
                        ("X", X, torch.complex128), ("info", info, torch.int32)):
        if not t.is_cuda:
            raise ValueError(f"{name} must be a CUDA tensor")
        if t.dtype != dt:
            raise ValueError(f"{name} must be {dt}, got {t.dtype}")
        if not t.is_contiguous():
            raise ValueError(f"{name} must be contiguous")
    batch = info.numel()
    for name, t, per in (("A", A, n * n), ("B", B, n * n), ("W", W, n), ("X", X, n * n)):
        if t.numel() != batch * per:
            raise ValueError(f"{name} has {t.numel()} elements, expected {batch * per} for batch {batch}")
    return batch


class Solver:
    """Runtime-n solver handle (mirrors NvrtcGeneigSolver, src/nvrtc/nvrtc_solver.hpp:81-217).

    batches_per_block: pairs per CTA of the QL stage (0 = auto).
    block_dim: threads per CTA of the CTA-per-pair stages, 128 or 256 (0 = auto).
    tuning: "suggested" (built-in schedule) or "autotune" (measured, persisted).
    cache: "auto" | "no_disk" | "none" (the autotune table's layers).
    precision: "fp64" (the plain drop-in) or "mixed" (complex64 tridiagonalisation and FP64
    eigensolve of that T, then FP64 Ogita-Aishima refinement against C on the FP64 tensor cores;
    n <= max_n("mixed") = 235 on B200).
    """

    def __init__(self, n: int, device: int = 0, *, precision: str = "fp64", batches_per_block: int = 0,
                 block_dim: int = 0, tuning: str = "suggested", cache: str = "auto", refine_steps: int = 0,
                 workspace_pairs: int = 0):
        lib = load()
        opts = SolverOptions()
        lib.sbg_solver_options_init(ctypes.byref(opts))
        opts.batches_per_block = batches_per_block
        opts.force_block_dim_x = block_dim
        opts.tuning_mode = _TUNING[tuning]
        opts.cache_mode = _CACHE[cache]
        opts.precision = PRECISIONS[precision]
        opts.refine_steps = refine_steps
        opts.workspace_pairs = workspace_pairs
        handle = ctypes.c_void_p()
        with torch.cuda.device(device):
            _check(lib.sbg_solver_create(n, device, ctypes.byref(opts), ctypes.byref(handle)), "sbg_solver_create")
        self._h = handle
        self._lib = lib
        self.n = n
        self.device = device
        self.precision = precision

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.sbg_solver_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def launch(self, A, B, W, X, info, stream=None) -> None:
        """Full solve of the pairs in A, B (device tensors) into W, X, info."""
        batch = _check_pair_buffers(self.n, A, B, W, X, info)
        _check(self._lib.sbg_solver_launch(self._h, _ptr(A), _ptr(B), _ptr(W), _ptr(X), _ptr(info), batch,
                                           _stream(stream)), "sbg_solver_launch")

    def launch_chunked(self, A, B, W, X, info, chunk_size: int, streams) -> None:
        """Round-robin chunks over several streams (NvrtcGeneigSolver::launch_chunked)."""
        batch = _check_pair_buffers(self.n, A, B, W, X, info)
        arr = (ctypes.c_void_p * len(streams))(*[s.cuda_stream for s in streams])
        _check(self._lib.sbg_solver_launch_chunked(self._h, _ptr(A), _ptr(B), _ptr(W), _ptr(X), _ptr(info), batch,
                                                   chunk_size, len(streams), arr), "sbg_solver_launch_chunked")

    def solve_host(self, A, B, W, X, info, chunk_size: int = 16384, num_streams: int = 4) -> None:
        """End-to-end solve of host (ideally pinned) CPU tensors; synchronous.  With B pinned
        (``pin_memory()``) only its lower triangle crosses the host link."""
        for name, t, dt in (("A", A, torch.complex128), ("B", B, torch.complex128), ("W", W, torch.float64),
                            ("X", X, torch.complex128), ("info", info, torch.int32)):
            if t.is_cuda or t.dtype != dt or not t.is_contiguous():
                raise ValueError(f"{name} must be a contiguous host {dt} tensor")
        batch = info.numel()
        _check(self._lib.sbg_solver_solve_host(self._h, _ptr(A), _ptr(B), _ptr(W), _ptr(X), _ptr(info), batch,
                                               chunk_size, num_streams), "sbg_solver_solve_host")

    def host_transfer_bytes(self):
        """(host->device, device->host) bytes of the last ``solve_host``: B's lower triangle only
        when B is pinned, device-mapped host memory (pulled by a kernel), all of B otherwise."""
        h2d, d2h = ctypes.c_longlong(), ctypes.c_longlong()
        _check(self._lib.sbg_solver_host_transfer_bytes(self._h, ctypes.byref(h2d), ctypes.byref(d2h)),
               "sbg_solver_host_transfer_bytes")
        return h2d.value, d2h.value

    def refine_redo_pairs(self, reset: bool = False) -> int:
        """Mixed form: pairs the refinement handed to the FP64 re-solve since creation (or the last
        reset); 0 for the FP64 form.  Waits for the device."""
        c = ctypes.c_longlong()
        _check(self._lib.sbg_solver_refine_redo_pairs(self._h, ctypes.byref(c), 1 if reset else 0),
               "sbg_solver_refine_redo_pairs")
        return c.value

    def enable_stage_timing(self, enable: bool = True) -> None:
        _check(self._lib.sbg_solver_enable_stage_timing(self._h, int(enable)), "sbg_solver_enable_stage_timing")

    STAGES = ("reduce", "tridiag", "eig", "back")

    def read_stage_times(self):
        """{stage: (ms, kernel launches)} since the last read, for the stages
        reduce (potrf + two-sided reduction), tridiag (Householder), eig (QL /
        QL + refinement) and back (Q Z and L^{-H})."""
        ms = (ctypes.c_double * 4)()
        nl = (ctypes.c_int * 4)()
        _check(self._lib.sbg_solver_read_stage_times(self._h, ms, nl), "sbg_solver_read_stage_times")
        return {k: (ms[i], nl[i]) for i, k in enumerate(self.STAGES)}

    def reserve(self, pairs: int, stream_slots: int = 1) -> None:
        _check(self._lib.sbg_solver_reserve(self._h, pairs, stream_slots), "sbg_solver_reserve")

    SCHEDULE_FIELDS = ("hetrd_threads", "pairs_per_cta", "col_exact", "back_lanes", "ql_warps", "chain_threads",
                       "back_qpass", "reduce_tc")

    @property
    def schedule(self) -> dict:
        """The launch schedule (sbg_solver_schedule): CTA shapes of the stage kernels."""
        out = (ctypes.c_int * len(self.SCHEDULE_FIELDS))()
        _check(self._lib.sbg_solver_schedule(self._h, out), "sbg_solver_schedule")
        return dict(zip(self.SCHEDULE_FIELDS, list(out)))

    @schedule.setter
    def schedule(self, sched: dict) -> None:
        cur = self.schedule
        cur.update(sched)
        vals = (ctypes.c_int * len(self.SCHEDULE_FIELDS))(*[int(cur[k]) for k in self.SCHEDULE_FIELDS])
        _check(self._lib.sbg_solver_set_schedule(self._h, vals), "sbg_solver_set_schedule")

    @property
    def batches_per_block(self) -> int:
        return int(self._lib.sbg_solver_batches_per_block(self._h))

    @property
    def block_dim_x(self) -> int:
        return int(self._lib.sbg_solver_block_dim_x(self._h))

    @property
    def shared_mem_bytes(self) -> int:
        return int(self._lib.sbg_solver_shared_mem_bytes(self._h))

    @property
    def was_autotuned(self) -> bool:
        return bool(self._lib.sbg_solver_was_autotuned(self._h))

    @property
    def autotune_sweep_ran(self) -> bool:
        return bool(self._lib.sbg_solver_autotune_sweep_ran(self._h))

    @property
    def cache_layer_used(self) -> str:
        return self._lib.sbg_solver_cache_layer_used(self._h).decode()


class Queue:
    """A planned batch of pairs of uneven order (sbg_queue_create / sbg_launch_queue).

    ns: the order of every pair, in batch order.  Buffers are packed: pair p's A, B and X
    are n[p] x n[p] column-major back to back (``offsets()`` gives where each starts), W
    holds n[p] eigenvalues per pair back to back, info one int per pair.  ``pack_pairs`` /
    ``unpack`` convert from / to lists of flat (n*n,) matrices.  One ``launch`` replays one
    CUDA graph with every n running concurrently.
    """

    def __init__(self, ns, device: int = 0, *, precision: str = "fp64", tuning: str = "suggested",
                 cache: str = "auto", refine_steps: int = 0, chunk_pairs: int = 0):
        lib = load()
        opts = SolverOptions()
        lib.sbg_solver_options_init(ctypes.byref(opts))
        opts.tuning_mode = _TUNING[tuning]
        opts.cache_mode = _CACHE[cache]
        opts.precision = PRECISIONS[precision]
        opts.refine_steps = refine_steps
        opts.workspace_pairs = chunk_pairs
        ns = [int(v) for v in ns]
        arr = (ctypes.c_int * max(1, len(ns)))(*ns)
        handle = ctypes.c_void_p()
        with torch.cuda.device(device):
            _check(lib.sbg_queue_create(arr, len(ns), device, ctypes.byref(opts), ctypes.byref(handle)),
                   "sbg_queue_create")
        self._h = handle
        self._lib = lib
        self.ns = ns
        self.device = device

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.sbg_queue_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        return int(self._lib.sbg_queue_size(self._h))

    @property
    def matrix_elements(self) -> int:
        return int(self._lib.sbg_queue_matrix_elements(self._h))

    @property
    def vector_elements(self) -> int:
        return int(self._lib.sbg_queue_vector_elements(self._h))

    @property
    def graph_builds(self) -> int:
        return int(self._lib.sbg_queue_graph_builds(self._h))

    def buckets(self):
        """[{n, count, chunk, precision, autotuned}] per distinct n, largest n first."""
        out = []
        for i in range(int(self._lib.sbg_queue_buckets(self._h))):
            v = [ctypes.c_int() for _ in range(5)]
            _check(self._lib.sbg_queue_bucket(self._h, i, *[ctypes.byref(x) for x in v]), "sbg_queue_bucket")
            out.append({"n": v[0].value, "count": v[1].value, "chunk": v[2].value,
                        "precision": "mixed" if v[3].value == 1 else "fp64", "autotuned": bool(v[4].value)})
        return out

    def offsets(self):
        """(matrix element offset, vector element offset) of every pair."""
        mo, vo, m, v = [], [], 0, 0
        for n in self.ns:
            mo.append(m); vo.append(v)
            m += n * n; v += n
        return mo, vo

    def launch(self, A, B, W, X, info, stream=None) -> None:
        for name, t, dt, size in (("A", A, torch.complex128, self.matrix_elements),
                                  ("B", B, torch.complex128, self.matrix_elements),
                                  ("W", W, torch.float64, self.vector_elements),
                                  ("X", X, torch.complex128, self.matrix_elements),
                                  ("info", info, torch.int32, len(self))):
            if not t.is_cuda or t.dtype != dt or not t.is_contiguous() or t.numel() != size:
                raise ValueError(f"{name} must be a contiguous CUDA {dt} tensor of {size} elements")
        _check(self._lib.sbg_launch_queue(self._h, _ptr(A), _ptr(B), _ptr(W), _ptr(X), _ptr(info), _stream(stream)),
               "sbg_launch_queue")


class SpinWave:
    """One spin-wave cell held on the GPU (sbg_spinwave_*): assembles A(q), B(q) per q, and
    contracts each eigenvector to an intensity, around the solve.

    sites: (nb, 2) int site pairs (i, j); coef: (nb, 5) float (Re a, Im a, Re b, Im b, c);
    disp: (nb, 3) bond displacements; pos: (N, 3) site positions or None; field: constant
    added to B's diagonal.  Per q: P_ij += a/2 e^{iq.d}, P_ji += conj(a/2 e^{iq.d}),
    Q_ij = Q_ji += b/2 e^{iq.d}, P_ii, P_jj -= c/2; A = diag(I, -I),
    B = [[P, Q], [conj Q, conj P]] + field I.  Intensity of eigenpair m:
    |sum_i e^{-iq.r_i} (x_m[i] + x_m[N+i])|^2 / (N |lambda_m|).
    q: (nq, 3) float64 tensors (device for the device calls, host for ``solve_host``).
    """

    def __init__(self, n_sites: int, sites, coef, disp, pos=None, field: float = 0.0, device: int = 0):
        import numpy as np
        lib = load()
        sites = np.ascontiguousarray(np.asarray(sites, dtype=np.int32).reshape(-1, 2))
        nb = sites.shape[0]
        coef = np.ascontiguousarray(np.asarray(coef, dtype=np.float64).reshape(nb, 5))
        disp = np.ascontiguousarray(np.asarray(disp, dtype=np.float64).reshape(nb, 3))
        posp = None
        if pos is not None:
            pos = np.ascontiguousarray(np.asarray(pos, dtype=np.float64).reshape(n_sites, 3))
            posp = pos.ctypes.data_as(ctypes.c_void_p)
        handle = ctypes.c_void_p()
        with torch.cuda.device(device):
            _check(lib.sbg_spinwave_create(n_sites, nb, sites.ctypes.data_as(ctypes.c_void_p),
                                           coef.ctypes.data_as(ctypes.c_void_p),
                                           disp.ctypes.data_as(ctypes.c_void_p), posp, float(field), device,
                                           ctypes.byref(handle)), "sbg_spinwave_create")
        self._h = handle
        self._lib = lib
        self.n_sites = n_sites
        self.n = 2 * n_sites
        self.device = device

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.sbg_spinwave_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _q(self, q, cuda: bool):
        if q.dtype != torch.float64 or not q.is_contiguous() or q.dim() != 2 or q.shape[1] != 3 \
                or q.is_cuda != cuda:
            raise ValueError(f"q must be a contiguous {'CUDA' if cuda else 'host'} float64 (nq, 3) tensor")
        return q.shape[0]

    @staticmethod
    def _buf(name, t, dt, numel, cuda: bool, optional: bool = False):
        if t is None:
            if optional:
                return
            raise ValueError(f"{name} is required")
        if t.is_cuda != cuda or t.dtype != dt or not t.is_contiguous() or t.numel() != numel:
            raise ValueError(f"{name} must be a contiguous {'CUDA' if cuda else 'host'} {dt} tensor "
                             f"of {numel} elements")

    def assemble(self, q, A=None, B=None, stream=None):
        """A(q), B(q) of every q into (nq, n*n) column-major device tensors (allocated when None;
        A is skipped when A is False).  Returns (A, B)."""
        nq = self._q(q, True)
        nn = self.n * self.n
        if B is None:
            B = torch.empty((nq, nn), dtype=torch.complex128, device=q.device)
        if A is None:
            A = torch.empty((nq, nn), dtype=torch.complex128, device=q.device)
        self._buf("B", B, torch.complex128, nq * nn, True)
        if A is not False:
            self._buf("A", A, torch.complex128, nq * nn, True)
        _check(self._lib.sbg_spinwave_assemble(self._h, _ptr(q), nq, None if A is False else _ptr(A), _ptr(B),
                                               _stream(stream)), "sbg_spinwave_assemble")
        return (None if A is False else A), B

    def intensities(self, q, W, X, info, I=None, stream=None):
        nq = self._q(q, True)
        if I is None:
            I = torch.empty((nq, self.n), dtype=torch.float64, device=q.device)
        self._buf("W", W, torch.float64, nq * self.n, True)
        self._buf("X", X, torch.complex128, nq * self.n * self.n, True)
        self._buf("info", info, torch.int32, nq, True)
        self._buf("I", I, torch.float64, nq * self.n, True)
        _check(self._lib.sbg_spinwave_intensities(self._h, _ptr(q), nq, _ptr(W), _ptr(X), _ptr(info), _ptr(I),
                                                  _stream(stream)), "sbg_spinwave_intensities")
        return I

    def solve(self, solver: Solver, q, W, info, X=None, I=None, stream=None) -> None:
        """Assemble + solve (+ intensities when I is given) for every q, on the device."""
        nq = self._q(q, True)
        self._buf("W", W, torch.float64, nq * self.n, True)
        self._buf("info", info, torch.int32, nq, True)
        self._buf("X", X, torch.complex128, nq * self.n * self.n, True, optional=True)
        self._buf("I", I, torch.float64, nq * self.n, True, optional=True)
        _check(self._lib.sbg_spinwave_solve(self._h, solver._h, _ptr(q), nq, _ptr(W), _ptr(X), _ptr(I), _ptr(info),
                                            _stream(stream)), "sbg_spinwave_solve")

    def solve_host(self, solver: Solver, q, W, info, X=None, I=None, chunk_size: int = 0,
                   num_streams: int = 2) -> None:
        """The same from (ideally pinned) host q into host W, info, X, I; synchronous."""
        nq = self._q(q, False)
        self._buf("W", W, torch.float64, nq * self.n, False)
        self._buf("info", info, torch.int32, nq, False)
        self._buf("X", X, torch.complex128, nq * self.n * self.n, False, optional=True)
        self._buf("I", I, torch.float64, nq * self.n, False, optional=True)
        _check(self._lib.sbg_spinwave_solve_host(self._h, solver._h, _ptr(q), nq, _ptr(W), _ptr(X), _ptr(I),
                                                 _ptr(info), chunk_size, num_streams), "sbg_spinwave_solve_host")


def pack_pairs(mats):
    """List of flat (n*n,) column-major matrices -> one packed 1-D tensor."""
    return torch.cat([m.reshape(-1) for m in mats])


def unpack(packed, ns, square: bool = True):
    """Packed 1-D tensor -> list of per-pair flat tensors (n*n each, or n each if not square)."""
    out, o = [], 0
    for n in ns:
        k = n * n if square else n
        out.append(packed[o:o + k])
        o += k
    return out


def solve(A, B, *, precision: str = "fp64", device: int = 0, solver: Solver | None = None, stream=None):
    """Solves every pair of A, B ((batch, n*n) column-major complex128, host or device).

    Host inputs are copied to the device and the results copied back (the
    end-to-end path); device inputs stay on the device.  Returns (W, X, info).
    """
    host = not (isinstance(A, torch.Tensor) and A.is_cuda)
    A = torch.as_tensor(A)
    B = torch.as_tensor(B)
    batch, nn = A.shape
    n = int(round(nn ** 0.5))
    if n * n != nn or B.shape != A.shape:
        raise ValueError("A and B must both be (batch, n*n)")
    dev = torch.device("cuda", device)
    if solver is None:
        solver = Solver(n, device, precision=precision)
    dA = A.to(dev, non_blocking=True)
    dB = B.to(dev, non_blocking=True)
    dW = torch.empty((batch, n), dtype=torch.float64, device=dev)
    dX = torch.empty((batch, nn), dtype=torch.complex128, device=dev)
    dinfo = torch.empty(batch, dtype=torch.int32, device=dev)
    solver.launch(dA, dB, dW, dX, dinfo, stream=stream)
    if host:
        return dW.cpu(), dX.cpu(), dinfo.cpu()
    return dW, dX, dinfo


# ------------------------------------------------------------------ fixed n = 54 drop-in

def geneig_full_n54_batched(A, B, W, X, info, stream=None) -> None:
    """geneig_full_n54_batched_launch (src/geneig_fixed.cu:474-492)."""
    batch = _check_pair_buffers(54, A, B, W, X, info)
    load().geneig_full_n54_batched_launch(_ptr(A), _ptr(B), _ptr(W), _ptr(X), _ptr(info), batch, _stream(stream))


def chol_n54(S, L, info, stream=None) -> None:
    load().chol_n54_launch(_ptr(S), _ptr(L), _ptr(info), _stream(stream))


def reduce_n54(H, S, M, info, stream=None) -> None:
    load().geneig_reduce_n54_launch(_ptr(H), _ptr(S), _ptr(M), _ptr(info), _stream(stream))


def reduce_eig_n54(H, S, W, V, info, stream=None) -> None:
    load().geneig_reduce_eig_n54_launch(_ptr(H), _ptr(S), _ptr(W), _ptr(V), _ptr(info), _stream(stream))


def full_n54(H, S, W, U, info, stream=None) -> None:
    load().geneig_full_n54_launch(_ptr(H), _ptr(S), _ptr(W), _ptr(U), _ptr(info), _stream(stream))


def finish_n54(L, M, W, U, info, batch: int, stream=None) -> None:
    load().geneig_finish_n54_launch(_ptr(L), _ptr(M), _ptr(W), _ptr(U), _ptr(info), batch, _stream(stream))


def fixed_n54_introspection() -> dict:
    lib = load()
    names = [k for k in _lib.SIGNATURES if k.endswith(("_block_dim_x", "_shared_mem_bytes", "_smem_bytes", "_workspace"))
             and "n54" in k]
    return {k: int(getattr(lib, k)()) for k in names}


def tuning_table_path(device: int = 0) -> str:
    buf = ctypes.create_string_buffer(4096)
    _check(load().sbg_tuning_table_path(device, buf, len(buf)), "sbg_tuning_table_path")
    return buf.value.decode()


def tuning_forget_in_process() -> None:
    _check(load().sbg_tuning_forget_in_process(), "sbg_tuning_forget_in_process")
