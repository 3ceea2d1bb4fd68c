/*
 * sbg/geneig.h — C ABI of the B200 batched Hermitian-definite generalized eigensolver
 *
 *     A x = lambda B x,   A Hermitian (may be indefinite), B Hermitian positive definite,
 *
 * for batches of complex128 n x n pairs, the spin-wave pairs Sunny.jl produces per q-point.
 * Drop-in for the launchers of riteshbhirud/sunny-batched-geneig:
 *   - the fixed n = 54 C ABI of src/geneig_fixed.cu (same names, signatures, layout), and
 *   - the runtime-n NvrtcGeneigSolver of src/nvrtc/nvrtc_solver.hpp:99-145, exposed as an
 *     opaque handle with the same construction options, launch / launch_chunked and getters.
 *
 * Conventions (identical to the reference):
 *   - matrices are column-major, leading dimension n, pairs contiguous (stride n*n elements);
 *   - A is read in full; only the lower triangle of B is read;
 *   - W[b*n + i] ascending; column i of X is the eigenvector of W[b*n+i], X^H B X = I,
 *     arbitrary phase per column;
 *   - every call is asynchronous on the given stream; the caller owns all device buffers.
 * Per-pair info (always written; the caller need not zero it):
 *   0            success
 *   1 .. n       the tridiagonal QL failed to converge (that many off-diagonals left),
 *                the zheev/zhegv convention
 *   n + i        the leading minor of order i of B is not positive definite (also NaN/Inf
 *                on B's diagonal path), the zhegv convention; W and X of that pair are NaN.
 *   The staged Cholesky / reduction launchers report the zpotrf convention (i, not n + i).
 *   The first failing stage wins (the reference's heev could overwrite a potrf failure).
 */
#ifndef SBG_GENEIG_H
#define SBG_GENEIG_H

#include <stddef.h>
#include <cuComplex.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef enum {
    SBG_OK = 0,
    SBG_ERR_INVALID_VALUE = 1,   /* bad n, batch, pointer or option */
    SBG_ERR_CUDA = 2,            /* a CUDA runtime call failed (see sbg_last_error) */
    SBG_ERR_NO_MEMORY = 3,       /* device workspace allocation failed */
    SBG_ERR_UNSUPPORTED = 4,     /* n outside the supported range for this form */
    SBG_ERR_CAPTURING = 5,       /* workspace growth needed while the stream is being captured */
    SBG_ERR_INTERNAL = 6         /* a C++ exception escaped (message in sbg_last_error) */
} sbg_status;

const char* sbg_status_string(int status);
/* Message of the last failed call on this host thread ("" if none). */
const char* sbg_last_error(void);

/* ------------------------------------------------------------------ fixed n = 54 drop-in */
/* Replaces src/geneig_fixed.cu:474-492: full solve of batch_size pairs. */
void geneig_full_n54_batched_launch(const cuDoubleComplex* d_H, const cuDoubleComplex* d_S,
                                    double* d_W, cuDoubleComplex* d_U, int* d_info,
                                    int batch_size, cudaStream_t stream);
/* Replace src/geneig_fixed.cu:494-497 (block size and dynamic shared memory of the
 * largest stage kernel of the batched solve). */
unsigned int geneig_full_n54_batched_block_dim_x(void);
unsigned int geneig_full_n54_batched_shared_mem_bytes(void);

/* Staged twins (debug / validation entry points, src/geneig_fixed.cu:106-152, 166-227,
 * 247-325, 339-405, 516-592).  The single-matrix ones process exactly one pair. */
/* geneig_fixed.cu:134-152: L = chol(S), lower, strict upper zeroed; info = zpotrf's. */
void chol_n54_launch(const cuDoubleComplex* d_S, cuDoubleComplex* d_L, int* d_info,
                     cudaStream_t stream);
unsigned int chol_n54_block_dim_x(void);
unsigned int chol_n54_shared_mem_bytes(void);
/* geneig_fixed.cu:208-227: M = L^{-1} H L^{-H}, lower, strict upper zeroed. */
void geneig_reduce_n54_launch(const cuDoubleComplex* d_H, const cuDoubleComplex* d_S,
                              cuDoubleComplex* d_M, int* d_info, cudaStream_t stream);
unsigned int geneig_reduce_n54_block_dim_x(void);
unsigned int geneig_reduce_n54_shared_mem_bytes(void);
/* geneig_fixed.cu:302-325: W, V = eig(M) (V: eigenvectors of the reduced matrix). */
void geneig_reduce_eig_n54_launch(const cuDoubleComplex* d_H, const cuDoubleComplex* d_S,
                                  double* d_W, cuDoubleComplex* d_V, int* d_info,
                                  cudaStream_t stream);
unsigned int geneig_reduce_eig_n54_block_dim_x(void);
unsigned int geneig_reduce_eig_n54_shared_mem_bytes(void);
/* Introspection twins of geneig_fixed.cu:320-324: shared memory of the Cholesky/reduction
 * stage, of the eigensolve stage, and the per-pair device workspace (complex128 elements). */
unsigned int geneig_reduce_eig_n54_chol_smem_bytes(void);
unsigned int geneig_reduce_eig_n54_heev_smem_bytes(void);
unsigned int geneig_reduce_eig_n54_heev_workspace(void);
/* geneig_fixed.cu:385-405: full solve of one pair. */
void geneig_full_n54_launch(const cuDoubleComplex* d_H, const cuDoubleComplex* d_S,
                            double* d_W, cuDoubleComplex* d_U, int* d_info, cudaStream_t stream);
unsigned int geneig_full_n54_block_dim_x(void);
unsigned int geneig_full_n54_shared_mem_bytes(void);
/* geneig_fixed.cu:569-592: from (L, M) (lower triangles read) -> W, U = L^{-H} eigvecs(M). */
void geneig_finish_n54_launch(const cuDoubleComplex* d_L, const cuDoubleComplex* d_M,
                              double* d_W, cuDoubleComplex* d_U, int* d_info, int batch_size,
                              cudaStream_t stream);
unsigned int geneig_finish_n54_block_dim_x(void);
unsigned int geneig_finish_n54_shared_mem_bytes(void);

/* ------------------------------------------------------------------ runtime-n solver */
/* Mirrors NvrtcGeneigSolver (src/nvrtc/nvrtc_solver.hpp:81-217).  The reference JIT-compiles
 * a kernel per (n, pairs per CTA, block size); here every kernel is compiled ahead of time
 * for sm_100a and construction only selects a schedule (and, with SBG_TUNING_AUTOTUNE,
 * measures the candidates and persists the winner). */
typedef struct sbg_solver sbg_solver;

enum { SBG_TUNING_SUGGESTED = 0, SBG_TUNING_AUTOTUNE = 1 };            /* TuningMode, hpp:38 */
enum { SBG_CACHE_AUTO = 0, SBG_CACHE_NO_DISK = 1, SBG_CACHE_NONE = 2 }; /* CacheMode, hpp:46 */
enum { SBG_PRECISION_FP64 = 0, SBG_PRECISION_MIXED = 1 };

typedef struct {
    int batches_per_block;    /* pairs per CTA; 0 = auto (ctor arg, hpp:99): of the warp-per-pair Cholesky and
                                 Householder kernels for n <= 65 (1, 2 or 4), of the QL rotation stage above */
    int force_block_dim_x;    /* threads per CTA of the CTA-per-pair Householder (66 <= n <= 84): 128 or 256;
                                 0 = auto (hpp:100) */
    int tuning_mode;          /* SBG_TUNING_*  (hpp:101) */
    int cache_mode;           /* SBG_CACHE_*   (hpp:102) */
    int precision;            /* SBG_PRECISION_FP64 (plain drop-in) or SBG_PRECISION_MIXED */
    int refine_steps;         /* mixed form: most Ogita-Aishima updates, 0 = default (5).  Each pass checks every
                                 residual (<= 256 eps ||C||_F) and the orthonormality (<= 1e-13) first and stops
                                 there; from complex64 two updates are typical.  A pair still short after the
                                 last update is solved again by the FP64 fallback */
    int workspace_pairs;      /* pairs per internal chunk; 0 = default */
} sbg_solver_options;

void sbg_solver_options_init(sbg_solver_options* opts);
/* NvrtcGeneigSolver ctor (nvrtc_solver.cpp:927-1047). opts may be NULL. */
int sbg_solver_create(int n, int device_id, const sbg_solver_options* opts, sbg_solver** out);
int sbg_solver_destroy(sbg_solver* s);
/* NvrtcGeneigSolver::launch (nvrtc_solver.cpp:1063-1076).  Any batch >= 0; no multiple-of-
 * pairs-per-CTA restriction (the reference's partial last block was unchecked).  The solver's
 * device scratch is kept per stream (one workspace slot for each distinct stream it is launched
 * on, the first stream taking slot 0), so launches on different streams may overlap, as the
 * reference's may; launches on the same stream are ordered by it. */
int sbg_solver_launch(sbg_solver* s, const cuDoubleComplex* d_A, const cuDoubleComplex* d_B,
                      double* d_W, cuDoubleComplex* d_X, int* d_info, int batch,
                      cudaStream_t stream);
/* NvrtcGeneigSolver::launch_chunked (nvrtc_solver.cpp:1078-1107): round-robin chunks of
 * chunk_size pairs over num_streams streams, no synchronisation between chunks. */
int sbg_solver_launch_chunked(sbg_solver* s, const cuDoubleComplex* d_A,
                              const cuDoubleComplex* d_B, double* d_W, cuDoubleComplex* d_X,
                              int* d_info, int total, int chunk_size, int num_streams,
                              const cudaStream_t* streams);
/* Pre-sizes the internal workspace (pairs per chunk, number of stream slots: the first
 * stream_slots distinct streams the solver is launched on) so later launches never allocate
 * (required before capturing a launch into a CUDA graph). */
int sbg_solver_reserve(sbg_solver* s, int pairs, int stream_slots);
/* End-to-end solve of HOST-resident pairs: chunks of chunk_size pairs are copied to the
 * device, solved and copied back, round-robin over num_streams internal streams so the
 * copies of one chunk overlap the kernels of another (the chunked multi-stream idea of
 * launch_chunked, nvrtc_solver.cpp:1078-1107, applied to host<->device traffic).
 * Synchronous: returns once W, X and info are on the host.  Host buffers should be
 * page-locked (cudaHostAlloc) for the copies to overlap.  Device staging buffers are
 * owned by the solver and grow on demand.  Only B's lower triangle crosses the host link
 * when h_B lies in one pinned, device-mapped allocation (cudaHostAlloc memory on 64-bit
 * systems): a kernel reads it in place; otherwise all of B is copied.  Calls on one solver are
 * serialised (they share its staging buffers); use one solver per host thread for overlap. */
int sbg_solver_solve_host(sbg_solver* s, const cuDoubleComplex* h_A, const cuDoubleComplex* h_B,
                          double* h_W, cuDoubleComplex* h_X, int* h_info, int batch,
                          int chunk_size, int num_streams);
/* Bytes the solver's last sbg_solver_solve_host moved host -> device and device -> host. */
int sbg_solver_host_transfer_bytes(const sbg_solver* s, long long* h2d_bytes, long long* d2h_bytes);

/* Mixed form: the number of pairs its refinement handed to the FP64 re-solve (did not reach the
 * gates within refine_steps updates, or the eigensolve of the complex64 T failed) over all launches
 * since the solver was created or the count last reset (reset != 0 clears it after reading).
 * Synchronous (waits for the device); 0 for an FP64 solver.  No counterpart in the reference. */
int sbg_solver_refine_redo_pairs(sbg_solver* s, long long* count, int reset);

/* Per-stage timing: when enabled, every launch records CUDA events around each stage
 * kernel on the launch stream.  sbg_solver_read_stage_times synchronizes on them and
 * returns, per stage (0 = Cholesky + two-sided reduction, 1 = Householder
 * tridiagonalisation, 2 = tridiagonal eigensolve (QL, or QL + refinement for the mixed
 * form), 3 = back-transform), the summed milliseconds and the number of kernel launches,
 * then clears the record. */
int sbg_solver_enable_stage_timing(sbg_solver* s, int enable);
int sbg_solver_read_stage_times(sbg_solver* s, double* ms_out4, int* launches_out4);

/* Device bytes of workspace per pair for a given n and precision. */
size_t sbg_workspace_bytes_per_pair(int n, int precision);
/* Exact device bytes of the workspace a solver allocates for `pairs` pairs of order n: the
 * per-pair bytes times pairs plus the 256-byte alignment of its seven regions (at most
 * 7 * 256 bytes more). */
size_t sbg_workspace_bytes(int n, int precision, int pairs);

/* The solver's schedule as eight ints (no counterpart in the reference, whose schedule is its
 * (batches per block, block size) pair): [0] threads per CTA of the CTA-per-pair Householder,
 * [1] pairs per CTA of the warp-per-pair Cholesky / Householder kernels, [2] 1 = the exact-n
 * column kernels where they exist (n = 32, 54), [3] lanes per column of the column back-transform
 * (1 or 2), [4] pairs per CTA of the QL rotation stage, [5] pairs per CTA of the QL scalar
 * chain, [6] reflectors per pass of the column back-transform's Q application (1 or 2), [7] 1 = the
 * triangular stages above n = 56 (Cholesky, reduction, X = L^{-H} Y) by the blocked kernels on the
 * FP64 tensor cores, and above n = 84 the Householder by its own one-pass kernel, 0 = by the
 * one-CTA / cluster kernels that also do the Householder (0 or 1).
 * set_schedule replaces it (values checked against their ranges and the device's shared memory;
 * SBG_ERR_INVALID_VALUE otherwise), for callers that tune outside the library. */
int sbg_solver_schedule(const sbg_solver* s, int* out8);
int sbg_solver_set_schedule(sbg_solver* s, const int* in8);

/* Getters (nvrtc_solver.hpp:128-145). */
int sbg_solver_matrix_size(const sbg_solver* s);
int sbg_solver_batches_per_block(const sbg_solver* s);
int sbg_solver_block_dim_x(const sbg_solver* s);
/* The largest dynamic shared memory per CTA among the stage kernels this solver launches (the
 * reference's was its one fused kernel's). */
unsigned int sbg_solver_shared_mem_bytes(const sbg_solver* s);
int sbg_solver_was_autotuned(const sbg_solver* s);
int sbg_solver_autotune_sweep_ran(const sbg_solver* s);
/* "in-process", "disk" or "compile" (here: "measured") — which layer supplied the schedule. */
const char* sbg_solver_cache_layer_used(const sbg_solver* s);
int sbg_solver_precision(const sbg_solver* s);

/* Largest n each form supports on this device (shared-memory bound).  FP64: 256 (n <= 84
 * one CTA or warp per pair; 84 < n <= 256 one CTA per pair with the pair's matrices in device
 * memory, or thread-block clusters in the scalar schedule); mixed: 235 (the
 * complex64 Householder takes one CTA per pair: n <= 63 one warp per pair and the refinement on
 * shared-memory tiles, 63 < n <= 235 one CTA per pair and the refinement on the pair's matrices in
 * the workspace, which then holds five more n x n complex matrices per pair). */
int sbg_max_n(int precision);

/* ------------------------------------------------------------------ uneven-n queue */
/* No counterpart in the reference, whose runtime-n solver (nvrtc_solver.hpp:99-145) serves one n
 * per instance; this replaces "one NvrtcGeneigSolver + one launch per n" for a mixed batch.
 * A queue is planned once for the orders n[0..count) of a batch and launched any number of times:
 *   - Packed layout: pair p's A, B and X are n[p] x n[p] column-major starting at element
 *     sum_{q<p} n[q]^2 of d_A / d_B / d_X; its eigenvalues at element sum_{q<p} n[q] of d_W; its
 *     info at d_info[p].  A and B are read as in sbg_solver_launch (A full, B lower).
 *   - Every n gets its own solver with the per-n schedule (opts->tuning_mode as in
 *     sbg_solver_create: the table, or the autotuner); opts->precision = MIXED applies to the
 *     n that the mixed form supports (sbg_max_n) and the others run FP64 (sbg_queue_bucket reports
 *     which); each bucket's chunk (staging + solver scratch) is sized from half the free device
 *     memory at creation, split over the buckets, 1 to 8 GiB each; opts->workspace_pairs > 0
 *     sets the pairs per chunk instead (for callers that must bound the queue's memory).
 *   - sbg_launch_queue is asynchronous on `stream`: it replays one CUDA graph in which all n run
 *     concurrently (captured on the first launch, and again when the buffers change).
 * All calls return an sbg_status. */
typedef struct sbg_queue sbg_queue;
int sbg_queue_create(const int* n, int count, int device_id, const sbg_solver_options* opts, sbg_queue** out);
int sbg_queue_destroy(sbg_queue* q);
int sbg_launch_queue(sbg_queue* q, const cuDoubleComplex* d_A, const cuDoubleComplex* d_B, double* d_W,
                     cuDoubleComplex* d_X, int* d_info, cudaStream_t stream);
int sbg_queue_size(const sbg_queue* q);
/* Complex elements of the packed A (= B, X) and doubles of the packed W. */
long long sbg_queue_matrix_elements(const sbg_queue* q);
long long sbg_queue_vector_elements(const sbg_queue* q);
/* Distinct n (buckets, largest n first) and, per bucket, its n, pair count, pairs per chunk,
 * precision and whether its schedule came from the autotuner. */
int sbg_queue_buckets(const sbg_queue* q);
int sbg_queue_bucket(const sbg_queue* q, int i, int* n, int* count, int* chunk, int* precision, int* was_autotuned);
/* How many times the launch graph was captured (1 while the buffers stay the same). */
int sbg_queue_graph_builds(const sbg_queue* q);

/* ------------------------------------------------------------------ spin-wave q-sweeps */
/* No counterpart in the reference: the steps either side of the solve when the pairs come from a
 * linear spin-wave model swept over q.  The reference's intended caller assembles A(q), B(q) on
 * the host and moves 2 x 16 n^2 bytes per q to the GPU and 16 n^2 bytes of eigenvectors back; a
 * model held on the GPU takes q (24 bytes) in and gives W and n intensities per q out.
 *   - Cell: n_sites = N sites, order n = 2N.  Bond k joins sites (i, j) = (sites[2k], sites[2k+1])
 *     with displacement d = disp[3k..3k+2] and coefficients a = coef[5k] + i coef[5k+1],
 *     b = coef[5k+2] + i coef[5k+3], c = coef[5k+4].  pos[3i..3i+2] is site i's position
 *     (NULL: all zero); field is a constant added to the diagonal of B.
 *   - Per q (q = d_q[3p..3p+2]): P_ij += a/2 e^{i q.d}, P_ji += conj(a/2 e^{i q.d}),
 *     Q_ij += b/2 e^{i q.d}, Q_ji += b/2 e^{i q.d}, P_ii -= c/2, P_jj -= c/2, summed in bond
 *     order; A = diag(I_N, -I_N) and B = [[P, Q], [conj Q, conj P]] + field I (column-major, as
 *     sbg_solver_launch reads them).
 *   - Intensity of eigenpair m of pair p: I_m = |sum_{i<N} e^{-i q.r_i} (x_m[i] + x_m[N+i])|^2
 *     / (N |lambda_m|), in W's order (d_I[n p + m]); NaN for a pair whose info != 0.
 *   - sbg_spinwave_solve runs assembly, the solve and the contraction on `stream`, chunk by
 *     chunk (the solver's chunk size), with the solver `s` (order 2N, same device).  d_X and d_I
 *     may each be NULL (eigenvectors / intensities not wanted); W and info are always written.
 *     Per stream it keeps one chunk of A, B and (when d_X is NULL) X scratch, grown on first
 *     use: run one sweep of the largest size on a stream before capturing it into a graph.
 *   - sbg_spinwave_solve_host takes page-locked host q, W, X (or NULL), I (or NULL) and info,
 *     overlaps the copies with the kernels over num_streams internal streams (chunk_size 0:
 *     the solver's chunk) and returns when the results are on the host; calls on one model are
 *     serialised (they share its staging buffers).
 * All calls return an sbg_status. */
typedef struct sbg_spinwave sbg_spinwave;
int sbg_spinwave_create(int n_sites, int n_bonds, const int* sites, const double* coef, const double* disp,
                        const double* pos, double field, int device_id, sbg_spinwave** out);
int sbg_spinwave_destroy(sbg_spinwave* m);
int sbg_spinwave_matrix_size(const sbg_spinwave* m);
/* A may be NULL (B only). */
int sbg_spinwave_assemble(sbg_spinwave* m, const double* d_q, int nq, cuDoubleComplex* d_A, cuDoubleComplex* d_B,
                          cudaStream_t stream);
int sbg_spinwave_intensities(sbg_spinwave* m, const double* d_q, int nq, const double* d_W,
                             const cuDoubleComplex* d_X, const int* d_info, double* d_I, cudaStream_t stream);
int sbg_spinwave_solve(sbg_spinwave* m, sbg_solver* s, const double* d_q, int nq, double* d_W,
                       cuDoubleComplex* d_X, double* d_I, int* d_info, cudaStream_t stream);
int sbg_spinwave_solve_host(sbg_spinwave* m, sbg_solver* s, const double* h_q, int nq, double* h_W,
                            cuDoubleComplex* h_X, double* h_I, int* h_info, int chunk_size, int num_streams);

/* ------------------------------------------------------------------ allocation-free solve */
/* This entry point has no counterpart in the reference.
 *
 * For callers that cannot let a library allocate device memory: frameworks that own every byte
 * of device memory through their own pool allocator, applications running under a fixed memory
 * budget they pre-allocated, and latency-sensitive loops that cannot absorb the device-wide
 * synchronisation of cudaMalloc/cudaFree.  It runs the same plain FP64 solve as
 * sbg_solver_launch, but its scratch is one fixed array compiled into the library,
 * SBG_NOALLOC_SCRATCH_BYTES long, which every GPU that loads the library keeps until process
 * exit.  The caller still provides A, B, W, X and info.
 *   - It allocates nothing (no cudaMalloc, cudaFree or allocating library call).
 *   - Limit: sbg_workspace_bytes(n, SBG_PRECISION_FP64, batch) must fit in
 *     SBG_NOALLOC_SCRATCH_BYTES (at n = 54 that is 533 pairs); larger batches are rejected with
 *     SBG_ERR_INVALID_VALUE and a message in sbg_last_error() — split them into slices.
 *   - The first call on a device looks up the array's device address (cudaGetSymbolAddress)
 *     and caches it; make that first call before any stream capture.  The cached address
 *     belongs to the device's current context: cudaDeviceReset on that device after the first
 *     call is not supported (the array would move and the cached address dangle).
 *   - All calls share the one array and it keeps the last call's contents (nothing in it needs
 *     to start at zero).  Calls that overlap on the GPU race on it: order them on one stream.
 * Returns an sbg_status. */
#define SBG_NOALLOC_SCRATCH_BYTES (64u << 20)
int sbg_geneig_full_noalloc_launch(int n, const cuDoubleComplex* d_A, const cuDoubleComplex* d_B,
                                   double* d_W, cuDoubleComplex* d_X, int* d_info, int batch,
                                   cudaStream_t stream);

/* Autotune table (the analogue of the reference's on-disk cubin cache,
 * nvrtc_solver.cpp:403-431): path of this device's table file, written into buf.
 * Directory: $SUNNY_GENEIG_CACHE_DIR, else $XDG_CACHE_HOME/sunny_geneig_b200, else
 * $HOME/.cache/sunny_geneig_b200. */
int sbg_tuning_table_path(int device_id, char* buf, size_t buflen);
/* Forgets the in-process autotune memo (the next autotuned construction reads the file). */
int sbg_tuning_forget_in_process(void);

/* ------------------------------------------------------------------ device self-test */
/* No counterpart in the reference.  Writes d_r[i] = the reciprocal of d_u[i] as the inverse
 * iteration computes it (Newton-Raphson from the hardware estimate, not a correctly rounded
 * division), i < count, on `stream`, so a test can compare it with 1.0 / u.  Returns an
 * sbg_status. */
int sbg_selftest_reciprocal(const double* d_u, double* d_r, int count, cudaStream_t stream);
/* No counterpart in the reference.  FP64 FMA throughput probe for the roofline's denominator:
 * `blocks` CTAs of 256 threads; every thread runs 8 independent dependent FMA chains of 4 * iters
 * FMAs each, so one launch executes blocks * 256 * 64 * iters FP64 flops.  d_out receives
 * blocks * 256 doubles (the chains' sums).  Time it with CUDA events on `stream`. */
int sbg_selftest_fp64_fma(double* d_out, int blocks, int iters, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* SBG_GENEIG_H */
