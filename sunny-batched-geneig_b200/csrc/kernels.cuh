// Kernel declarations and the workspace layout shared by the host launchers.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <cstddef>

namespace sbg {

// Per-pair scratch between the three stage kernels (struct of arrays over pairs).
//   LV  n*n complex   column-major, ld = n: the Cholesky factor L in the lower
//                     triangle (diagonal included) and the Householder vectors of
//                     the tridiagonalisation along the rows above the
//                     superdiagonal: LV(k, i) = v_k(i) for i >= k + 2
//   tau n   complex   reflector scalars
//   d,e n   real      tridiagonal diagonal / subdiagonal
// The tridiagonal eigenvectors Z (n*n real) are written into the caller's X buffer,
// which the back-transform kernel then overwrites with X in place.
//   log  cap entries (16 B)  the QL rotation log of the pair (ql_chain)
//   perm n int               sort permutation of the QL eigenvalues
//   flag 1 int               1 if the log overflowed (the apply kernel then runs the
//                            warp-per-pair QL for that pair)
struct Workspace {
    double2* LV = nullptr;
    double2* tau = nullptr;
    double* d = nullptr;
    double* e = nullptr;
    void* log = nullptr;
    int* perm = nullptr;
    int* flag = nullptr;
    int log_cap = 0;    // entries per pair the QL may log
    int log_stride = 0; // entries per pair of the log region (>= log_cap; the mixed form's stash lives there)
    int capacity = 0;   // pairs
    int n = 0;
    // Mixed form for kMixedMaxN < n <= kMixedBigMaxN only (null otherwise): the refinement's
    // per-pair n x n complex matrices (column-major, ld = n) -- the FP64 copy of C, the second
    // eigenvector buffer, P = C Y (then the correction E), G = Y^H Y, S = Y^H P -- and its per-pair
    // outcome rstat (kRefine* below).
    double2* rfC = nullptr;
    double2* rfY = nullptr;
    double2* rfP = nullptr;
    double2* rfG = nullptr;
    double2* rfS = nullptr;
    int* rstat = nullptr;
    // Pair selection: when sel is set, the stage kernels that honour it (the FP64 kernels for
    // 57 <= n <= 256) run pair b only if bit sel[b] of sel_mask is set, and leave every other
    // pair's outputs and scratch untouched.  The mixed form uses it to re-solve in FP64 only the
    // pairs its refinement gave up on.
    const int* sel = nullptr;
    int sel_mask = 0;
    // Mixed form: running count of the pairs its refinement handed to the FP64 re-solve (the
    // solver's; null for workspaces without one).
    unsigned long long* redo_count = nullptr;
};

// Outcome of the mixed form's refinement for kMixedMaxN < n <= kMixedBigMaxN (Workspace::rstat).
enum RefineStatus : int {
    kRefineActive = 0,     // not decided yet (only while the refinement runs)
    kRefineDone = 1,       // converged: W and Y (in X) final, X = L^{-H} Y still to come
    kRefineRedo = 2,       // to be solved again by the FP64 kernels
    kRefineSkip = 3,       // an earlier stage failed (B not positive definite, copy timeout)
};

#ifdef __CUDACC__
__device__ __forceinline__ bool pair_selected(const Workspace& ws, int b) {
    return ws.sel == nullptr || ((ws.sel_mask >> ws.sel[b]) & 1) != 0;
}
#endif

// Rotation-log capacity per pair: ~1.1 n^2 rotations are typical (about two QL sweeps per
// eigenvalue); pairs that need more fall back to the warp-per-pair QL.  The environment
// variable SBG_QL_LOG_CAPACITY lowers it (a testing knob that forces the fallback).
int ql_log_capacity(int n);

// Mixed form: the FP64 refinement's tiles are n padded to a multiple of 8 (the FP64 MMA shape),
// stored planar (re and im planes), column-major with leading dimension refine_ld(n) (which keeps
// the MMA fragment loads free of bank conflicts).  Its copy of C (both planes, full Hermitian,
// zero padding) is the pair's stash: refine_stash_entries(n) 16-byte entries of the log region.
__host__ __device__ constexpr int refine_np(int n) { return (n + 7) / 8 * 8; }
__host__ __device__ constexpr int refine_ld(int n) { return refine_np(n) + 4; }
__host__ __device__ constexpr int refine_stash_entries(int n) { return refine_np(n) * refine_ld(n); }
constexpr int kMixedMaxN = 63;       // inverse iteration (no rotation log, so the stash is free)
// Entries of the rotation-log region the tensor-core kernels of n > 56 use as scratch between the
// eigensolves (csrc/reduce_tc.cu): the inverted 32 x 32 diagonal blocks of L, and above n = 84 the
// Q application's copy of Z (n^2 doubles), block of reflectors (n x 32), T (32 x 32) and V^H Y
// (32 x n).  Never more than the default rotation-log capacity (3 n^2 / 2 + 8 n + 16); the region
// is kept at least this large when a smaller log capacity is asked for.
__host__ __device__ constexpr int tc_scratch_entries(int n) {
    return n <= 56 ? 0
                   : (n <= 84 ? (n + 31) / 32 * 1024
                              : ((n + 31) / 32 * 1024 > (n * n + 1) / 2 + (2 * n + 32) * 32
                                     ? (n + 31) / 32 * 1024
                                     : (n * n + 1) / 2 + (2 * n + 32) * 32));
}
// Mixed form above kMixedMaxN: the refinement runs on per-pair matrices in the workspace
// (csrc/mixed_big.cu); the largest n is where the complex64 Householder's packed tile still fits one
// CTA's shared memory (sbg_max_n reports it: 235 with B200's 227 KB per CTA).
constexpr int kMixedBigMaxN = 256;
inline bool mixed_big(int n, bool mixed) { return mixed && n > kMixedMaxN; }

// Bytes per pair of the workspace of a solver of order n (mixed: the mixed form's).
size_t workspace_bytes_per_pair(int n, bool mixed = false);
// Carves a Workspace for `capacity` pairs of size n out of `base` (256-byte aligned).  Each of
// its regions (seven; thirteen for the mixed form above kMixedMaxN) starts on a 256-byte boundary.
Workspace carve_workspace(void* base, int n, int capacity, bool mixed = false);
// Exact bytes carve_workspace(base, n, capacity, mixed) spans from base: every allocation that
// backs a workspace is sized by this (at most workspace_bytes_per_pair(n, mixed) * capacity +
// 13 * 256).
size_t workspace_bytes(int n, int capacity, bool mixed = false);

enum ReduceMode : int {
    kReduceFull = 0,      // potrf + hegst          -> L into ws.LV (lower), C lower into out
    kReduceChol = 1,      // potrf only             -> out (L, strict upper zeroed)
    kReduceHegst = 2,     // potrf + hegst          -> out (M lower, strict upper zeroed)
    kReduceFromLM = 3,    // given L                -> L copied into ws.LV (lower)
    kReduceMixed = 4,     // potrf + hegst          -> as kReduceFull, but for n > kSmallMaxN the
                          //                           reduction stops before the tridiagonalisation
};
enum BackMode : int {
    kBackFull = 0,        // X = L^{-H} Q Z
    kBackQOnly = 1,       // V = Q Z (eigenvectors of the reduced matrix)
    kBackLOnly = 2,       // X = L^{-H} Y, Y complex in the X buffer (mixed form)
};

// Launch shape of the stage kernels, the part of a schedule the autotuner varies:
//   threads     threads per CTA of k_hetrd (66 <= n <= 84): 128 or 256
//   pair_warps  pairs (one warp each) per CTA of k_potrf_warp, k_hetrd_warp, k_hetrd_warp_c64
//               (n <= 65): 1, 2 or 4 -- the reference's "batches per block"
//   col_exact   k_hegst_col / k_back_col: the exact-n instantiation where one exists (n = 32, 54)
//               instead of the one for the next larger NMAX
//   back_lanes  lanes per column of k_back_col (n <= 56): 1 or 2
//   back_qpass  reflectors per pass of k_back_col's Q application (n <= 56): 1 or 2
//   reduce_tc   n > 56: the triangular stages on the FP64 tensor cores -- Cholesky and reduction by
//               the blocked kernel k_reduce_tc (above kSmallMaxN, FP64 form, then the Householder
//               alone by k_hetrd_l2 instead of k_reduce_mid / k_reduce_big doing all three), and
//               X = L^{-H} Y by k_back_tc after the Q-only back-transform, which above kSmallMaxN is
//               the compact-WY tensor-core kernel k_back_q_tc
struct LaunchShape {
    int threads = 256;
    int pair_warps = 2;
    int col_exact = 1;
    int back_lanes = 1;
    int back_qpass = 1;
    int reduce_tc = 0;
};

// Launchers (asynchronous on `stream`; return cudaSuccess or the launch error).
cudaError_t launch_reduce(int mode, const double2* A, const double2* B, int n, int batch,
                          const Workspace& ws, double2* out, int* info, const LaunchShape& shape, cudaStream_t stream);
// Householder tridiagonalisation of C (lower triangle read, column-major, ld = n) ->
// reflectors into ws.LV (rows above the superdiagonal), tau, d, e.  Pairs with info != 0 skip.
cudaError_t launch_hetrd(int n, int batch, const double2* C, const Workspace& ws, int* info, const LaunchShape& shape,
                         cudaStream_t stream);
size_t hetrd_smem_bytes(int n, int threads);
// Two-kernel QL: thread-per-pair scalar chain logging rotations, then a warp-per-pair
// application of the log to Z (single = FP32 chain and Z, the mixed form's first half).
cudaError_t launch_ql_logged(int n, int batch, const Workspace& ws, double* W, double2* X, int* info,
                             bool single, int chain_threads, int apply_warps, cudaStream_t stream);
// Mixed form (n <= kMixedMaxN), after the FP64 reduction left C in X:
//   launch_hetrd_c64     complex64 Householder (warp per pair); FP64-promoted reflectors, tau (made
//                        unitary in FP64) and T into the workspace, C into the pair's stash;
//   launch_eig_mixed     eigenpairs of that T (launch_eig_invit, FP64), Y = Q Z
//                        (launch_back(kBackQOnly)), then launch_refine_mixed: FP64 Ogita-Aishima
//                        refinement of (W, Y) against the stashed C on the FP64 tensor cores, and
//                        the FP64 fallback for pairs it cannot take;
//   launch_back(kBackLOnly)  X = L^{-H} Y.
cudaError_t launch_hetrd_c64(int n, int batch, const double2* C, const Workspace& ws, int* info,
                             const LaunchShape& shape, cudaStream_t stream);
cudaError_t launch_refine_mixed(int n, int batch, const Workspace& ws, double* W, double2* X, int* info,
                                int refine_steps, cudaStream_t stream);
cudaError_t launch_eig_mixed(int n, int batch, const Workspace& ws, double* W, double2* X, int* info,
                             int refine_steps, int chain_threads, const LaunchShape& shape, cudaStream_t stream);
size_t hetrd_c64_smem_bytes(int n);
// Dynamic shared memory of a CTA of the warp-per-pair kernels (k_potrf_warp, k_hetrd_warp,
// k_hetrd_warp_c64) with pair_warps pairs.
size_t pair_kernels_smem_bytes(int n, int pair_warps);
size_t refine_c_smem_bytes(int n);
size_t mixed_fallback_smem_bytes(int n);
// Host-buffer path: copies `count` pairs of n x n column-major matrices from pinned host memory
// that the GPU can address (src is its device-side address) into device memory, either every
// element or only rows j..n-1 of each column j (lower, for B, whose upper triangle no kernel
// reads).  The kernel's loads cross the host link; one CTA per SM keeps enough of them in flight.
cudaError_t launch_pull_pairs(const double2* src, double2* dst, int count, int n, bool lower, cudaStream_t stream);
cudaError_t launch_back(int mode, int n, int batch, const Workspace& ws, double2* X, int* info,
                        const LaunchShape& shape, cudaStream_t stream);

// Pairs with n <= kSmallMaxN are solved by CTA-per-pair (or warp-per-pair) stage kernels;
// kSmallMaxN < n <= kBigMaxN by the cluster kernels of bigsolve.cu.  For those the reduce
// launch (kReduceFull only) also tridiagonalises, so launch_hetrd has nothing left to do,
// and the reflectors are stored along the columns of LV's strict upper triangle
// (v_k(k+1+s) = LV(s, n-1-k)) instead of its rows.
constexpr int kSmallMaxN = 84;
constexpr int kBigMaxN = 256;
bool big_path(int n);
size_t big_reduce_smem_bytes(int n);
size_t ql_rows_smem_bytes(int n, bool single);
// Largest dynamic shared memory per CTA among the FP64 kernels a solve of order n > kSmallMaxN
// launches: tc = the schedule's reduce_tc, chain_threads its QL chain width.
size_t big_stage_smem_bytes(int n, bool tc, int chain_threads);
// mode: kBigFull (Cholesky, reduction, Householder: k_reduce_mid / k_reduce_big), kBigHegstOnly (the
// same kernels, stopping after C = L^{-1} A L^{-H}: C's lower triangle in X, L in LV) or kBigHetrdOnly
// (the Householder alone by k_hetrd_l2, from C's lower triangle in X with L already in LV, as
// k_reduce_tc leaves them; pairs with info != 0 are skipped).
enum BigReduceMode : int { kBigFull = 0, kBigHegstOnly = 1, kBigHetrdOnly = 2 };
cudaError_t launch_reduce_big(const double2* A, const double2* B, int n, int batch, const Workspace& ws, double2* X,
                              int* info, cudaStream_t stream, int mode = kBigFull);
// Mixed form for kMixedMaxN < n <= kMixedBigMaxN (csrc/mixed_big.cu), after
// launch_reduce(kReduceMixed) left L in LV and C's lower triangle in X:
//   launch_hetrd_c64_big   complex64 Householder, one CTA per pair: FP64-promoted reflectors (in the
//                          layout launch_back expects for n), tau made unitary in FP64, d, e; C
//                          (FP64, full Hermitian) into ws.rfC;
//   launch_refine_big      after the FP64 eigenpairs of that T and Y = Q Z in X: Ogita-Aishima
//                          refinement of (W, Y) against rfC, every product on the FP64 tensor
//                          cores; ws.rstat gets each pair's outcome.
cudaError_t launch_hetrd_c64_big(int n, int batch, const double2* C, const Workspace& ws, int* info,
                                 cudaStream_t stream);
// The FP64 Householder alone for n > kSmallMaxN after launch_reduce_tc (C's lower triangle in X),
// one CTA per pair with the packed triangle in the pair's rotation-log region (L2-resident global
// memory): reflectors to LV's columns, d, e, tau; pairs with info != 0 are skipped.
cudaError_t launch_hetrd_l2(int n, int batch, const double2* C, const Workspace& ws, int* info,
                           cudaStream_t stream);
// Blocked FP64 Cholesky and reduction on the FP64 tensor cores (csrc/reduce_tc.cu), one CTA per
// pair: L into LV's lower triangle, C = L^{-1} A L^{-H} (lower triangle) into X, info as the other
// reduce kernels (n + i for a leading minor i that is not positive definite).  Uses the pair's
// rotation-log region as scratch.  Honours the pair selection.
cudaError_t launch_reduce_tc(const double2* A, const double2* B, int n, int batch, const Workspace& ws, double2* X,
                             int* info, cudaStream_t stream);
// X = L^{-H} Y in place (Y complex in X) by the blocked backward substitution on the FP64 tensor
// cores (csrc/reduce_tc.cu), one CTA per pair; NaN for pairs whose B was not positive definite.
// Uses the pair's rotation-log region as scratch.  Honours the pair selection.
cudaError_t launch_back_tc(int n, int batch, const Workspace& ws, double2* X, const int* info, cudaStream_t stream);
// Y = Q Z in place (Z real in X, Y complex over it) for n > kSmallMaxN: the reflectors of the big-n
// Householder applied in compact-WY blocks of 32 (zlarft's T) as tile products on the FP64 tensor
// cores (csrc/reduce_tc.cu), one CTA per pair; NaN for pairs whose B was not positive definite.
// Uses the pair's rotation-log region as scratch.  Honours the pair selection.
cudaError_t launch_back_q_tc(int n, int batch, const Workspace& ws, double2* X, const int* info,
                             cudaStream_t stream);
cudaError_t launch_refine_big(int n, int batch, const Workspace& ws, double* W, double2* X, int* info,
                              int refine_steps, cudaStream_t stream);
size_t hetrd_c64_big_smem_bytes(int n);
size_t refine_big_smem_bytes();
cudaError_t launch_ql_rows(int n, int batch, const Workspace& ws, double* W, double2* X, int* info, bool single,
                           int chain_threads, cudaStream_t stream);
cudaError_t launch_back_big(int mode, int n, int batch, const Workspace& ws, double2* X, const int* info,
                            cudaStream_t stream);
// The QL scalar chain alone (thread per pair): W, the rotation log, perm, flag.
// redo: only pairs with ws.flag == 2 (flagged by launch_eig_invit); they keep 2, or get 3 on a
// log overflow.
cudaError_t launch_ql_chain(int n, int batch, const Workspace& ws, double* W, int* info, bool single,
                            int chain_threads, cudaStream_t stream, bool redo = false);

// Kernels one full reduce launch (kReduceFull) issues for order n: the warp Cholesky and the
// column hegst kernel for n <= 56; above kSmallMaxN with the tensor-core reduction (tc), k_reduce_tc
// and the Householder kernel; one kernel otherwise.
inline int reduce_kernel_count(int n, bool tc = false) { return n <= 56 || (n > kSmallMaxN && tc) ? 2 : 1; }
// (57 <= n <= 84 with tc: k_reduce_tc alone, the Householder being its own stage there.)
// FP64 eigenvectors by inverse iteration (k_ql_values + k_tridiag_invit) for n <= kInvitMaxN, with
// the warp QL inside the kernel for pairs it cannot take, and for kSmallMaxN < n <= kInvitBigMaxN,
// where such pairs are flagged and the rotation-log QL (k_ql_chain + k_ql_apply_rows) redone for
// them only; the rotation-log QL for every other n and for the mixed form.
constexpr int kInvitMaxN = 63;
constexpr int kInvitBigMaxN = 128;
inline bool eig_by_inverse_iteration(int n, bool single) {
    return !single && (n <= kInvitMaxN || (n > kSmallMaxN && n <= kInvitBigMaxN));
}
// Kernels one eigensolve stage launches for order n.
inline int eig_kernel_count(int n, bool single) {
    if (single) return 5;          // k_ql_values, k_tridiag_invit, Q-apply, refinement, fallback
    if (n <= kInvitMaxN) return 2;
    return n > kSmallMaxN && n <= kInvitBigMaxN ? 4 : 2;
}
// Eigenvalues (k_ql_values) and inverse-iteration eigenvectors (k_tridiag_invit) of every pair;
// flag_redo: pairs it cannot take get ws.flag = 2 (and no output) instead of the in-kernel QL.
cudaError_t launch_eig_invit(int n, int batch, const Workspace& ws, double* W, double2* X, int* info,
                             int chain_threads, bool flag_redo, cudaStream_t stream);

size_t reduce_smem_bytes(int mode, int n);
size_t ql_chain_smem_bytes(int n, int threads, bool single);
size_t ql_apply_smem_bytes(int n, int warps_per_cta, bool single);
size_t back_smem_bytes(int n);
size_t invit_smem_bytes(int n, bool with_tile);
// r[i] = recip_nr(u[i]) for i < count (device self-test of the inverse iteration's reciprocal).
cudaError_t launch_selftest_recip(const double* u, double* r, int count, cudaStream_t stream);
// FP64 FMA throughput probe: `blocks` CTAs of 256 threads, each thread 8 chains x 4 x iters FMAs;
// out holds blocks * 256 doubles.
cudaError_t launch_selftest_fp64_fma(double* out, int blocks, int iters, cudaStream_t stream);
// Largest dynamic shared memory a block may opt into on the CURRENT device (queried once per
// device ordinal; 0 if the query fails).
int max_smem_optin();

// Per-kernel record of the dynamic shared-memory limit raised on each device.
// cudaFuncSetAttribute acts on the device current at the call, so one process that launches on
// several GPUs has to raise it on each of them.  Ordinals beyond kDevices are raised every call.
struct SmemOptIn {
    static constexpr int kDevices = 64;
    std::atomic<int> raised[kDevices] = {};
};
// Raises `kernel`'s dynamic shared-memory limit to `bytes` on the current device unless the
// record shows it done there already.
void set_smem_limit(const void* kernel, SmemOptIn& rec, int bytes);

}  // namespace sbg
