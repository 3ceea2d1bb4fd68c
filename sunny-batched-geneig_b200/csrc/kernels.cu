// Stage kernels of the batched generalized eigensolve for n <= 84, and the launchers
// that route larger n to the cluster kernels of bigsolve.cu.
//
//   reduce   k_potrf_warp + k_hegst_col (n <= 56) or k_reduce (57..84): B = L L^H and
//            C = L^{-1} A L^{-H}; L into the workspace, C into the caller's X buffer.
//   hetrd    k_hetrd_warp (n <= 65) or k_hetrd: Householder tridiagonalisation of C,
//            reflectors and (d, e, tau) into the workspace; the mixed form (n <= 56) runs it
//            in complex64 (k_hetrd_warp_c64).
//   eig      FP64, n <= 63 (and 85..128, launched from bigsolve.cu): k_ql_values (the
//            implicit-QL recurrence, one thread per pair, eigenvalues only) and
//            k_tridiag_invit (eigenvectors by inverse iteration, one warp per pair).
//            Otherwise k_ql_chain logs the recurrence's rotations and k_ql_apply /
//            k_ql_apply_reg replay the log onto Z (W ascending).  The mixed form refines
//            Y = Q Z against C afterwards (refine.cu).
//   back     k_back_col (n <= 56) or k_back: X = L^{-H} Q Z, written over Z (the mixed
//            form: Y = Q Z, then X = L^{-H} Y after the refinement).
//
// The split follows where the work is latency bound: the QL recurrence is a
// dependent scalar chain per pair, so it runs with many pairs per SM, while the
// BLAS2-shaped stages run a warp or a CTA per pair.
#include "kernels.cuh"
#include "stages.cuh"
#include "colsolve.cuh"

#include <algorithm>
#include <cstdlib>
#include <atomic>
#include <mutex>

namespace sbg {

namespace {

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Shared-memory carve-up of k_reduce.
struct ReduceSmem {
    size_t Ls, As, invd, bar, total;
    __host__ __device__ ReduceSmem(int n) {
        const size_t ld = static_cast<size_t>(tile_ld(n));
        size_t o = 0;
        Ls = o;   o += 16 * ld * n;
        As = o;   o += 16 * ld * n;
        invd = o; o += align_up(8 * n, 16);
        bar = o;  o += 16;
        total = o;
    }
};


// Waits for the bulk copies of this CTA; on the (never expected) timeout it flags
// the pair (every thread that timed out ORs the bit into the pair's info word, when one is
// given) and waits once more, bounded, so no copy lands after the CTA exits.  The stage then
// runs on whatever landed; the flag (info > n) makes the back-transform write NaN for the pair
// and every later stage skip it.
__device__ inline bool wait_copies(uint64_t* bar, int* info_word) {
    if (mbar_wait_bounded(bar, 0, kMaxPolls)) return true;
    if (info_word) atomicOr(info_word, kInfoCopyTimeout);
    mbar_wait_bounded(bar, 0, kMaxPolls);
    return false;
}

// ----------------------------------------------------------------------------- k_reduce
template <int T, int G, int RM>
__global__ void __launch_bounds__(T, RM <= 8 ? 2 : 1) k_reduce(int mode, const double2* __restrict__ A,
                                              const double2* __restrict__ B, int n, int batch,
                                              Workspace ws, double2* __restrict__ out,
                                              int* __restrict__ info) {
    const int b = blockIdx.x;
    if (b >= batch || !pair_selected(ws, b)) return;
    extern __shared__ __align__(16) unsigned char smem[];
    const ReduceSmem lay(n);
    const int ld = tile_ld(n);
    double2* Ls = reinterpret_cast<double2*>(smem + lay.Ls);
    double2* As = reinterpret_cast<double2*>(smem + lay.As);
    double* invd = reinterpret_cast<double*>(smem + lay.invd);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + lay.bar);

    const int tid = threadIdx.x;
    const size_t mat = static_cast<size_t>(n) * n;
    const double2* Ab = A + mat * b;     // A (unused in kReduceChol / kReduceFromLM)
    const double2* Bb = B + mat * b;     // B, or L in kReduceFromLM
    const bool need_a = mode != kReduceChol && mode != kReduceFromLM;

    // ---- stage the pair into shared memory: B (lower part of each column) and A
    if (tid == 0) { mbar_init(bar, 1); fence_mbar_init(); }
    __syncthreads();
    if (tid < 32) {
        if (tid == 0) {
            uint32_t bytes = static_cast<uint32_t>(16 * (static_cast<size_t>(n) * (n + 1) / 2));
            if (need_a) bytes += static_cast<uint32_t>(16 * mat);
            mbar_arrive_expect_tx(bar, bytes);
        }
        __syncwarp();
        for (int j = tid; j < n; j += 32) {
            bulk_g2s(Ls + j + static_cast<size_t>(j) * ld, Bb + j + static_cast<size_t>(j) * n, 16u * (n - j), bar);
            if (need_a) bulk_g2s(As + static_cast<size_t>(j) * ld, Ab + static_cast<size_t>(j) * n, 16u * n, bar);
        }
    }
    // the first stage: info[b] is written only at the end (with the timeout bit of thread 0's wait)
    const int copy_status = wait_copies(bar, nullptr) ? 0 : kInfoCopyTimeout;

    int st = 0;
    if (mode == kReduceFromLM) {
        for (int i = tid; i < n; i += T) invd[i] = 1.0 / Ls[i + i * ld].x;
        __syncthreads();
    } else {
        st = potrf_lower(Ls, ld, n, invd);
    }
    if (st != 0) {
        if (tid == 0) info[b] = ((mode == kReduceFull) ? n + st : st) | copy_status;
        return;
    }
    if (mode == kReduceChol) {
        for (size_t idx = tid; idx < mat; idx += T) {
            const int j = static_cast<int>(idx / n), i = static_cast<int>(idx - static_cast<size_t>(j) * n);
            out[mat * b + idx] = (i >= j) ? Ls[i + j * ld] : make_double2(0.0, 0.0);
        }
        if (tid == 0) info[b] = copy_status;
        return;
    }
    if (mode != kReduceFromLM) {
        const int g = tid % G;
        double2 y[RM];
        {   // W = L^{-1} A: column j = tid / G, rows g + G r in registers
            const int j = tid / G;
            const bool valid = j < n;
#pragma unroll
            for (int r = 0; r < RM; ++r) {
                const int i = g + G * r;
                y[r] = (valid && i < n) ? As[i + j * ld] : make_double2(0.0, 0.0);
            }
            seg_trsm_lower<G, RM>(Ls, ld, invd, y, n, g);
            if (valid) {
#pragma unroll
                for (int r = 0; r < RM; ++r) {
                    const int i = g + G * r;
                    if (i < n) As[i + j * ld] = y[r];
                }
            }
        }
        __syncthreads();
        {   // C = W L^{-H} (lower part): row i = tid / G, columns g + G r in registers
            const int i = tid / G;
            const bool valid = i < n;
            const int kmax = min(n - 1, (tid | 31) / G);
#pragma unroll
            for (int r = 0; r < RM; ++r) {
                const int kk = g + G * r;
                y[r] = (valid && kk < n) ? As[i + kk * ld] : make_double2(0.0, 0.0);
            }
            seg_trsm_right_lowerH<G, RM>(Ls, ld, invd, y, kmax, valid ? i : -1, g);
            if (valid) {
#pragma unroll
                for (int r = 0; r < RM; ++r) {
                    const int kk = g + G * r;
                    if (kk <= i) As[i + kk * ld] = y[r];
                }
            }
        }
        __syncthreads();
    }
    if (mode == kReduceHegst || mode == kReduceFull) {
        double2* Mg = out + mat * b;
        for (size_t idx = tid; idx < mat; idx += T) {
            const int j = static_cast<int>(idx / n), i = static_cast<int>(idx - static_cast<size_t>(j) * n);
            double2 v = make_double2(0.0, 0.0);
            if (i >= j) { v = As[i + j * ld]; if (i == j) v.y = 0.0; }
            if (i >= j || mode == kReduceHegst) Mg[idx] = v;
        }
    }
    if (mode == kReduceFull || mode == kReduceFromLM) {
        // L into the lower triangle of the pair's LV tile (the reflectors fill the upper part later)
        double2* LVg = ws.LV + mat * b;
        for (size_t idx = tid; idx < mat; idx += T) {
            const int j = static_cast<int>(idx / n), i = static_cast<int>(idx - static_cast<size_t>(j) * n);
            if (i >= j) LVg[idx] = Ls[i + j * ld];
        }
    }
    if (tid == 0) info[b] = copy_status;
}

struct BackSmem {
    size_t LVs, invd, tau, cpair, bar, total;
    __host__ __device__ BackSmem(int n, int tile_ld_override = 0) {
        const size_t ld = static_cast<size_t>(tile_ld_override > 0 ? tile_ld_override : tile_ld(n));
        size_t o = 0;
        LVs = o;  o += 16 * ld * n;
        invd = o; o += align_up(8 * n, 16);
        tau = o;  o += 16 * n;
        cpair = o; o += 16 * n;
        bar = o;  o += 16;
        total = o;
    }
};

// ----------------------------------------------------------------------------- k_potrf_warp
// One WARP per pair (n <= 64): B's lower triangle bulk-copied into a packed tile,
// Cholesky by potrf_warp_packed; L goes to `out` (strict upper zeroed, the staged
// Cholesky) or to the lower triangle of the pair's LV tile (the full solve).
__host__ __device__ inline size_t potrf_warp_bytes(int n) {
    return align_up(16 * static_cast<size_t>(n) * (n + 1) / 2, 16) + align_up(8 * n, 16) + 16;
}
constexpr int kMaxPairWarps = 4;      // warp-per-pair kernels: 1, 2 or 4 pairs (warps) per CTA
constexpr int kColMaxN = 56;      // column-per-thread kernels: y[NMAX] in registers, NMAX in {32, 48, 56}

__global__ void __launch_bounds__(32 * kMaxPairWarps) k_potrf_warp(int mode, const double2* __restrict__ B, int n,
                                                                      int batch, Workspace ws, double2* __restrict__ out,
                                                                      int* __restrict__ info) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x * (blockDim.x >> 5) + warp;
    if (b >= batch) return;
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char* base = smem + potrf_warp_bytes(n) * warp;
    double2* P = reinterpret_cast<double2*>(base);
    double* invd = reinterpret_cast<double*>(base + align_up(16 * static_cast<size_t>(n) * (n + 1) / 2, 16));
    uint64_t* bar = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(invd) + align_up(8 * n, 16));
    const size_t mat = static_cast<size_t>(n) * n;
    const double2* Bb = B + mat * b;
    if (lane == 0) { mbar_init(bar, 1); fence_mbar_init(); }
    __syncwarp();
    if (lane == 0) mbar_arrive_expect_tx(bar, static_cast<uint32_t>(16 * (static_cast<size_t>(n) * (n + 1) / 2)));
    __syncwarp();
    for (int j = lane; j < n; j += 32)
        bulk_g2s(P + pk(j, n), Bb + j + static_cast<size_t>(j) * n, 16u * (n - j), bar);
    // the first stage: info[b] is written only at the end, with the timeout bit of lane 0's wait
    const int copy_status = wait_copies(bar, nullptr) ? 0 : kInfoCopyTimeout;
    const int st = potrf_warp_packed<double>(P, n, invd);
    if (st != 0) {
        if (lane == 0) info[b] = ((mode == kReduceFull) ? n + st : st) | copy_status;
        return;
    }
    __syncwarp();
    double2* dst = (mode == kReduceChol) ? out + mat * b : ws.LV + mat * b;
    for (int j = 0; j < n; ++j) {
        const double2* col = P + pk(j, n) - j;     // col[i] = L(i, j), i >= j
        for (int i = lane; i < n; i += 32) {
            if (i >= j) dst[i + static_cast<size_t>(j) * n] = col[i];
            else if (mode == kReduceChol) dst[i + static_cast<size_t>(j) * n] = make_double2(0.0, 0.0);
        }
    }
    if (lane == 0) info[b] = copy_status;
}

// ----------------------------------------------------------------------------- k_hegst_col
// One CTA of NMAX threads per pair (n <= NMAX): C = L^{-1} A L^{-H}.  Thread j solves
// column j of W = L^{-1} A in registers and stores it to the pair's X slice (in L2);
// after the barrier thread i reads row i of W back and solves row i of C = W L^{-H},
// columns k <= i, writing C's lower triangle over its own row.  Only the packed L
// lives in shared memory.  kReduceHegst also zeroes the strict upper triangle.
__host__ __device__ inline size_t hegst_col_bytes(int n) {
    return align_up(16 * static_cast<size_t>(n) * (n + 1) / 2, 16) + align_up(8 * n, 16) + 16;
}

// EXACT: n == NMAX is a compile-time constant (the common sizes get their own
// instantiation, so every row-bound test folds away).
template <int NMAX, bool EXACT>
__global__ void __launch_bounds__(NMAX, 4) k_hegst_col(int mode, const double2* __restrict__ A, const Workspace ws,
                                                    double2* __restrict__ out, int n_arg, int batch,
                                                    int* __restrict__ info) {
    const int n = EXACT ? NMAX : n_arg;
    const int b = blockIdx.x;
    if (b >= batch) return;
    if (info[b] != 0) return;
    extern __shared__ __align__(16) unsigned char smem[];
    double2* Lp = reinterpret_cast<double2*>(smem);
    double* invd = reinterpret_cast<double*>(smem + align_up(16 * static_cast<size_t>(n) * (n + 1) / 2, 16));
    uint64_t* bar = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(invd) + align_up(8 * n, 16));
    const int tid = threadIdx.x;
    const size_t mat = static_cast<size_t>(n) * n;
    const double2* Lg = ws.LV + mat * b;
    const double2* Ab = A + mat * b;
    double2* Ob = out + mat * b;
    if (tid == 0) { mbar_init(bar, 1); fence_mbar_init(); }
    __syncthreads();
    if (tid < 32) {
        if (tid == 0) mbar_arrive_expect_tx(bar, static_cast<uint32_t>(16 * (static_cast<size_t>(n) * (n + 1) / 2)));
        __syncwarp();
        for (int j = tid; j < n; j += 32)
            bulk_g2s(Lp + pk(j, n), Lg + j + static_cast<size_t>(j) * n, 16u * (n - j), bar);
    }
    const bool own = tid < n;
    double2 y[NMAX];
#pragma unroll
    for (int i = 0; i < NMAX; ++i)
        y[i] = (own && i < n) ? Ab[i + static_cast<size_t>(tid) * n] : make_double2(0.0, 0.0);
    wait_copies(bar, info + b);
    for (int i = tid; i < n; i += NMAX) invd[i] = 1.0 / Lp[pk(i, n)].x;
    __syncthreads();
    if (own) col_trsm_lower2<NMAX>(Lp, invd, y, n, [&](int k, double2 w) { Ob[k + static_cast<size_t>(tid) * n] = w; });
    __syncthreads();
    if (own) {
        const int i = tid;
#pragma unroll
        for (int kk = 0; kk < NMAX; ++kk) y[kk] = (kk <= i) ? Ob[i + static_cast<size_t>(kk) * n] : make_double2(0.0, 0.0);
        const int kmax = min(n - 1, (tid | 31));            // the warp's largest row: uniform loop bound
        row_trsm_right_lowerH2<NMAX>(Lp, invd, y, n, i, kmax, [&](int k, double2 c) {
            if (k == i) c.y = 0.0;
            Ob[i + static_cast<size_t>(k) * n] = c;
        });
        if (mode == kReduceHegst)
            for (int k = i + 1; k < n; ++k) Ob[i + static_cast<size_t>(k) * n] = make_double2(0.0, 0.0);
    }
}

// ----------------------------------------------------------------------------- k_back_col
// One CTA per pair (n <= NMAX): the G adjacent lanes of group j hold column j of Z in
// registers (rows G r + g), apply Q and L^{-H}, and store X(:, j) (kBackQOnly: Q Z).  The
// CTA is rounded up to whole warps; lanes of columns j >= n run the sweeps on zeros (the
// group shuffles need the full warp) and store nothing.
template <int NMAX, int G>
__host__ __device__ constexpr int back_col_threads() { return (NMAX * G + 31) / 32 * 32; }

template <int NMAX, int G, bool EXACT, int QP>
__global__ void __launch_bounds__(back_col_threads<NMAX, G>(), G == 1 ? 4 : 3) k_back_col(int mode, int n_arg, int batch,
                                                                            Workspace ws, double2* __restrict__ X,
                                                                            int* __restrict__ info) {
    const int n = EXACT ? NMAX : n_arg;              // EXACT: n is a compile-time constant
    constexpr int T = back_col_threads<NMAX, G>();
    constexpr int RM = (NMAX + G - 1) / G;
    // tile_ld(NMAX) as a compile-time stride: every row slot's offset is an immediate
    constexpr int LDC = (((NMAX | 1) & 7) == 7) ? (NMAX | 1) + 2 : (NMAX | 1);
    const int b = blockIdx.x;
    if (b >= batch) return;
    const size_t mat = static_cast<size_t>(n) * n;
    double2* Xb = X + mat * b;
    const int tid = threadIdx.x;
    if (info[b] > n || info[b] < 0) {
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        for (size_t idx = tid; idx < mat; idx += T) Xb[idx] = make_double2(nan, nan);
        return;
    }
    extern __shared__ __align__(16) unsigned char smem[];
    const BackSmem lay(n, LDC);
    constexpr int ld = LDC;
    double2* LVs = reinterpret_cast<double2*>(smem + lay.LVs);
    double* invd = reinterpret_cast<double*>(smem + lay.invd);
    double2* tau_s = reinterpret_cast<double2*>(smem + lay.tau);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + lay.bar);
    const double2* LVg = ws.LV + mat * b;
    if (tid == 0) { mbar_init(bar, 1); fence_mbar_init(); }
    __syncthreads();
    if (tid < 32) {
        if (tid == 0) mbar_arrive_expect_tx(bar, static_cast<uint32_t>(16 * mat));
        __syncwarp();
        for (int j = tid; j < n; j += 32)
            bulk_g2s(LVs + static_cast<size_t>(j) * ld, LVg + static_cast<size_t>(j) * n, 16u * n, bar);
    }
    const int col = tid / G, g = tid - col * G;
    const bool own = col < n;
    const double* Zg = reinterpret_cast<const double*>(Xb);
    double2 y[RM];
    if (mode == kBackLOnly) {                        // complex Y in the X buffer
#pragma unroll
        for (int r = 0; r < RM; ++r) {
            const int i = G * r + g;
            y[r] = (own && i < n) ? Xb[i + static_cast<size_t>(col) * n] : make_double2(0.0, 0.0);
        }
    } else {                                         // real Z in the X buffer
#pragma unroll
        for (int r = 0; r < RM; ++r) {
            const int i = G * r + g;
            y[r] = make_double2((own && i < n) ? Zg[i + static_cast<size_t>(col) * n] : 0.0, 0.0);
        }
    }
    for (int i = tid; i < n; i += T) tau_s[i] = ws.tau[static_cast<size_t>(n) * b + i];
    wait_copies(bar, info + b);
    for (int i = tid; i < n; i += T) invd[i] = 1.0 / LVs[i + i * ld].x;
    double2* cpair = reinterpret_cast<double2*>(smem + lay.cpair);
    if (QP == 2 && mode != kBackLOnly) reflector_couplings<double>(LVs, ld, n, cpair, T);
    __syncthreads();               // all of Z is in registers before any X is stored over it
    if (mode != kBackLOnly) {
        if constexpr (QP == 2) grp_apply_q2<G, RM, double>(LVs, ld, tau_s, cpair, y, n, g);
        else grp_apply_q<G, RM, double>(LVs, ld, tau_s, y, n, g);
    }
    double2* xcol = Xb + static_cast<size_t>(col) * n;
    if (mode == kBackFull || mode == kBackLOnly) {
        grp_trsm_lowerH2<G, RM>(LVs, ld, invd, y, n, g, [&](int k, double2 x) { if (own) xcol[k] = x; });
    } else if (own) {
#pragma unroll
        for (int r = 0; r < RM; ++r) {
            const int i = G * r + g;
            if (i < n) xcol[i] = y[r];
        }
    }
}

// ----------------------------------------------------------------------------- k_hetrd
// One CTA per pair, one tile: C (lower triangle) staged by TMA bulk copies, reduced
// to tridiagonal form; the reflectors go to the upper part of the pair's LV tile.
struct HetrdSmem {
    size_t As, vw, pbuf, ww, d, e, tau, bar, total;
    __host__ __device__ HetrdSmem(int n, int threads) {
        const size_t ld = static_cast<size_t>(tile_ld(n));
        const size_t nw = static_cast<size_t>(threads / 32);
        size_t o = 0;
        As = o;   o += 16 * ld * n;
        vw = o;   o += 16 * n * nw;
        pbuf = o; o += 32 * n;
        ww = o;   o += 16 * n * nw;
        d = o;    o += align_up(8 * n, 16);
        e = o;    o += align_up(8 * n, 16);
        tau = o;  o += 16 * n;
        bar = o;  o += 16;
        total = o;
    }
};
template <int T>
__global__ void __launch_bounds__(T) k_hetrd(int n, int batch, const double2* __restrict__ C, Workspace ws,
                                             int* __restrict__ info) {
    const int b = blockIdx.x;
    if (b >= batch || !pair_selected(ws, b)) return;
    if (info[b] != 0) return;
    extern __shared__ __align__(16) unsigned char smem[];
    const HetrdSmem lay(n, T);
    const int ld = tile_ld(n);
    double2* As = reinterpret_cast<double2*>(smem + lay.As);
    double2* vw = reinterpret_cast<double2*>(smem + lay.vw);
    double2* pbuf = reinterpret_cast<double2*>(smem + lay.pbuf);
    double2* ww = reinterpret_cast<double2*>(smem + lay.ww);
    double* d_s = reinterpret_cast<double*>(smem + lay.d);
    double* e_s = reinterpret_cast<double*>(smem + lay.e);
    double2* tau_s = reinterpret_cast<double2*>(smem + lay.tau);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + lay.bar);
    const int tid = threadIdx.x;
    const size_t mat = static_cast<size_t>(n) * n;
    const double2* Cb = C + mat * b;
    if (tid == 0) { mbar_init(bar, 1); fence_mbar_init(); }
    __syncthreads();
    if (tid < 32) {
        if (tid == 0) mbar_arrive_expect_tx(bar, static_cast<uint32_t>(16 * (static_cast<size_t>(n) * (n + 1) / 2)));
        __syncwarp();
        for (int j = tid; j < n; j += 32)
            bulk_g2s(As + j + static_cast<size_t>(j) * ld, Cb + j + static_cast<size_t>(j) * n, 16u * (n - j), bar);
    }
    wait_copies(bar, info + b);
    hetrd_lower(As, ld, n, d_s, e_s, tau_s, vw, pbuf, ww);
    // reflector k, component i >= k+2, sits at A(i, k); it goes to LV(k, i)
    double2* LVg = ws.LV + mat * b;
    for (size_t idx = tid; idx < mat; idx += T) {
        const int i = static_cast<int>(idx / n), k = static_cast<int>(idx - static_cast<size_t>(i) * n);
        if (i >= k + 2) LVg[k + static_cast<size_t>(i) * n] = As[i + k * ld];
        else if (i == k + 1) LVg[k + static_cast<size_t>(i) * n] = make_double2(1.0, 0.0);
    }
    for (int i = tid; i < n; i += T) {
        ws.d[static_cast<size_t>(n) * b + i] = d_s[i];
        ws.e[static_cast<size_t>(n) * b + i] = e_s[i];
        ws.tau[static_cast<size_t>(n) * b + i] = (i + 1 < n) ? tau_s[i] : make_double2(0.0, 0.0);
    }
}

// ----------------------------------------------------------------------------- k_hetrd_warp
// One WARP per pair (n <= 65): C's lower triangle is bulk-copied column by column into
// a packed lower-triangular tile (n(n+1)/2 complex; 23.8 KB at n = 54, so eight pairs
// fit an SM) and reduced by hetrd_warp_packed with warp-level synchronisation only.
__host__ __device__ inline size_t hetrd_warp_bytes(int n) {
    return align_up(16 * static_cast<size_t>(n) * (n + 1) / 2, 16) + 16 * 4 * n + 16;
}
constexpr int kHetrdWarpMaxN = 65;

__global__ void __launch_bounds__(32 * kMaxPairWarps) k_hetrd_warp(int n, int batch, const double2* __restrict__ C,
                                                                  Workspace ws, int* __restrict__ info) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x * (blockDim.x >> 5) + warp;
    if (b >= batch || !pair_selected(ws, b)) return;
    if (info[b] != 0) return;
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char* base = smem + hetrd_warp_bytes(n) * warp;
    double2* P = reinterpret_cast<double2*>(base);
    double2* vb = reinterpret_cast<double2*>(base + align_up(16 * static_cast<size_t>(n) * (n + 1) / 2, 16));
    double2* wb = vb + n;
    double2* vb2 = wb + n;
    double2* wb2 = vb2 + n;
    uint64_t* bar = reinterpret_cast<uint64_t*>(wb2 + n);
    const size_t mat = static_cast<size_t>(n) * n;
    const double2* Cb = C + mat * b;
    if (lane == 0) { mbar_init(bar, 1); fence_mbar_init(); }
    __syncwarp();
    if (lane == 0) mbar_arrive_expect_tx(bar, static_cast<uint32_t>(16 * (static_cast<size_t>(n) * (n + 1) / 2)));
    __syncwarp();
    for (int j = lane; j < n; j += 32)
        bulk_g2s(P + pk(j, n), Cb + j + static_cast<size_t>(j) * n, 16u * (n - j), bar);
    wait_copies(bar, info + b);
    // d, e and tau go straight to the workspace (global memory): that keeps the per-pair shared
    // memory at what eight pairs per SM allow
    double* dg = ws.d + static_cast<size_t>(n) * b;
    double* eg = ws.e + static_cast<size_t>(n) * b;
    double2* taug = ws.tau + static_cast<size_t>(n) * b;
    hetrd_warp_packed<double>(P, n, dg, eg, taug, vb, wb, vb2, wb2);
    double2* LVg = ws.LV + mat * b;
    for (int k = 0; k + 1 < n; ++k) {                    // LV(k, k+1) = v_k(k+1) = 1
        const double2* col = P + pk(k, n) - k;           // col[i] = A(i, k), i >= k
        for (int i = k + 1 + lane; i < n; i += 32)
            LVg[k + static_cast<size_t>(i) * n] = (i == k + 1) ? make_double2(1.0, 0.0) : col[i];
    }
    if (lane == 0) taug[n - 1] = make_double2(0.0, 0.0);
}

// ----------------------------------------------------------------------------- k_hetrd_warp_c64
// Mixed form, Householder stage in complex64: one WARP per pair (n <= 65).  C's lower triangle
// (FP64, in the X buffer) is rounded to complex64 into a packed tile (8 B per entry: 11.9 KB at
// n = 54, half of k_hetrd_warp's, so twice the pairs fit an SM) and tridiagonalised by
// hetrd_warp_packed<float>.  Outputs go where k_hetrd_warp puts them, promoted to FP64, so the
// FP64 eigen- and back-transform kernels run on them unchanged: reflectors in LV's rows above the
// superdiagonal, (d, e), and tau rescaled in FP64 so that each H = I - tau v v^H is unitary to
// FP64 rounding for the promoted v (|tau|^2 ||v||^2 = 2 Re tau; the FP32 tau satisfies it only to
// ~1e-7), which keeps the refinement's Y = Q Z orthonormal to the level of Z.  C itself (FP64) is
// also written to the pair's stash in the refinement's tile format (refine_stash_entries), since
// X, where the reduction left it, is overwritten before the refinement runs.
__host__ __device__ inline size_t hetrd_c64_bytes(int n) {
    return align_up(8 * static_cast<size_t>(n) * (n + 1) / 2, 16) + 8 * 4 * n + 2 * align_up(4 * n, 16) +
           align_up(8 * n, 16) + 16;
}

__device__ __forceinline__ double2* refine_stash(const Workspace& ws, int b) {
    return reinterpret_cast<double2*>(static_cast<char*>(ws.log) + 16 * static_cast<size_t>(ws.log_stride) * b);
}

__global__ void __launch_bounds__(32 * kMaxPairWarps) k_hetrd_warp_c64(int n, int batch,
                                                                              const double2* __restrict__ C,
                                                                              Workspace ws, int* __restrict__ info) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x * (blockDim.x >> 5) + warp;
    if (b >= batch) return;
    if (info[b] != 0) return;
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char* base = smem + hetrd_c64_bytes(n) * warp;
    float2* P = reinterpret_cast<float2*>(base);
    float2* vb = reinterpret_cast<float2*>(base + align_up(8 * static_cast<size_t>(n) * (n + 1) / 2, 16));
    float2* wb = vb + n;
    float2* vb2 = wb + n;
    float2* wb2 = vb2 + n;
    float* d_s = reinterpret_cast<float*>(wb2 + n);
    float* e_s = d_s + align_up(4 * n, 16) / 4;
    float2* tau_s = reinterpret_cast<float2*>(e_s + align_up(4 * n, 16) / 4);
    const size_t mat = static_cast<size_t>(n) * n;
    const double2* Cb = C + mat * b;
    // stash: C full Hermitian, planar (re plane, then im plane), column-major, ld = LD, zero padded
    const int NP = refine_np(n), LD = refine_ld(n);
    double* sre = reinterpret_cast<double*>(refine_stash(ws, b));
    double* sim = sre + static_cast<size_t>(NP) * LD;
    for (int j = 0; j < NP; ++j) {
        float2* col = P + pk(j, n) - j;
        for (int i = j + lane; i < NP; i += 32) {
            const bool in = i < n && j < n;
            double2 v = in ? Cb[i + static_cast<size_t>(j) * n] : make_double2(0.0, 0.0);
            if (i == j) v.y = 0.0;
            if (in) col[i] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
            sre[j * LD + i] = v.x;
            sim[j * LD + i] = v.y;
            if (i != j) { sre[i * LD + j] = v.x; sim[i * LD + j] = -v.y; }
        }
    }
    __syncwarp();
    hetrd_warp_packed<float, false>(P, n, d_s, e_s, tau_s, vb, wb, vb2, wb2);
    double2* LVg = ws.LV + mat * b;
    for (int k = 0; k + 1 < n; ++k) {                    // LV(k, k+1) = v_k(k+1) = 1
        const float2* col = P + pk(k, n) - k;            // col[i] = v_k(i), i >= k + 2
        double s2 = 0.0;
        for (int i = k + 1 + lane; i < n; i += 32) {
            const double2 v = (i == k + 1) ? make_double2(1.0, 0.0)
                                           : make_double2(static_cast<double>(col[i].x), static_cast<double>(col[i].y));
            LVg[k + static_cast<size_t>(i) * n] = v;
            s2 = fma(v.x, v.x, fma(v.y, v.y, s2));
        }
        s2 = warp_sum(s2);
        if (lane == 0) {
            const double tr = tau_s[k].x, ti = tau_s[k].y, t2 = tr * tr + ti * ti;
            const double sc = t2 > 0.0 ? 2.0 * tr / (t2 * s2) : 0.0;
            ws.tau[static_cast<size_t>(n) * b + k] = make_double2(tr * sc, ti * sc);
        }
    }
    for (int i = lane; i < n; i += 32) {
        ws.d[static_cast<size_t>(n) * b + i] = d_s[i];
        ws.e[static_cast<size_t>(n) * b + i] = (i + 1 < n) ? static_cast<double>(e_s[i]) : 0.0;
        if (i + 1 == n) ws.tau[static_cast<size_t>(n) * b + i] = make_double2(0.0, 0.0);
    }
}

// ----------------------------------------------------------------------------- k_ql_chain
// One THREAD per pair: the scalar QL recurrence with (d, e) in shared memory
// interleaved over the CTA, rotations appended to the pair's log.  All 32 lanes of
// a warp do useful work, so the FP64 pipe runs the chains of 32 pairs at once.
// redo: only the pairs k_tridiag_invit flagged (ws.flag == 2); they keep 2, or 3 on a log overflow.
template <typename R>
__global__ void k_ql_chain(int n, int batch, Workspace ws, double* __restrict__ W, int* __restrict__ info,
                           int redo) {
    const int tid = threadIdx.x, T = blockDim.x;
    const int b = blockIdx.x * T + tid;
    extern __shared__ __align__(16) unsigned char smem[];
    R* d = reinterpret_cast<R*>(smem) + tid;
    R* e = reinterpret_cast<R*>(smem) + static_cast<size_t>(n) * T + tid;
    if (b >= batch || !pair_selected(ws, b)) return;
    if (redo) {
        if (ws.flag[b] != 2) return;
        if (info[b] > 0 && info[b] <= n) info[b] = 0;          // QL non-convergence: run it again here
    }
    double* Wb = W + static_cast<size_t>(n) * b;
    cplx<R>* log = reinterpret_cast<cplx<R>*>(ws.log) + static_cast<size_t>(ws.log_cap) * b;
    if (!redo) ws.flag[b] = 0;
    if (info[b] != 0) {
        for (int i = 0; i < n; ++i) Wb[i] = __longlong_as_double(0x7ff8000000000000ll);
        log[0] = mk<R>(R(-1), R(0));
        return;
    }
    for (int i = 0; i < n; ++i) {
        d[i * T] = static_cast<R>(ws.d[static_cast<size_t>(n) * b + i]);
        e[i * T] = static_cast<R>(ws.e[static_cast<size_t>(n) * b + i]);
    }
    const int r = ql_chain<R>(n, d, e, T, log, ws.log_cap, ws.perm + static_cast<size_t>(n) * b, Wb);
    if (r < 0) ws.flag[b] = redo ? 3 : 1;
    else if (r > 0) info[b] = r;
}

// ----------------------------------------------------------------------------- k_ql_apply
// Applies each pair's rotation log to Z = I.  Rows of Z are independent, so a pair
// gets ceil(n / 32) warps and every lane owns ONE row (Z row-major in shared memory,
// odd leading dimension); the warps of a pair stream the log independently and never
// synchronise with each other.  The log is read 32 entries at a time (one coalesced
// load, staged in a per-warp shared buffer, read back by broadcast); within a sweep
// the rotation at column i loads z_i and carries z_{i+1} in a register.  Columns are
// written out in the sorted order of the eigenvalues.  A pair whose log overflowed is
// solved by the warp-per-pair QL on warp 0 of that pair instead.
template <typename R>
__host__ __device__ inline size_t ql_apply_pair_bytes(int n) {
    const int wpp = (n + 31) / 32;
    return align_up(sizeof(R) * static_cast<size_t>(n) * tile_ld(n), 16) +
           static_cast<size_t>(wpp) * 2 * 32 * sizeof(cplx<R>) + align_up(sizeof(R) * 2 * n, 16);
}

template <typename R>
__global__ void k_ql_apply(int n, int batch, Workspace ws, double* __restrict__ W, double2* __restrict__ X,
                           int* __restrict__ info) {
    using C = cplx<R>;
    const int wpp = (n + 31) / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pair_in_cta = warp / wpp, wip = warp - pair_in_cta * wpp;
    const int pairs_per_cta = (blockDim.x >> 5) / wpp;
    const int b = blockIdx.x * pairs_per_cta + pair_in_cta;
    extern __shared__ __align__(16) unsigned char smem[];
    const int ldz = tile_ld(n);
    unsigned char* base = smem + ql_apply_pair_bytes<R>(n) * pair_in_cta;
    R* Z = reinterpret_cast<R*>(base);
    C* stage = reinterpret_cast<C*>(base + align_up(sizeof(R) * static_cast<size_t>(n) * ldz, 16)) + wip * 64;
    R* dd = reinterpret_cast<R*>(base + align_up(sizeof(R) * static_cast<size_t>(n) * ldz, 16) +
                                 static_cast<size_t>(wpp) * 2 * 32 * sizeof(C));
    R* ee = dd + n;
    const bool live = b < batch && pair_selected(ws, b) && !(info[b] > n || info[b] < 0);
    const int row = wip * 32 + lane;
    const bool own = live && row < n;
    R* zrow = Z + row * ldz;
    if (own)
        for (int c = 0; c < n; ++c) zrow[c] = (row == c) ? R(1) : R(0);
    __syncthreads();      // every row is initialised before a fallback warp rotates all of them
    const bool fallback = live && ws.flag[b] != 0;
    if (live && !fallback)
        ql_log_apply_row<R>(reinterpret_cast<const C*>(ws.log) + static_cast<size_t>(ws.log_cap) * b, ws.log_cap,
                            stage, zrow, own);
    if (fallback && wip == 0) {
        for (int i = lane; i < n; i += 32) {
            dd[i] = static_cast<R>(ws.d[static_cast<size_t>(n) * b + i]);
            ee[i] = static_cast<R>(ws.e[static_cast<size_t>(n) * b + i]);
        }
        __syncwarp();
        const int unconv = tridiag_ql<R>(n, dd, ee, Z, ldz);
        for (int i = lane; i < n; i += 32) W[static_cast<size_t>(n) * b + i] = static_cast<double>(dd[i]);
        if (lane == 0 && unconv) info[b] = unconv;
    }
    __syncthreads();      // the fallback's warp wrote every row; all rows are final
    if (own) {
        const size_t mat = static_cast<size_t>(n) * n;
        R* Zg = reinterpret_cast<R*>(X + mat * b);
        const int* perm = ws.perm + static_cast<size_t>(n) * b;
        for (int k = 0; k < n; ++k) Zg[row + static_cast<size_t>(k) * n] = zrow[fallback ? k : perm[k]];
    }
}

// ----------------------------------------------------------------------------- k_ql_apply_reg
// The rotation log applied with each lane's row of Z in REGISTERS (n <= NMAX = 32): a sweep
// of rotations at columns col, col-1, ... enters an unrolled descending chain at case col
// (every register index static) and updates (z_i, z_{i+1}) in place; the stage buffer
// streaming is ql_log_apply_row's.  The columns are stored through the inverse sort
// permutation (z[c] -> column pinv[c]), so no register is ever indexed at run time.  A pair
// whose log overflowed is solved by the warp QL on its first warp with Z in the second half
// of the pair's X slice (no shared-memory Z tile is kept for it).
template <typename R>
__host__ __device__ inline size_t ql_apply_reg_pair_bytes(int n) {
    const int wpp = (n + 31) / 32;
    return static_cast<size_t>(wpp) * 2 * 32 * sizeof(cplx<R>) + align_up(4 * static_cast<size_t>(n), 16) +
           align_up(sizeof(R) * 2 * static_cast<size_t>(n), 16);
}

template <int NMAX, typename R>
__global__ void k_ql_apply_reg(int n, int batch, Workspace ws, double* __restrict__ W, double2* __restrict__ X,
                               int* __restrict__ info) {
    using C = cplx<R>;
    const int wpp = (n + 31) / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pair_in_cta = warp / wpp, wip = warp - pair_in_cta * wpp;
    const int pairs_per_cta = (blockDim.x >> 5) / wpp;
    const int b = blockIdx.x * pairs_per_cta + pair_in_cta;
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char* base = smem + ql_apply_reg_pair_bytes<R>(n) * pair_in_cta;
    C* stage = reinterpret_cast<C*>(base) + wip * 64;
    int* pinv = reinterpret_cast<int*>(base + static_cast<size_t>(wpp) * 2 * 32 * sizeof(C));
    R* dd = reinterpret_cast<R*>(base + static_cast<size_t>(wpp) * 2 * 32 * sizeof(C) + align_up(4 * static_cast<size_t>(n), 16));
    R* ee = dd + n;
    const bool live = b < batch && !(info[min(b, batch - 1)] > n || info[min(b, batch - 1)] < 0);
    const bool fallback = live && ws.flag[b] != 0;
    const int row = wip * 32 + lane;
    const bool own = live && row < n;
    R z[NMAX];
#pragma unroll
    for (int c = 0; c < NMAX; ++c) z[c] = (row == c) ? R(1) : R(0);
    if (live && !fallback) {
        const C* log = reinterpret_cast<const C*>(ws.log) + static_cast<size_t>(ws.log_cap) * b;
        const int cap = ws.log_cap;
        int loaded = 0, buf = 0, remaining = 0, col = 0;
        C pre = log[lane];
        bool done = false;
        while (!done) {
            stage[buf * 32 + lane] = pre;
            __syncwarp();
            loaded += 32;
            if (loaded < cap) pre = log[min(loaded + lane, cap - 1)];
            const C* st = stage + buf * 32;
            int k = 0;
            while (k < 32) {
                if (remaining == 0) {
                    const C h = st[k++];
                    const int top = static_cast<int>(h.x);
                    if (top < 0) { done = true; break; }
                    remaining = static_cast<int>(h.y);
                    col = top;
                    continue;
                }
                const int take = min(remaining, 32 - k);
                const C* e = st + k;
                int rem = take;
                // rotation at column I: (z_I, z_{I+1}) <- (c z_I - s z_{I+1}, s z_I + c z_{I+1})
#define SBG_ROT(I) case I: if constexpr ((I) + 1 < NMAX) { if (rem == 0) break; const C cs = *e++; \
                const R zi = z[I], zj = z[(I) + 1]; z[(I) + 1] = fma(cs.y, zi, cs.x * zj); \
                z[I] = fma(cs.x, zi, -cs.y * zj); --rem; }
                switch (col) { SBG_DESC64(SBG_ROT) default: break; }
#undef SBG_ROT
                k += take;
                col -= take;
                remaining -= take;
            }
            __syncwarp();
            buf ^= 1;
            if (!done && loaded >= cap) done = true;      // malformed log guard (never reached)
        }
    }
    // inverse sort permutation, by the pair's threads
    if (live && !fallback) {
        const int* perm = ws.perm + static_cast<size_t>(n) * b;
        for (int i = wip * 32 + lane; i < n; i += wpp * 32) pinv[perm[i]] = i;
    }
    __syncthreads();
    const size_t mat = static_cast<size_t>(n) * n;
    if (fallback) {
        if (wip != 0) return;
        R* Zs = reinterpret_cast<R*>(reinterpret_cast<unsigned char*>(X + mat * b) + 8 * mat);   // row-major, ld n
        for (size_t idx = lane; idx < mat; idx += 32) Zs[idx] = (idx / n == idx % n) ? R(1) : R(0);
        for (int i = lane; i < n; i += 32) {
            dd[i] = static_cast<R>(ws.d[static_cast<size_t>(n) * b + i]);
            ee[i] = static_cast<R>(ws.e[static_cast<size_t>(n) * b + i]);
        }
        __syncwarp();
        const int unconv = tridiag_ql<R>(n, dd, ee, Zs, n);
        for (int i = lane; i < n; i += 32) W[static_cast<size_t>(n) * b + i] = static_cast<double>(dd[i]);
        if (lane == 0 && unconv) info[b] = unconv;
        __syncwarp();
        R* Zg = reinterpret_cast<R*>(X + mat * b);
        for (int r = lane; r < n; r += 32)
            for (int k = 0; k < n; ++k) Zg[r + static_cast<size_t>(k) * n] = Zs[static_cast<size_t>(r) * n + k];
        return;
    }
    if (own) {
        R* Zg = reinterpret_cast<R*>(X + mat * b);
#pragma unroll
        for (int c = 0; c < NMAX; ++c)
            if (c < n) Zg[row + static_cast<size_t>(pinv[c]) * n] = z[c];
    }
}

// ----------------------------------------------------------------------------- k_ql_values
// The QL chain of k_ql_chain (one thread per pair) for the eigenvalues only: no rotation log,
// no permutation; W ascending.  Feeds k_tridiag_invit.
__global__ void k_ql_values(int n, int batch, Workspace ws, double* __restrict__ W, int* __restrict__ info) {
    const int tid = threadIdx.x, T = blockDim.x;
    const int b = blockIdx.x * T + tid;
    extern __shared__ __align__(16) unsigned char smem[];
    double* d = reinterpret_cast<double*>(smem) + tid;
    double* e = reinterpret_cast<double*>(smem) + static_cast<size_t>(n) * T + tid;
    if (b >= batch || !pair_selected(ws, b)) return;
    double* Wb = W + static_cast<size_t>(n) * b;
    if (info[b] != 0) {
        for (int i = 0; i < n; ++i) Wb[i] = __longlong_as_double(0x7ff8000000000000ll);
        return;
    }
    for (int i = 0; i < n; ++i) {
        d[i * T] = ws.d[static_cast<size_t>(n) * b + i];
        e[i * T] = ws.e[static_cast<size_t>(n) * b + i];
    }
    const int r = ql_chain<double, false>(n, d, e, T, nullptr, 0, nullptr, Wb);
    if (r > 0) info[b] = r;
}

// ----------------------------------------------------------------------------- k_tridiag_invit
// Eigenvectors of the tridiagonal T (d, e) from its FP64 eigenvalues (k_ql_values) by inverse
// iteration, one warp per pair, one lane per eigenvector at a time (LAPACK dstein's method):
// T - lambda_j I = L U without pivoting, a pivot below eps ||T|| replaced by that size, two
// solves from a fixed pseudo-random start, each followed by normalisation.  That is O(n) work
// per vector against the O(n^2) of applying every QL rotation to it.  The vectors of
// eigenvalues closer than kInvitOrtol ||T|| (a cluster) are computed in order, one lane per
// cluster, with three solves each orthogonalised against the cluster's earlier vectors
// (modified Gram-Schmidt); the other vectors' orthogonality is ~eps ||T|| / gap.  Every
// vector must pass ||T z - lambda z|| <= kInvitTol ||T||; a pair with a failed vector, a
// cluster of more than kInvitMaxCluster eigenvalues (a spectrum dominated by one huge
// eigenvalue), or a QL chain that did not converge is recomputed by the warp QL instead.
// Per-lane scratch (1/u and the vector) is interleaved [i * 33 + lane]: lane-parallel
// recurrences read consecutive words, and the warp's column-by-column copy to the caller's X
// buffer (Z, column k = vector k) reads it across lanes without bank conflicts.
constexpr double kInvitOrtol = 3e-4;
constexpr int kInvitMaxCluster = 8;
constexpr double kInvitTol = 256.0 * 1.1102230246251565e-16;
constexpr int kInvitLd = 33;            // lane scratch [i * 33 + lane]: rows also read across lanes

struct InvitSmem {
    size_t scr, dd, ee, lam, cls, mem, flag, per_warp;
    // with_tile: the scratch also holds the in-kernel fallback QL's Z tile
    __host__ __device__ explicit InvitSmem(int n, bool with_tile = true) {
        size_t o = 0;
        const size_t lanes = 2 * kInvitLd * static_cast<size_t>(n), tile = static_cast<size_t>(n) * tile_ld(n);
        scr = o;  o += 8 * (with_tile && tile > lanes ? tile : lanes);
        dd = o;   o += 8 * static_cast<size_t>(n);
        ee = o;   o += 8 * static_cast<size_t>(n);
        lam = o;  o += 8 * static_cast<size_t>(n);
        cls = o;  o += align_up(4 * static_cast<size_t>(n), 16);
        mem = o;  o += 4 * 32;
        flag = o; o += 16;
        per_warp = o;
    }
};

__device__ __forceinline__ double invit_start(int j, int i) {
    unsigned h = static_cast<unsigned>(i + 1) * 0x9E3779B1u ^ static_cast<unsigned>(j + 1) * 0x85EBCA77u;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    return static_cast<double>(h & 0xFFFFFu) * (2.0 / 1048575.0) - 1.0;
}

// Per-lane pieces of inverse iteration on T - lam I; invu and z are the lane's columns of the
// interleaved scratch ([i * kInvitLd + lane]).
#define SBG_IU(i) invu[(i) * kInvitLd + lane]
#define SBG_ZV(i) z[(i) * kInvitLd + lane]
// T - lam I = L U without pivoting (pivots below `tiny` raised to it): keeps 1/u_i.  Each step's
// operands are loaded one step ahead, so the dependent chain is only the recurrence itself.
__device__ __forceinline__ void invit_factor(int n, double lam, const double* __restrict__ dd,
                                             const double* __restrict__ ee, double tiny, double* __restrict__ invu) {
    const int lane = threadIdx.x & 31;
    double u = dd[0] - lam;
    if (fabs(u) < tiny) u = copysign(tiny, u);
    double iu = recip_nr(u);
    SBG_IU(0) = iu;
    double dn = n > 1 ? dd[1] - lam : 0.0, en = n > 1 ? ee[0] * ee[0] : 0.0;
    for (int i = 1; i < n; ++i) {
        const double di = dn, e2 = en;
        if (i + 1 < n) { dn = dd[i + 1] - lam; en = ee[i] * ee[i]; }
        u = fma(-e2, iu, di);
        if (fabs(u) < tiny) u = copysign(tiny, u);
        iu = recip_nr(u);
        SBG_IU(i) = iu;
    }
}
// z <- (T - lam I)^{-1} x with the factors above, x = sc z, or (GEN) the start vector of eigenvalue
// j; returns ||z||^2 (summed in the backward pass).  Operands are loaded one step ahead.
template <bool GEN>
__device__ __forceinline__ double invit_solve(int n, const double* __restrict__ ee, const double* __restrict__ invu,
                                              double* __restrict__ z, double sc, int j) {
    const int lane = threadIdx.x & 31;
    auto xin = [&](int i) { if constexpr (GEN) return invit_start(j, i); else return sc * SBG_ZV(i); };
    double y = xin(0);
    SBG_ZV(0) = y;
    double xn = n > 1 ? xin(1) : 0.0, cn = n > 1 ? ee[0] * SBG_IU(0) : 0.0;
    for (int i = 1; i < n; ++i) {                      // L y = x  (L(i, i-1) = e_{i-1} / u_{i-1})
        const double x = xn, c = cn;
        if (i + 1 < n) { xn = xin(i + 1); cn = ee[i] * SBG_IU(i); }
        y = fma(-c, y, x);
        SBG_ZV(i) = y;
    }
    double zn = y * SBG_IU(n - 1);                     // U z = y  (U(i, i+1) = e_i)
    SBG_ZV(n - 1) = zn;
    double s2 = zn * zn;
    double yp = n > 1 ? SBG_ZV(n - 2) : 0.0, ep = n > 1 ? ee[n - 2] : 0.0, ip = n > 1 ? SBG_IU(n - 2) : 0.0;
    for (int i = n - 2; i >= 0; --i) {
        const double yi = yp, ei = ep, ii = ip;
        if (i > 0) { yp = SBG_ZV(i - 1); ep = ee[i - 1]; ip = SBG_IU(i - 1); }
        zn = fma(-ei, zn, yi) * ii;
        SBG_ZV(i) = zn;
        s2 = fma(zn, zn, s2);
    }
    return s2;
}
// z <- sc z in place; returns ||T z - lam z||^2 of the scaled vector (one pass).
__device__ __forceinline__ double invit_scale_residual(int n, double lam, const double* __restrict__ dd,
                                                       const double* __restrict__ ee, double* __restrict__ z,
                                                       double sc) {
    const int lane = threadIdx.x & 31;
    double zp = 0.0, zc = SBG_ZV(0), r2 = 0.0;
    for (int i = 0; i < n; ++i) {
        const double zx = i + 1 < n ? SBG_ZV(i + 1) : 0.0;
        double v = (dd[i] - lam) * zc;
        if (i > 0) v = fma(ee[i - 1], zp, v);
        if (i + 1 < n) v = fma(ee[i], zx, v);
        r2 = fma(v, v, r2);
        SBG_ZV(i) = zc * sc;
        zp = zc;
        zc = zx;
    }
    return r2 * sc * sc;
}
#undef SBG_IU
#undef SBG_ZV

// flag_redo: a pair the kernel cannot take gets ws.flag = 2 and no output (the rotation-log QL is
// then run for the flagged pairs); otherwise the warp QL runs here, on a Z tile in the scratch.
__global__ void __launch_bounds__(32) k_tridiag_invit(int n, int batch, Workspace ws, double* __restrict__ W,
                                                      double2* __restrict__ X, int* __restrict__ info,
                                                      int flag_redo) {
    const int b = blockIdx.x, lane = threadIdx.x & 31;
    if (b >= batch || !pair_selected(ws, b)) return;
    if (flag_redo && lane == 0) ws.flag[b] = 0;
    const int inf = info[b];
    if (inf > n || inf < 0) return;                   // an earlier stage failed: W and X are NaN
    extern __shared__ __align__(16) unsigned char smem[];
    const InvitSmem lay(n, !flag_redo);
    double* scr = reinterpret_cast<double*>(smem + lay.scr);
    double* dd = reinterpret_cast<double*>(smem + lay.dd);
    double* ee = reinterpret_cast<double*>(smem + lay.ee);
    double* lam = reinterpret_cast<double*>(smem + lay.lam);
    int* cls = reinterpret_cast<int*>(smem + lay.cls);
    int* members = reinterpret_cast<int*>(smem + lay.mem);
    int* sflag = reinterpret_cast<int*>(smem + lay.flag);
    double* Wb = W + static_cast<size_t>(n) * b;
    double* Zg = reinterpret_cast<double*>(X + static_cast<size_t>(n) * n * b);
    double rs = 0.0;
    for (int i = lane; i < n; i += 32) {
        dd[i] = ws.d[static_cast<size_t>(n) * b + i];
        ee[i] = ws.e[static_cast<size_t>(n) * b + i];
        lam[i] = Wb[i];
    }
    __syncwarp();
    for (int i = lane; i < n; i += 32) {
        double v = fabs(dd[i]);
        if (i > 0) v += fabs(ee[i - 1]);
        if (i + 1 < n) v += fabs(ee[i]);
        rs = fmax(rs, v);
    }
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) rs = fmax(rs, shfl_xor(rs, m));
    const double tnorm = rs > 0.0 && isfinite(rs) ? rs : 1.0;
    const double tiny = 1.1102230246251565e-16 * tnorm;
    if (lane == 0) {                                  // clusters: cls[j] = index of the first member
        int start = 0, biggest = 1, cnt = 0;
        for (int j = 0; j < n; ++j) {
            if (j > 0 && !(lam[j] - lam[j - 1] <= kInvitOrtol * tnorm)) start = j;
            cls[j] = start;
            biggest = max(biggest, j - start + 1);
            if (start != j) { if (cnt < 32) members[cnt] = j; ++cnt; }
        }
        sflag[0] = biggest;
        sflag[1] = cnt;
    }
    __syncwarp();
    const int cnt = sflag[1];
    bool fallback = inf != 0 || sflag[0] > kInvitMaxCluster || cnt > 32;
    if (!fallback) {
        bool ok = true;
        double* invu = scr;
        double* zs = scr + kInvitLd * n;
        // (1) each cluster's first vector and every singleton: factor, two solves from a fixed
        // pseudo-random start, residual test; 32 at a time, then copied out column by column
        for (int base = 0; base < n; base += 32) {
            const int j = base + lane;
            if (j < n && cls[j] == j) {
                invit_factor(n, lam[j], dd, ee, tiny, invu);
                double s2 = invit_solve<true>(n, ee, invu, zs, 1.0, j);
                const bool f1 = s2 > 0.0 && isfinite(s2);
                s2 = invit_solve<false>(n, ee, invu, zs, f1 ? 1.0 / sqrt(s2) : 1.0, j);
                const bool f2 = s2 > 0.0 && isfinite(s2);
                const double r2 = invit_scale_residual(n, lam[j], dd, ee, zs, f2 ? 1.0 / sqrt(s2) : 1.0);
                ok &= f1 && f2 && sqrt(r2) <= kInvitTol * tnorm;
            }
            __syncwarp();
            const int top = min(32, n - base);
            for (int L = 0; L < top; ++L) {
                const int jj = base + L;
                if (cls[jj] != jj) continue;          // uniform
                double* zc = Zg + static_cast<size_t>(jj) * n;
                for (int i = lane; i < n; i += 32) zc[i] = zs[i * kInvitLd + L];
            }
            __syncwarp();
        }
        ok = __all_sync(0xffffffffu, ok);              // from here on `ok` is the same on every lane
        // (2) the other cluster members, one lane each, all at once: three rounds of a solve
        // (every lane its own member) and modified Gram-Schmidt in index order (the whole warp,
        // lanes over rows) against the cluster's first vector and its earlier members
        if (ok && cnt > 0) {
            const int jm = lane < cnt ? members[lane] : -1;
            if (jm >= 0) {
                invit_factor(n, lam[jm], dd, ee, tiny, invu);
            }
            for (int it = 0; it < 3 && ok; ++it) {        // each round's input is unit (Gram-Schmidt below)
                if (jm >= 0) {
                    if (it == 0) invit_solve<true>(n, ee, invu, zs, 1.0, jm);
                    else invit_solve<false>(n, ee, invu, zs, 1.0, jm);
                }
                __syncwarp();
                for (int m = 0; m < cnt && ok; ++m) {
                    const int j = members[m], s0 = cls[j];
                    const double* q0 = Zg + static_cast<size_t>(s0) * n;
                    double c = 0.0;
                    for (int i = lane; i < n; i += 32) c = fma(q0[i], zs[i * kInvitLd + m], c);
                    c = warp_sum(c);
                    for (int i = lane; i < n; i += 32) zs[i * kInvitLd + m] = fma(-c, q0[i], zs[i * kInvitLd + m]);
                    for (int m2 = 0; m2 < m; ++m2) {
                        if (cls[members[m2]] != s0) continue;     // uniform
                        double c2 = 0.0;
                        for (int i = lane; i < n; i += 32) c2 = fma(zs[i * kInvitLd + m2], zs[i * kInvitLd + m], c2);
                        c2 = warp_sum(c2);
                        for (int i = lane; i < n; i += 32)
                            zs[i * kInvitLd + m] = fma(-c2, zs[i * kInvitLd + m2], zs[i * kInvitLd + m]);
                    }
                    double s2 = 0.0;
                    for (int i = lane; i < n; i += 32) s2 = fma(zs[i * kInvitLd + m], zs[i * kInvitLd + m], s2);
                    s2 = warp_sum(s2);
                    if (!(s2 > 0.0) || !isfinite(s2)) { ok = false; break; }     // uniform
                    const double inv = 1.0 / sqrt(s2);
                    for (int i = lane; i < n; i += 32) zs[i * kInvitLd + m] *= inv;
                }
                __syncwarp();
            }
            if (jm >= 0 && ok) ok &= sqrt(invit_scale_residual(n, lam[jm], dd, ee, zs, 1.0)) <= kInvitTol * tnorm;
            for (int m = 0; m < cnt; ++m) {
                double* zc = Zg + static_cast<size_t>(members[m]) * n;
                for (int i = lane; i < n; i += 32) zc[i] = zs[i * kInvitLd + m];
            }
        }
        fallback = !__all_sync(0xffffffffu, ok);
    }
    if (fallback && flag_redo) {
        if (lane == 0) ws.flag[b] = 2;
        return;
    }
    if (fallback) {                                   // the warp QL, Z tile over the lane scratch
        const int ldz = tile_ld(n);
        __syncwarp();
        for (int r = lane; r < n; r += 32)
            for (int c = 0; c < n; ++c) scr[r * ldz + c] = (r == c) ? 1.0 : 0.0;
        for (int i = lane; i < n; i += 32) {
            dd[i] = ws.d[static_cast<size_t>(n) * b + i];
            ee[i] = ws.e[static_cast<size_t>(n) * b + i];
        }
        __syncwarp();
        const int unconv = tridiag_ql<double>(n, dd, ee, scr, ldz);
        __syncwarp();
        for (int i = lane; i < n; i += 32) Wb[i] = dd[i];
        for (int r = lane; r < n; r += 32)
            for (int k = 0; k < n; ++k) Zg[r + static_cast<size_t>(k) * n] = scr[r * ldz + k];
        if (lane == 0) info[b] = unconv;
    }
}

// ----------------------------------------------------------------------------- k_back
// One CTA per pair: X = L^{-H} Q Z.  Column j of Z is held in registers by a group
// of G lanes (lane g owns rows g + G r), read straight from the X buffer; only the
// LV tile (L below, reflectors above the superdiagonal) is staged in shared memory
// by TMA bulk copies.  The result is written over Z.

template <int T, int G, int RM>
__global__ void __launch_bounds__(T, RM <= 8 ? 2 : 1) k_back(int mode, int n, int batch, Workspace ws,
                                            double2* __restrict__ X, int* __restrict__ info) {
    const int b = blockIdx.x;
    if (b >= batch || !pair_selected(ws, b)) return;
    const size_t mat = static_cast<size_t>(n) * n;
    double2* Xb = X + mat * b;
    const int tid = threadIdx.x;
    if (info[b] > n || info[b] < 0) {     // B not positive definite: nothing to transform
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        for (size_t idx = tid; idx < mat; idx += T) Xb[idx] = make_double2(nan, nan);
        return;
    }
    extern __shared__ __align__(16) unsigned char smem[];
    const BackSmem lay(n);
    const int ld = tile_ld(n);
    double2* LVs = reinterpret_cast<double2*>(smem + lay.LVs);
    double* invd = reinterpret_cast<double*>(smem + lay.invd);
    double2* tau_s = reinterpret_cast<double2*>(smem + lay.tau);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + lay.bar);

    const double2* LVg = ws.LV + mat * b;
    if (tid == 0) { mbar_init(bar, 1); fence_mbar_init(); }
    __syncthreads();
    if (tid < 32) {
        if (tid == 0) mbar_arrive_expect_tx(bar, static_cast<uint32_t>(16 * mat));
        __syncwarp();
        for (int j = tid; j < n; j += 32)
            bulk_g2s(LVs + static_cast<size_t>(j) * ld, LVg + static_cast<size_t>(j) * n, 16u * n, bar);
    }
    const int g = tid % G, j = tid / G;
    const bool valid = j < n;
    const double* Zg = reinterpret_cast<const double*>(Xb);
    double2 y[RM];
#pragma unroll
    for (int r = 0; r < RM; ++r) {
        const int i = g + G * r;
        if (mode == kBackLOnly)            // complex Y in the X buffer
            y[r] = (valid && i < n) ? Xb[i + static_cast<size_t>(j) * n] : make_double2(0.0, 0.0);
        else                               // real Z in the X buffer
            y[r] = make_double2((valid && i < n) ? Zg[i + static_cast<size_t>(j) * n] : 0.0, 0.0);
    }
    for (int i = tid; i < n; i += T) tau_s[i] = ws.tau[static_cast<size_t>(n) * b + i];
    wait_copies(bar, info + b);
    for (int i = tid; i < n; i += T) invd[i] = 1.0 / LVs[i + i * ld].x;
    __syncthreads();              // also: every thread has read its Z before any X is written
    if (mode != kBackLOnly) seg_apply_q<G, RM>(LVs, ld, tau_s, y, n, g);
    if (mode == kBackFull || mode == kBackLOnly) seg_trsm_lowerH<G, RM>(LVs, ld, invd, y, n, g);
    if (valid) {
#pragma unroll
        for (int r = 0; r < RM; ++r) {
            const int i = g + G * r;
            if (i < n) Xb[i + static_cast<size_t>(j) * n] = y[r];
        }
    }
}

// Pairs (warps) per CTA of the warp-per-pair kernels: 1, 2 or 4 (anything else: the default 2).
inline int pair_warps_of(const LaunchShape& s) {
    return (s.pair_warps == 1 || s.pair_warps == 2 || s.pair_warps == 4) ? s.pair_warps : 2;
}

template <class K>
void set_max_smem_once(K kernel, SmemOptIn& rec) {
    set_smem_limit(reinterpret_cast<const void*>(kernel), rec, max_smem_optin());
}

}  // namespace

// ============================================================================== host side

int ql_log_capacity(int n) {
    const int dflt = (3 * n * n) / 2 + 8 * n + 16;
    if (const char* v = std::getenv("SBG_QL_LOG_CAPACITY")) {
        const int c = std::atoi(v);
        if (c >= 16 && c < dflt) return c;
    }
    return dflt;
}

size_t workspace_bytes_per_pair(int n, bool mixed) {
    const size_t nn = static_cast<size_t>(n) * n;
    // the default (largest) rotation-log capacity, or the mixed form's stash if that is larger
    const size_t cap = static_cast<size_t>(std::max((3 * n * n) / 2 + 8 * n + 16, refine_stash_entries(n)));
    const size_t refine = mixed_big(n, mixed) ? 5 * 16 * nn + 4 : 0;
    return 16 * nn + 16 * n + 8 * n * 2 + 16 * cap + 4 * n + 4 + refine;
}

namespace {
// Byte offsets of the workspace's regions from its base, each rounded up to 256 bytes: seven,
// and for the mixed form above kMixedMaxN six more (the refinement's matrices and status).
struct WorkspaceLayout {
    size_t LV, tau, d, e, log, perm, flag, rfC = 0, rfY = 0, rfP = 0, rfG = 0, rfS = 0, rstat = 0, end;
    int log_cap, log_stride;
    bool refine;
    WorkspaceLayout(int n, int capacity, bool mixed) {
        const size_t nn = static_cast<size_t>(n) * n, cap = static_cast<size_t>(capacity);
        log_cap = ql_log_capacity(n);
        log_stride = std::max(std::max(log_cap, refine_stash_entries(n)), tc_scratch_entries(n));
        refine = mixed_big(n, mixed);
        size_t o = 0;
        auto take = [&](size_t bytes) { const size_t q = o; o += align_up(bytes, 256); return q; };
        LV = take(16 * nn * cap);
        tau = take(16 * n * cap);
        d = take(8 * n * cap);
        e = take(8 * n * cap);
        log = take(16 * static_cast<size_t>(log_stride) * cap);
        perm = take(4 * n * cap);
        flag = take(4 * cap);
        if (refine) {
            rfC = take(16 * nn * cap);
            rfY = take(16 * nn * cap);
            rfP = take(16 * nn * cap);
            rfG = take(16 * nn * cap);
            rfS = take(16 * nn * cap);
            rstat = take(4 * cap);
        }
        end = o;
    }
};
}  // namespace

size_t workspace_bytes(int n, int capacity, bool mixed) { return WorkspaceLayout(n, capacity, mixed).end; }

Workspace carve_workspace(void* base, int n, int capacity, bool mixed) {
    const WorkspaceLayout lay(n, capacity, mixed);
    char* p = static_cast<char*>(base);
    Workspace w;
    w.n = n;
    w.capacity = capacity;
    w.LV = reinterpret_cast<double2*>(p + lay.LV);
    w.tau = reinterpret_cast<double2*>(p + lay.tau);
    w.d = reinterpret_cast<double*>(p + lay.d);
    w.e = reinterpret_cast<double*>(p + lay.e);
    w.log_cap = lay.log_cap;
    w.log_stride = lay.log_stride;
    w.log = p + lay.log;
    w.perm = reinterpret_cast<int*>(p + lay.perm);
    w.flag = reinterpret_cast<int*>(p + lay.flag);
    if (lay.refine) {
        w.rfC = reinterpret_cast<double2*>(p + lay.rfC);
        w.rfY = reinterpret_cast<double2*>(p + lay.rfY);
        w.rfP = reinterpret_cast<double2*>(p + lay.rfP);
        w.rfG = reinterpret_cast<double2*>(p + lay.rfG);
        w.rfS = reinterpret_cast<double2*>(p + lay.rfS);
        w.rstat = reinterpret_cast<int*>(p + lay.rstat);
    }
    return w;
}

int max_smem_optin() {
    // per device ordinal (devices can differ); 0 = not yet queried
    static std::atomic<int> cache[SmemOptIn::kDevices];
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return 0; }
    if (dev >= 0 && dev < SmemOptIn::kDevices && (v = cache[dev].load(std::memory_order_relaxed)) > 0) return v;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (dev >= 0 && dev < SmemOptIn::kDevices) cache[dev].store(v, std::memory_order_relaxed);
    return v;
}

void set_smem_limit(const void* kernel, SmemOptIn& rec, int bytes) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return; }
    const bool tracked = dev >= 0 && dev < SmemOptIn::kDevices;
    if (tracked && rec.raised[dev].load(std::memory_order_acquire) >= bytes) return;
    // Idempotent: two threads that race here both set the same limit.  A failure is left for
    // the launch to report (it fails with the limit unraised).
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    if (!tracked) return;
    int cur = rec.raised[dev].load(std::memory_order_relaxed);
    while (cur < bytes && !rec.raised[dev].compare_exchange_weak(cur, bytes, std::memory_order_acq_rel)) {
    }
}

size_t reduce_smem_bytes(int, int n) { return ReduceSmem(n).total; }
size_t back_smem_bytes(int n) { return BackSmem(n).total; }
size_t invit_smem_bytes(int n, bool with_tile) { return InvitSmem(n, with_tile).per_warp; }

// The register-segment kernels: (threads T, lanes per column G, rows per lane RM) by
// size: n <= 32 -> (256, 8, 4), n <= 64 -> (512, 8, 8), else (512, 4, 22) (n <= 88).
#define SBG_DISPATCH_BY_N(n, KERNEL, ...)                                              \
    do {                                                                               \
        if ((n) <= 32) { KERNEL<256, 8, 4>(__VA_ARGS__); }                             \
        else if ((n) <= 64) { KERNEL<512, 8, 8>(__VA_ARGS__); }                        \
        else { KERNEL<512, 4, 22>(__VA_ARGS__); }                                      \
    } while (0)

template <int T, int G, int RM>
void run_reduce(int mode, const double2* A, const double2* B, int n, int batch, const Workspace& ws, double2* out,
                int* info, size_t smem, cudaStream_t stream) {
    static SmemOptIn f;
    set_max_smem_once(k_reduce<T, G, RM>, f);
    k_reduce<T, G, RM><<<batch, T, smem, stream>>>(mode, A, B, n, batch, ws, out, info);
}

template <int T, int G, int RM>
void run_back(int mode, int n, int batch, const Workspace& ws, double2* X, int* info, size_t smem,
              cudaStream_t stream) {
    static SmemOptIn f;
    set_max_smem_once(k_back<T, G, RM>, f);
    k_back<T, G, RM><<<batch, T, smem, stream>>>(mode, n, batch, ws, X, info);
}

template <int NMAX, bool EXACT = false>
void run_hegst_col(int mode, const double2* A, const Workspace& ws, double2* out, int n, int batch, int* info,
                   cudaStream_t stream) {
    static SmemOptIn f;
    set_max_smem_once(k_hegst_col<NMAX, EXACT>, f);
    k_hegst_col<NMAX, EXACT><<<batch, NMAX, hegst_col_bytes(n), stream>>>(mode, A, ws, out, n, batch, info);
}

cudaError_t launch_reduce(int mode, const double2* A, const double2* B, int n, int batch,
                          const Workspace& ws, double2* out, int* info, const LaunchShape& shape, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    // kReduceMixed is kReduceFull that, above kSmallMaxN, stops before the tridiagonalisation
    // (below it the reduction never tridiagonalises)
    const bool hegst_only = mode == kReduceMixed;
    if (hegst_only) mode = kReduceFull;
    if (!B || !info) return cudaErrorInvalidValue;
    if ((mode == kReduceChol || mode == kReduceHegst || mode == kReduceFull) && !out) return cudaErrorInvalidValue;
    if ((mode == kReduceHegst || mode == kReduceFull) && !A) return cudaErrorInvalidValue;
    if ((mode == kReduceFull || mode == kReduceFromLM) && !ws.LV) return cudaErrorInvalidValue;
    if (n > kSmallMaxN) {
        if (mode != kReduceFull) return cudaErrorInvalidValue;
        if (shape.reduce_tc) {                       // tensor-core Cholesky + reduction, then the Householder
            cudaError_t err = launch_reduce_tc(A, B, n, batch, ws, out, info, stream);
            if (err != cudaSuccess || hegst_only) return err;
            return launch_reduce_big(A, B, n, batch, ws, out, info, stream, kBigHetrdOnly);
        }
        return launch_reduce_big(A, B, n, batch, ws, out, info, stream, hegst_only ? kBigHegstOnly : kBigFull);
    }
    // The two-kernel path hands L from k_potrf_warp to k_hegst_col through ws.LV, so it
    // needs a workspace (the staged Cholesky alone does not).
    if (n <= kColMaxN && mode != kReduceFromLM && (mode == kReduceChol || ws.LV != nullptr)) {
        const int pw = pair_warps_of(shape);
        static SmemOptIn fp;
        set_max_smem_once(k_potrf_warp, fp);
        const int grid = (batch + pw - 1) / pw;
        k_potrf_warp<<<grid, 32 * pw, potrf_warp_bytes(n) * pw, stream>>>(mode, B, n, batch, ws, out, info);
        if (mode == kReduceChol) return cudaGetLastError();
        if (n == 32 && shape.col_exact) run_hegst_col<32, true>(mode, A, ws, out, n, batch, info, stream);
        else if (n == 54 && shape.col_exact) run_hegst_col<54, true>(mode, A, ws, out, n, batch, info, stream);
        else if (n <= 32) run_hegst_col<32>(mode, A, ws, out, n, batch, info, stream);
        else if (n <= 48) run_hegst_col<48>(mode, A, ws, out, n, batch, info, stream);
        else run_hegst_col<56>(mode, A, ws, out, n, batch, info, stream);
        return cudaGetLastError();
    }
    // 57 <= n <= 84 with the tensor-core triangular stages: the blocked Cholesky and reduction
    // (the Householder is a separate kernel here anyway)
    if (shape.reduce_tc && mode == kReduceFull) return launch_reduce_tc(A, B, n, batch, ws, out, info, stream);
    const size_t smem = reduce_smem_bytes(mode, n);
    if (smem > static_cast<size_t>(max_smem_optin())) return cudaErrorInvalidValue;
    SBG_DISPATCH_BY_N(n, run_reduce, mode, A, B, n, batch, ws, out, info, smem, stream);
    return cudaGetLastError();
}

size_t hetrd_smem_bytes(int n, int threads) { return HetrdSmem(n, threads).total; }

cudaError_t launch_hetrd(int n, int batch, const double2* C, const Workspace& ws, int* info, const LaunchShape& shape,
                         cudaStream_t stream) {
    const int threads = shape.threads;
    if (batch <= 0) return cudaSuccess;
    if (!C || !info || !ws.LV || !ws.d || !ws.e || !ws.tau) return cudaErrorInvalidValue;
    if (n > kSmallMaxN) return big_path(n) ? cudaSuccess : cudaErrorInvalidValue;   // done by the reduce kernel
    if (n <= kHetrdWarpMaxN) {
        const int pw = pair_warps_of(shape);
        const size_t smem = hetrd_warp_bytes(n) * pw;
        if (smem > static_cast<size_t>(max_smem_optin())) return cudaErrorInvalidValue;
        static SmemOptIn fw;
        set_max_smem_once(k_hetrd_warp, fw);
        k_hetrd_warp<<<(batch + pw - 1) / pw, 32 * pw, smem, stream>>>(n, batch, C, ws, info);
        return cudaGetLastError();
    }
    const size_t smem = hetrd_smem_bytes(n, threads == 128 ? 128 : 256);
    if (smem > static_cast<size_t>(max_smem_optin())) return cudaErrorInvalidValue;
    static SmemOptIn f128, f256;
    if (threads == 128) {
        set_max_smem_once(k_hetrd<128>, f128);
        k_hetrd<128><<<batch, 128, smem, stream>>>(n, batch, C, ws, info);
    } else {
        set_max_smem_once(k_hetrd<256>, f256);
        k_hetrd<256><<<batch, 256, smem, stream>>>(n, batch, C, ws, info);
    }
    return cudaGetLastError();
}


size_t ql_chain_smem_bytes(int n, int threads, bool single) {
    return (single ? 4 : 8) * 2 * static_cast<size_t>(n) * threads;
}
// pairs_per_cta pairs of ceil(n / 32) warps each share a CTA.
size_t ql_apply_smem_bytes(int n, int pairs_per_cta, bool single) {
    return (single ? ql_apply_pair_bytes<float>(n) : ql_apply_pair_bytes<double>(n)) * pairs_per_cta;
}

cudaError_t launch_ql_chain(int n, int batch, const Workspace& ws, double* W, int* info, bool single,
                            int chain_threads, cudaStream_t stream, bool redo) {
    if (batch <= 0) return cudaSuccess;
    if (!W || !info || !ws.d || !ws.e || !ws.log || !ws.perm || !ws.flag) return cudaErrorInvalidValue;
    const size_t cs = ql_chain_smem_bytes(n, chain_threads, single);
    if (cs > static_cast<size_t>(max_smem_optin())) return cudaErrorInvalidValue;
    const int cgrid = (batch + chain_threads - 1) / chain_threads;
    static SmemOptIn fcd, fcf;
    if (single) {
        set_max_smem_once(k_ql_chain<float>, fcf);
        k_ql_chain<float><<<cgrid, chain_threads, cs, stream>>>(n, batch, ws, W, info, redo ? 1 : 0);
    } else {
        set_max_smem_once(k_ql_chain<double>, fcd);
        k_ql_chain<double><<<cgrid, chain_threads, cs, stream>>>(n, batch, ws, W, info, redo ? 1 : 0);
    }
    return cudaGetLastError();
}

cudaError_t launch_eig_invit(int n, int batch, const Workspace& ws, double* W, double2* X, int* info,
                             int chain_threads, bool flag_redo, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (!W || !X || !info || !ws.d || !ws.e || !ws.flag) return cudaErrorInvalidValue;
    const size_t vs = ql_chain_smem_bytes(n, chain_threads, false);
    const size_t is = InvitSmem(n, !flag_redo).per_warp;
    if (vs > static_cast<size_t>(max_smem_optin()) || is > static_cast<size_t>(max_smem_optin()))
        return cudaErrorInvalidValue;
    static SmemOptIn fv, fi;
    set_max_smem_once(k_ql_values, fv);
    set_max_smem_once(k_tridiag_invit, fi);
    k_ql_values<<<(batch + chain_threads - 1) / chain_threads, chain_threads, vs, stream>>>(n, batch, ws, W, info);
    k_tridiag_invit<<<batch, 32, is, stream>>>(n, batch, ws, W, X, info, flag_redo ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_ql_logged(int n, int batch, const Workspace& ws, double* W, double2* X, int* info,
                             bool single, int chain_threads, int apply_warps, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (!W || !X || !info || !ws.d || !ws.e || !ws.log || !ws.perm || !ws.flag) return cudaErrorInvalidValue;
    if (n > kSmallMaxN) return launch_ql_rows(n, batch, ws, W, X, info, single, chain_threads, stream);
    if (eig_by_inverse_iteration(n, single))                        // eigenvalues by QL, vectors by inverse iteration
        return launch_eig_invit(n, batch, ws, W, X, info, chain_threads, false, stream);
    const size_t cs = ql_chain_smem_bytes(n, chain_threads, single);
    const size_t as = ql_apply_smem_bytes(n, apply_warps, single);
    if (cs > static_cast<size_t>(max_smem_optin()) || as > static_cast<size_t>(max_smem_optin()))
        return cudaErrorInvalidValue;
    const int cgrid = (batch + chain_threads - 1) / chain_threads;
    const int agrid = (batch + apply_warps - 1) / apply_warps;     // apply_warps = pairs per CTA
    const int athreads = 32 * ((n + 31) / 32) * apply_warps;
    if (n <= 32) {                                                  // Z rows in registers
        // (measured: at n = 32 this beats the shared-memory Z tile by ~4 %; at n = 54 it is 30 %
        // slower: 148 registers a lane and the per-chunk jump into the rotation chain cost more)
        cudaError_t err = launch_ql_chain(n, batch, ws, W, info, single, chain_threads, stream);
        if (err != cudaSuccess) return err;
        // one pair per CTA: ~150 registers a lane, so small CTAs pack the SM best
        const size_t rs = single ? ql_apply_reg_pair_bytes<float>(n) : ql_apply_reg_pair_bytes<double>(n);
        const int rgrid = batch, rthreads = 32 * ((n + 31) / 32);
        static SmemOptIn r32d, r32f;
#define SBG_RUN_REG(NM, R, FLAG)                                                                 \
        { set_max_smem_once(k_ql_apply_reg<NM, R>, FLAG);                                          \
          k_ql_apply_reg<NM, R><<<rgrid, rthreads, rs, stream>>>(n, batch, ws, W, X, info); }
        if (single) SBG_RUN_REG(32, float, r32f)
        else SBG_RUN_REG(32, double, r32d)
#undef SBG_RUN_REG
        return cudaGetLastError();
    }
    static SmemOptIn fcd, fcf, fad, faf;
    if (single) {
        set_max_smem_once(k_ql_chain<float>, fcf);
        set_max_smem_once(k_ql_apply<float>, faf);
        k_ql_chain<float><<<cgrid, chain_threads, cs, stream>>>(n, batch, ws, W, info, 0);
        k_ql_apply<float><<<agrid, athreads, as, stream>>>(n, batch, ws, W, X, info);
    } else {
        set_max_smem_once(k_ql_chain<double>, fcd);
        set_max_smem_once(k_ql_apply<double>, fad);
        k_ql_chain<double><<<cgrid, chain_threads, cs, stream>>>(n, batch, ws, W, info, 0);
        k_ql_apply<double><<<agrid, athreads, as, stream>>>(n, batch, ws, W, X, info);
    }
    return cudaGetLastError();
}

size_t hetrd_c64_smem_bytes(int n) { return hetrd_c64_bytes(n) * kMaxPairWarps; }

size_t pair_kernels_smem_bytes(int n, int pair_warps) {
    const size_t per = std::max(potrf_warp_bytes(n), std::max(hetrd_warp_bytes(n), hetrd_c64_bytes(n)));
    return per * static_cast<size_t>(pair_warps);
}

cudaError_t launch_hetrd_c64(int n, int batch, const double2* C, const Workspace& ws, int* info,
                             const LaunchShape& shape, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (n < 1 || n > kMixedMaxN || !C || !info || !ws.LV || ws.log_stride < refine_stash_entries(n))
        return cudaErrorInvalidValue;
    const int pw = pair_warps_of(shape);
    const size_t smem = hetrd_c64_bytes(n) * pw;
    if (smem > static_cast<size_t>(max_smem_optin())) return cudaErrorInvalidValue;
    static SmemOptIn f;
    set_max_smem_once(k_hetrd_warp_c64, f);
    k_hetrd_warp_c64<<<(batch + pw - 1) / pw, 32 * pw, smem, stream>>>(n, batch, C, ws, info);
    return cudaGetLastError();
}

template <int NMAX, int G, bool EXACT = false>
void run_back_col_g(int mode, int n, int batch, const Workspace& ws, double2* X, int* info, size_t smem,
                    cudaStream_t stream, int qpass) {
    smem = BackSmem(n, (((NMAX | 1) & 7) == 7) ? (NMAX | 1) + 2 : (NMAX | 1)).total;
    if (qpass == 2) {
        static SmemOptIn f2;
        set_max_smem_once(k_back_col<NMAX, G, EXACT, 2>, f2);
        k_back_col<NMAX, G, EXACT, 2><<<batch, back_col_threads<NMAX, G>(), smem, stream>>>(mode, n, batch, ws, X, info);
    } else {
        static SmemOptIn f1;
        set_max_smem_once(k_back_col<NMAX, G, EXACT, 1>, f1);
        k_back_col<NMAX, G, EXACT, 1><<<batch, back_col_threads<NMAX, G>(), smem, stream>>>(mode, n, batch, ws, X, info);
    }
}


// ----------------------------------------------------------------------------- k_pull_pairs
// Pairs are walked grid-stride, each by the whole CTA; every thread keeps 4 independent 16-byte
// loads in flight (their latency is the host link's, about a microsecond), then stores them.
constexpr int kPullThreads = 256;
constexpr int kPullDepth = 4;

__global__ void __launch_bounds__(kPullThreads) k_pull_pairs(const double2* __restrict__ src,
                                                             double2* __restrict__ dst, int count, int n,
                                                             int lower) {
    const int nn = n * n;
    for (int p = blockIdx.x; p < count; p += gridDim.x) {
        const double2* s = src + static_cast<size_t>(nn) * p;
        double2* d = dst + static_cast<size_t>(nn) * p;
        for (int base = 0; base < nn; base += kPullDepth * kPullThreads) {
            double2 v[kPullDepth];
            int at[kPullDepth];
#pragma unroll
            for (int u = 0; u < kPullDepth; ++u) {
                const int e = base + u * kPullThreads + threadIdx.x;
                const int col = e / n, row = e - col * n;
                at[u] = (e < nn && (!lower || row >= col)) ? e : -1;
                if (at[u] >= 0) v[u] = s[e];
            }
#pragma unroll
            for (int u = 0; u < kPullDepth; ++u)
                if (at[u] >= 0) d[at[u]] = v[u];
        }
    }
}

cudaError_t launch_pull_pairs(const double2* src, double2* dst, int count, int n, bool lower, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_pull_pairs<<<std::min(count, sms), kPullThreads, 0, stream>>>(src, dst, count, n, lower ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_back(int mode, int n, int batch, const Workspace& ws, double2* X, int* info,
                        const LaunchShape& shape, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (!X || !info || !ws.LV || !ws.tau) return cudaErrorInvalidValue;
    if (n > kSmallMaxN) {
        if (shape.reduce_tc) {                          // Q Z and L^{-H} on the tensor cores
            if (mode != kBackLOnly) {
                const cudaError_t err = launch_back_q_tc(n, batch, ws, X, info, stream);
                if (err != cudaSuccess || mode == kBackQOnly) return err;
            }
            return launch_back_tc(n, batch, ws, X, info, stream);
        }
        return launch_back_big(mode, n, batch, ws, X, info, stream);
    }
    const size_t smem = back_smem_bytes(n);
    if (smem > static_cast<size_t>(max_smem_optin())) return cudaErrorInvalidValue;
    if (n <= kColMaxN) {
        const bool two = shape.back_lanes == 2;
        const int qp = shape.back_qpass == 2 ? 2 : 1;
        if (n == 32 && shape.col_exact) {
            if (two) run_back_col_g<32, 2, true>(mode, n, batch, ws, X, info, smem, stream, qp);
            else run_back_col_g<32, 1, true>(mode, n, batch, ws, X, info, smem, stream, qp);
        } else if (n == 54 && shape.col_exact) {
            if (two) run_back_col_g<54, 2, true>(mode, n, batch, ws, X, info, smem, stream, qp);
            else run_back_col_g<54, 1, true>(mode, n, batch, ws, X, info, smem, stream, qp);
        } else if (n <= 32) {
            if (two) run_back_col_g<32, 2>(mode, n, batch, ws, X, info, smem, stream, qp);
            else run_back_col_g<32, 1>(mode, n, batch, ws, X, info, smem, stream, qp);
        } else if (n <= 48) {
            if (two) run_back_col_g<48, 2>(mode, n, batch, ws, X, info, smem, stream, qp);
            else run_back_col_g<48, 1>(mode, n, batch, ws, X, info, smem, stream, qp);
        } else {
            if (two) run_back_col_g<56, 2>(mode, n, batch, ws, X, info, smem, stream, qp);
            else run_back_col_g<56, 1>(mode, n, batch, ws, X, info, smem, stream, qp);
        }
        return cudaGetLastError();
    }
    if (shape.reduce_tc && mode != kBackQOnly) {        // Q Z by the CTA kernel, L^{-H} on the tensor cores
        if (mode == kBackFull) {
            SBG_DISPATCH_BY_N(n, run_back, kBackQOnly, n, batch, ws, X, info, smem, stream);
            const cudaError_t err = cudaGetLastError();
            if (err != cudaSuccess) return err;
        }
        return launch_back_tc(n, batch, ws, X, info, stream);
    }
    SBG_DISPATCH_BY_N(n, run_back, mode, n, batch, ws, X, info, smem, stream);
    return cudaGetLastError();
}

// Device self-test of recip_nr (the inverse iteration's reciprocal): r[i] = recip_nr(u[i]).
__global__ void k_selftest_recip(const double* __restrict__ u, double* __restrict__ r, int count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) r[i] = recip_nr(u[i]);
}

cudaError_t launch_selftest_recip(const double* u, double* r, int count, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const int blocks = std::min((count + 255) / 256, 148 * 8);
    k_selftest_recip<<<blocks, 256, 0, stream>>>(u, r, count);
    return cudaGetLastError();
}

// FP64 FMA throughput probe: every thread runs kFmaChains independent dependent chains of
// fma(a, x, y) (x, y runtime values, so nothing folds) for `iters` rounds and stores their sum.
// Flops = 2 * kFmaChains * iters * threads.  Enough independent chains per warp cover the FMA
// latency, so the FP64 pipe, not the chain, bounds it.
constexpr int kFmaChains = 8;
__global__ void __launch_bounds__(256) k_selftest_fp64_fma(double* __restrict__ out, int iters, double x, double y) {
    double a[kFmaChains];
#pragma unroll
    for (int c = 0; c < kFmaChains; ++c) a[c] = threadIdx.x * 1e-3 + c;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
            for (int c = 0; c < kFmaChains; ++c) a[c] = fma(a[c], x, y);
        }
    }
    double sum = 0.0;
#pragma unroll
    for (int c = 0; c < kFmaChains; ++c) sum += a[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = sum;
}

cudaError_t launch_selftest_fp64_fma(double* out, int blocks, int iters, cudaStream_t stream) {
    if (blocks <= 0 || iters <= 0) return cudaErrorInvalidValue;
    k_selftest_fp64_fma<<<blocks, 256, 0, stream>>>(out, iters, 0.999999, 1e-7);
    return cudaGetLastError();
}

}  // namespace sbg
