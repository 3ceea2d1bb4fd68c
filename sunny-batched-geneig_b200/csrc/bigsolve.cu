// Stage kernels for pairs beyond one CTA-per-pair tile of the small path (84 < n <= 256).
//
//   k_reduce_mid     84 < n <= 160: one CTA per pair on the packed lower triangle (potrf,
//                    hegst, hetrd; see below).
//   k_reduce_big     160 < n <= 256: one CLUSTER of CS CTAs per pair.  Column j of every n x n operand
//                    lives in CTA j % CS of the cluster (cyclic, so the work of the
//                    triangular stages is spread evenly), in that CTA's shared memory:
//                    the lower triangle of B / L packed by columns, and A / W / C as full
//                    columns.  It runs
//                      potrf  B = L L^H, right-looking; the pivot column is read by every
//                             CTA from its owner over DSMEM; one cluster barrier per column;
//                      hegst  W = L^{-1} A and C = L^{-1} W^H (C is Hermitian, so
//                             C = (W L^{-H})^H): warp-per-column register solves with L staged
//                             a panel of columns at a time from the owners over DSMEM; W^H is
//                             formed through the pair's X buffer (L2-resident);
//                      hetrd  the owner of column k forms reflector k; every CTA reads it over
//                             DSMEM, forms its share of the Hermitian matvec from its own
//                             columns, the shares are summed over DSMEM, and each CTA applies
//                             the rank-2 update to its own columns (two cluster barriers per
//                             column);
//                    and writes L, the reflectors, d, e, tau and info.
//   k_ql_apply_rows  the QL rotation log applied to one 32-row block of Z per CTA (a pair's
//                    n x n Z does not fit one SM here); a pair whose log overflowed is solved
//                    by the warp QL of its first block with Z in the X buffer's second half.
//                    In FP64 for n <= 128 the eigenvectors come from inverse iteration
//                    (k_tridiag_invit, kernels.cu) and this kernel, with the log, only redoes
//                    the pairs inverse iteration flagged.
//   k_back_big       a cluster of ceil(n / 32) CTAs per pair, each CTA a contiguous block of
//                    32 columns: X = L^{-H} Q Z with 8 (n <= 160) or 16 lanes per column
//                    (a column's rows in registers across its lane group), the
//                    reflectors and L staged a panel at a time from ws.LV.  The (cluster)
//                    barrier only orders every CTA's read of Z before any write of X (they alias).
//
// Workspace use (big n): ws.LV holds L in its lower triangle (diagonal included) and
// reflector v_k packed along column n-1-k of the strict upper triangle:
// v_k(k+1+s) = LV(s, n-1-k), s = 0 .. n-2-k (v_k(k+1) = 1 stored explicitly).
#include "kernels.cuh"
#include "stages.cuh"
#include "colsolve.cuh"

#include <cooperative_groups.h>
#include <mutex>

namespace cg = cooperative_groups;

namespace sbg {

namespace {

__host__ __device__ inline size_t big_align(size_t x, size_t a) { return (x + a - 1) / a * a; }

constexpr int kBigThreads = 256;
constexpr int kBigWarps = kBigThreads / 32;
constexpr int kBigPanel = 4;        // L columns / reflectors staged per panel of the register solves

// Own columns of cluster rank r: global j = t * CS + r, t = 0 .. own_cols - 1.
__host__ __device__ inline int own_cols(int n, int cs, int r) { return n > r ? (n - r + cs - 1) / cs : 0; }
// Packed offset of own column t (rows j .. n-1 of global column j = t * cs + r).
__host__ __device__ inline int own_off(int t, int n, int cs, int r) { return t * (n - r) - cs * t * (t - 1) / 2; }

template <typename T>
__device__ __forceinline__ T* peer(T* p, int rank) {
    return cg::this_cluster().map_shared_rank(p, static_cast<unsigned>(rank));
}
template <int CS>
__device__ __forceinline__ void cluster_barrier() {
    if constexpr (CS == 1) __syncthreads();
    else cg::this_cluster().sync();
}

// Visits the packed-lower elements (i >= j) of own columns t0 .. nc-1, spread over the
// CTA's threads: f(t, j, i).
template <class F>
__device__ __forceinline__ void for_own_lower(int n, int cs, int r, int t0, int nc, F&& f) {
    if (t0 >= nc) return;
    const int base = own_off(t0, n, cs, r);
    const int total = own_off(nc, n, cs, r) - base;
    int t = t0, tbeg = 0, tend = n - (t0 * cs + r);          // flat range of column t
    for (int p = threadIdx.x; p < total; p += blockDim.x) {
        while (p >= tend) { ++t; tbeg = tend; tend += n - (t * cs + r); }
        const int j = t * cs + r;
        f(t, j, j + (p - tbeg));
    }
}

__device__ __forceinline__ double2 block_sum2(double2 v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v.x = warp_sum(v.x);
    v.y = warp_sum(v.y);
    __syncthreads();                     // red is free (its previous readers are done)
    if (lane == 0) { red[2 * warp] = v.x; red[2 * warp + 1] = v.y; }
    __syncthreads();
    double2 s = make_double2(0.0, 0.0);
    for (int w = 0; w < kBigWarps; ++w) { s.x += red[2 * w]; s.y += red[2 * w + 1]; }
    return s;
}

// ----------------------------------------------------------------------------- k_reduce_big
struct BigReduceSmem {
    size_t Lp, Cc, panel, invd, sdot, red, misc, bar, total;
    __host__ __device__ BigReduceSmem(int n, int cs) {
        const int nc0 = (n + cs - 1) / cs;
        size_t o = 0;
        Lp = o;    o += big_align(16 * static_cast<size_t>(own_off(nc0, n, cs, 0)), 16);
        Cc = o;    o += 16 * static_cast<size_t>(nc0) * n;
        panel = o; o += 16 * static_cast<size_t>(kBigPanel) * n;      // >= 3 n: v, w, p of hetrd
        invd = o;  o += big_align(8 * static_cast<size_t>(n), 16);
        sdot = o;  o += 16 * static_cast<size_t>(nc0);
        red = o;   o += 16 * kBigWarps;
        misc = o;  o += 48;                                           // fail flag; tau by step parity
        bar = o;   o += 16;
        total = o;
    }
};

// y <- L^{-1} y for the warp's columns y[c], c < ncw (rows lane + 32 q in registers),
// L distributed over the cluster (packed own columns Lp); columns of L are staged a
// panel at a time into `panel` by the whole CTA.  Every thread of the CTA must call it.
template <int CS, int RM, int NCW>
__device__ __forceinline__ void big_lower_solve(double2 (&y)[NCW][RM], int ncw, int n, double2* Lp, double2* panel,
                                                const double* invd) {
    const int tid = threadIdx.x, lane = tid & 31;
    for (int k0 = 0; k0 < n; k0 += kBigPanel) {
        __syncthreads();                                  // the previous panel is consumed
        for (int q = 0; q < kBigPanel && k0 + q < n; ++q) {
            const int k = k0 + q, o = k % CS;
            const double2* src = peer(Lp, o) + own_off(k / CS, n, CS, o) - k;   // src[i] = L(i, k)
            for (int i = k + 1 + tid; i < n; i += kBigThreads) panel[q * n + i] = src[i];
        }
        __syncthreads();
        for (int q = 0; q < kBigPanel; ++q) {
            const int k = k0 + q;
            if (k >= n) break;
            const double ik = invd[k];
            double2 lv[RM];
#pragma unroll
            for (int r = 0; r < RM; ++r) {
                const int i = lane + 32 * r;
                lv[r] = (i > k && i < n) ? panel[q * n + i] : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int c = 0; c < NCW; ++c) {
                if (c < ncw) {
                    double2 piv = cshfl(seg_get(y[c], k >> 5), k & 31);
                    piv = cscale(piv, ik);
                    if (lane == (k & 31)) seg_set(y[c], k >> 5, piv);
#pragma unroll
                    for (int r = 0; r < RM; ++r)
                        if (lane + 32 * r > k) y[c][r] = cfms(lv[r], piv, y[c][r]);
                }
            }
        }
    }
}

template <int CS, int RM>
__global__ void __launch_bounds__(kBigThreads) k_reduce_big(const double2* __restrict__ A,
                                                            const double2* __restrict__ B, int n, int batch,
                                                            Workspace ws, double2* __restrict__ X,
                                                            int* __restrict__ info, int mode) {
    constexpr int NCW = ((32 * RM + CS - 1) / CS + kBigWarps - 1) / kBigWarps;   // own columns per warp (max)
    const int r = CS == 1 ? 0 : static_cast<int>(cg::this_cluster().block_rank());
    const int b = blockIdx.x / CS;                     // grid = batch * CS: b < batch
    if (!pair_selected(ws, b)) return;                 // uniform over the pair's cluster
    extern __shared__ __align__(16) unsigned char smem[];
    const BigReduceSmem lay(n, CS);
    double2* Lp = reinterpret_cast<double2*>(smem + lay.Lp);
    double2* Cc = reinterpret_cast<double2*>(smem + lay.Cc);
    double2* panel = reinterpret_cast<double2*>(smem + lay.panel);
    double* invd = reinterpret_cast<double*>(smem + lay.invd);
    double2* sdot = reinterpret_cast<double2*>(smem + lay.sdot);
    double* red = reinterpret_cast<double*>(smem + lay.red);
    int* s_fail = reinterpret_cast<int*>(smem + lay.misc);
    double2* s_tau = reinterpret_cast<double2*>(smem + lay.misc + 16);    // [2]
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + lay.bar);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nc = own_cols(n, CS, r);
    const size_t mat = static_cast<size_t>(n) * n;
    const double2* Ab = A + mat * b;
    const double2* Bb = B + mat * b;
    double2* Xb = X + mat * b;
    double2* LVb = ws.LV + mat * b;
    double* db = ws.d + static_cast<size_t>(n) * b;
    double* eb = ws.e + static_cast<size_t>(n) * b;
    double2* taub = ws.tau + static_cast<size_t>(n) * b;

    // ---- stage own columns: lower part of B (packed) and all of A
    if (tid == 0) { *s_fail = 0; mbar_init(bar, 1); fence_mbar_init(); }
    __syncthreads();
    if (warp == 0) {
        if (lane == 0) mbar_arrive_expect_tx(bar, 16u * static_cast<uint32_t>(own_off(nc, n, CS, r) + n * nc));
        __syncwarp();
        for (int t = lane; t < nc; t += 32) {
            const int j = t * CS + r;
            bulk_g2s(Lp + own_off(t, n, CS, r), Bb + j + static_cast<size_t>(j) * n, 16u * (n - j), bar);
            bulk_g2s(Cc + static_cast<size_t>(t) * n, Ab + static_cast<size_t>(j) * n, 16u * n, bar);
        }
    }
    int status = 0;
    if (!mbar_wait_bounded(bar, 0, kMaxPolls)) {
        status = kInfoCopyTimeout;
        mbar_wait_bounded(bar, 0, kMaxPolls);
    }
    cluster_barrier<CS>();                             // every CTA of the cluster is running

    // ---- potrf (right-looking, cyclic columns)
    int fail = 0;
    for (int k = 0; k < n; ++k) {
        const int o = k % CS;
        if (r == o) {
            double2* col = Lp + own_off(k / CS, n, CS, r);             // col[i - k] = B(i, k)
            const double dkk = col[0].x;
            __syncthreads();                                            // dkk read before it is replaced
            if (!(dkk > 0.0)) {
                if (tid == 0) *s_fail = k + 1;
            } else {
                const double dsq = sqrt(dkk), inv = 1.0 / dsq;
                for (int i = 1 + tid; i < n - k; i += kBigThreads) col[i] = cscale(col[i], inv);
                if (tid == 0) col[0] = make_double2(dsq, 0.0);
            }
        }
        cluster_barrier<CS>();
        fail = *peer(s_fail, o);
        if (fail) break;                                                // uniform over the cluster
        const int m = n - k - 1;
        if (m == 0) break;
        const double2* lk = peer(Lp, o) + own_off(k / CS, n, CS, o) + 1;   // lk[i'] = L(k+1+i', k)
        for (int i = tid; i < m; i += kBigThreads) panel[i] = lk[i];
        __syncthreads();
        const int t0 = k + 1 > r ? (k + 1 - r + CS - 1) / CS : 0;
        for_own_lower(n, CS, r, t0, nc, [&](int t, int j, int i) {
            double2* a = Lp + own_off(t, n, CS, r) + (i - j);
            *a = cfmsc(panel[i - k - 1], panel[j - k - 1], *a);
        });
        __syncthreads();
    }

    if (!fail) {
        {                                               // Cholesky done: W and C here
            for (int k = tid; k < n; k += kBigThreads) {
                const int o = k % CS;
                invd[k] = 1.0 / peer(Lp, o)[own_off(k / CS, n, CS, o)].x;
            }
            // ---- W = L^{-1} A on own columns (warp w: own columns t = w + 8 c)
            const int ncw = nc > warp ? (nc - warp + kBigWarps - 1) / kBigWarps : 0;
            double2 y[NCW][RM];
    #pragma unroll
            for (int c = 0; c < NCW; ++c)
    #pragma unroll
                for (int q = 0; q < RM; ++q) {
                    const int i = lane + 32 * q, t = warp + kBigWarps * c;
                    y[c][q] = (c < ncw && i < n) ? Cc[static_cast<size_t>(t) * n + i] : make_double2(0.0, 0.0);
                }
            big_lower_solve<CS, RM, NCW>(y, ncw, n, Lp, panel, invd);
    #pragma unroll
            for (int c = 0; c < NCW; ++c)
    #pragma unroll
                for (int q = 0; q < RM; ++q) {
                    const int i = lane + 32 * q, j = (warp + kBigWarps * c) * CS + r;
                    if (c < ncw && i < n) Xb[i + static_cast<size_t>(j) * n] = y[c][q];
                }
            __threadfence();
            cluster_barrier<CS>();                          // all of W is in X
            // ---- C = L^{-1} W^H: column j of W^H is conj(row j of W)
    #pragma unroll
            for (int c = 0; c < NCW; ++c)
    #pragma unroll
                for (int q = 0; q < RM; ++q) {
                    const int i = lane + 32 * q, j = (warp + kBigWarps * c) * CS + r;
                    y[c][q] = (c < ncw && i < n) ? cconj(Xb[j + static_cast<size_t>(i) * n]) : make_double2(0.0, 0.0);
                }
            big_lower_solve<CS, RM, NCW>(y, ncw, n, Lp, panel, invd);
    #pragma unroll
            for (int c = 0; c < NCW; ++c)
    #pragma unroll
                for (int q = 0; q < RM; ++q) {
                    const int i = lane + 32 * q, t = warp + kBigWarps * c, j = t * CS + r;
                    double2 v = y[c][q];
                    if (i == j) v.y = 0.0;
                    if (c < ncw && i < n) Cc[static_cast<size_t>(t) * n + i] = v;
                }
            __syncthreads();
        }
        if (mode == kBigHegstOnly) {                    // mixed form: C's lower triangle and L out
            cluster_barrier<CS>();                      // every CTA has read its rows of W from X
            for_own_lower(n, CS, r, 0, nc, [&](int t, int j, int i) {
                LVb[i + static_cast<size_t>(j) * n] = Lp[own_off(t, n, CS, r) + (i - j)];
                Xb[i + static_cast<size_t>(j) * n] = Cc[static_cast<size_t>(t) * n + i];
            });
            if (r == 0 && tid == 0) info[b] = status;
            cluster_barrier<CS>();                      // no CTA leaves while a peer may read its memory
            return;
        }

        // ---- hetrd (LAPACK zhetd2's steps, lower)
        double2* vl = panel;                 // v_k(k+1+i'), i' < m
        double2* wl = panel + n;             // w(k+1+i')
        double2* pb = panel + 2 * n;         // this CTA's share of A22 v
        for (int k = 0; k + 1 < n; ++k) {
            const int m = n - k - 1, o = k % CS, tk_loc = k / CS;
            if (r == o && warp == 0) {
                double2* x = Cc + static_cast<size_t>(tk_loc) * n + (k + 1);   // x[i'] = C(k+1+i', k)
                double s2 = 0.0;
                for (int i = 1 + lane; i < m; i += 32) s2 += cabs2(x[i]);
                s2 = warp_sum(s2);
                const double2 alpha = x[0];
                double2 tk, scale;
                double beta;
                if (s2 == 0.0 && alpha.y == 0.0) {
                    tk = make_double2(0.0, 0.0); beta = alpha.x; scale = make_double2(0.0, 0.0);
                } else {
                    const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + s2);
                    beta = alpha.x >= 0.0 ? -nrm : nrm;
                    tk = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
                    const double ar = alpha.x - beta, ai = alpha.y, den = ar * ar + ai * ai;
                    scale = make_double2(ar / den, -ai / den);
                }
                __syncwarp();                                               // alpha read by every lane
                if (tk.x != 0.0 || tk.y != 0.0) {
                    for (int i = 1 + lane; i < m; i += 32) x[i] = cmul(x[i], scale);
                    if (lane == 0) x[0] = make_double2(1.0, 0.0);
                }
                if (lane == 0) {
                    s_tau[k & 1] = tk;
                    db[k] = Cc[static_cast<size_t>(tk_loc) * n + k].x;
                    eb[k] = beta;
                    taub[k] = tk;
                }
            }
            cluster_barrier<CS>();
            const double2 tk = peer(s_tau, o)[k & 1];
            if (tk.x == 0.0 && tk.y == 0.0) continue;                       // H_k = I (uniform)
            const double2* vsrc = peer(Cc, o) + static_cast<size_t>(tk_loc) * n + (k + 1);
            for (int i = tid; i < m; i += kBigThreads) vl[i] = vsrc[i];
            __syncthreads();
            const int t0 = k + 1 > r ? (k + 1 - r + CS - 1) / CS : 0;
            // own column j > k: sdot[t] = sum_{i > j} conj(C(i, j)) v_i   (the mirrored upper part)
            for (int t = t0 + warp; t < nc; t += kBigWarps) {
                const int j = t * CS + r;
                const double2* col = Cc + static_cast<size_t>(t) * n;
                double2 acc = make_double2(0.0, 0.0);
                for (int i = j + 1 + lane; i < n; i += 32) acc = cfmac(col[i], vl[i - k - 1], acc);
                acc.x = warp_sum(acc.x);
                acc.y = warp_sum(acc.y);
                if (lane == 0) sdot[t] = acc;
            }
            __syncthreads();
            // row i = k+1+i': sum over own columns k < j <= i of C(i, j) v_j, plus sdot for i's own column
            for (int ii = tid; ii < m; ii += kBigThreads) {
                const int i = k + 1 + ii;
                double2 acc = make_double2(0.0, 0.0);
                for (int t = t0; t < nc; ++t) {
                    const int j = t * CS + r;
                    if (j > i) break;
                    const double2 c = Cc[static_cast<size_t>(t) * n + i];
                    const double2 vj = vl[j - k - 1];
                    if (j == i) { acc.x = fma(c.x, vj.x, acc.x); acc.y = fma(c.x, vj.y, acc.y); }
                    else acc = cfma(c, vj, acc);
                }
                if (i >= r && (i - r) % CS == 0) acc = cadd(acc, sdot[(i - r) / CS]);
                pb[ii] = acc;
            }
            cluster_barrier<CS>();
            // p = tau * (sum of the shares); alpha2 = -tau/2 (p^H v); w = p + alpha2 v
            double2 dl = make_double2(0.0, 0.0);
            for (int ii = tid; ii < m; ii += kBigThreads) {
                double2 s = make_double2(0.0, 0.0);
#pragma unroll
                for (int q = 0; q < CS; ++q) s = cadd(s, peer(pb, q)[ii]);
                const double2 p = cmul(tk, s);
                wl[ii] = p;
                dl = cfmac(p, vl[ii], dl);
            }
            const double2 dot = block_sum2(dl, red);
            const double2 a2 = cscale(cmul(tk, dot), -0.5);
            for (int ii = tid; ii < m; ii += kBigThreads) wl[ii] = cfma(a2, vl[ii], wl[ii]);
            __syncthreads();
            // own trailing columns: C(i, j) -= v_i conj(w_j) + w_i conj(v_j), i >= j
            for_own_lower(n, CS, r, t0, nc, [&](int t, int j, int i) {
                double2* a = Cc + static_cast<size_t>(t) * n + i;
                const int ii = i - k - 1, jj = j - k - 1;
                double2 v = cfmsc(vl[ii], wl[jj], *a);
                v = cfmsc(wl[ii], vl[jj], v);
                if (i == j) v.y = 0.0;
                *a = v;
            });
            __syncthreads();
        }
        if (r == (n - 1) % CS && tid == 0) {
            db[n - 1] = Cc[static_cast<size_t>((n - 1) / CS) * n + (n - 1)].x;
            eb[n - 1] = 0.0;
            taub[n - 1] = make_double2(0.0, 0.0);
        }
        // ---- L -> LV lower; reflector k -> LV(s, n-1-k), s = i - k - 1
        for_own_lower(n, CS, r, 0, nc, [&](int t, int j, int i) {
            LVb[i + static_cast<size_t>(j) * n] = Lp[own_off(t, n, CS, r) + (i - j)];
            if (i > j) LVb[(i - j - 1) + static_cast<size_t>(n - 1 - j) * n] = Cc[static_cast<size_t>(t) * n + i];
        });
    }
    if (r == 0 && tid == 0) info[b] = (fail ? n + fail : 0) | status;
    cluster_barrier<CS>();                              // no CTA leaves while a peer may read its memory
}

// ----------------------------------------------------------------------------- k_reduce_mid
// One CTA per pair for 84 < n <= kMidMaxN, where the packed lower triangle (n(n+1)/2 complex,
// 206 KB at n = 160) fits one SM's shared memory, so no cluster barrier is needed:
//   potrf   B's lower triangle (TMA bulk copies, packed) factored in place, right-looking;
//   hegst   W = L^{-1} A, then C = L^{-1} W^H with kMidLanes lanes per column (rows g + 8 r in
//           registers), L read from the packed tile; W is parked in the pair's LV slot and C's
//           lower triangle in its X slot (both L2-resident), L then goes to LV's lower triangle;
//   hetrd   C's lower triangle is loaded into the tile and tridiagonalised (zhetd2's steps);
//           reflector k goes to LV's column n-1-k (the big path's convention).
// The Cholesky and rank-2 updates walk the balanced row pairs (q, m-1-q) of the trailing
// matrix, each pair's fused walk split over kMidGroup threads; the Hermitian matvec splits the
// pair's row walk and mirrored column walk the same way and combines by shuffles.
constexpr int kMidThreads = 256;
constexpr int kMidGroup = 4;            // threads per row pair
constexpr int kMidLanes = 8;            // lanes per column in the triangular solves

// A22(r, j) of the trailing matrix starting at c0 (packed by columns, order m) is at
// c0 + mid_off(j, m) + r; the address advances by m - j - 1 from column j to j + 1.
__device__ __forceinline__ int mid_off(int j, int m) { return j * m - j * (j - 1) / 2 - j; }

struct MidSmem {
    size_t P, vb, wb, pb, invd, red, misc, bar, total;
    __host__ __device__ explicit MidSmem(int n) {
        size_t o = 0;
        P = o;    o += big_align(16 * static_cast<size_t>(n) * (n + 1) / 2, 16);
        vb = o;   o += 16 * static_cast<size_t>(n);
        wb = o;   o += 16 * static_cast<size_t>(n);
        pb = o;   o += 16 * static_cast<size_t>(n);
        invd = o; o += big_align(8 * static_cast<size_t>(n), 16);
        red = o;  o += 16 * kBigWarps;
        misc = o; o += 48;                // fail flag; tau by step parity
        bar = o;  o += 16;
        total = o;
    }
};

// f(a, row, j) on the packed-lower elements A22(row, j), j <= row, of the row pairs
// (q, m-1-q): each pair's walk (row q's q+1 terms, then row m-1-q's) split into kMidGroup chunks.
template <class T, class F>
__device__ __forceinline__ void mid_pair_walk(T* c0, int m, F&& f) {
    const int h = (m + 1) >> 1;
    const int grp = threadIdx.x / kMidGroup, sub = threadIdx.x % kMidGroup;
    for (int q = grp; q < h; q += kMidThreads / kMidGroup) {
        const int r1 = q, r2 = m - 1 - q;
        const int tot = (r2 != r1) ? m + 1 : r1 + 1;
        const int t0 = sub * tot / kMidGroup, t1 = (sub + 1) * tot / kMidGroup;
        int row = t0 <= r1 ? r1 : r2;
        int jj = t0 <= r1 ? t0 : t0 - r1 - 1;
        T* a = c0 + mid_off(jj, m) + row;
        for (int t = t0; t < t1; ++t) {
            if (t == r1 + 1) { row = r2; jj = 0; a = c0 + r2; }
            f(a, row, jj);
            a += m - jj - 1;
            ++jj;
        }
    }
}

// zhetd2's steps on the packed lower triangle P (order n, packed by columns) by one CTA of
// kMidThreads threads, four CTA barriers per step: reflector and v by warp 0 | the Hermitian
// matvec over the balanced row pairs (row walk and mirrored column walk split over kMidGroup
// threads, combined by shuffles) with the dot product's per-warp partials | w | rank-2 update.
// Reflector k stays in column k below the diagonal (its first component, 1, at A(k+1, k)); d, e
// and tau go to dout, eout, tout as they are formed.  R = double for the plain form
// (k_reduce_mid), float for the mixed form's complex64 Householder (k_hetrd_c64_big).
template <typename R, typename RD, typename CT>
__device__ void mid_hetrd(cplx<R>* P, int n, cplx<R>* vb, cplx<R>* wb, cplx<R>* pb, R* red, cplx<R>* s_tk,
                          RD* dout, RD* eout, CT* tout) {
    using C = cplx<R>;
    const C zero = mk<R>(R(0), R(0));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int grp = tid / kMidGroup, sub = tid % kMidGroup;
    for (int k = 0; k + 1 < n; ++k) {
        const int m = n - k - 1;
        C* x = P + pk(k, n) + 1;                            // x[i] = A(k+1+i, k)
        if (warp == 0) {
            R s2 = R(0);
            for (int i = 1 + lane; i < m; i += 32) s2 += cabs2(x[i]);
            s2 = warp_sum(s2);
            const C alpha = x[0];
            C tk, scale;
            R beta;
            if (s2 == R(0) && alpha.y == R(0)) {
                tk = zero; beta = alpha.x; scale = zero;
            } else {
                const R nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + s2);
                beta = alpha.x >= R(0) ? -nrm : nrm;
                tk = mk<R>((beta - alpha.x) / beta, -alpha.y / beta);
                const R ar = alpha.x - beta, ai = alpha.y, den = ar * ar + ai * ai;
                scale = mk<R>(ar / den, -ai / den);
            }
            if (tk.x != R(0) || tk.y != R(0)) {
                __syncwarp();                                     // every lane has read alpha
                for (int i = lane; i < m; i += 32) {
                    const C v = (i == 0) ? mk<R>(R(1), R(0)) : cmul(x[i], scale);
                    vb[i] = v;
                    x[i] = v;
                }
            }
            if (lane == 0) {
                s_tk[k & 1] = tk;
                dout[k] = P[pk(k, n)].x;
                eout[k] = beta;
                tout[k] = tk;
            }
        }
        __syncthreads();
        const C tk = s_tk[k & 1];
        if (tk.x == R(0) && tk.y == R(0)) continue;                 // H_k = I (uniform)
        // p = tau A22 v over the row pairs; warp-uniform loop (the group shuffles need whole warps)
        C* c0 = P + pk(k + 1, n);
        const int h = (m + 1) >> 1;
        C dpart = zero;                   // this lane's share of p^H v
        for (int qb = 0; qb < h; qb += kMidThreads / kMidGroup) {
            const int q = qb + grp;
            const bool act = q < h;
            const int r1 = q, r2 = m - 1 - q;
            const bool two = act && r2 != r1;
            C lo1 = zero, lo2 = lo1, up1 = lo1, up2 = lo1;
            if (act) {
                // lower row walk: row r1's r1 terms, then row r2's r2 terms
                const int tot = two ? r1 + r2 : r1;
                const int t0 = sub * tot / kMidGroup, t1 = (sub + 1) * tot / kMidGroup;
                int jj = t0 < r1 ? t0 : t0 - r1;
                const C* a = c0 + mid_off(jj, m) + (t0 < r1 ? r1 : r2);
                for (int t = t0; t < t1; ++t) {
                    if (t == r1) { jj = 0; a = c0 + r2; }
                    if (t < r1) lo1 = cfma(*a, vb[jj], lo1); else lo2 = cfma(*a, vb[jj], lo2);
                    a += m - jj - 1;
                    ++jj;
                }
                // mirrored column walk: column r1 below the diagonal (m-1-r1 terms), then column r2's
                const int sw = m - 1 - r1;
                const int tot2 = two ? m - 1 : sw;
                const int u0 = sub * tot2 / kMidGroup, u1 = (sub + 1) * tot2 / kMidGroup;
                const C* d1 = c0 + mid_off(r1, m) + r1;
                const C* d2 = c0 + mid_off(r2, m) + r2;
                for (int t = u0; t < u1; ++t) {
                    if (t < sw) up1 = cfmac(d1[t + 1], vb[r1 + t + 1], up1);
                    else up2 = cfmac(d2[t - sw + 1], vb[r2 + t - sw + 1], up2);
                }
            }
#pragma unroll
            for (int o = 1; o < kMidGroup; o <<= 1) {
                lo1.x += shfl_xor(lo1.x, o); lo1.y += shfl_xor(lo1.y, o);
                lo2.x += shfl_xor(lo2.x, o); lo2.y += shfl_xor(lo2.y, o);
                up1.x += shfl_xor(up1.x, o); up1.y += shfl_xor(up1.y, o);
                up2.x += shfl_xor(up2.x, o); up2.y += shfl_xor(up2.y, o);
            }
            if (act && sub == 0) {
                const C* d1 = c0 + mid_off(r1, m) + r1;
                C s = cadd(lo1, up1);
                s.x = fma(d1[0].x, vb[r1].x, s.x);
                s.y = fma(d1[0].x, vb[r1].y, s.y);
                const C p1 = cmul(tk, s);
                pb[r1] = p1;
                dpart = cfmac(p1, vb[r1], dpart);
                if (two) {
                    const C* d2 = c0 + mid_off(r2, m) + r2;
                    C s2v = cadd(lo2, up2);
                    s2v.x = fma(d2[0].x, vb[r2].x, s2v.x);
                    s2v.y = fma(d2[0].x, vb[r2].y, s2v.y);
                    const C p2 = cmul(tk, s2v);
                    pb[r2] = p2;
                    dpart = cfmac(p2, vb[r2], dpart);
                }
            }
        }
        dpart.x = warp_sum(dpart.x);
        dpart.y = warp_sum(dpart.y);
        if (lane == 0) { red[2 * warp] = dpart.x; red[2 * warp + 1] = dpart.y; }
        __syncthreads();
        // w = p - tau/2 (p^H v) v
        C dot = zero;
#pragma unroll
        for (int w8 = 0; w8 < kBigWarps; ++w8) { dot.x += red[2 * w8]; dot.y += red[2 * w8 + 1]; }
        const C a2 = cscale(cmul(tk, dot), R(-0.5));
        for (int i = tid; i < m; i += kMidThreads) wb[i] = cfma(a2, vb[i], pb[i]);
        __syncthreads();
        // A22 -= v w^H + w v^H (lower)
        mid_pair_walk(c0, m, [&](C* a, int row, int j) {
            C v = cfmsc(vb[row], wb[j], *a);
            v = cfmsc(wb[row], vb[j], v);
            if (row == j) v.y = R(0);
            *a = v;
        });
        __syncthreads();
    }
    if (tid == 0) {
        dout[n - 1] = P[pk(n - 1, n)].x;
        eout[n - 1] = R(0);
        tout[n - 1] = zero;
    }
}

template <int RM>
__global__ void __launch_bounds__(kMidThreads) k_reduce_mid(const double2* __restrict__ A,
                                                            const double2* __restrict__ B, int n, int batch,
                                                            Workspace ws, double2* __restrict__ X,
                                                            int* __restrict__ info, int mode) {
    const int b = blockIdx.x;
    if (b >= batch || !pair_selected(ws, b)) return;
    extern __shared__ __align__(16) unsigned char smem[];
    const MidSmem lay(n);
    double2* P = reinterpret_cast<double2*>(smem + lay.P);
    double2* vb = reinterpret_cast<double2*>(smem + lay.vb);
    double2* wb = reinterpret_cast<double2*>(smem + lay.wb);
    double2* pb = reinterpret_cast<double2*>(smem + lay.pb);
    double* invd = reinterpret_cast<double*>(smem + lay.invd);
    double* red = reinterpret_cast<double*>(smem + lay.red);
    int* s_fail = reinterpret_cast<int*>(smem + lay.misc);
    double2* s_tk = reinterpret_cast<double2*>(smem + lay.misc + 16);      // [2]
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + lay.bar);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const size_t mat = static_cast<size_t>(n) * n;
    const double2* Ab = A + mat * b;
    const double2* Bb = B + mat * b;
    double2* Xb = X + mat * b;
    double2* LVb = ws.LV + mat * b;
    double* db = ws.d + static_cast<size_t>(n) * b;
    double* eb = ws.e + static_cast<size_t>(n) * b;
    double2* taub = ws.tau + static_cast<size_t>(n) * b;

    int status = 0;
    {                                                             // Cholesky and reduction
        if (tid == 0) { *s_fail = 0; mbar_init(bar, 1); fence_mbar_init(); }
        __syncthreads();
        if (warp == 0) {
            if (lane == 0) mbar_arrive_expect_tx(bar, static_cast<uint32_t>(16 * (static_cast<size_t>(n) * (n + 1) / 2)));
            __syncwarp();
            for (int j = lane; j < n; j += 32)
                bulk_g2s(P + pk(j, n), Bb + j + static_cast<size_t>(j) * n, 16u * (n - j), bar);
        }
        if (!mbar_wait_bounded(bar, 0, kMaxPolls)) {
            status = kInfoCopyTimeout;
            mbar_wait_bounded(bar, 0, kMaxPolls);
        }

        // ---- potrf
        for (int k = 0; k < n; ++k) {
            double2* col = P + pk(k, n);                              // col[i - k] = A(i, k)
            const double dkk = col[0].x;
            __syncthreads();                                          // every thread has read dkk
            if (!(dkk > 0.0)) { if (tid == 0) *s_fail = k + 1; break; }     // uniform
            const double dsq = sqrt(dkk), inv = 1.0 / dsq;
            const int m = n - k - 1;
            for (int i = 1 + tid; i <= m; i += kMidThreads) col[i] = cscale(col[i], inv);
            if (tid == 0) { col[0] = make_double2(dsq, 0.0); invd[k] = inv; }
            __syncthreads();
            if (m == 0) break;
            const double2* l = col + 1;                               // l[r] = L(k+1+r, k)
            mid_pair_walk(P + pk(k + 1, n), m, [&](double2* a, int row, int j) { *a = cfmsc(l[row], l[j], *a); });
            __syncthreads();
        }
        __syncthreads();
        const int fail = *s_fail;
        if (fail) {
            if (tid == 0) info[b] = (n + fail) | status;
            return;
        }

        // ---- hegst: 8 lanes per column, 32 columns per pass
        {
            const int g = tid % kMidLanes;
            const int cpp = kMidThreads / kMidLanes;
            for (int c0 = 0; c0 < n; c0 += cpp) {                     // W = L^{-1} A -> LV slot
                const int j = c0 + tid / kMidLanes;
                const bool own = j < n;
                double2 y[RM];
    #pragma unroll
                for (int r = 0; r < RM; ++r) {
                    const int i = g + kMidLanes * r;
                    y[r] = (own && i < n) ? Ab[i + static_cast<size_t>(j) * n] : make_double2(0.0, 0.0);
                }
                grp_trsm_lower_packed<kMidLanes, RM, double>(P, invd, y, n, g);
    #pragma unroll
                for (int r = 0; r < RM; ++r) {
                    const int i = g + kMidLanes * r;
                    if (own && i < n) LVb[i + static_cast<size_t>(j) * n] = y[r];
                }
            }
            __syncthreads();
            for (int c0 = 0; c0 < n; c0 += cpp) {                     // C = L^{-1} W^H -> X slot (lower)
                const int j = c0 + tid / kMidLanes;
                const bool own = j < n;
                double2 y[RM];
    #pragma unroll
                for (int r = 0; r < RM; ++r) {
                    const int i = g + kMidLanes * r;
                    y[r] = (own && i < n) ? cconj(LVb[j + static_cast<size_t>(i) * n]) : make_double2(0.0, 0.0);
                }
                grp_trsm_lower_packed<kMidLanes, RM, double>(P, invd, y, n, g);
    #pragma unroll
                for (int r = 0; r < RM; ++r) {
                    const int i = g + kMidLanes * r;
                    double2 v = y[r];
                    if (i == j) v.y = 0.0;
                    if (own && i < n && i >= j) Xb[i + static_cast<size_t>(j) * n] = v;
                }
            }
            __syncthreads();
        }
        // L -> LV lower (W is no longer needed), then C's lower triangle -> the tile
        for (size_t idx = tid; idx < mat; idx += kMidThreads) {
            const int j = static_cast<int>(idx / n), i = static_cast<int>(idx - static_cast<size_t>(j) * n);
            if (i >= j) LVb[idx] = P[pk(j, n) + i - j];
        }
        __syncthreads();
    }
    if (mode == kBigHegstOnly) {                                   // mixed form: C stays in X
        if (tid == 0) info[b] = status;
        return;
    }
    for (size_t idx = tid; idx < mat; idx += kMidThreads) {
        const int j = static_cast<int>(idx / n), i = static_cast<int>(idx - static_cast<size_t>(j) * n);
        if (i >= j) P[pk(j, n) + i - j] = Xb[idx];
    }
    __syncthreads();
    mid_hetrd<double>(P, n, vb, wb, pb, red, s_tk, db, eb, taub);
    // reflector k (rows k+1 .. n-1 of column k) -> LV(s, n-1-k), s = i - k - 1
    for (size_t idx = tid; idx < mat; idx += kMidThreads) {
        const int k = static_cast<int>(idx / n), i = static_cast<int>(idx - static_cast<size_t>(k) * n);
        if (i > k) LVb[(i - k - 1) + static_cast<size_t>(n - 1 - k) * n] = P[pk(k, n) + i - k];
    }
    if (tid == 0) info[b] = status;
}

// ----------------------------------------------------------------------------- k_hetrd_c64_big
// Mixed form, kMixedMaxN < n <= kMixedBigMaxN: the Householder stage in complex64, one CTA per
// pair.  C's lower triangle (FP64, left in X by the reduction) is rounded to complex64 into a
// packed tile (8 B per entry: 66 KB at n = 128, half of what the FP64 tile takes) and
// tridiagonalised by mid_hetrd<float>; C itself, full Hermitian and FP64, goes to ws.rfC for the
// refinement (X is overwritten before it runs).  The outputs go where the FP64 kernels put theirs,
// promoted to FP64, so the FP64 eigensolve of T and the back-transform run on them unchanged:
// reflector k along LV's row k above the superdiagonal for n <= kSmallMaxN, along LV's column
// n-1-k beyond (v_k(k+1) = 1 stored), d and e, and tau rescaled in FP64 so that each
// H = I - tau v v^H is unitary to FP64 rounding for the promoted v (|tau|^2 ||v||^2 = 2 Re tau).
struct C64BigSmem {
    size_t P, vb, wb, pb, red, tk, d, e, tau, total;
    __host__ __device__ explicit C64BigSmem(int n) {
        size_t o = 0;
        P = o;   o += big_align(8 * static_cast<size_t>(n) * (n + 1) / 2, 16);
        vb = o;  o += big_align(8 * static_cast<size_t>(n), 16);
        wb = o;  o += big_align(8 * static_cast<size_t>(n), 16);
        pb = o;  o += big_align(8 * static_cast<size_t>(n), 16);
        red = o; o += 8 * kBigWarps;
        tk = o;  o += 16;
        d = o;   o += big_align(4 * static_cast<size_t>(n), 16);
        e = o;   o += big_align(4 * static_cast<size_t>(n), 16);
        tau = o; o += big_align(8 * static_cast<size_t>(n), 16);
        total = o;
    }
};

__global__ void __launch_bounds__(kMidThreads) k_hetrd_c64_big(int n, int batch, const double2* __restrict__ C,
                                                               Workspace ws, int* __restrict__ info) {
    const int b = blockIdx.x;
    if (b >= batch) return;
    if (info[b] != 0) return;                                     // an earlier stage failed (uniform)
    extern __shared__ __align__(16) unsigned char smem[];
    const C64BigSmem lay(n);
    float2* P = reinterpret_cast<float2*>(smem + lay.P);
    float2* vb = reinterpret_cast<float2*>(smem + lay.vb);
    float2* wb = reinterpret_cast<float2*>(smem + lay.wb);
    float2* pb = reinterpret_cast<float2*>(smem + lay.pb);
    float* red = reinterpret_cast<float*>(smem + lay.red);
    float2* s_tk = reinterpret_cast<float2*>(smem + lay.tk);
    float* d_s = reinterpret_cast<float*>(smem + lay.d);
    float* e_s = reinterpret_cast<float*>(smem + lay.e);
    float2* tau_s = reinterpret_cast<float2*>(smem + lay.tau);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const size_t mat = static_cast<size_t>(n) * n;
    const double2* Cb = C + mat * b;
    double2* Sb = ws.rfC + mat * b;
    for (size_t idx = tid; idx < mat; idx += kMidThreads) {
        const int j = static_cast<int>(idx / n), i = static_cast<int>(idx - static_cast<size_t>(j) * n);
        if (i < j) continue;
        double2 v = Cb[idx];
        if (i == j) v.y = 0.0;
        P[pk(j, n) + i - j] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
        Sb[idx] = v;
        if (i != j) Sb[j + static_cast<size_t>(i) * n] = make_double2(v.x, -v.y);
    }
    __syncthreads();
    mid_hetrd<float>(P, n, vb, wb, pb, red, s_tk, d_s, e_s, tau_s);
    __syncthreads();
    const bool rows = n <= kSmallMaxN;                            // the small path's reflector layout
    double2* LVb = ws.LV + mat * b;
    for (int k = warp; k + 1 < n; k += kBigWarps) {              // one warp per reflector
        const float2* col = P + pk(k, n) - k;                     // col[i] = v_k(i), i >= k + 2
        double s2 = 0.0;
        for (int i = k + 1 + lane; i < n; i += 32) {
            const double2 v = (i == k + 1) ? make_double2(1.0, 0.0)
                                           : make_double2(static_cast<double>(col[i].x), static_cast<double>(col[i].y));
            if (rows) LVb[k + static_cast<size_t>(i) * n] = v;
            else LVb[(i - k - 1) + static_cast<size_t>(n - 1 - k) * n] = v;
            s2 = fma(v.x, v.x, fma(v.y, v.y, s2));
        }
        s2 = warp_sum(s2);
        if (lane == 0) {
            const double tr = tau_s[k].x, ti = tau_s[k].y, t2 = tr * tr + ti * ti;
            const double sc = t2 > 0.0 ? 2.0 * tr / (t2 * s2) : 0.0;
            ws.tau[static_cast<size_t>(n) * b + k] = make_double2(tr * sc, ti * sc);
        }
    }
    for (int i = tid; i < n; i += kMidThreads) {
        ws.d[static_cast<size_t>(n) * b + i] = d_s[i];
        ws.e[static_cast<size_t>(n) * b + i] = (i + 1 < n) ? static_cast<double>(e_s[i]) : 0.0;
        if (i + 1 == n) ws.tau[static_cast<size_t>(n) * b + i] = make_double2(0.0, 0.0);
    }
}

// ----------------------------------------------------------------------------- k_hetrd_l2
// The FP64 Householder alone (after k_reduce_tc), one CTA per pair, with the packed lower triangle
// in global memory -- the pair's rotation-log region, free until the eigensolve -- instead of shared
// memory, so no shared-memory tile limits how large n may be (the FP64 tile no longer fits one SM
// above n = 160).  zhetd2's steps, with ONE pass over the trailing triangle per step instead of a
// matvec walk that reads it twice and an update walk that reads and writes it: step k-1's rank-2
// update is applied lazily, to column k by warp 0 just before it forms reflector k from that
// column, and to columns k+1.. by all warps in the same walk that forms the Hermitian matvec with
// reflector k.  The walk goes down columns (pairs of a long and a short column per warp), a warp
// reading 32 consecutive rows at a time; lane l owns the rows i = l (mod 32), so the matvec's
// row sums stay in its registers and only the column sums need a warp reduction.
// Reflector k goes to LV's column n-1-k (the big path's layout), d, e, tau as k_reduce_mid's.
// 3 CTAs per SM (80 registers; 92 unbounded, 2 CTAs) measured fastest: 1.12x over 2, 1.06x over 4
// (64 registers, with spills), at n = 192.
constexpr int kL2Slots = kBigMaxN / 32;         // 32-row chunks of a column

struct L2HetrdSmem {
    size_t v, w, p, col, rows, red, tk, total;
    __host__ __device__ explicit L2HetrdSmem(int n) {
        size_t o = 0;
        v = o;    o += 16 * 2 * static_cast<size_t>(n);            // reflectors k and k-1, by absolute row
        w = o;    o += 16 * static_cast<size_t>(n);                // w of the pending update
        p = o;    o += 16 * static_cast<size_t>(n);
        col = o;  o += 16 * static_cast<size_t>(n);                // column sums of the matvec
        rows = o; o += 16 * static_cast<size_t>(kBigWarps) * n;    // row sums, per warp
        red = o;  o += 16 * kBigWarps;
        tk = o;   o += 32;
        total = o;
    }
};

__global__ void __launch_bounds__(kMidThreads, 3) k_hetrd_l2(int n, int batch, const double2* __restrict__ C,
                                                             Workspace ws, int* __restrict__ info) {
    const int b = blockIdx.x;
    if (b >= batch || !pair_selected(ws, b)) return;
    if (info[b] != 0) return;                                     // the Cholesky failed (uniform)
    extern __shared__ __align__(16) unsigned char smem[];
    const L2HetrdSmem L(n);
    double2* vbuf = reinterpret_cast<double2*>(smem + L.v);
    double2* wb = reinterpret_cast<double2*>(smem + L.w);
    double2* pb = reinterpret_cast<double2*>(smem + L.p);
    double2* colp = reinterpret_cast<double2*>(smem + L.col);
    double2* prow = reinterpret_cast<double2*>(smem + L.rows);
    double* red = reinterpret_cast<double*>(smem + L.red);
    double2* s_tk = reinterpret_cast<double2*>(smem + L.tk);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const size_t mat = static_cast<size_t>(n) * n;
    const double2* Cb = C + mat * b;
    double2* P = static_cast<double2*>(ws.log) + static_cast<size_t>(ws.log_stride) * b;
    double* dout = ws.d + static_cast<size_t>(n) * b;
    double* eout = ws.e + static_cast<size_t>(n) * b;
    double2* tout = ws.tau + static_cast<size_t>(n) * b;
    for (int j = warp; j < n; j += kBigWarps)                     // C's lower triangle, packed by columns
        for (int i = j + lane; i < n; i += 32) {
            double2 v = Cb[i + static_cast<size_t>(j) * n];
            if (i == j) v.y = 0.0;
            P[pk(j, n) + i - j] = v;
        }
    __syncthreads();
    const double2 zero = make_double2(0.0, 0.0);
    bool upd = false;                                             // step k-1's update pending (uniform)
    for (int k = 0; k + 1 < n; ++k) {
        double2* vb = vbuf + (k & 1) * n;                         // reflector k, vb[i] for rows i > k
        const double2* vp = vbuf + ((k + 1) & 1) * n;             // reflector k-1 (while upd)
        const int m = n - k - 1;
        double2* ck = P + pk(k, n) - k;                           // ck[i] = A(i, k), i >= k
        if (warp == 0) {
            if (upd) {
                const double2 wk = wb[k], vk = vp[k];
                for (int i = k + lane; i < n; i += 32) {
                    double2 a = cfmsc(vp[i], wk, ck[i]);
                    a = cfmsc(wb[i], vk, a);
                    if (i == k) a.y = 0.0;
                    ck[i] = a;
                }
                __syncwarp();
            }
            double2* x = ck + k + 1;                              // x[i] = A(k+1+i, k)
            double s2 = 0.0;
            for (int i = 1 + lane; i < m; i += 32) s2 += cabs2(x[i]);
            s2 = warp_sum(s2);
            const double2 alpha = x[0];
            double2 tk, scale;
            double beta;
            if (s2 == 0.0 && alpha.y == 0.0) {
                tk = zero; beta = alpha.x; scale = zero;
            } else {
                const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + s2);
                beta = alpha.x >= 0.0 ? -nrm : nrm;
                tk = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
                const double ar = alpha.x - beta, ai = alpha.y, den = ar * ar + ai * ai;
                scale = make_double2(ar / den, -ai / den);
            }
            if (tk.x != 0.0 || tk.y != 0.0) {
                __syncwarp();                                     // every lane has read alpha
                for (int i = lane; i < m; i += 32) {
                    const double2 v = (i == 0) ? make_double2(1.0, 0.0) : cmul(x[i], scale);
                    vb[k + 1 + i] = v;
                    x[i] = v;
                }
            }
            if (lane == 0) {
                s_tk[k & 1] = tk;
                dout[k] = ck[k].x;
                eout[k] = beta;
                tout[k] = tk;
            }
        }
        __syncthreads();
        const double2 tk = s_tk[k & 1];
        const bool mv = tk.x != 0.0 || tk.y != 0.0;
        if (!upd && !mv) continue;                                // nothing to apply or form (uniform)
        double2 acc[kL2Slots];
#pragma unroll
        for (int s = 0; s < kL2Slots; ++s) acc[s] = zero;
        const int npair = (m + 1) >> 1;                           // columns k+1+q and n-1-q
        for (int q = warp; q < npair; q += kBigWarps) {
            for (int h = 0; h < 2; ++h) {
                const int j = h == 0 ? k + 1 + q : n - 1 - q;
                if (h == 1 && j == k + 1 + q) break;              // the middle column, once
                double2* cj = P + pk(j, n) - j;                   // cj[i] = A(i, j), i >= j
                const double2 vj = vb[j];
                double2 wj = zero, vpj = zero;
                if (upd) { wj = wb[j]; vpj = vp[j]; }
                double2 cs = zero;
#pragma unroll
                for (int s = 0; s < kL2Slots; ++s) {
                    if (32 * s >= n) break;                       // uniform
                    if (32 * s + 31 < j) continue;                // uniform: the chunk is above the diagonal
                    const int i = 32 * s + lane;
                    if (i >= j && i < n) {
                        double2 a = cj[i];
                        if (upd) {
                            a = cfmsc(vp[i], wj, a);
                            a = cfmsc(wb[i], vpj, a);
                            if (i == j) a.y = 0.0;
                            cj[i] = a;
                        }
                        if (mv) {
                            if (i == j) {
                                acc[s].x = fma(a.x, vj.x, acc[s].x);
                                acc[s].y = fma(a.x, vj.y, acc[s].y);
                            } else {
                                acc[s] = cfma(a, vj, acc[s]);
                                cs = cfmac(a, vb[i], cs);
                            }
                        }
                    }
                }
                if (mv) {
                    cs.x = warp_sum(cs.x);
                    cs.y = warp_sum(cs.y);
                    if (lane == 0) colp[j] = cs;
                }
            }
        }
        if (mv) {
#pragma unroll
            for (int s = 0; s < kL2Slots; ++s) {
                const int i = 32 * s + lane;
                if (i > k && i < n) prow[warp * n + i] = acc[s];
            }
        }
        __syncthreads();
        if (!mv) { upd = false; continue; }                       // H_k = I: nothing pending (uniform)
        // p = tau A22 v, then w = p - tau/2 (p^H v) v
        double2 dpart = zero;
        for (int i = k + 1 + tid; i < n; i += kMidThreads) {
            double2 sum = colp[i];
#pragma unroll
            for (int w8 = 0; w8 < kBigWarps; ++w8) sum = cadd(sum, prow[w8 * n + i]);
            const double2 p = cmul(tk, sum);
            pb[i] = p;
            dpart = cfmac(p, vb[i], dpart);
        }
        dpart.x = warp_sum(dpart.x);
        dpart.y = warp_sum(dpart.y);
        if (lane == 0) { red[2 * warp] = dpart.x; red[2 * warp + 1] = dpart.y; }
        __syncthreads();
        double2 dot = zero;
#pragma unroll
        for (int w8 = 0; w8 < kBigWarps; ++w8) { dot.x += red[2 * w8]; dot.y += red[2 * w8 + 1]; }
        const double2 a2 = cscale(cmul(tk, dot), -0.5);
        for (int i = k + 1 + tid; i < n; i += kMidThreads) wb[i] = cfma(a2, vb[i], pb[i]);
        __syncthreads();
        upd = true;
    }
    if (tid == 0) {
        double2* cl = P + pk(n - 1, n);
        double2 a = cl[0];
        if (upd) {                                                // step n-2's update of A(n-1, n-1)
            const double2* vl = vbuf + ((n - 2) & 1) * n;
            a = cfmsc(vl[n - 1], wb[n - 1], a);
            a = cfmsc(wb[n - 1], vl[n - 1], a);
            a.y = 0.0;
            cl[0] = a;
        }
        dout[n - 1] = a.x;
        eout[n - 1] = 0.0;
        tout[n - 1] = zero;
    }
    __syncthreads();
    double2* LVb = ws.LV + mat * b;
    for (int k = warp; k + 1 < n; k += kBigWarps) {               // reflector k below the diagonal of column k
        const double2* ck = P + pk(k, n) - k;
        for (int i = k + 1 + lane; i < n; i += 32) LVb[(i - k - 1) + static_cast<size_t>(n - 1 - k) * n] = ck[i];
    }
}

// ----------------------------------------------------------------------------- k_ql_apply_rows
template <typename R>
__host__ __device__ inline size_t ql_rows_bytes(int n) {
    return big_align(sizeof(R) * 32 * static_cast<size_t>(tile_ld(n)), 16) + 64 * sizeof(cplx<R>) +
           big_align(sizeof(R) * 2 * static_cast<size_t>(n), 16);
}

// redo: only the pairs flagged by k_tridiag_invit (ws.flag 2, or 3 after a log overflow).
template <typename R>
__global__ void __launch_bounds__(32) k_ql_apply_rows(int n, int batch, Workspace ws, double* __restrict__ W,
                                                      double2* __restrict__ X, int* __restrict__ info, int redo) {
    using C = cplx<R>;
    const int nrb = (n + 31) / 32;                     // row blocks per pair
    const int b = blockIdx.x / nrb, rb = blockIdx.x - b * nrb, lane = threadIdx.x;
    if (b >= batch || !pair_selected(ws, b)) return;
    if (redo && ws.flag[b] < 2) return;
    if (info[b] > n || info[b] < 0) return;            // B not positive definite: the back stage writes NaN
    extern __shared__ __align__(16) unsigned char smem[];
    const int ldz = tile_ld(n);
    R* Z = reinterpret_cast<R*>(smem);
    C* stage = reinterpret_cast<C*>(smem + big_align(sizeof(R) * 32 * static_cast<size_t>(ldz), 16));
    R* dd = reinterpret_cast<R*>(reinterpret_cast<unsigned char*>(stage) + 64 * sizeof(C));
    R* ee = dd + n;
    const size_t mat = static_cast<size_t>(n) * n;
    R* Zg = reinterpret_cast<R*>(X + mat * b);
    if (ws.flag[b] != 0 && ws.flag[b] != 2) {          // log overflow: warp QL on block 0
        if (rb != 0) return;
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
        for (int row = lane; row < n; row += 32)
            for (int k = 0; k < n; ++k) Zg[row + static_cast<size_t>(k) * n] = Zs[static_cast<size_t>(row) * n + k];
        return;
    }
    const int row = rb * 32 + lane;
    const bool own = row < n;
    R* zrow = Z + lane * ldz;
    if (own)
        for (int c = 0; c < n; ++c) zrow[c] = (row == c) ? R(1) : R(0);
    __syncwarp();
    ql_log_apply_row<R>(reinterpret_cast<const C*>(ws.log) + static_cast<size_t>(ws.log_cap) * b, ws.log_cap, stage,
                        zrow, own);
    if (own) {
        const int* perm = ws.perm + static_cast<size_t>(n) * b;
        for (int k = 0; k < n; ++k) Zg[row + static_cast<size_t>(k) * n] = zrow[perm[k]];
    }
}

// ----------------------------------------------------------------------------- k_back_big
struct BigBackSmem {
    size_t panel, tau, invd, total;
    __host__ __device__ explicit BigBackSmem(int n) {
        size_t o = 0;
        panel = o; o += 16 * static_cast<size_t>(kBigPanel) * n;
        tau = o;   o += 16 * static_cast<size_t>(n);
        invd = o;  o += big_align(8 * static_cast<size_t>(n), 16);
        total = o;
    }
};

// Group grp (G consecutive lanes) of the CTA holds local columns grp + (256 / G) w, w < NCW,
// rows g + G q in y[w][q]; every dot product combines over the group with log2 G shuffles.
// The k loops are uniform over the CTA and inactive columns run on zeros (the group shuffles
// need whole warps).
template <int CS, int G, int RM, int NCW>
__global__ void __launch_bounds__(kBigThreads) k_back_big(int mode, int n, int batch, Workspace ws,
                                                          double2* __restrict__ X, const int* __restrict__ info) {
    constexpr int GROUPS = kBigThreads / G;
    const int r = CS == 1 ? 0 : static_cast<int>(cg::this_cluster().block_rank());
    const int b = blockIdx.x / CS;
    if (!pair_selected(ws, b)) return;                  // uniform over the pair's cluster
    extern __shared__ __align__(16) unsigned char smem[];
    const BigBackSmem lay(n);
    double2* panel = reinterpret_cast<double2*>(smem + lay.panel);
    double2* taus = reinterpret_cast<double2*>(smem + lay.tau);
    double* invd = reinterpret_cast<double*>(smem + lay.invd);
    const int tid = threadIdx.x, lane = tid & 31;
    const int grp = tid / G, g = tid - grp * G;
    const size_t mat = static_cast<size_t>(n) * n;
    double2* Xb = X + mat * b;
    const double2* LVb = ws.LV + mat * b;
    const int nb = (n + CS - 1) / CS, c0 = r * nb, nc = max(0, min(n, c0 + nb) - c0);
    const bool bad = info[b] > n || info[b] < 0;
    double2 y[NCW][RM];
    const double* Zg = reinterpret_cast<const double*>(Xb);
#pragma unroll
    for (int w = 0; w < NCW; ++w)
#pragma unroll
        for (int q = 0; q < RM; ++q) {
            const int i = g + G * q, lc = grp + GROUPS * w;
            const bool in = !bad && lc < nc && i < n;
            if (mode == kBackLOnly)                     // complex Y in the X buffer
                y[w][q] = in ? Xb[i + static_cast<size_t>(c0 + lc) * n] : make_double2(0.0, 0.0);
            else                                        // real Z in the X buffer
                y[w][q] = make_double2(in ? Zg[i + static_cast<size_t>(c0 + lc) * n] : 0.0, 0.0);
        }
    if (!bad) {
        for (int k = tid; k < n; k += kBigThreads) {
            taus[k] = ws.tau[static_cast<size_t>(n) * b + k];
            invd[k] = 1.0 / LVb[k + static_cast<size_t>(k) * n].x;
        }
    }
    cluster_barrier<CS>();                              // every CTA has read its Z before X is written
    if (bad) {
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        for (int idx = tid; idx < n * nc; idx += kBigThreads)
            Xb[static_cast<size_t>(c0) * n + idx] = make_double2(nan, nan);
        return;
    }
    // ---- Y = Q Z: H_k for k = n-2 .. 0 (kBackLOnly: Y given)
    for (int k0 = mode == kBackLOnly ? -1 : n - 2; k0 >= 0; k0 -= kBigPanel) {
        __syncthreads();
        for (int p = 0; p < kBigPanel && k0 - p >= 0; ++p) {
            const int k = k0 - p;
            const double2* src = LVb + static_cast<size_t>(n - 1 - k) * n - (k + 1);    // src[i] = v_k(i)
            for (int i = k + 1 + tid; i < n; i += kBigThreads) panel[p * n + i] = src[i];
        }
        __syncthreads();
#pragma unroll 1
        for (int p = 0; p < kBigPanel; ++p) {
            const int k = k0 - p;
            if (k < 0) break;
            const double2 tk = taus[k];
            if (tk.x == 0.0 && tk.y == 0.0) continue;
            double2 lv[RM];
#pragma unroll
            for (int q = 0; q < RM; ++q) {
                const int i = g + G * q;
                lv[q] = (i > k && i < n) ? panel[p * n + i] : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int w = 0; w < NCW; ++w) {
                double2 a0 = make_double2(0.0, 0.0), a1 = a0;
#pragma unroll
                for (int q = 0; q < RM; ++q) {
                    if (q & 1) a1 = cfmac(lv[q], y[w][q], a1); else a0 = cfmac(lv[q], y[w][q], a0);
                }
                double2 acc = cadd(a0, a1);
#pragma unroll
                for (int o = 1; o < G; o <<= 1) { acc.x += shfl_xor(acc.x, o); acc.y += shfl_xor(acc.y, o); }
                const double2 sc = cmul(tk, acc);
#pragma unroll
                for (int q = 0; q < RM; ++q) y[w][q] = cfms(lv[q], sc, y[w][q]);
            }
        }
    }
    // ---- X = L^{-H} Y: x_k = (y_k - sum_{i > k} conj(L(i, k)) x_i) / L(k, k), k = n-1 .. 0
    if (mode == kBackFull || mode == kBackLOnly) {
        for (int k0 = n - 1; k0 >= 0; k0 -= kBigPanel) {
            __syncthreads();
            for (int p = 0; p < kBigPanel && k0 - p >= 0; ++p) {
                const int k = k0 - p;
                const double2* src = LVb + static_cast<size_t>(k) * n;           // src[i] = L(i, k)
                for (int i = k + 1 + tid; i < n; i += kBigThreads) panel[p * n + i] = src[i];
            }
            __syncthreads();
#pragma unroll 1
            for (int p = 0; p < kBigPanel; ++p) {
                const int k = k0 - p;
                if (k < 0) break;
                const double ik = invd[k];
                const int rk = k / G, gk = k - rk * G;
                double2 lv[RM];
#pragma unroll
                for (int q = 0; q < RM; ++q) {
                    const int i = g + G * q;
                    lv[q] = (i > k && i < n) ? panel[p * n + i] : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int w = 0; w < NCW; ++w) {
                    double2 a0 = make_double2(0.0, 0.0), a1 = a0;
#pragma unroll
                    for (int q = 0; q < RM; ++q) {
                        if (q & 1) a1 = cfmac(lv[q], y[w][q], a1); else a0 = cfmac(lv[q], y[w][q], a0);
                    }
                    double2 acc = cadd(a0, a1);
#pragma unroll
                    for (int o = 1; o < G; o <<= 1) { acc.x += shfl_xor(acc.x, o); acc.y += shfl_xor(acc.y, o); }
                    double2 xk = cshfl(seg_get(y[w], rk), (lane & ~(G - 1)) | gk);
                    xk = cscale(csub(xk, acc), ik);
                    if (g == gk) seg_set(y[w], rk, xk);
                }
            }
        }
    }
#pragma unroll
    for (int w = 0; w < NCW; ++w)
#pragma unroll
        for (int q = 0; q < RM; ++q) {
            const int i = g + G * q, lc = grp + GROUPS * w;
            if (lc < nc && i < n) Xb[i + static_cast<size_t>(c0 + lc) * n] = y[w][q];
        }
}

template <class K>
void set_big_smem_once(K kernel, SmemOptIn& rec, size_t bytes) {
    set_smem_limit(reinterpret_cast<const void*>(kernel), rec, static_cast<int>(bytes));
}

template <typename... KArgs, typename... Args>
cudaError_t launch_clustered(void (*kernel)(KArgs...), int cs, int grid, int threads, size_t smem,
                             cudaStream_t stream, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(static_cast<unsigned>(threads));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(cs);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// (cluster size, rows per lane) by n: n <= 96 -> (4, 3), <= 128 -> (4, 4), <= 160 -> (8, 5),
// <= 192 -> (8, 6), <= 256 -> (8, 8).
#define SBG_BIG_DISPATCH(n, FN, ...)                                              \
    do {                                                                          \
        if ((n) <= 96) FN<4, 3>(__VA_ARGS__);                                     \
        else if ((n) <= 128) FN<4, 4>(__VA_ARGS__);                               \
        else if ((n) <= 160) FN<8, 5>(__VA_ARGS__);                               \
        else if ((n) <= 192) FN<8, 6>(__VA_ARGS__);                               \
        else FN<8, 8>(__VA_ARGS__);                                               \
    } while (0)

template <int CS, int RM>
void run_reduce_big(cudaError_t* err, const double2* A, const double2* B, int n, int batch, const Workspace& ws,
                    double2* X, int* info, cudaStream_t stream, int mode) {
    const size_t smem = BigReduceSmem(n, CS).total;
    static SmemOptIn f;
    set_big_smem_once(k_reduce_big<CS, RM>, f, static_cast<size_t>(max_smem_optin()));
    *err = launch_clustered(k_reduce_big<CS, RM>, CS, batch * CS, kBigThreads, smem, stream, A, B, n, batch, ws, X,
                            info, mode);
}

template <int CS, int G, int RM, int NCW>
void run_back_big(cudaError_t* err, int mode, int n, int batch, const Workspace& ws, double2* X, const int* info,
                  cudaStream_t stream) {
    const size_t smem = BigBackSmem(n).total;
    static SmemOptIn f;
    set_big_smem_once(k_back_big<CS, G, RM, NCW>, f, static_cast<size_t>(max_smem_optin()));
    *err = launch_clustered(k_back_big<CS, G, RM, NCW>, CS, batch * CS, kBigThreads, smem, stream, mode, n, batch,
                            ws, X, info);
}

template <int CS, int RM>
void big_smem_of(size_t* out, int n) { *out = BigReduceSmem(n, CS).total; }

constexpr int kMidMaxN = 160;             // the packed tile + buffers fit 227 KB up to here

template <int RM>
void run_reduce_mid(const double2* A, const double2* B, int n, int batch, const Workspace& ws, double2* X, int* info,
                    cudaStream_t stream, int mode) {
    static SmemOptIn f;
    set_big_smem_once(k_reduce_mid<RM>, f, static_cast<size_t>(max_smem_optin()));
    k_reduce_mid<RM><<<batch, kMidThreads, MidSmem(n).total, stream>>>(A, B, n, batch, ws, X, info, mode);
}

}  // namespace

bool big_path(int n) { return n > kSmallMaxN && n <= kBigMaxN; }

size_t big_reduce_smem_bytes(int n) {
    if (n <= kMidMaxN) return MidSmem(n).total;
    size_t s = 0;
    SBG_BIG_DISPATCH(n, big_smem_of, &s, n);
    return s;
}

cudaError_t launch_reduce_big(const double2* A, const double2* B, int n, int batch, const Workspace& ws, double2* X,
                              int* info, cudaStream_t stream, int mode) {
    if (batch <= 0) return cudaSuccess;
    if (!A || !B || !X || !info || !ws.LV || !ws.d || !ws.e || !ws.tau) return cudaErrorInvalidValue;
    if (!big_path(n) || mode < kBigFull || mode > kBigHetrdOnly) return cudaErrorInvalidValue;
    // the Householder alone: one CTA per pair, one pass over the L2-resident packed triangle per step
    // (k_hetrd_l2), measured faster than both the shared-memory tile of k_reduce_mid (1.04x at
    // n = 96, 1.3x at n = 128 and 160, whole reduce stage) and the 8-CTA cluster (4.7x at n = 192)
    if (mode == kBigHetrdOnly) return launch_hetrd_l2(n, batch, X, ws, info, stream);
    if (n <= kMidMaxN) {                     // one CTA per pair: no cluster barriers
        if (n <= 96) run_reduce_mid<12>(A, B, n, batch, ws, X, info, stream, mode);
        else if (n <= 128) run_reduce_mid<16>(A, B, n, batch, ws, X, info, stream, mode);
        else run_reduce_mid<20>(A, B, n, batch, ws, X, info, stream, mode);
        return cudaGetLastError();
    }
    cudaError_t err = cudaSuccess;
    SBG_BIG_DISPATCH(n, run_reduce_big, &err, A, B, n, batch, ws, X, info, stream, mode);
    return err != cudaSuccess ? err : cudaGetLastError();
}

size_t hetrd_c64_big_smem_bytes(int n) { return C64BigSmem(n).total; }

cudaError_t launch_hetrd_c64_big(int n, int batch, const double2* C, const Workspace& ws, int* info,
                                 cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (n <= kMixedMaxN || n > kMixedBigMaxN) return cudaErrorInvalidValue;
    if (!C || !info || !ws.LV || !ws.d || !ws.e || !ws.tau || !ws.rfC) return cudaErrorInvalidValue;
    const size_t smem = C64BigSmem(n).total;
    if (smem > static_cast<size_t>(max_smem_optin())) return cudaErrorInvalidValue;
    static SmemOptIn f;
    set_big_smem_once(k_hetrd_c64_big, f, smem);
    k_hetrd_c64_big<<<batch, kMidThreads, smem, stream>>>(n, batch, C, ws, info);
    return cudaGetLastError();
}

cudaError_t launch_hetrd_l2(int n, int batch, const double2* C, const Workspace& ws, int* info,
                           cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (n <= kSmallMaxN || n > kBigMaxN || !C || !info || !ws.LV || !ws.d || !ws.e || !ws.tau || !ws.log)
        return cudaErrorInvalidValue;
    if (static_cast<size_t>(ws.log_stride) < static_cast<size_t>(n) * (n + 1) / 2) return cudaErrorInvalidValue;
    const size_t smem = L2HetrdSmem(n).total;
    if (smem > static_cast<size_t>(max_smem_optin())) return cudaErrorInvalidValue;
    static SmemOptIn f;
    set_big_smem_once(k_hetrd_l2, f, smem);
    k_hetrd_l2<<<batch, kMidThreads, smem, stream>>>(n, batch, C, ws, info);
    return cudaGetLastError();
}

size_t ql_rows_smem_bytes(int n, bool single) { return single ? ql_rows_bytes<float>(n) : ql_rows_bytes<double>(n); }

size_t big_stage_smem_bytes(int n, bool tc, int chain_threads) {
    size_t m = std::max(ql_rows_smem_bytes(n, false), ql_chain_smem_bytes(n, chain_threads, false));
    if (eig_by_inverse_iteration(n, false)) m = std::max(m, invit_smem_bytes(n, false));
    if (tc) return std::max(m, L2HetrdSmem(n).total);       // k_reduce_tc / k_back_*_tc: static only
    return std::max(m, std::max(big_reduce_smem_bytes(n), BigBackSmem(n).total));
}

cudaError_t launch_ql_rows(int n, int batch, const Workspace& ws, double* W, double2* X, int* info, bool single,
                           int chain_threads, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (!W || !X || !info || !ws.d || !ws.e || !ws.log || !ws.perm || !ws.flag) return cudaErrorInvalidValue;
    const size_t cs = ql_chain_smem_bytes(n, chain_threads, single);
    const size_t as = ql_rows_smem_bytes(n, single);
    if (cs > static_cast<size_t>(max_smem_optin()) || as > static_cast<size_t>(max_smem_optin()))
        return cudaErrorInvalidValue;
    // FP64 up to kInvitBigMaxN: inverse iteration for every pair it can take, then the rotation-log
    // QL below for the pairs it flagged only
    const bool redo = eig_by_inverse_iteration(n, single);
    if (redo) {
        cudaError_t err = launch_eig_invit(n, batch, ws, W, X, info, chain_threads, true, stream);
        if (err != cudaSuccess) return err;
    }
    cudaError_t err = launch_ql_chain(n, batch, ws, W, info, single, chain_threads, stream, redo);
    if (err != cudaSuccess) return err;
    const int grid = ((n + 31) / 32) * batch;
    static SmemOptIn fd, ff;
    if (single) {
        set_big_smem_once(k_ql_apply_rows<float>, ff, static_cast<size_t>(max_smem_optin()));
        k_ql_apply_rows<float><<<grid, 32, as, stream>>>(n, batch, ws, W, X, info, 0);
    } else {
        set_big_smem_once(k_ql_apply_rows<double>, fd, static_cast<size_t>(max_smem_optin()));
        k_ql_apply_rows<double><<<grid, 32, as, stream>>>(n, batch, ws, W, X, info, redo ? 1 : 0);
    }
    return cudaGetLastError();
}

cudaError_t launch_back_big(int mode, int n, int batch, const Workspace& ws, double2* X, const int* info,
                            cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (!X || !info || !ws.LV || !ws.tau) return cudaErrorInvalidValue;
    if (!big_path(n)) return cudaErrorInvalidValue;
    cudaError_t err = cudaSuccess;
    // (CTAs per pair, rows per lane, columns per lane group): 8 lanes per column, rows 8 q + g
    // (CTAs per pair, lanes per column, rows per lane, columns per lane group): one column
    // per 8-lane group (32 columns per CTA) up to n = 160, two per 16-lane group above
    if (n <= 96) run_back_big<3, 8, 12, 1>(&err, mode, n, batch, ws, X, info, stream);
    else if (n <= 128) run_back_big<4, 8, 16, 1>(&err, mode, n, batch, ws, X, info, stream);
    else if (n <= 160) run_back_big<5, 8, 20, 1>(&err, mode, n, batch, ws, X, info, stream);
    else run_back_big<8, 16, 16, 2>(&err, mode, n, batch, ws, X, info, stream);
    return err != cudaSuccess ? err : cudaGetLastError();
}

}  // namespace sbg
