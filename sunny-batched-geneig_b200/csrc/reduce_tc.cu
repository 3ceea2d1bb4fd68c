// Blocked FP64 Cholesky and two-sided reduction on the FP64 tensor cores, one CTA (4 warps) per
// pair, for n > kSmallMaxN, where the scalar kernels that hold a pair's triangle in shared memory
// (k_reduce_mid) or spread it over a cluster (k_reduce_big) run at a few percent of the FP64 peak.
//
//   k_reduce_tc   B = L L^H, W = L^{-1} A, C = L^{-1} W^H (= L^{-1} A L^{-H}), in 32 x 32 blocks:
//                   Cholesky, left-looking: T(:, K) = B(:, K) - L(:, <K) L(K, <K)^H (tile products),
//                     the diagonal block factored in shared memory (zpotrf's steps), inverted there
//                     (ztrti2's steps), the panel L(I, K) = T(I, K) L(K, K)^{-H} a tile product with
//                     that inverse;
//                   W, block row by block row: T(I, :) = A(I, :) - L(I, <I) W(<I, :), then
//                     W(I, :) = L(I, I)^{-1} T(I, :) (a tile product with the inverted diagonal
//                     block, the blocked trsm of GPU solver libraries);
//                   C, lower blocks only: T(I, J) = W(J, I)^H - L(I, <I) C(<I, J), where C(K, J)
//                     above the diagonal is read as C(J, K)^H, then C(I, J) = L(I, I)^{-1} T(I, J).
//                 Every product goes through tiles.cuh (32 x 32 output tiles, mma.sync.m8n8k4.f64).
//                 L goes to LV's lower triangle, C's lower triangle to X (over W, whose blocks below
//                 the diagonal are no longer read once the block row of C that overwrites them is
//                 formed); the inverted diagonal blocks live in the pair's rotation-log region
//                 (free until the eigensolve).  The outputs are those of the other reduce kernels in
//                 kReduceMixed mode: info = n + i for a leading minor i that is not positive definite
//                 (the pair's outputs are then left to the later stages' NaN handling).
#include "kernels.cuh"
#include "tiles.cuh"

namespace sbg {

namespace {

constexpr int kNB = kTile;               // block size of the blocked algorithm
constexpr int kDLD = kNB + 1;            // the diagonal block in shared memory (odd stride)

struct TcSmem {
    TileSmem t;
    double2 D[kNB * kDLD];
};

// The diagonal block (bs x bs lower triangle of T at (c0, c0), padded to 32 with the identity)
// factored in place, D = L_KK (zpotrf 'L', right-looking).  Returns 0, or the local column + 1 of
// the first pivot that is not positive (also NaN); uniform over the CTA.
__device__ int factor_diag(TcSmem& sm, const double2* L, int n, int c0, int bs) {
    const int tid = threadIdx.x;
    for (int e = tid; e < kNB * kNB; e += kTileThreads) {
        const int i = e % kNB, j = e / kNB;
        double2 v = make_double2(i == j ? 1.0 : 0.0, 0.0);
        if (i < bs && j < bs && i >= j) v = ldcg2(L + (c0 + i) + static_cast<size_t>(c0 + j) * n);
        sm.D[i + j * kDLD] = v;
    }
    __syncthreads();
    for (int k = 0; k < kNB; ++k) {
        const double dkk = sm.D[k + k * kDLD].x;
        __syncthreads();                                  // every thread has read the pivot
        if (!(dkk > 0.0)) return k + 1;                   // uniform
        const double dsq = sqrt(dkk), inv = 1.0 / dsq;
        if (tid > k && tid < kNB) sm.D[tid + k * kDLD] = cscale(sm.D[tid + k * kDLD], inv);
        if (tid == 0) sm.D[k + k * kDLD] = make_double2(dsq, 0.0);
        __syncthreads();
        for (int e = tid; e < kNB * kNB; e += kTileThreads) {
            const int i = e % kNB, j = e / kNB;
            if (j > k && i >= j)
                sm.D[i + j * kDLD] = cfmsc(sm.D[i + k * kDLD], sm.D[j + k * kDLD], sm.D[i + j * kDLD]);
        }
        __syncthreads();
    }
    return 0;
}

// D = L_KK^{-1} in place (ztrti2 'L', non-unit): for j = 31 .. 0, with the block below and right of
// (j, j) already inverted, column j becomes -L22^{-1} l_j / l_jj and (j, j) becomes 1 / l_jj.
__device__ void invert_diag(TcSmem& sm) {
    const int tid = threadIdx.x;
    for (int j = kNB - 1; j >= 0; --j) {
        double2 acc = make_double2(0.0, 0.0);
        if (tid > j && tid < kNB)
            for (int l = j + 1; l <= tid; ++l) acc = cfma(sm.D[tid + l * kDLD], sm.D[l + j * kDLD], acc);
        const double inv = 1.0 / sm.D[j + j * kDLD].x;
        __syncthreads();                                  // column j and the pivot are read
        if (tid > j && tid < kNB) sm.D[tid + j * kDLD] = cscale(acc, -inv);
        if (tid == 0) sm.D[j + j * kDLD] = make_double2(inv, 0.0);
        __syncthreads();
    }
}

// One 32 x 32 tile of a block product into a column-major n x n matrix: acc (already holding the
// tile's initial value) plus the products the caller adds, stored at (r0, c0) (lower: only
// entries on or below the global diagonal).
__device__ __forceinline__ void store_tile(const Quarter& acc, double2* M, int n, int r0, int c0, bool lower) {
    quarter_store(acc, M + r0 + static_cast<size_t>(c0) * n, n, n - r0, n - c0, lower, r0, c0);
}

__global__ void __launch_bounds__(kTileThreads, 3) k_reduce_tc(const double2* A, const double2* B, int n, int batch,
                                                               Workspace ws, double2* X, int* info) {
    __shared__ TcSmem sm;
    const int b = blockIdx.x;
    if (b >= batch || !pair_selected(ws, b)) return;
    const int tid = threadIdx.x;
    const size_t mat = static_cast<size_t>(n) * n;
    const double2* Ab = A + mat * b;
    const double2* Bb = B + mat * b;
    double2* Xb = X + mat * b;
    double2* L = ws.LV + mat * b;
    double2* Linv = static_cast<double2*>(ws.log) + static_cast<size_t>(ws.log_stride) * b;   // kNB^2 per block
    const int nbk = (n + kNB - 1) / kNB;
    const MatView none{nullptr, 1, 0, 0};

    // ---- Cholesky, left-looking by blocks of 32 columns
    for (int K = 0; K < nbk; ++K) {
        const int c0 = kNB * K, bs = min(kNB, n - c0);
        for (int I = K; I < nbk; ++I) {                       // T(I, K) = B(I, K) - L(I, <K) L(K, <K)^H
            const int r0 = kNB * I;
            Quarter acc[1];
            quarter_load<kOpN>(acc[0], sub_view(Bb, n, n, n, r0, c0));     // B's upper part is never stored
            if (K > 0)
                tile_mm<kOpN, kOpC, 1>(acc, sub_view(L, n, n, n, r0, 0), sub_view(L, n, n, n, c0, 0), none, c0,
                                       sm.t, true);
            store_tile(acc[0], L, n, r0, c0, I == K);
        }
        __syncthreads();
        const int f = factor_diag(sm, L, n, c0, bs);
        if (f) {                                              // uniform: the leading minor c0 + f is not PD
            if (tid == 0) info[b] = n + c0 + f;
            return;
        }
        for (int e = tid; e < kNB * kNB; e += kTileThreads) {
            const int i = e % kNB, j = e / kNB;
            if (i < bs && j < bs && i >= j) L[(c0 + i) + static_cast<size_t>(c0 + j) * n] = sm.D[i + j * kDLD];
        }
        invert_diag(sm);
        double2* LiK = Linv + static_cast<size_t>(K) * kNB * kNB;
        for (int e = tid; e < kNB * kNB; e += kTileThreads) {
            const int i = e % kNB, j = e / kNB;
            LiK[e] = i >= j ? sm.D[i + j * kDLD] : make_double2(0.0, 0.0);
        }
        __syncthreads();
        const MatView inv{LiK, kNB, kNB, kNB};
        for (int I = K + 1; I < nbk; ++I) {                   // L(I, K) = T(I, K) L(K, K)^{-H}, in place
            const int r0 = kNB * I;
            Quarter acc[1];
            acc[0].zero();
            tile_mm<kOpN, kOpC, 1>(acc, sub_view(L, n, n, n, r0, c0), inv, none, bs, sm.t);
            store_tile(acc[0], L, n, r0, c0, false);
        }
        __syncthreads();
    }

    // ---- W = L^{-1} A, block row by block row, into X
    for (int I = 0; I < nbk; ++I) {
        const int r0 = kNB * I, bs = min(kNB, n - r0);
        for (int C = 0; C < nbk; ++C) {                       // T(I, :) = A(I, :) - L(I, <I) W(<I, :)
            const int cc = kNB * C;
            Quarter acc[1];
            quarter_load<kOpN>(acc[0], sub_view(Ab, n, n, n, r0, cc));
            if (I > 0)
                tile_mm<kOpN, kOpN, 1>(acc, sub_view(L, n, n, n, r0, 0), sub_view(Xb, n, n, n, 0, cc), none, r0,
                                       sm.t, true);
            store_tile(acc[0], Xb, n, r0, cc, false);
        }
        __syncthreads();
        const MatView inv{Linv + static_cast<size_t>(I) * kNB * kNB, kNB, kNB, kNB};
        for (int C = 0; C < nbk; ++C) {                       // W(I, :) = L(I, I)^{-1} T(I, :), in place
            const int cc = kNB * C;
            Quarter acc[1];
            acc[0].zero();
            tile_mm<kOpN, kOpN, 1>(acc, inv, sub_view(Xb, n, n, n, r0, cc), none, bs, sm.t);
            store_tile(acc[0], Xb, n, r0, cc, false);
        }
        __syncthreads();
    }

    // ---- C = L^{-1} W^H, lower blocks, over X.  Block (I, J), J <= I:
    //   T(I, J) = W(J, I)^H - L(I, <J) C(<J, J) - L(I, J..I-1) C(J..I-1, J),
    // where C(K, J) for K < J lies above the diagonal and is read as C(J, K)^H (block row J is done;
    // for J = I its blocks K < I were formed earlier in this row), then C(I, J) = L(I, I)^{-1} T(I, J).
    // W(J, I) with J < I is above the diagonal, which C never overwrites; W(I, I) is read before
    // C(I, I) replaces it.
    for (int I = 0; I < nbk; ++I) {
        const int r0 = kNB * I, bs = min(kNB, n - r0);
        const MatView inv{Linv + static_cast<size_t>(I) * kNB * kNB, kNB, kNB, kNB};
        for (int J = 0; J <= I; ++J) {
            const int cj = kNB * J;
            Quarter acc[1];
            quarter_load<kOpC>(acc[0], sub_view(Xb, n, n, n, cj, r0));     // W(cj + j, r0 + i)^*
            if (J > 0)
                tile_mm<kOpN, kOpC, 1>(acc, sub_view(L, n, n, n, r0, 0), sub_view(Xb, n, n, n, cj, 0), none, cj,
                                       sm.t, true);
            if (r0 > cj)
                tile_mm<kOpN, kOpN, 1>(acc, sub_view(L, n, n, n, r0, cj), sub_view(Xb, n, n, n, cj, cj), none,
                                       r0 - cj, sm.t, true);
            __syncthreads();                                  // every read of the tile's W^H done
            store_tile(acc[0], Xb, n, r0, cj, false);
            __syncthreads();
            acc[0].zero();
            tile_mm<kOpN, kOpN, 1>(acc, inv, sub_view(Xb, n, n, n, r0, cj), none, bs, sm.t);
            store_tile(acc[0], Xb, n, r0, cj, false);
            __syncthreads();
        }
    }
    for (int i = tid; i < n; i += kTileThreads) Xb[i + static_cast<size_t>(i) * n].y = 0.0;   // Hermitian C
    if (tid == 0) info[b] = 0;
}

// X = L^{-H} Y in place over the X buffer (Y complex there), one CTA per pair, for n > kSmallMaxN:
// the backward substitution by blocks of 32, from the last block row up,
//   T(I, :) = Y(I, :) - L(>I, I)^H X(>I, :),   X(I, :) = L(I, I)^{-H} T(I, :),
// every product a tile product on the FP64 tensor cores; the diagonal blocks of L (LV's lower
// triangle) inverted in shared memory into the pair's rotation-log region (free again after the
// eigensolve).  Pairs with info outside 0..n get NaN (B was not positive definite); pairs not
// selected are left alone.
__global__ void __launch_bounds__(kTileThreads, 3) k_back_tc(int n, int batch, Workspace ws, double2* X,
                                                             const int* info) {
    __shared__ TcSmem sm;
    const int b = blockIdx.x;
    if (b >= batch || !pair_selected(ws, b)) return;
    const int tid = threadIdx.x;
    const size_t mat = static_cast<size_t>(n) * n;
    double2* Xb = X + mat * b;
    if (info[b] > n || info[b] < 0) {                         // uniform
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        for (size_t idx = tid; idx < mat; idx += kTileThreads) Xb[idx] = make_double2(nan, nan);
        return;
    }
    const double2* L = ws.LV + mat * b;
    double2* Linv = static_cast<double2*>(ws.log) + static_cast<size_t>(ws.log_stride) * b;
    const int nbk = (n + kNB - 1) / kNB;
    const MatView none{nullptr, 1, 0, 0};
    for (int K = 0; K < nbk; ++K) {                           // the diagonal blocks of L, inverted
        const int c0 = kNB * K, bs = min(kNB, n - c0);
        for (int e = tid; e < kNB * kNB; e += kTileThreads) {
            const int i = e % kNB, j = e / kNB;
            double2 v = make_double2(i == j ? 1.0 : 0.0, 0.0);
            if (i < bs && j < bs && i >= j) v = ldcg2(L + (c0 + i) + static_cast<size_t>(c0 + j) * n);
            sm.D[i + j * kDLD] = v;
        }
        __syncthreads();
        invert_diag(sm);
        double2* LiK = Linv + static_cast<size_t>(K) * kNB * kNB;
        for (int e = tid; e < kNB * kNB; e += kTileThreads) {
            const int i = e % kNB, j = e / kNB;
            LiK[e] = i >= j ? sm.D[i + j * kDLD] : make_double2(0.0, 0.0);
        }
        __syncthreads();
    }
    for (int I = nbk - 1; I >= 0; --I) {
        const int r0 = kNB * I, bs = min(kNB, n - r0), below = n - r0 - bs;
        if (below > 0) {
            for (int C = 0; C < nbk; ++C) {                   // T(I, :) = Y(I, :) - L(>I, I)^H X(>I, :)
                const int cc = kNB * C;
                Quarter acc[1];
                quarter_load<kOpN>(acc[0], sub_view(Xb, n, n, n, r0, cc));
                tile_mm<kOpC, kOpN, 1>(acc, sub_view(L, n, n, n, r0 + bs, r0), sub_view(Xb, n, n, n, r0 + bs, cc),
                                       none, below, sm.t, true);
                store_tile(acc[0], Xb, n, r0, cc, false);
            }
            __syncthreads();
        }
        const MatView inv{Linv + static_cast<size_t>(I) * kNB * kNB, kNB, kNB, kNB};
        for (int C = 0; C < nbk; ++C) {                       // X(I, :) = L(I, I)^{-H} T(I, :), in place
            const int cc = kNB * C;
            Quarter acc[1];
            acc[0].zero();
            tile_mm<kOpC, kOpN, 1>(acc, inv, sub_view(Xb, n, n, n, r0, cc), none, bs, sm.t);
            store_tile(acc[0], Xb, n, r0, cc, false);
        }
        __syncthreads();
    }
}

// Y = Q Z for n > kSmallMaxN (Z real in the X buffer, Y complex over it), Q = H_0 H_1 ... H_{n-2}
// from the reflectors the big-n Householder stores (v_k(k+1+s) = LV(s, n-1-k), v_k(k+1) = 1) and
// tau: blocks of 32 reflectors in compact WY form, Q_blk = I - V T V^H with T upper triangular
// (LAPACK zlarft, forward, columnwise: T(i, i) = tau_i, T(0:i, i) = -tau_i T(0:i, 0:i) V^H v_i),
// applied from the last block to the first, Y(rows below the block) -= V (T (V^H Y)), every product
// a tile product on the FP64 tensor cores.  One CTA per pair; the pair's rotation-log region (free
// after the eigensolve) holds a copy of Z, the block's V (n x 32), T (32 x 32) and V^H Y (32 x n).
// Pairs with info outside 0..n get NaN; pairs not selected are left alone.
__global__ void __launch_bounds__(kTileThreads, 3) k_back_q_tc(int n, int batch, Workspace ws, double2* X,
                                                               const int* info) {
    __shared__ TcSmem sm;
    __shared__ double2 s_tau[kNB];
    const int b = blockIdx.x;
    if (b >= batch || !pair_selected(ws, b)) return;
    const int tid = threadIdx.x;
    const size_t mat = static_cast<size_t>(n) * n;
    double2* Xb = X + mat * b;
    if (info[b] > n || info[b] < 0) {                         // uniform
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        for (size_t idx = tid; idx < mat; idx += kTileThreads) Xb[idx] = make_double2(nan, nan);
        return;
    }
    const double2* LV = ws.LV + mat * b;
    const double2* taub = ws.tau + static_cast<size_t>(n) * b;
    double2* scr = static_cast<double2*>(ws.log) + static_cast<size_t>(ws.log_stride) * b;
    double* Zc = reinterpret_cast<double*>(scr);                              // n^2 doubles
    double2* Vb = scr + (mat + 1) / 2;                                        // n x 32, ld n
    double2* Tb = Vb + static_cast<size_t>(n) * kNB;                          // 32 x 32
    double2* Wb = Tb + kNB * kNB;                                             // 32 x n, ld 32
    const MatView none{nullptr, 1, 0, 0};
    // ---- Y = Z as complex (through a copy of Z: the complex Y overwrites the real Z it is made of)
    const double* Zg = reinterpret_cast<const double*>(Xb);
    for (size_t idx = tid; idx < mat; idx += kTileThreads) Zc[idx] = Zg[idx];
    __syncthreads();
    for (size_t idx = tid; idx < mat; idx += kTileThreads) Xb[idx] = make_double2(Zc[idx], 0.0);
    __syncthreads();
    const int nref = n - 1;                                   // reflectors 0 .. n-2
    const int nblk = (nref + kNB - 1) / kNB;
    for (int blk = nblk - 1; blk >= 0; --blk) {
        const int j0 = kNB * blk, kb = min(kNB, nref - j0), r0 = j0 + 1, m = n - r0;
        // V: rows r0 .. n-1 of reflectors j0 .. j0 + kb - 1 (zero above each one's leading 1)
        for (int e = tid; e < m * kNB; e += kTileThreads) {
            const int r = e % m, jj = e / m, k = j0 + jj, i = r0 + r;
            double2 v = make_double2(0.0, 0.0);
            if (jj < kb) {
                if (i == k + 1) v = make_double2(1.0, 0.0);
                else if (i > k + 1) v = ldcg2(LV + (i - k - 1) + static_cast<size_t>(n - 1 - k) * n);
            }
            Vb[r + static_cast<size_t>(jj) * n] = v;
        }
        if (tid < kNB) s_tau[tid] = tid < kb ? ldcg2(taub + j0 + tid) : make_double2(0.0, 0.0);
        __syncthreads();
        const MatView vview{Vb, n, m, kNB};
        {                                                     // G = V^H V into D
            Quarter acc[1];
            acc[0].zero();
            tile_mm<kOpC, kOpN, 1>(acc, vview, vview, none, m, sm.t);
            quarter_store(acc[0], Tb, kNB, kNB, kNB);
        }
        __syncthreads();
        for (int e = tid; e < kNB * kNB; e += kTileThreads) sm.D[(e % kNB) + (e / kNB) * kDLD] = ldcg2(Tb + e);
        __syncthreads();
        // T over G's strict upper part (G(l, j) is read only for l < j, T(i, l) only for i <= l < j)
        for (int j = 0; j < kNB; ++j) {
            double2 t = make_double2(0.0, 0.0);
            if (tid < j) {
                for (int l = tid; l < j; ++l) {
                    const double2 til = l == tid ? s_tau[tid] : sm.D[l + tid * kDLD];    // T(tid, l), stored transposed
                    t = cfma(til, sm.D[l + j * kDLD], t);
                }
                t = cmul(t, make_double2(-s_tau[j].x, -s_tau[j].y));
            }
            __syncthreads();                                  // column j of G is read
            if (tid < j) sm.D[j + tid * kDLD] = t;            // T(tid, j) kept at D(j, tid), below the diagonal
            __syncthreads();
        }
        for (int e = tid; e < kNB * kNB; e += kTileThreads) {
            const int i = e % kNB, j = e / kNB;
            double2 v = make_double2(0.0, 0.0);
            if (i == j) v = s_tau[i];
            else if (i < j) v = sm.D[j + i * kDLD];
            Tb[e] = v;                                        // T(i, j), upper triangular
        }
        __syncthreads();
        const MatView tview{Tb, kNB, kNB, kNB};
        for (int cc = 0; cc < n; cc += kTile) {               // W = V^H Y(r0:, :)
            Quarter acc[1];
            acc[0].zero();
            tile_mm<kOpC, kOpN, 1>(acc, vview, sub_view(Xb, n, n, n, r0, cc), none, m, sm.t);
            quarter_store(acc[0], Wb + static_cast<size_t>(cc) * kNB, kNB, kNB, n - cc);
        }
        __syncthreads();
        for (int cc = 0; cc < n; cc += kTile) {               // W = T W, in place
            Quarter acc[1];
            acc[0].zero();
            tile_mm<kOpN, kOpN, 1>(acc, tview, sub_view(Wb, kNB, kNB, n, 0, cc), none, kb, sm.t);
            quarter_store(acc[0], Wb + static_cast<size_t>(cc) * kNB, kNB, kNB, n - cc);
        }
        __syncthreads();
        for (int rr = 0; rr < m; rr += kTile)                 // Y(r0:, :) -= V W
            for (int cc = 0; cc < n; cc += kTile) {
                Quarter acc[1];
                quarter_load<kOpN>(acc[0], sub_view(Xb, n, n, n, r0 + rr, cc));
                tile_mm<kOpN, kOpN, 1>(acc, sub_view(Vb, n, m, kNB, rr, 0), sub_view(Wb, kNB, kNB, n, 0, cc), none,
                                       kb, sm.t, true);
                store_tile(acc[0], Xb, n, r0 + rr, cc, false);
            }
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_reduce_tc(const double2* A, const double2* B, int n, int batch, const Workspace& ws, double2* X,
                             int* info, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (n < 1 || n > kBigMaxN || !A || !B || !X || !info || !ws.LV || !ws.log) return cudaErrorInvalidValue;
    // the inverted diagonal blocks take ceil(n / 32) x 32 x 32 entries of the rotation-log region
    if (static_cast<size_t>(ws.log_stride) < static_cast<size_t>((n + kNB - 1) / kNB) * kNB * kNB)
        return cudaErrorInvalidValue;
    k_reduce_tc<<<batch, kTileThreads, 0, stream>>>(A, B, n, batch, ws, X, info);
    return cudaGetLastError();
}

cudaError_t launch_back_tc(int n, int batch, const Workspace& ws, double2* X, const int* info, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (n < 1 || n > kBigMaxN || !X || !info || !ws.LV || !ws.log) return cudaErrorInvalidValue;
    if (static_cast<size_t>(ws.log_stride) < static_cast<size_t>((n + kNB - 1) / kNB) * kNB * kNB)
        return cudaErrorInvalidValue;
    k_back_tc<<<batch, kTileThreads, 0, stream>>>(n, batch, ws, X, info);
    return cudaGetLastError();
}

cudaError_t launch_back_q_tc(int n, int batch, const Workspace& ws, double2* X, const int* info,
                             cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (n <= kSmallMaxN || n > kBigMaxN || !X || !info || !ws.LV || !ws.tau || !ws.log) return cudaErrorInvalidValue;
    // Z's copy, V, T and V^H Y in the rotation-log region
    const size_t need = (static_cast<size_t>(n) * n + 1) / 2 + static_cast<size_t>(2 * n + kNB) * kNB;
    if (static_cast<size_t>(ws.log_stride) < need) return cudaErrorInvalidValue;
    k_back_q_tc<<<batch, kTileThreads, 0, stream>>>(n, batch, ws, X, info);
    return cudaGetLastError();
}

}  // namespace sbg
