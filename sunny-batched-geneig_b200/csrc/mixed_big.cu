// Mixed form above kMixedMaxN (kMixedMaxN < n <= kMixedBigMaxN): the FP64 Ogita-Aishima
// refinement of the complex64 eigen-decomposition of C = L^{-1} A L^{-H}, for orders whose C and
// eigenvector matrix no longer fit one SM's shared memory together (at n = 128 each is 256 KB).
//
//   k_refine_big   one CTA (4 warps) per pair.  The pair's n x n matrices live in the workspace
//                  (column-major, ld = n): C (ws.rfC, written by k_hetrd_c64_big), the
//                  eigenvectors Y (the X buffer and ws.rfY, alternating as Y is updated), P = C Y
//                  (ws.rfP, later the correction E), G = Y^H Y (ws.rfG), S = Y^H P (ws.rfS).
//                  Every product is computed 32 x 32 output tile by tile: 16-deep panels of both
//                  operands staged in shared memory (the next panel prefetched into registers
//                  while the current one is multiplied), each warp a 16 x 16 quarter of the tile as
//                  2 x 2 blocks of mma.sync.m8n8k4.f64 (a complex product as four real ones).  G
//                  and S are Hermitian: only their lower tiles are formed, both in one pass over
//                  Y^H.  Each pair's outcome goes to ws.rstat (kRefineDone, kRefineRedo,
//                  kRefineSkip).
#include "kernels.cuh"
#include "stages.cuh"
#include "tiles.cuh"

namespace sbg {

namespace {

constexpr int kRfThreads = kTileThreads;
constexpr int kRfTile = kTile;
constexpr int kRfWarps = kTileWarps;
constexpr double kRfEps = 1.1102230246251565e-16;
constexpr double kRfOrthTol = 1e-13;     // max |(Y^H Y - I)_ij| accepted

struct RfSmem {
    TileSmem t;
    double lam[kMixedBigMaxN];
    double red[4 * kRfWarps];
    int order[kMixedBigMaxN];
};

// The tile at (r0, c0) of products of the pair's n x n matrices: acc[o] += op(A) B_o with op(A) = A
// or A^H (CONJA), summed over all of k.
template <bool CONJA, int NOUT>
__device__ __forceinline__ void rf_tile_mm(Quarter (&acc)[NOUT], const double2* A, const double2* B0,
                                           const double2* B1, int n, int r0, int c0, RfSmem& sm) {
    const MatView a = CONJA ? sub_view(A, n, n, n, 0, r0) : sub_view(A, n, n, n, r0, 0);
    const MatView b0 = sub_view(B0, n, n, n, 0, c0);
    const MatView b1 = NOUT == 2 ? sub_view(B1, n, n, n, 0, c0) : b0;
    tile_mm<CONJA ? kOpC : kOpN, kOpN, NOUT>(acc, a, b0, b1, n, sm.t);
}

__device__ __forceinline__ void rf_store(const Quarter& acc, double2* M, int n, int r0, int c0) {
    quarter_store(acc, M + r0 + static_cast<size_t>(c0) * n, n, n - r0, n - c0);
}

// Block-wide sums of v[0], v[1] and the max of v[2]; every thread gets them.
__device__ __forceinline__ void block_sum2_max(double (&v)[3], double* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v[0] = warp_sum(v[0]);
    v[1] = warp_sum(v[1]);
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v[2] = fmax(v[2], shfl_xor(v[2], m));
    __syncthreads();                                          // red is free
    if (lane == 0) { red[4 * w] = v[0]; red[4 * w + 1] = v[1]; red[4 * w + 2] = v[2]; }
    __syncthreads();
    double a = 0.0, b = 0.0, c = 0.0;
#pragma unroll
    for (int i = 0; i < kRfWarps; ++i) { a += red[4 * i]; b += red[4 * i + 1]; c = fmax(c, red[4 * i + 2]); }
    v[0] = a; v[1] = b; v[2] = c;
}

// The Ogita-Aishima iteration on Y (Ogita & Aishima, "Iterative refinement for symmetric
// eigenvalue decomposition", Japan J. Indust. Appl. Math. 35 (2018), Algorithm 1, for a
// Hermitian C), each pass's products also deciding whether to stop:
//   P = C Y;  G = Y^H Y, S = Y^H P (lower tiles);  lam_i = S_ii / G_ii  (Rayleigh quotients);
//   stop when every column has ||P_j - lam_j y_j|| <= 256 eps ||C||_F ||y_j|| and
//   max |R_ij| <= kRfOrthTol (R = I - G);
//   else delta = max(2 (||S - diag lam||_F + ||C||_F ||R||_F), floor ||C||_F),
//   E_ij = (S_ij + lam_j R_ij) / (lam_j - lam_i) where |lam_j - lam_i| > delta, else R_ij / 2,
//   Y <- Y + Y E.  floor = 1e-2 once only the orthogonality is missing (eigenvalues closer than
//   1e-2 ||C||_F are then only orthogonalised).
// A pair not converged after max_updates updates gets kRefineRedo (the FP64 kernels solve it
// again); a pair whose eigensolve of the complex64 T did not converge likewise.
__global__ void __launch_bounds__(kRfThreads, 3) k_refine_big(int n, int batch, Workspace ws, double* W, double2* X,
                                                               int* info, int max_updates) {
    __shared__ RfSmem sm;
    const int b = blockIdx.x;
    if (b >= batch) return;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int inf = info[b];
    if (inf > n || inf < 0) {                                 // B not positive definite, or a copy timed out
        if (tid == 0) ws.rstat[b] = kRefineSkip;
        return;
    }
    if (inf != 0) {                                           // the FP64 eigensolve of the complex64 T failed
        if (tid == 0) {
            ws.rstat[b] = kRefineRedo;
            info[b] = 0;
            if (ws.redo_count) atomicAdd(ws.redo_count, 1ull);
        }
        return;
    }
    const size_t mat = static_cast<size_t>(n) * n;
    const double2* Cb = ws.rfC + mat * b;
    double2* Pb = ws.rfP + mat * b;
    double2* Gb = ws.rfG + mat * b;
    double2* Sb = ws.rfS + mat * b;
    double2* Y = X + mat * b;                                 // the current eigenvectors
    double2* Yn = ws.rfY + mat * b;                           // the next ones
    const int nt = (n + kRfTile - 1) / kRfTile;
    // ||C||_F
    double cn[3] = {0.0, 0.0, 0.0};
    for (size_t idx = tid; idx < mat; idx += kRfThreads) {
        const double2 v = ldcg2(Cb + idx);
        cn[0] = fma(v.x, v.x, fma(v.y, v.y, cn[0]));
    }
    block_sum2_max(cn, sm.red);
    const double cnorm = sqrt(cn[0]);
    for (int it = 0;; ++it) {
        // ---- P = C Y
        for (int tile = 0; tile < nt * nt; ++tile) {
            const int r0 = kRfTile * (tile % nt), c0 = kRfTile * (tile / nt);
            Quarter acc[1];
            acc[0].zero();
            rf_tile_mm<false, 1>(acc, Cb, Y, nullptr, n, r0, c0, sm);
            rf_store(acc[0], Pb, n, r0, c0);
        }
        __syncthreads();                                      // P complete (global, this CTA's writes)
        // ---- G = Y^H Y and S = Y^H P, lower tiles
        for (int tr = 0; tr < nt; ++tr)
            for (int tc = 0; tc <= tr; ++tc) {
                Quarter acc[2];
                acc[0].zero();
                acc[1].zero();
                rf_tile_mm<true, 2>(acc, Y, Y, Pb, n, kRfTile * tr, kRfTile * tc, sm);
                rf_store(acc[0], Gb, n, kRfTile * tr, kRfTile * tc);
                rf_store(acc[1], Sb, n, kRfTile * tr, kRfTile * tc);
            }
        __syncthreads();
        // ---- Rayleigh quotients
        for (int i = tid; i < n; i += kRfThreads) {
            const size_t di = i + static_cast<size_t>(i) * n;
            sm.lam[i] = ldcg2(Sb + di).x / ldcg2(Gb + di).x;
        }
        __syncthreads();
        // ---- every column's residual: ||P_j - lam_j y_j||^2 against (256 eps ||C||_F)^2 ||y_j||^2
        bool res_ok = true;
        for (int j = w; j < n; j += kRfWarps) {
            double rr = 0.0, yy = 0.0;
            const double lj = sm.lam[j];
            for (int i = lane; i < n; i += 32) {
                const size_t idx = i + static_cast<size_t>(j) * n;
                const double2 y = ldcg2(Y + idx), p = ldcg2(Pb + idx);
                const double dr = fma(-lj, y.x, p.x), di = fma(-lj, y.y, p.y);
                rr = fma(dr, dr, fma(di, di, rr));
                yy = fma(y.x, y.x, fma(y.y, y.y, yy));
            }
            rr = warp_sum(rr);
            yy = warp_sum(yy);
            const double tol = 256.0 * kRfEps * cnorm;
            if (!(rr <= tol * tol * yy)) res_ok = false;
        }
        res_ok = __syncthreads_and(res_ok);
        // ---- ||S - diag lam||_F^2, ||R||_F^2 and max |R_ij| over the lower triangle (off-diagonal twice)
        double acc3[3] = {0.0, 0.0, 0.0};
        for (size_t idx = tid; idx < mat; idx += kRfThreads) {
            const int j = static_cast<int>(idx / n), i = static_cast<int>(idx - static_cast<size_t>(j) * n);
            if (i < j) continue;
            const double2 gv = ldcg2(Gb + idx), sv = ldcg2(Sb + idx);
            const double wgt = i == j ? 1.0 : 2.0;
            const double sr = (i == j) ? sv.x - sm.lam[i] : sv.x;
            const double rr = (i == j ? 1.0 : 0.0) - gv.x, ri = gv.y;
            acc3[0] += wgt * fma(sr, sr, sv.y * sv.y);
            acc3[1] += wgt * fma(rr, rr, ri * ri);
            acc3[2] = fmax(acc3[2], fabs(rr) + fabs(ri));
        }
        block_sum2_max(acc3, sm.red);
        const bool orth_ok = acc3[2] <= kRfOrthTol;
        if (res_ok && orth_ok) break;
        if (it >= max_updates) {
            if (tid == 0) {                                   // the FP64 kernels solve it again
                ws.rstat[b] = kRefineRedo;
                if (ws.redo_count) atomicAdd(ws.redo_count, 1ull);
            }
            return;
        }
        const double floor_rel = res_ok ? 1e-2 : 0.0;
        const double delta = fmax(2.0 * (sqrt(acc3[0]) + cnorm * sqrt(acc3[1])), floor_rel * cnorm);
        // ---- E over P (no longer read): each lower entry gives E_ij and, mirrored, E_ji
        __syncthreads();                                      // every residual read of P is done
        for (size_t idx = tid; idx < mat; idx += kRfThreads) {
            const int j = static_cast<int>(idx / n), i = static_cast<int>(idx - static_cast<size_t>(j) * n);
            if (i < j) continue;
            const double2 gv = ldcg2(Gb + idx), sv = ldcg2(Sb + idx);
            const double rr = (i == j ? 1.0 : 0.0) - gv.x, ri = -gv.y;
            const double li = sm.lam[i], lj = sm.lam[j], gap = lj - li;
            double er, ei, fr, fi;                            // E_ij, E_ji
            if (i != j && fabs(gap) > delta) {
                const double inv = 1.0 / gap;
                er = fma(lj, rr, sv.x) * inv;
                ei = fma(lj, ri, sv.y) * inv;
                fr = -fma(li, rr, sv.x) * inv;                // (conj S_ij + lam_i conj R_ij) / (lam_i - lam_j)
                fi = fma(li, ri, sv.y) * inv;
            } else {
                er = 0.5 * rr; ei = 0.5 * ri;
                fr = 0.5 * rr; fi = -0.5 * ri;
            }
            __stcg(Pb + idx, make_double2(er, ei));
            if (i != j) __stcg(Pb + j + static_cast<size_t>(i) * n, make_double2(fr, fi));
        }
        __syncthreads();                                      // E complete
        // ---- Y_next = Y + Y E
        for (int tile = 0; tile < nt * nt; ++tile) {
            const int r0 = kRfTile * (tile % nt), c0 = kRfTile * (tile / nt);
            Quarter acc[1];
            quarter_load<kOpN>(acc[0], sub_view(Y, n, n, n, r0, c0));
            rf_tile_mm<false, 1>(acc, Y, Pb, nullptr, n, r0, c0, sm);
            rf_store(acc[0], Yn, n, r0, c0);
        }
        __syncthreads();
        double2* tmp = Y;
        Y = Yn;
        Yn = tmp;
    }
    // ---- converged: W ascending and Y's columns alike, into W and X
    if (tid == 0) {
        for (int j = 0; j < n; ++j) sm.order[j] = j;
        for (int j = 1; j < n; ++j) {                         // insertion sort by lam (stable)
            const int o = sm.order[j];
            const double v = sm.lam[o];
            int k = j - 1;
            while (k >= 0 && sm.lam[sm.order[k]] > v) { sm.order[k + 1] = sm.order[k]; --k; }
            sm.order[k + 1] = o;
        }
    }
    __syncthreads();
    double2* Xb = X + mat * b;
    const double2* src = Y;
    if (Y == Xb) {                                            // permute through the other buffer
        for (size_t idx = tid; idx < mat; idx += kRfThreads) __stcg(Yn + idx, ldcg2(Y + idx));
        __syncthreads();
        src = Yn;
    }
    for (int j = tid; j < n; j += kRfThreads) W[static_cast<size_t>(n) * b + j] = sm.lam[sm.order[j]];
    for (size_t idx = tid; idx < mat; idx += kRfThreads) {
        const int c = static_cast<int>(idx / n), r = static_cast<int>(idx - static_cast<size_t>(c) * n);
        Xb[idx] = ldcg2(src + r + static_cast<size_t>(sm.order[c]) * n);
    }
    if (tid == 0) ws.rstat[b] = kRefineDone;
}

}  // namespace

size_t refine_big_smem_bytes() { return sizeof(RfSmem); }

cudaError_t launch_refine_big(int n, int batch, const Workspace& ws, double* W, double2* X, int* info,
                              int refine_steps, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (n <= kMixedMaxN || n > kMixedBigMaxN || refine_steps < 1) return cudaErrorInvalidValue;
    if (!W || !X || !info || !ws.rfC || !ws.rfY || !ws.rfP || !ws.rfG || !ws.rfS || !ws.rstat)
        return cudaErrorInvalidValue;
    k_refine_big<<<batch, kRfThreads, 0, stream>>>(n, batch, ws, W, X, info, refine_steps);
    return cudaGetLastError();
}

}  // namespace sbg
