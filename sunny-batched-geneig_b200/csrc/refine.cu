// Mixed form, second half: FP64 refinement of the complex64 eigen-decomposition of
// C = L^{-1} A L^{-H} (Ogita-Aishima iteration) with every matrix product on the FP64 tensor
// cores (mma.sync m8n8k4 f64), and the FP64 fallback for pairs the refinement cannot take.
//
//   k_refine_c<NP>       one CTA per pair, NP / 8 warps; C (from the pair's stash) and the
//                        eigenvector matrix Y = Q Z (from the X buffer) held in shared memory as
//                        planar FP64 tiles (re and im planes, column-major, ld = NP + 4, zero
//                        padded to NP = n rounded up to 8).  Warp w owns rows 8w..8w+7 of every
//                        strip product (all NP columns): P = C Y and Y' = Y + Y E; the Hermitian
//                        G = Y^H Y and S = Y^H P are computed as lower-triangle 8 x 8 blocks dealt
//                        round-robin over the warps.  Writes the refined Y over X and W, or flags
//                        the pair (ws.flag = 2).
//   k_mixed_fallback     flagged pairs only: FP64 Householder, FP64 QL and Y = Q Z in one CTA,
//                        from the stashed C (Y into X, W).  The back-transform X = L^{-H} Y runs
//                        after both, for every pair.
#include "kernels.cuh"
#include "stages.cuh"

#include <algorithm>

namespace sbg {

namespace {

__host__ __device__ constexpr size_t align16(size_t x) { return (x + 15) / 16 * 16; }

// D(8x8) += A(8x4) B(4x8), FP64, one warp.  Lane (g, t) = (lane / 4, lane % 4) holds
// a = A(g, t), b = B(t, g) and d0, d1 = D(g, 2t), D(g, 2t + 1).
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

// One warp's 8 x NP strip of a complex product in the MMA accumulator layout: lane (g, t) holds
// row 8w + g, columns 8 cb + 2t + q (q = 0, 1) of every column block cb.
template <int NB>
struct Strip {
    double re[NB][2], im[NB][2];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int c = 0; c < NB; ++c) { re[c][0] = re[c][1] = im[c][0] = im[c][1] = 0.0; }
    }
    __device__ __forceinline__ void load(const double* Mre, const double* Mim, int ld, int row0) {
        const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int c = 0; c < NB; ++c)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int idx = (8 * c + 2 * t + q) * ld + row0 + g;
                re[c][q] = Mre[idx];
                im[c][q] = Mim[idx];
            }
    }
    __device__ __forceinline__ void store(double* Mre, double* Mim, int ld, int row0) const {
        const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int c = 0; c < NB; ++c)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int idx = (8 * c + 2 * t + q) * ld + row0 + g;
                Mre[idx] = re[c][q];
                Mim[idx] = im[c][q];
            }
    }
};

// acc += A(rows row0..row0+7, :) B over k in [0, 8 NB).  A(r, k) is M(r, k) of the stored matrix,
// or conj(M(k, r)) when CONJT; B(k, c) is the stored matrix N(k, c).  Every operand load is a
// column-major planar read with ld = NP + 4, which spreads the 16 lanes of each half-warp over 16
// distinct 8-byte banks for both fragment shapes.
template <int NB, bool CONJT>
__device__ __forceinline__ void cgemm(Strip<NB>& acc, const double* __restrict__ Mre, const double* __restrict__ Mim,
                                      const double* __restrict__ Nre, const double* __restrict__ Nim, int ld, int row0) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll 2
    for (int k0 = 0; k0 < 8 * NB; k0 += 4) {
        const int ia = CONJT ? (row0 + g) * ld + k0 + t : (k0 + t) * ld + row0 + g;
        const double ar = Mre[ia];
        const double ai = CONJT ? -Mim[ia] : Mim[ia];
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            const int ib = (8 * c + g) * ld + k0 + t;
            const double br = Nre[ib], bi = Nim[ib];
            dmma(acc.re[c][0], acc.re[c][1], ar, br);
            dmma(acc.re[c][0], acc.re[c][1], -ai, bi);
            dmma(acc.im[c][0], acc.im[c][1], ar, bi);
            dmma(acc.im[c][0], acc.im[c][1], ai, br);
        }
    }
}

// The lower-triangle 8 x 8 blocks of the Hermitian products G = Y^H Y and S = Y^H P:
// NB (NB + 1) / 2 blocks, block q being (row block r, column block c), r >= c, in row-major order of
// the lower triangle, dealt round-robin to the NB warps (warp w takes q = w, w + NB, ...; at most KB).
template <int NB>
struct Gram {
    static constexpr int kTotal = NB * (NB + 1) / 2;
    static constexpr int KB = (kTotal + NB - 1) / NB;
    double gre[KB][2], gim[KB][2], sre[KB][2], sim[KB][2];
};

__device__ __forceinline__ void lower_block(int q, int& r, int& c) {
    r = 0;
    while ((r + 1) * (r + 2) / 2 <= q) ++r;
    c = q - r * (r + 1) / 2;
}

// G and S (lower blocks of this warp) in one pass: both share the A operand Y^H.
template <int NB>
__device__ __forceinline__ void gram_lower(Gram<NB>& gm, const double* __restrict__ Yre, const double* __restrict__ Yim,
                                           const double* __restrict__ Pre, const double* __restrict__ Pim, int ld) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    int ra[Gram<NB>::KB], cb[Gram<NB>::KB];
#pragma unroll
    for (int k = 0; k < Gram<NB>::KB; ++k) {
        const int q = w + k * NB;
        ra[k] = 0;
        cb[k] = 0;
        if (q < Gram<NB>::kTotal) lower_block(q, ra[k], cb[k]);
        gm.gre[k][0] = gm.gre[k][1] = gm.gim[k][0] = gm.gim[k][1] = 0.0;
        gm.sre[k][0] = gm.sre[k][1] = gm.sim[k][0] = gm.sim[k][1] = 0.0;
    }
#pragma unroll 2
    for (int k0 = 0; k0 < 8 * NB; k0 += 4) {
#pragma unroll
        for (int k = 0; k < Gram<NB>::KB; ++k) {
            if (w + k * NB >= Gram<NB>::kTotal) continue;          // uniform over the warp
            const int ia = (8 * ra[k] + g) * ld + k0 + t;
            const int ib = (8 * cb[k] + g) * ld + k0 + t;
            const double ar = Yre[ia], ai = -Yim[ia];
            const double yr = Yre[ib], yi = Yim[ib], pr = Pre[ib], pi = Pim[ib];
            dmma(gm.gre[k][0], gm.gre[k][1], ar, yr);
            dmma(gm.gre[k][0], gm.gre[k][1], -ai, yi);
            dmma(gm.gim[k][0], gm.gim[k][1], ar, yi);
            dmma(gm.gim[k][0], gm.gim[k][1], ai, yr);
            dmma(gm.sre[k][0], gm.sre[k][1], ar, pr);
            dmma(gm.sre[k][0], gm.sre[k][1], -ai, pi);
            dmma(gm.sim[k][0], gm.sim[k][1], ar, pi);
            dmma(gm.sim[k][0], gm.sim[k][1], ai, pr);
        }
    }
}

// Block-wide sums of four values (one slot row per warp in red[4 * NW]); every thread gets them.
template <int NW>
__device__ __forceinline__ void block_sum4(double (&v)[4], double* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = warp_sum(v[q]);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q) red[4 * w + q] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double s = 0.0;
        for (int i = 0; i < NW; ++i) s += red[4 * i + q];
        v[q] = s;
    }
    __syncthreads();
}

// Block-wide sums of v[0], v[1] and max of v[2] (same slots as block_sum4).
template <int NW>
__device__ __forceinline__ void block_sum2_max(double (&v)[4], double* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v[0] = warp_sum(v[0]);
    v[1] = warp_sum(v[1]);
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v[2] = fmax(v[2], shfl_xor(v[2], m));
    if (lane == 0) { red[4 * w] = v[0]; red[4 * w + 1] = v[1]; red[4 * w + 2] = v[2]; }
    __syncthreads();
    double a = 0.0, b = 0.0, c = 0.0;
    for (int i = 0; i < NW; ++i) { a += red[4 * i]; b += red[4 * i + 1]; c = fmax(c, red[4 * i + 2]); }
    v[0] = a; v[1] = b; v[2] = c;
    __syncthreads();
}

template <int NP>
struct RefineCSmem {
    static constexpr int LD = NP + 4;
    static constexpr size_t plane = sizeof(double) * NP * LD;
    static constexpr size_t Cre = 0, Cim = plane, Yre = 2 * plane, Yim = 3 * plane, Pre = 4 * plane,
                            Pim = 5 * plane, lam = 6 * plane;
    static constexpr size_t red = lam + align16(sizeof(double) * NP);
    static constexpr size_t order = red + align16(sizeof(double) * 4 * (NP / 8));
    static constexpr size_t bar = order + align16(sizeof(int) * NP);
    static constexpr size_t total = bar + 16;
};

constexpr double kEps = 1.1102230246251565e-16;
constexpr double kOrthTol = 1e-13;       // max |(Y^H Y - I)_ij| accepted

// The Ogita-Aishima iteration on Y (Ogita & Aishima, "Iterative refinement for symmetric
// eigenvalue decomposition", Japan J. Indust. Appl. Math. 35 (2018), Algorithm 1, here for a
// Hermitian C), arranged so that the products of each pass also decide whether to stop:
//   P = C Y;  G = Y^H Y, S = Y^H P (lower blocks);  lam_i = S_ii / G_ii  (Rayleigh quotients);
//   stop when every column has ||P_j - lam_j y_j|| <= 256 eps ||C||_F ||y_j|| and
//   max |R_ij| <= kOrthTol (R = I - G);
//   else delta = max(2 (||S - diag lam||_F + ||C||_F ||R||_F), floor ||C||_F),
//   E_ij = (S_ij + lam_j R_ij) / (lam_j - lam_i) where |lam_j - lam_i| > delta, else R_ij / 2,
//   Y <- Y + Y E.  floor = 1e-2 once only the orthogonality is missing: eigenvalues closer than
//   1e-2 ||C||_F are then only orthogonalised (their O(eps ||C|| / gap) corrections would undo it).
// A start from complex64 typically stops after one update (two passes of products).  Returns
// true when it stopped converged within max_updates updates.
template <int NP>
__device__ bool refine(int n, const double* Cre, const double* Cim, double* Yre, double* Yim, double* Pre, double* Pim,
                       double* lam, double* red, double cnorm, int max_updates) {
    constexpr int NB = NP / 8, LD = NP + 4, NT = NP * 4;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = lane >> 2, t = lane & 3;
    const int row0 = 8 * w;
    for (int it = 0;; ++it) {
        {
            Strip<NB> P;
            P.zero();
            cgemm<NB, false>(P, Cre, Cim, Yre, Yim, LD, row0);
            P.store(Pre, Pim, LD, row0);      // the P tile is free: the previous E was consumed
        }
        __syncthreads();
        Gram<NB> gm;
        gram_lower<NB>(gm, Yre, Yim, Pre, Pim, LD);
        int rb[Gram<NB>::KB], cbk[Gram<NB>::KB];
#pragma unroll
        for (int k = 0; k < Gram<NB>::KB; ++k) {
            rb[k] = cbk[k] = 0;
            if (w + k * NB < Gram<NB>::kTotal) lower_block(w + k * NB, rb[k], cbk[k]);
        }
#pragma unroll
        for (int k = 0; k < Gram<NB>::KB; ++k)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int i = 8 * rb[k] + g;
                if (w + k * NB < Gram<NB>::kTotal && rb[k] == cbk[k] && 2 * t + q == g && i < n)
                    lam[i] = gm.sre[k][q] / gm.gre[k][q];
            }
        __syncthreads();                       // lam visible; every warp is done reading P as an operand
        // norms and the largest departure from orthonormality (lower blocks; off-diagonal blocks twice)
        double acc[4] = {0.0, 0.0, 0.0, 0.0};  // ||S - diag lam||^2, ||R||^2, max|R_ij|, -
#pragma unroll
        for (int k = 0; k < Gram<NB>::KB; ++k)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int i = 8 * rb[k] + g, j = 8 * cbk[k] + 2 * t + q;
                if (w + k * NB < Gram<NB>::kTotal && i < n && j < n) {
                    const double wgt = rb[k] == cbk[k] ? 1.0 : 2.0;
                    const double sr = (i == j) ? gm.sre[k][q] - lam[i] : gm.sre[k][q];
                    const double rr = (i == j ? 1.0 : 0.0) - gm.gre[k][q], ri = gm.gim[k][q];
                    acc[0] += wgt * fma(sr, sr, gm.sim[k][q] * gm.sim[k][q]);
                    acc[1] += wgt * fma(rr, rr, ri * ri);
                    acc[2] = fmax(acc[2], fabs(rr) + fabs(ri));
                }
            }
        // residual of every column: ||P_j - lam_j y_j||^2 against (256 eps ||C||_F)^2 ||y_j||^2
        bool res_ok = true;
        for (int j = tid; j < n; j += NT) {
            double rr = 0.0, yy = 0.0;
            const double lj = lam[j];
            for (int i = 0; i < n; ++i) {
                const double yr = Yre[j * LD + i], yi = Yim[j * LD + i];
                const double dr = fma(-lj, yr, Pre[j * LD + i]), di = fma(-lj, yi, Pim[j * LD + i]);
                rr = fma(dr, dr, fma(di, di, rr));
                yy = fma(yr, yr, fma(yi, yi, yy));
            }
            const double tol = 256.0 * kEps * cnorm;
            if (!(rr <= tol * tol * yy)) res_ok = false;
        }
        res_ok = __syncthreads_and(res_ok);
        block_sum2_max<NB>(acc, red);           // acc[0], acc[1] summed, acc[2] the block's max
        const bool orth_ok = acc[2] <= kOrthTol;
        if (res_ok && orth_ok) return true;
        if (it >= max_updates) return false;
        const double floor_rel = res_ok ? 1e-2 : 0.0;
        const double delta = fmax(2.0 * (sqrt(acc[0]) + cnorm * sqrt(acc[1])), floor_rel * cnorm);
        // E over the P tile (P is no longer read): each lower block gives E_ij and, mirrored, E_ji
#pragma unroll
        for (int k = 0; k < Gram<NB>::KB; ++k) {
            if (w + k * NB >= Gram<NB>::kTotal) continue;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int i = 8 * rb[k] + g, j = 8 * cbk[k] + 2 * t + q;
                double er = 0.0, ei = 0.0, fr = 0.0, fi = 0.0;     // E_ij, E_ji
                if (i < n && j < n) {
                    const double rr = (i == j ? 1.0 : 0.0) - gm.gre[k][q], ri = -gm.gim[k][q];
                    const double gap = lam[j] - lam[i];
                    if (i != j && fabs(gap) > delta) {
                        const double inv = 1.0 / gap;
                        er = fma(lam[j], rr, gm.sre[k][q]) * inv;
                        ei = fma(lam[j], ri, gm.sim[k][q]) * inv;
                        fr = -fma(lam[i], rr, gm.sre[k][q]) * inv;  // (conj S_ij + lam_i conj R_ij) / (lam_i - lam_j)
                        fi = fma(lam[i], ri, gm.sim[k][q]) * inv;
                    } else {
                        er = 0.5 * rr; ei = 0.5 * ri;
                        fr = 0.5 * rr; fi = -0.5 * ri;
                    }
                }
                Pre[j * LD + i] = er;
                Pim[j * LD + i] = ei;
                if (rb[k] != cbk[k]) {
                    Pre[i * LD + j] = fr;
                    Pim[i * LD + j] = fi;
                }
            }
        }
        __syncthreads();                       // E visible
        Strip<NB> Yn;
        Yn.load(Yre, Yim, LD, row0);
        cgemm<NB, false>(Yn, Yre, Yim, Pre, Pim, LD, row0);
        __syncthreads();                       // every warp is done reading Y
        Yn.store(Yre, Yim, LD, row0);
        __syncthreads();
    }
}

template <int NP>
__global__ void __launch_bounds__(NP * 4, 1) k_refine_c(int n, int batch, Workspace ws, double* __restrict__ W,
                                                      double2* __restrict__ X, int* __restrict__ info,
                                                      int max_updates) {
    constexpr int NB = NP / 8, LD = NP + 4, NT = NP * 4;
    using L = RefineCSmem<NP>;
    const int b = blockIdx.x;
    if (b >= batch) return;
    const int tid = threadIdx.x;
    const int inf = info[b];
    if (inf > n || inf < 0) return;            // B not positive definite (or a copy timed out)
    if (inf != 0) {                            // the FP64 eigensolve of the complex64 T did not converge
        if (tid == 0) {
            ws.flag[b] = 2;
            info[b] = 0;
            if (ws.redo_count) atomicAdd(ws.redo_count, 1ull);
        }
        return;
    }
    extern __shared__ __align__(16) unsigned char smem[];
    double* Cre = reinterpret_cast<double*>(smem + L::Cre);
    double* Cim = reinterpret_cast<double*>(smem + L::Cim);
    double* Yre = reinterpret_cast<double*>(smem + L::Yre);
    double* Yim = reinterpret_cast<double*>(smem + L::Yim);
    double* Pre = reinterpret_cast<double*>(smem + L::Pre);
    double* Pim = reinterpret_cast<double*>(smem + L::Pim);
    double* lam = reinterpret_cast<double*>(smem + L::lam);
    double* red = reinterpret_cast<double*>(smem + L::red);
    int* order = reinterpret_cast<int*>(smem + L::order);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::bar);
    const size_t mat = static_cast<size_t>(n) * n;
    double2* Xb = X + mat * b;
    // ---- C (both planes, one bulk copy of the stash) and Y (the X buffer, complex -> planar)
    if (tid == 0) { mbar_init(bar, 1); fence_mbar_init(); }
    __syncthreads();
    if (tid == 0) {
        const uint32_t bytes = static_cast<uint32_t>(2 * L::plane);
        mbar_arrive_expect_tx(bar, bytes);
        bulk_g2s(Cre, static_cast<const char*>(ws.log) + 16 * static_cast<size_t>(ws.log_stride) * b, bytes, bar);
    }
    for (int idx = tid; idx < NP * NP; idx += NT) {
        const int c = idx / NP, r = idx - c * NP;
        const double2 v = (r < n && c < n) ? Xb[r + static_cast<size_t>(c) * n] : make_double2(0.0, 0.0);
        Yre[c * LD + r] = v.x;
        Yim[c * LD + r] = v.y;
    }
    if (!mbar_wait_bounded(bar, 0, kMaxPolls)) {
        atomicOr(info + b, kInfoCopyTimeout);
        mbar_wait_bounded(bar, 0, kMaxPolls);
    }
    __syncthreads();
    double cn[4] = {0.0, 0.0, 0.0, 0.0};
    for (int idx = tid; idx < NP * NP; idx += NT) {
        const int c = idx / NP, r = idx - c * NP;
        cn[0] = fma(Cre[c * LD + r], Cre[c * LD + r], fma(Cim[c * LD + r], Cim[c * LD + r], cn[0]));
    }
    block_sum4<NB>(cn, red);
    const double cnorm = sqrt(cn[0]);
    if (!refine<NP>(n, Cre, Cim, Yre, Yim, Pre, Pim, lam, red, cnorm, max_updates)) {
        if (tid == 0) {                        // the FP64 fallback redoes this pair
            ws.flag[b] = 2;
            if (ws.redo_count) atomicAdd(ws.redo_count, 1ull);
        }
        return;
    }
    if (tid == 0) ws.flag[b] = 0;
    // ---- outputs: W ascending and Y's columns alike (a swap can only come from eigenvalues the
    // complex64 start ordered within its rounding; the columns follow their eigenvalues)
    if (tid == 0) {
        for (int j = 0; j < n; ++j) order[j] = j;
        for (int j = 1; j < n; ++j) {                      // insertion sort by lam (stable)
            const int o = order[j];
            const double v = lam[o];
            int k = j - 1;
            while (k >= 0 && lam[order[k]] > v) { order[k + 1] = order[k]; --k; }
            order[k + 1] = o;
        }
    }
    __syncthreads();
    for (int j = tid; j < n; j += NT) W[static_cast<size_t>(n) * b + j] = lam[order[j]];
    for (int idx = tid; idx < n * n; idx += NT) {
        const int c = idx / n, r = idx - c * n;
        const int src = order[c] * LD + r;
        Xb[idx] = make_double2(Yre[src], Yim[src]);
    }
}

// ---------------------------------------------------------------------------- k_mixed_fallback
// Pairs flagged by k_refine_c (ws.flag == 2): the plain FP64 eigensolve of C in one CTA, from the
// stashed C: Householder (hetrd_lower), QL with the rotations applied to Z (tridiag_ql, one
// warp), then Y = Q Z; Y into the X buffer, W ascending.  Rare (near-singular B, where FP32
// cannot resolve the small eigenvalues), so it is written for clarity, not speed.
struct FallbackSmem {
    size_t As, Y, Z, vw, pbuf, ww, d, e, tau, total;
    __host__ __device__ FallbackSmem(int n, int threads) {
        const size_t ld = static_cast<size_t>(tile_ld(n)), nw = static_cast<size_t>(threads / 32);
        size_t o = 0;
        As = o;   o += align16(16 * ld * n);
        Y = o;    o += align16(16 * ld * n);
        Z = o;    o += align16(8 * ld * n);
        vw = o;   o += align16(16 * n * nw);
        pbuf = o; o += align16(32 * n);
        ww = o;   o += align16(16 * n * nw);
        d = o;    o += align16(8 * n);
        e = o;    o += align16(8 * n);
        tau = o;  o += align16(16 * n);
        total = o;
    }
};
constexpr int kFallbackThreads = 128;

__global__ void __launch_bounds__(kFallbackThreads) k_mixed_fallback(int n, int batch, Workspace ws,
                                                                     double* __restrict__ W,
                                                                     double2* __restrict__ X, int* __restrict__ info) {
    const int b = blockIdx.x;
    if (b >= batch || ws.flag[b] != 2) return;
    const int inf = info[b];
    if (inf > n || inf < 0) return;
    extern __shared__ __align__(16) unsigned char smem[];
    const FallbackSmem lay(n, kFallbackThreads);
    const int ld = tile_ld(n), tid = threadIdx.x;
    double2* As = reinterpret_cast<double2*>(smem + lay.As);
    double2* Y = reinterpret_cast<double2*>(smem + lay.Y);
    double* Z = reinterpret_cast<double*>(smem + lay.Z);
    double2* vw = reinterpret_cast<double2*>(smem + lay.vw);
    double2* pbuf = reinterpret_cast<double2*>(smem + lay.pbuf);
    double2* ww = reinterpret_cast<double2*>(smem + lay.ww);
    double* d = reinterpret_cast<double*>(smem + lay.d);
    double* e = reinterpret_cast<double*>(smem + lay.e);
    double2* tau = reinterpret_cast<double2*>(smem + lay.tau);
    const int LDS = refine_ld(n), NP = refine_np(n);
    const double* sre = reinterpret_cast<const double*>(static_cast<const char*>(ws.log) +
                                                        16 * static_cast<size_t>(ws.log_stride) * b);
    const double* sim = sre + static_cast<size_t>(NP) * LDS;
    for (int idx = tid; idx < n * n; idx += kFallbackThreads) {
        const int c = idx / n, r = idx - c * n;
        As[r + c * ld] = make_double2(sre[c * LDS + r], sim[c * LDS + r]);
    }
    __syncthreads();
    hetrd_lower<double>(As, ld, n, d, e, tau, vw, pbuf, ww);
    __syncthreads();
    for (int idx = tid; idx < n * ld; idx += kFallbackThreads) Z[idx] = 0.0;   // identity, either layout
    __syncthreads();
    for (int i = tid; i < n; i += kFallbackThreads) Z[i + i * ld] = 1.0;
    __syncthreads();
    int unconv = 0;
    if (tid < 32) unconv = tridiag_ql<double>(n, d, e, Z, ld);
    __syncthreads();
    // Y = Q Z = H_0 (H_1 (... H_{n-2} Z)), thread per column (tridiag_ql keeps Z row-major:
    // Z(r, c) at Z[r * ld + c])
    for (int idx = tid; idx < n * n; idx += kFallbackThreads) {
        const int c = idx / n, r = idx - c * n;
        Y[r + c * ld] = make_double2(Z[r * ld + c], 0.0);
    }
    __syncthreads();
    for (int k = n - 2; k >= 0; --k) {
        const double2 tk = tau[k];
        if (tk.x == 0.0 && tk.y == 0.0) continue;
        for (int c = tid; c < n; c += kFallbackThreads) {
            double2* y = Y + c * ld;
            double2 s = y[k + 1];                                 // v(k+1) = 1
            for (int i = k + 2; i < n; ++i) s = cfmac(As[i + k * ld], y[i], s);     // v^H y
            const double2 ts = cmul(tk, s);
            y[k + 1] = csub(y[k + 1], ts);
            for (int i = k + 2; i < n; ++i) y[i] = cfms(As[i + k * ld], ts, y[i]);
        }
        __syncthreads();
    }
    double2* Xb = X + static_cast<size_t>(n) * n * b;
    for (int idx = tid; idx < n * n; idx += kFallbackThreads) {
        const int c = idx / n, r = idx - c * n;
        Xb[idx] = Y[r + c * ld];
    }
    for (int i = tid; i < n; i += kFallbackThreads) W[static_cast<size_t>(n) * b + i] = d[i];
    if (tid == 0) {
        if (unconv) info[b] = unconv;
        ws.flag[b] = 0;
    }
}

template <int NP>
cudaError_t run_refine_c(int n, int batch, const Workspace& ws, double* W, double2* X, int* info, int steps,
                         cudaStream_t stream) {
    static SmemOptIn f;
    const size_t smem = RefineCSmem<NP>::total;
    if (smem > static_cast<size_t>(max_smem_optin())) return cudaErrorInvalidValue;
    set_smem_limit(reinterpret_cast<const void*>(k_refine_c<NP>), f, static_cast<int>(smem));
    k_refine_c<NP><<<batch, NP * 4, smem, stream>>>(n, batch, ws, W, X, info, steps);
    return cudaGetLastError();
}

}  // namespace

size_t refine_c_smem_bytes(int n) {
    switch (refine_np(n)) {
        case 8: return RefineCSmem<8>::total;
        case 16: return RefineCSmem<16>::total;
        case 24: return RefineCSmem<24>::total;
        case 32: return RefineCSmem<32>::total;
        case 40: return RefineCSmem<40>::total;
        case 48: return RefineCSmem<48>::total;
        case 56: return RefineCSmem<56>::total;
        case 64: return RefineCSmem<64>::total;
        default: return 0;
    }
}

size_t mixed_fallback_smem_bytes(int n) { return FallbackSmem(n, kFallbackThreads).total; }

cudaError_t launch_refine_mixed(int n, int batch, const Workspace& ws, double* W, double2* X, int* info,
                                int refine_steps, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if (n < 1 || n > kMixedMaxN || refine_steps < 1) return cudaErrorInvalidValue;
    if (!W || !X || !info || !ws.log || !ws.flag || ws.log_stride < refine_stash_entries(n))
        return cudaErrorInvalidValue;
    cudaError_t err = cudaSuccess;
    switch (refine_np(n)) {
        case 8: err = run_refine_c<8>(n, batch, ws, W, X, info, refine_steps, stream); break;
        case 16: err = run_refine_c<16>(n, batch, ws, W, X, info, refine_steps, stream); break;
        case 24: err = run_refine_c<24>(n, batch, ws, W, X, info, refine_steps, stream); break;
        case 32: err = run_refine_c<32>(n, batch, ws, W, X, info, refine_steps, stream); break;
        case 40: err = run_refine_c<40>(n, batch, ws, W, X, info, refine_steps, stream); break;
        case 48: err = run_refine_c<48>(n, batch, ws, W, X, info, refine_steps, stream); break;
        case 56: err = run_refine_c<56>(n, batch, ws, W, X, info, refine_steps, stream); break;
        case 64: err = run_refine_c<64>(n, batch, ws, W, X, info, refine_steps, stream); break;
        default: return cudaErrorInvalidValue;
    }
    if (err != cudaSuccess) return err;
    static SmemOptIn ff;
    const size_t fs = mixed_fallback_smem_bytes(n);
    if (fs > static_cast<size_t>(max_smem_optin())) return cudaErrorInvalidValue;
    set_smem_limit(reinterpret_cast<const void*>(k_mixed_fallback), ff, static_cast<int>(fs));
    k_mixed_fallback<<<batch, kFallbackThreads, fs, stream>>>(n, batch, ws, W, X, info);
    return cudaGetLastError();
}

cudaError_t launch_eig_mixed(int n, int batch, const Workspace& ws, double* W, double2* X, int* info,
                             int refine_steps, int chain_threads, const LaunchShape& shape, cudaStream_t stream) {
    cudaError_t err = launch_eig_invit(n, batch, ws, W, X, info, chain_threads, false, stream);
    if (err == cudaSuccess) err = launch_back(kBackQOnly, n, batch, ws, X, info, shape, stream);
    if (err == cudaSuccess) err = launch_refine_mixed(n, batch, ws, W, X, info, refine_steps, stream);
    return err;
}

}  // namespace sbg
