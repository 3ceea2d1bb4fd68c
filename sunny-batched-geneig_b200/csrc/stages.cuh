// Stage device functions of the generalized Hermitian-definite eigensolve
//   A x = lambda B x,  B = L L^H,  C = L^{-1} A L^{-H} = Q T Q^H,  T Z = Z Lambda,
//   X = L^{-H} Q Z.
//
// Each function runs on one CTA ("team") over tiles that live in shared memory
// (column-major, leading dimension ld = n | 1 so row walks are bank-conflict
// free).  The stage boundaries are the reference's (src/geneig_fixed.cu:455-464):
// potrf on B, the two-sided triangular reduction, the Hermitian eigensolve and
// the back substitution; the eigensolve is split into Householder
// tridiagonalisation, implicit QL on the real tridiagonal, and the reflector
// back-application.
#pragma once

#include "common.cuh"

namespace sbg {

// ============================================================================ potrf
// In-place lower Cholesky of the tile L (only the lower triangle is read, as
// zpotrf 'L'). Right-looking, one CTA barrier per column: in phase k every
// thread updates the trailing lower triangle with the unscaled column k divided
// by L_kk, and the scaling of column k itself is deferred to phase k+1, when no
// thread reads it any more.  invd[k] receives 1 / L_kk.
// Returns 0, or k+1 for the first leading minor that is not positive definite
// (also for NaN), the zpotrf convention.  Reference: Cholesky54, geneig_fixed.cu:17-26.
template <typename R>
__device__ int potrf_lower(cplx<R>* L, int ld, int n, R* invd) {
    using C = cplx<R>;
    const int tid = threadIdx.x, T = blockDim.x;
    R pd = R(0), pinv = R(0);
    for (int k = 0; k < n; ++k) {
        const R dkk = L[k + k * ld].x;
        if (!(dkk > R(0))) return k + 1;           // uniform: every thread reads the same word
        const R d = sqrt(dkk);
        const R inv = R(1) / d;
        const R invdd = inv * inv;
        if (k > 0) {                                // deferred scaling of column k-1
            for (int i = k + tid; i < n; i += T) L[i + (k - 1) * ld] = cscale(L[i + (k - 1) * ld], pinv);
            if (tid == 0) L[(k - 1) + (k - 1) * ld] = mk<R>(pd, R(0));
        }
        if (tid == 0) invd[k] = inv;
        const int m = n - k - 1;
        const C* colk = L + k * ld;
        // thread (row r, column chunk c) updates L(k+1+r, k+1+j) for j in its chunk, j <= r
        const int chunks = max(1, T / max(m, 1));
        const int cw = (m + chunks - 1) / chunks;
        for (int t = tid; t < m * chunks; t += T) {
            const int r = t % m, c = t / m;
            const int i = k + 1 + r;
            const C lik = cscale(colk[i], invdd);
            const int j1 = min(r + 1, (c + 1) * cw);
            C* Li = L + i + (k + 1) * ld;
            for (int jj = c * cw; jj < j1; ++jj)
                Li[jj * ld] = cfmsc(lik, colk[k + 1 + jj], Li[jj * ld]);
        }
        __syncthreads();
        pd = d; pinv = inv;
    }
    if (tid == 0) L[(n - 1) + (n - 1) * ld] = mk<R>(pd, R(0));
    __syncthreads();
    return 0;
}

// ============================================================================ hetrd (lower)
// Householder reduction of the Hermitian tile A (lower triangle valid) to real
// symmetric tridiagonal form T = Q^H A Q, Q = H_0 H_1 ... H_{n-2},
// H_k = I - tau_k v_k v_k^H with v_k = (0_{k+1}, 1, A(k+2:n, k)) stored in place.
// Outputs d[0:n], e[0:n-1] (real), tau[0:n-1].  The steps are LAPACK zhetd2's
// (reflector as zlarfg, p = tau A22 v, w = p - tau/2 (p^H v) v,
// A22 -= v w^H + w v^H).  Two CTA barriers per step: every warp computes the
// reflector and w itself (into its own slices of vw / ww, n complex per warp), so no
// warp waits on another for those; the barriers only separate the Hermitian matvec
// (a row walk over the lower part and a column walk over the mirrored upper part,
// partial sums in pbuf, 2n complex) from the rank-2 update, and the update from the
// next step.
template <typename R>
__device__ void hetrd_lower(cplx<R>* A, int lda, int n, R* d, R* e, cplx<R>* tau,
                            cplx<R>* vw_all, cplx<R>* pbuf, cplx<R>* ww_all) {
    using C = cplx<R>;
    const int tid = threadIdx.x, T = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5;
    C* vw = vw_all + warp * n;
    C* ww = ww_all + warp * n;
    for (int k = 0; k + 1 < n; ++k) {
        const int m = n - k - 1;
        C* x = A + (k + 1) + k * lda;                    // x[0..m) = A(k+1:n, k)
        // ---- reflector (every warp)
        R s2 = R(0);
        for (int i = 1 + lane; i < m; i += 32) s2 += cabs2(x[i]);
        s2 = warp_sum(s2);
        const C alpha = x[0];
        C tk, scale;
        R beta;
        if (s2 == R(0) && alpha.y == R(0)) {
            tk = mk<R>(R(0), R(0)); beta = alpha.x; scale = mk<R>(R(0), R(0));
        } else {
            const R nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + s2);
            beta = alpha.x >= R(0) ? -nrm : nrm;
            tk = mk<R>((beta - alpha.x) / beta, -alpha.y / beta);
            const R ar = alpha.x - beta, ai = alpha.y;   // scale = 1 / (alpha - beta)
            const R den = ar * ar + ai * ai;
            scale = mk<R>(ar / den, -ai / den);
        }
        if (tid == 0) { e[k] = beta; tau[k] = tk; }
        if (tk.x == R(0) && tk.y == R(0)) continue;      // H_k = I (uniform: same value in every warp)
        for (int i = lane; i < m; i += 32) vw[i] = (i == 0) ? mk<R>(R(1), R(0)) : cmul(x[i], scale);
        __syncwarp();
        // ---- p partial sums: part 0 = sum_{j<=r} A22(r,j) v_j, part 1 = sum_{j>r} conj(A22(j,r)) v_j
        C* A22 = A + (k + 1) + (k + 1) * lda;
        for (int t = tid; t < 2 * m; t += T) {
            const int part = t >= m, r = t - part * m;
            C acc0 = mk<R>(R(0), R(0)), acc1 = mk<R>(R(0), R(0));
            if (part == 0) {
                int j = 0;
                for (; j + 1 < r; j += 2) {
                    acc0 = cfma(A22[r + j * lda], vw[j], acc0);
                    acc1 = cfma(A22[r + (j + 1) * lda], vw[j + 1], acc1);
                }
                for (; j < r; ++j) acc0 = cfma(A22[r + j * lda], vw[j], acc0);
                const R drr = A22[r + r * lda].x;
                acc0.x = fma(drr, vw[r].x, acc0.x);
                acc0.y = fma(drr, vw[r].y, acc0.y);
            } else {
                const C* col = A22 + r * lda;
                int j = r + 1;
                for (; j + 1 < m; j += 2) {
                    acc0 = cfmac(col[j], vw[j], acc0);
                    acc1 = cfmac(col[j + 1], vw[j + 1], acc1);
                }
                for (; j < m; ++j) acc0 = cfmac(col[j], vw[j], acc0);
            }
            pbuf[t] = cadd(acc0, acc1);
        }
        __syncthreads();
        // the scaled reflector replaces x (nobody reads column k after the barrier above)
        if (warp == 0)
            for (int i = 1 + lane; i < m; i += 32) x[i] = vw[i];
        // ---- p = tau (part0 + part1); alpha2 = -tau/2 (p^H v); w = p + alpha2 v (every warp)
        C dot = mk<R>(R(0), R(0));
        for (int r = lane; r < m; r += 32) {
            const C p = cmul(tk, cadd(pbuf[r], pbuf[m + r]));
            ww[r] = p;
            dot = cfmac(p, vw[r], dot);
        }
        dot.x = warp_sum(dot.x);
        dot.y = warp_sum(dot.y);
        const C a2 = cscale(cmul(tk, dot), R(-0.5));
        for (int r = lane; r < m; r += 32) ww[r] = cfma(a2, vw[r], ww[r]);
        __syncwarp();
        // ---- A22 -= v w^H + w v^H on the lower triangle; thread (row r, column chunk c)
        {
            const int chunks = max(1, T / m);
            const int cw = (m + chunks - 1) / chunks;
            for (int t = tid; t < m * chunks; t += T) {
                const int r = t % m, c = t / m;
                const C vr = vw[r], wr = ww[r];
                const int j0 = c * cw, j1 = min(r + 1, (c + 1) * cw);
                for (int j = j0; j < j1; ++j) {
                    C a = A22[r + j * lda];
                    a = cfmsc(vr, ww[j], a);
                    a = cfmsc(wr, vw[j], a);
                    if (j == r) a.y = R(0);
                    A22[r + j * lda] = a;
                }
            }
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += T) d[i] = A[i + i * lda].x;
    if (tid == 0 && n >= 1) e[n - 1] = R(0);
    __syncthreads();
}

// ============================================================================ tridiagonal QL
// Eigen-decomposition of the real symmetric tridiagonal (d, e) by implicit QL
// with Wilkinson-type shifts, accumulating the rotations into Z (row-major,
// Z[r * ldz + c], initialised to I by the caller).  One warp per problem: every
// lane runs the same scalar recurrence (so no broadcast is needed) and applies
// each rotation to the rows it owns (r = lane + 32 q).  The deflation test is
// LAPACK dsteqr's relative one, |e_m|^2 <= eps^2 |d_m| |d_{m+1}| + safmin, and the
// matrix is scaled to unit max-norm first (dsteqr scales only at the range
// limits; scaling always keeps the single-precision variant safe).
// Eigenvalues come back ascending with Z's columns permuted alike (dsteqr's
// final selection sort).  Returns the number of off-diagonals that failed to
// converge within 30 iterations per eigenvalue (0 on success).
// d, e live in shared memory private to the warp; only lane 0 writes them.
template <typename R>
__device__ int tridiag_ql(int n, R* d, R* e, R* Z, int ldz) {
    const int lane = threadIdx.x & 31;
    const R eps = sizeof(R) == 8 ? R(1.1102230246251565e-16) : R(5.9604645e-08);
    const R eps2 = eps * eps;
    const R safmin = sizeof(R) == 8 ? R(2.2250738585072014e-308) : R(1.17549435e-38);
    // scale to unit max-norm
    R anorm = R(0);
    for (int i = 0; i < n; ++i) anorm = fmax(anorm, fabs(d[i]));
    for (int i = 0; i + 1 < n; ++i) anorm = fmax(anorm, fabs(e[i]));
    if (!(anorm > R(0)) || !isfinite(anorm)) anorm = R(1);
    const R sc = R(1) / anorm;
    __syncwarp();
    if (lane == 0) {
        for (int i = 0; i < n; ++i) d[i] *= sc;
        for (int i = 0; i + 1 < n; ++i) e[i] *= sc;
        e[n - 1] = R(0);
    }
    __syncwarp();
    int unconverged = 0;
    const int maxit = 30;
    for (int l = 0; l < n; ++l) {
        int iter = 0;
        for (;;) {
            int m = l;
            for (; m < n - 1; ++m) {
                const R em = e[m];
                if (em * em <= (eps2 * fabs(d[m])) * fabs(d[m + 1]) + safmin) break;
            }
            if (m == l) break;
            if (iter == maxit) { ++unconverged; break; }
            ++iter;
            const R el = e[l], dl = d[l];
            R g = (d[l + 1] - dl) / (R(2) * el);
            R r = sqrt(fma(g, g, R(1)));
            g = d[m] - dl + el / (g + copysign(r, g));
            R s = R(1), c = R(1), p = R(0);
            bool early = false;
            for (int i = m - 1; i >= l; --i) {
                const R ei = e[i];
                const R f = s * ei, b = c * ei;
                const R rr = fma(f, f, g * g);
                if (rr == R(0)) {
                    __syncwarp();
                    if (lane == 0) { d[i + 1] -= p; e[m] = R(0); }
                    __syncwarp();
                    early = true;
                    break;
                }
                const R ri = rsqrt(rr);
                r = rr * ri;
                s = f * ri;
                c = g * ri;
                const R di1 = d[i + 1];
                g = di1 - p;
                r = fma(d[i] - g, s, R(2) * c * b);
                p = s * r;
                __syncwarp();
                if (lane == 0) { e[i + 1] = rr * ri; d[i + 1] = g + p; }
                g = fma(c, r, -b);
                // rotate columns i, i+1 of the rows this lane owns
                for (int row = lane; row < n; row += 32) {
                    R* zr = Z + row * ldz;
                    const R zi = zr[i], zi1 = zr[i + 1];
                    zr[i + 1] = fma(s, zi, c * zi1);
                    zr[i] = fma(c, zi, -s * zi1);
                }
                __syncwarp();
            }
            if (early) continue;
            __syncwarp();
            if (lane == 0) { d[l] -= p; e[l] = g; e[m] = R(0); }
            __syncwarp();
        }
    }
    // sort ascending (selection sort, as dsteqr)
    for (int i = 0; i + 1 < n; ++i) {
        int k = i;
        R pmin = d[i];
        for (int j = i + 1; j < n; ++j) if (d[j] < pmin) { k = j; pmin = d[j]; }
        if (k != i) {
            __syncwarp();
            if (lane == 0) { d[k] = d[i]; d[i] = pmin; }
            for (int row = lane; row < n; row += 32) {
                R* zr = Z + row * ldz;
                const R t = zr[i]; zr[i] = zr[k]; zr[k] = t;
            }
            __syncwarp();
        }
    }
    __syncwarp();
    if (lane == 0) for (int i = 0; i < n; ++i) d[i] *= anorm;
    __syncwarp();
    return unconverged;
}

// ============================================================================ QL, scalar chain only
// The same implicit QL as tridiag_ql, run by ONE thread for one pair, with d and
// e in shared memory interleaved over the CTA (element i of thread t at
// [i * stride + t]).  Instead of rotating Z, every rotation (c, s) is appended
// to a per-pair log in global memory: a sweep is a header entry
// (top = m - 1, count) followed by `count` rotations acting on column pairs
// (i, i+1), i = top, top-1, ..., top-count+1.  A header with count = 0 and
// top = -1 ends the log.  The eigenvalues are sorted ascending and perm[k]
// receives the pre-sort column index of eigenvalue k.
// Returns the number of unconverged off-diagonals, or -1 if the log capacity
// (cap entries) would be exceeded (the caller then falls back to tridiag_ql).
// LOG = false: eigenvalues only (no log, no permutation; log, cap and perm are ignored).
template <typename R, bool LOG = true>
__device__ int ql_chain(int n, R* d, R* e, int stride, cplx<R>* log, int cap, int* perm, double* W) {
    using C = cplx<R>;
    const R eps = sizeof(R) == 8 ? R(1.1102230246251565e-16) : R(5.9604645e-08);
    const R eps2 = eps * eps;
    const R safmin = sizeof(R) == 8 ? R(2.2250738585072014e-308) : R(1.17549435e-38);
#define D(i) d[(i) * stride]
#define E(i) e[(i) * stride]
    R anorm = R(0);
    for (int i = 0; i < n; ++i) anorm = fmax(anorm, fabs(D(i)));
    for (int i = 0; i + 1 < n; ++i) anorm = fmax(anorm, fabs(E(i)));
    if (!(anorm > R(0)) || !isfinite(anorm)) anorm = R(1);
    const R sc = R(1) / anorm;
    for (int i = 0; i < n; ++i) D(i) *= sc;
    for (int i = 0; i + 1 < n; ++i) E(i) *= sc;
    E(n - 1) = R(0);
    int pos = 0, unconverged = 0;
    const int maxit = 30;
    for (int l = 0; l < n; ++l) {
        int iter = 0;
        for (;;) {
            int m = l;
            for (; m < n - 1; ++m) {
                const R em = E(m);
                if (em * em <= (eps2 * fabs(D(m))) * fabs(D(m + 1)) + safmin) break;
            }
            if (m == l) break;
            if (iter == maxit) { ++unconverged; break; }
            ++iter;
            int hdr = 0;
            if constexpr (LOG) {
                if (pos + (m - l) + 2 > cap) return -1;
                hdr = pos++;
            }
            const R el = E(l), dl = D(l);
            R g = (D(l + 1) - dl) / (R(2) * el);
            R r = sqrt(fma(g, g, R(1)));
            g = D(m) - dl + el / (g + copysign(r, g));
            R s = R(1), c = R(1), p = R(0);
            bool early = false;
            int i = m - 1;
            R ei = E(i), di = D(i);
            for (; i >= l; --i) {
                const R f = s * ei, b = c * ei;
                const R rr = fma(f, f, g * g);
                if (rr == R(0)) { D(i + 1) -= p; E(m) = R(0); early = true; break; }
                const R di1 = D(i + 1);
                const R ei_next = (i > l) ? E(i - 1) : R(0);     // prefetch: not written in this sweep
                const R di_next = (i > l) ? D(i - 1) : R(0);
                const R ri = rsqrt(rr);
                E(i + 1) = rr * ri;
                s = f * ri;
                c = g * ri;
                g = di1 - p;
                r = fma(di - g, s, R(2) * c * b);
                p = s * r;
                D(i + 1) = g + p;
                g = fma(c, r, -b);
                if constexpr (LOG) log[pos++] = mk<R>(c, s);
                ei = ei_next; di = di_next;
            }
            if constexpr (LOG) log[hdr] = mk<R>(R(m - 1), R(early ? (m - 1 - i) : (m - l)));
            if (early) continue;
            D(l) -= p; E(l) = g; E(m) = R(0);
        }
    }
    if constexpr (LOG) log[pos] = mk<R>(R(-1), R(0));
    // selection sort with the permutation recorded
    if constexpr (LOG) for (int k = 0; k < n; ++k) perm[k] = k;
    for (int k = 0; k + 1 < n; ++k) {
        int j = k;
        R pmin = D(k);
        for (int t = k + 1; t < n; ++t) if (D(t) < pmin) { j = t; pmin = D(t); }
        if (j != k) {
            D(j) = D(k); D(k) = pmin;
            if constexpr (LOG) { const int tp = perm[k]; perm[k] = perm[j]; perm[j] = tp; }
        }
    }
    for (int k = 0; k < n; ++k) W[k] = static_cast<double>(D(k) * anorm);
#undef D
#undef E
    return unconverged;
}

// ============================================================================ register-segment solvers
// Column (or row) work where the G lanes of a group share one column and lane g keeps
// the entries of rows i = g + G r, r < RM, in registers for the whole stage; only L
// or the reflectors are read from shared memory (the same address for every group:
// a broadcast).  Requires n <= G * RM and n <= (threads / G) columns per pass.

// Selects seg[r] for a runtime r (unrolled, so seg stays in registers).
template <int RM, typename C>
__device__ __forceinline__ C seg_get(const C (&seg)[RM], int r) {
    C v = seg[0];
#pragma unroll
    for (int q = 1; q < RM; ++q) if (q == r) v = seg[q];
    return v;
}
template <int RM, typename C>
__device__ __forceinline__ void seg_set(C (&seg)[RM], int r, C v) {
#pragma unroll
    for (int q = 0; q < RM; ++q) if (q == r) seg[q] = v;
}

// y <- L^{-1} y (forward substitution) on the column segment; L column-major in smem.
template <int G, int RM, typename C, typename R>
__device__ __forceinline__ void seg_trsm_lower(const C* L, int ldl, const R* invd, C (&y)[RM], int n, int g) {
    for (int k = 0; k < n; ++k) {
        const int owner = k % G, rk = k / G;
        C wk = seg_get(y, rk);
        wk = cscale(wk, invd[k]);
        if (g == owner) seg_set(y, rk, wk);
        wk = cshfl(wk, owner, G);
        const C* lk = L + k * ldl;
#pragma unroll
        for (int r = RM - 1; r >= 0; --r) {          // active rows i > k form a suffix of r
            const int i = g + G * r;
            if (i <= k) break;
            if (i < n) y[r] = cfms(lk[i], wk, y[r]);
        }
    }
}

// Row segment of W (columns kk = g + G r of row i) <- W L^{-H}, only kk <= i formed.
template <int G, int RM, typename C, typename R>
__device__ __forceinline__ void seg_trsm_right_lowerH(const C* L, int ldl, const R* invd, C (&y)[RM], int kmax,
                                                      int i, int g) {
    for (int k = 0; k <= kmax; ++k) {
        const int owner = k % G, rk = k / G;
        C ck = seg_get(y, rk);
        ck = cscale(ck, invd[k]);
        if (g == owner && k <= i) seg_set(y, rk, ck);
        ck = cshfl(ck, owner, G);
        const C* lk = L + k * ldl;
#pragma unroll
        for (int r = RM - 1; r >= 0; --r) {          // active columns k < kk <= i
            const int kk = g + G * r;
            if (kk <= k) break;
            if (kk <= i) y[r] = cfmsc(ck, lk[kk], y[r]);
        }
    }
}

// y <- Q y, Q = H_0 ... H_{n-2}, with the reflectors along the rows of LV: component i >= k+2
// of v_k sits at LV(k, i) (above the superdiagonal); v_k(k+1) = 1 is implicit.
template <int G, int RM, typename C>
__device__ __forceinline__ void seg_apply_q(const C* LV, int ld, const C* tau, C (&y)[RM], int n, int g) {
    using R = decltype(C().x);
    for (int k = n - 2; k >= 0; --k) {
        const C tk = tau[k];
        if (tk.x == R(0) && tk.y == R(0)) continue;
        const C* vrow = LV + k;                    // v_k(i) = LV(k, i) = vrow[i * ld], i >= k + 2
        C s = mk<R>(R(0), R(0));
#pragma unroll
        for (int r = RM - 1; r >= 0; --r) {          // active rows i > k form a suffix of r
            const int i = g + G * r;
            if (i <= k) break;
            if (i < n) {
                const C vi = (i == k + 1) ? mk<R>(R(1), R(0)) : vrow[i * ld];
                s = cfmac(vi, y[r], s);
            }
        }
        s.x = group_sum(s.x, G);
        s.y = group_sum(s.y, G);
        s = cmul(tk, s);
#pragma unroll
        for (int r = RM - 1; r >= 0; --r) {
            const int i = g + G * r;
            if (i <= k) break;
            if (i < n) {
                const C vi = (i == k + 1) ? mk<R>(R(1), R(0)) : vrow[i * ld];
                y[r] = cfms(vi, s, y[r]);
            }
        }
    }
}

// y <- L^{-H} y (backward substitution) on the column segment.
template <int G, int RM, typename C, typename R>
__device__ __forceinline__ void seg_trsm_lowerH(const C* L, int ldl, const R* invd, C (&y)[RM], int n, int g) {
    for (int k = n - 1; k >= 0; --k) {
        const int owner = k % G, rk = k / G;
        C xk = seg_get(y, rk);
        xk = cscale(xk, invd[k]);
        if (g == owner) seg_set(y, rk, xk);
        xk = cshfl(xk, owner, G);
        const C* lrow = L + k;                     // L(k, i) = lrow[i * ldl], i < k
#pragma unroll
        for (int r = 0; r < RM; ++r) {               // active rows i < k form a prefix of r
            const int i = g + G * r;
            if (i >= k) break;
            y[r] = cfms(cconj(lrow[i * ldl]), xk, y[r]);
        }
    }
}

// ============================================================================ QL log application
// Applies one pair's rotation log (ql_chain's format: a header (top, count), then count
// rotations (c, s) for columns top, top-1, ...; a header with top < 0 ends the log) to
// the row zrow of Z owned by this lane (own = false: the lane only helps stream the
// log).  The log is read 32 entries at a time with one coalesced load into the warp's
// stage buffer (64 entries, double-buffered) and read back by broadcast; within a sweep
// the rotation at column i loads z_i and carries z_{i+1} in a register.
template <typename R>
__device__ __forceinline__ void ql_log_apply_row(const cplx<R>* log, int cap, cplx<R>* stage, R* zrow, bool own) {
    using C = cplx<R>;
    const int lane = threadIdx.x & 31;
    int loaded = 0, buf = 0, remaining = 0, col = 0;
    C pre = log[lane];
    R carry = R(0);
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
                if (own && remaining > 0) carry = zrow[col + 1];
                continue;
            }
            const int take = min(remaining, 32 - k);
            if (own) {
                for (int t = 0; t < take; ++t) {
                    const C cs = st[k + t];
                    const R zi = zrow[col - t];
                    zrow[col - t + 1] = fma(cs.y, zi, cs.x * carry);
                    carry = fma(cs.x, zi, -cs.y * carry);
                }
            }
            k += take;
            col -= take;
            remaining -= take;
            if (remaining == 0 && own) zrow[col + 1] = carry;
        }
        __syncwarp();
        buf ^= 1;
        if (!done && loaded >= cap) done = true;      // malformed log guard (never reached)
    }
}

// ============================================================================ hetrd, one warp, packed
// Column-major packed lower triangle: A(i, j), i >= j, at P[pk(j, n) + i - j].
__host__ __device__ __forceinline__ int pk(int j, int n) { return j * n - (j * (j - 1)) / 2; }

// ---- warp helpers of hetrd_warp_packed (one warp, packed lower triangle, lane rows L and m-1-L)

// LAPACK zlarfg on x[0..m) (x[0] = alpha): beta, tau, and the scale that turns x[1..m) into the
// reflector's tail (v = (1, x[1..m) * scale)).  Every lane gets the same values.
template <typename R>
struct WarpReflector { cplx<R> tau, scale; R beta; };

template <typename R>
__device__ __forceinline__ WarpReflector<R> warp_reflector(const cplx<R>* x, int m) {
    const int lane = threadIdx.x & 31;
    R s2 = R(0);
    for (int i = 1 + lane; i < m; i += 32) s2 += cabs2(x[i]);
    s2 = warp_sum(s2);
    const cplx<R> alpha = x[0];
    WarpReflector<R> f;
    if (s2 == R(0) && alpha.y == R(0)) {
        f.tau = mk<R>(R(0), R(0)); f.beta = alpha.x; f.scale = mk<R>(R(0), R(0));
    } else {
        const R nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + s2);
        f.beta = alpha.x >= R(0) ? -nrm : nrm;
        const R ib = R(1) / f.beta;                      // two reciprocals instead of four divisions
        f.tau = mk<R>((f.beta - alpha.x) * ib, -alpha.y * ib);
        const R ar = alpha.x - f.beta, ai = alpha.y;
        const R id = R(1) / (ar * ar + ai * ai);
        f.scale = mk<R>(ar * id, -ai * id);
    }
    return f;
}

// The reflector's vector into vb[0..m) (and its tail over x[1..m)); with tau = 0 (H = I) vb = e_0.
template <typename R>
__device__ __forceinline__ void warp_store_reflector(cplx<R>* x, int m, const WarpReflector<R>& f, cplx<R>* vb) {
    const int lane = threadIdx.x & 31;
    const bool id = f.tau.x == R(0) && f.tau.y == R(0);
    __syncwarp();                                        // every lane has read x[0] and the norm terms
    for (int i = lane; i < m; i += 32) {
        if (id) { vb[i] = mk<R>(i == 0 ? R(1) : R(0), R(0)); continue; }
        const cplx<R> v = (i == 0) ? mk<R>(R(1), R(0)) : cmul(x[i], f.scale);
        vb[i] = v;
        if (i > 0) x[i] = v;
    }
}

// (A22 v)_r for the lane's rows r1 = lane and r2 = m-1-lane of the packed trailing matrix whose
// column 0 starts at c0 (order m).  Each lane walks its two rows in ONE loop of uniform length (row
// r1's terms, then row r2's), so no lane waits for the others' longer row: the pair has m-1 terms
// in the lower row walk, m-1 in the mirrored column walk.  A22(r, j) sits at
// c0 + r - j + sum_{t<j} (m - t): the address advances by (m - j - 1) from column j to j + 1.
template <typename R>
__device__ __forceinline__ void warp_hemv_rows(const cplx<R>* c0, int m, const cplx<R>* vb, cplx<R>& s1, cplx<R>& s2) {
    using C = cplx<R>;
    const int lane = threadIdx.x & 31;
    const int h = (m + 1) >> 1;
    const int r1 = lane, r2 = m - 1 - lane;
    const bool own2 = lane < h && r2 != r1;
    const C zero = mk<R>(R(0), R(0));
    s1 = zero;
    s2 = zero;
    if (lane >= h) return;
    const int tot = own2 ? r1 + r2 : r1;                 // lower walk length
    const int sw = m - 1 - r1;
    const int tot2 = own2 ? m - 1 : sw;                  // column walk length (== tot when own2)
    const C* diag1 = c0 + (r1 * m - r1 * (r1 - 1) / 2); // A22(r1, r1)
    const C* diag2 = c0 + (r2 * m - r2 * (r2 - 1) / 2); // A22(r2, r2)
    C acc = zero, low1 = zero, u = zero, up1 = zero;
    const C* pa = c0 + r1;
    int jj = 0;
    const C* cp = diag1 + 1;                             // next column-walk element
    const C* vp = vb + r1 + 1;                           // its partner in v
    bool lsw = false, usw = false;
    const int both = tot < tot2 ? tot : tot2;
    int t = 0;
    for (; t < both; ++t) {
        if (t == r1) { low1 = acc; acc = zero; pa = c0 + r2; jj = 0; lsw = true; }
        if (t == sw) { up1 = u; u = zero; cp = diag2 + 1; vp = vb + r2 + 1; usw = true; }
        acc = cfma(*pa, vb[jj], acc);
        u = cfmac(*cp, *vp, u);
        pa += m - jj - 1;
        ++jj;
        ++cp;
        ++vp;
    }
    for (; t < tot; ++t) {                               // (only when the lengths differ)
        if (t == r1) { low1 = acc; acc = zero; pa = c0 + r2; jj = 0; lsw = true; }
        acc = cfma(*pa, vb[jj], acc);
        pa += m - jj - 1;
        ++jj;
    }
    for (; t < tot2; ++t) {
        if (t == sw) { up1 = u; u = zero; cp = diag2 + 1; vp = vb + r2 + 1; usw = true; }
        u = cfmac(*cp, *vp, u);
        ++cp;
        ++vp;
    }
    C low2 = zero, up2 = zero;
    if (lsw) low2 = acc; else low1 = acc;
    if (usw) up2 = u; else up1 = u;
    C a1 = up1;
    a1.x = fma(diag1[0].x, vb[r1].x, a1.x);
    a1.y = fma(diag1[0].x, vb[r1].y, a1.y);
    s1 = cadd(low1, a1);
    if (own2) {
        C a2 = up2;
        a2.x = fma(diag2[0].x, vb[r2].x, a2.x);
        a2.y = fma(diag2[0].x, vb[r2].y, a2.y);
        s2 = cadd(low2, a2);
    }
}

// A22 -= sum_q (v_q w_q^H + w_q v_q^H), q < NP, on the lane's rows r1 = lane and r2 = m-1-lane of the
// packed trailing matrix at c0 (order m): r1 + 1 terms of row r1 (diagonal last), then r2 + 1 of row
// r2, in one loop.  The terms of each entry are applied in q order; the diagonal entries stay real.
template <typename R, int NP>
__device__ __forceinline__ void warp_her2_rows(cplx<R>* c0, int m, const cplx<R>* const (&vq)[NP],
                                               const cplx<R>* const (&wq)[NP]) {
    using C = cplx<R>;
    const int lane = threadIdx.x & 31;
    const int h = (m + 1) >> 1;
    const int r1 = lane, r2 = m - 1 - lane;
    if (lane >= h) return;
    const bool own2 = r2 != r1;
    const int tot = own2 ? r1 + r2 + 2 : r1 + 1;
    C* a = c0 + r1;
    C vr[NP], wr[NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) { vr[q] = vq[q][r1]; wr[q] = wq[q][r1]; }
    int jj = 0;
    C* dg1 = nullptr;
    for (int t = 0; t < tot; ++t) {
        if (t == r1 + 1) {
            dg1 = a - (m - jj);
            a = c0 + r2;
#pragma unroll
            for (int q = 0; q < NP; ++q) { vr[q] = vq[q][r2]; wr[q] = wq[q][r2]; }
            jj = 0;
        }
        C tv = *a;
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            tv = cfmsc(vr[q], wq[q][jj], tv);
            tv = cfmsc(wr[q], vq[q][jj], tv);
        }
        *a = tv;
        a += m - jj - 1;
        ++jj;
    }
    // the diagonal entries (each row's last term) stay real
    if (dg1 == nullptr) dg1 = a - (m - jj);
    else a[-(m - jj)].y = R(0);
    dg1->y = R(0);
}

// The Householder tridiagonalisation of hetrd_lower (LAPACK zhetd2's steps) run by ONE warp on a
// packed lower triangle, for n <= 65, two steps per pass over the trailing triangle.  At step k
// lane L owns trailing rows L and m-1-L (m = n-k-1), which balances both the Hermitian matvec
// (m terms per row) and the rank-2 update (r+1 terms for row r).  Step k's rank-2 update
// A22 -= v w^H + w v^H is applied at once only to column k+1 (which step k+1 turns into its
// reflector); step k+1's matvec runs on the trailing matrix without step k's update and corrects
// it with two dot products, p' = tau' (A22 v' - v^ (w^^H v') - w^ (v^^H v')) (v^, w^: v, w without
// their first entry), and one pass then applies both steps' updates.  The trailing triangle is so
// read and written once per two steps instead of once per step (the walks are bound by shared-
// memory traffic).  Only __syncwarp is needed.  The scaled reflector replaces A(k+2:n, k).
// d, e, tau may be global memory (written by lane 0 as they are formed, d at the end);
// vb, wb, vb2, wb2: n complex of shared scratch each (vb2, wb2 unused when !TWO_STEP).
// TWO_STEP = false runs one step per pass (zhetd2's own order): measured better for complex64,
// whose walks are bound by instruction issue rather than shared-memory traffic (twice the pairs
// per SM, half the bytes), so the deferral's extra dot products and column pass cost more than
// the halved update traffic saves (49.2 against 42.8 ms per 262,144 pairs at n = 54).
template <typename R, bool TWO_STEP = true>
__device__ void hetrd_warp_packed(cplx<R>* P, int n, R* d, R* e, cplx<R>* tau, cplx<R>* vb, cplx<R>* wb,
                                  cplx<R>* vb2, cplx<R>* wb2) {
    using C = cplx<R>;
    const int lane = threadIdx.x & 31;
    const C zero = mk<R>(R(0), R(0));
    int k = 0;
    while (k + 1 < n) {
        const int m = n - k - 1;
        C* x = P + pk(k, n) + 1;                        // x[i] = A(k+1+i, k)
        // ---- step k: reflector, p = tau A22 v, w = p - tau/2 (p^H v) v
        const WarpReflector<R> f = warp_reflector<R>(x, m);
        if (lane == 0) { e[k] = f.beta; tau[k] = f.tau; }
        warp_store_reflector<R>(x, m, f, vb);
        __syncwarp();
        C* c0 = P + pk(k + 1, n);
        const int r1 = lane, r2 = m - 1 - lane, h = (m + 1) >> 1;
        const bool own1 = lane < h, own2 = own1 && r2 != r1;
        {
            C s1, s2;
            warp_hemv_rows<R>(c0, m, vb, s1, s2);
            const C p1 = cmul(f.tau, s1), p2 = cmul(f.tau, s2);
            C dot = zero;
            if (own1) dot = cfmac(p1, vb[r1], dot);
            if (own2) dot = cfmac(p2, vb[r2], dot);
            dot.x = warp_sum(dot.x);
            dot.y = warp_sum(dot.y);
            const C a2 = cscale(cmul(f.tau, dot), R(-0.5));
            if (own1) wb[r1] = cfma(a2, vb[r1], p1);     // (tau = 0: p = 0, w = 0)
            if (own2) wb[r2] = cfma(a2, vb[r2], p2);
        }
        __syncwarp();
        if (!TWO_STEP || k + 2 >= n) {                  // one step: apply its update alone
            const C* vq[1] = {vb};
            const C* wq[1] = {wb};
            warp_her2_rows<R, 1>(c0, m, vq, wq);
            __syncwarp();
            k += 1;
            continue;
        }
        if constexpr (TWO_STEP) {
            // ---- column k+1 takes step k's update: A22(r, 0) -= v_r conj(w_0) + w_r conj(v_0)
            for (int r = lane; r < m; r += 32) {
                C t = cfmsc(vb[r], wb[0], c0[r]);
                t = cfmsc(wb[r], vb[0], t);
                if (r == 0) t.y = R(0);
                c0[r] = t;
            }
            __syncwarp();
            // ---- step k+1 on the trailing matrix A22' (rows and columns >= k+2, order m1) without
            // step k's update: p' = tau' (A22' v' - v^ (w^^H v') - w^ (v^^H v'))
            const int m1 = m - 1;
            C* x1 = c0 + 1;                                 // x1[i] = A(k+2+i, k+1)
            const WarpReflector<R> f1 = warp_reflector<R>(x1, m1);
            if (lane == 0) { e[k + 1] = f1.beta; tau[k + 1] = f1.tau; }
            warp_store_reflector<R>(x1, m1, f1, vb2);
            __syncwarp();
            C* c1 = P + pk(k + 2, n);
            const C* vh = vb + 1;                           // v^, w^ over the rows of A22'
            const C* wh = wb + 1;
            {
                C g1 = zero, g2 = zero;                     // w^^H v', v^^H v'
                for (int i = lane; i < m1; i += 32) {
                    g1 = cfmac(wh[i], vb2[i], g1);
                    g2 = cfmac(vh[i], vb2[i], g2);
                }
                g1.x = warp_sum(g1.x); g1.y = warp_sum(g1.y);
                g2.x = warp_sum(g2.x); g2.y = warp_sum(g2.y);
                C s1, s2;
                warp_hemv_rows<R>(c1, m1, vb2, s1, s2);
                const int q1 = lane, q2 = m1 - 1 - lane, hh = (m1 + 1) >> 1;
                const bool o1 = lane < hh, o2 = o1 && q2 != q1;
                C p1 = zero, p2 = zero;
                if (o1) { s1 = cfms(vh[q1], g1, s1); s1 = cfms(wh[q1], g2, s1); p1 = cmul(f1.tau, s1); }
                if (o2) { s2 = cfms(vh[q2], g1, s2); s2 = cfms(wh[q2], g2, s2); p2 = cmul(f1.tau, s2); }
                C dot = zero;
                if (o1) dot = cfmac(p1, vb2[q1], dot);
                if (o2) dot = cfmac(p2, vb2[q2], dot);
                dot.x = warp_sum(dot.x);
                dot.y = warp_sum(dot.y);
                const C a2 = cscale(cmul(f1.tau, dot), R(-0.5));
                if (o1) wb2[q1] = cfma(a2, vb2[q1], p1);
                if (o2) wb2[q2] = cfma(a2, vb2[q2], p2);
            }
            __syncwarp();
            // ---- both updates on A22': step k's, then step k+1's
            {
                const C* vq[2] = {vh, vb2};
                const C* wq[2] = {wh, wb2};
                warp_her2_rows<R, 2>(c1, m1, vq, wq);
            }
            __syncwarp();
            k += 2;
        }
    }
    for (int i = lane; i < n; i += 32) d[i] = P[pk(i, n)].x;
    if (lane == 0 && n >= 1) e[n - 1] = R(0);
    __syncwarp();
}

}  // namespace sbg
