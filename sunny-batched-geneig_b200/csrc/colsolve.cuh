// Column-per-thread stage functions for n <= NMAX (NMAX = 32 or 64).
//
// One thread owns a whole column (or row) of the n x n operand in registers,
// y[0..NMAX).  Every sweep over the rows is a switch fall-through chain: it enters
// at the first active row (n - 1 or k - 1, the same for every thread of the warp),
// each case handles one row with a compile-time register index, and a `break` out
// of the switch ends the sweep at the active range's edge.  The pivot a
// substitution needs next is carried out of the sweep in a register, so no dynamic
// register index is ever formed, and each value that becomes final is stored
// straight to its destination.  L and the Householder reflectors are read from
// shared memory; all threads of the CTA read the same address at the same time
// (a broadcast).
//
// Packed lower-triangular tiles use column-major packing: A(i, j), i >= j, at
// P[pk(j, n) + i - j] (pk in stages.cuh).
#pragma once

#include "stages.cuh"

// Row-slot sequences.  SBG_DESC64(C) expands to C(63) C(62) ... C(0) (a one-jump
// select, e.g. of a pivot); SBG_BLOCKS(K) expands to K(7) ... K(0), one `case` per block
// of 8 rows, so that the rows of a block are straight-line code the scheduler can
// interleave, and SBG_ROWS8(S, B) expands to S(8B+7) ... S(8B) inside a block.
#define SBG_DESC64(C) C(63) C(62) C(61) C(60) C(59) C(58) C(57) C(56) C(55) C(54) C(53) C(52) C(51) C(50) C(49) C(48) C(47) C(46) C(45) C(44) C(43) C(42) C(41) C(40) C(39) C(38) C(37) C(36) C(35) C(34) C(33) C(32) C(31) C(30) C(29) C(28) C(27) C(26) C(25) C(24) C(23) C(22) C(21) C(20) C(19) C(18) C(17) C(16) C(15) C(14) C(13) C(12) C(11) C(10) C(9) C(8) C(7) C(6) C(5) C(4) C(3) C(2) C(1) C(0)
#define SBG_BLOCKS(K) K(7) K(6) K(5) K(4) K(3) K(2) K(1) K(0)
#define SBG_ROWS8(S, B) S((B) * 8 + 7) S((B) * 8 + 6) S((B) * 8 + 5) S((B) * 8 + 4) \
                        S((B) * 8 + 3) S((B) * 8 + 2) S((B) * 8 + 1) S((B) * 8 + 0)

namespace sbg {

// ---------------------------------------------------------------- potrf, one warp, packed
// Right-looking lower Cholesky of the packed tile P by one warp (n <= 65), two columns per pass:
// column k is scaled, column k+1 takes column k's update and is scaled, then ONE pass over the
// trailing triangle (rows and columns >= k+2) subtracts both rank-1 terms, in the order the
// one-column algorithm would (so the result is the same bit for bit) but reading and writing
// each trailing entry once per two columns instead of once per column.  Lane L updates the
// trailing rows L and m-1-L (balanced pairs, as in hetrd_warp_packed).  invd[k] = 1 / L_kk.
// Returns 0 or the order of the first non-positive (or NaN) leading minor, the zpotrf convention.
template <typename R>
__device__ int potrf_warp_packed(cplx<R>* P, int n, R* invd) {
    using C = cplx<R>;
    const int lane = threadIdx.x & 31;
    for (int k = 0; k < n; k += 2) {
        C* colk = P + pk(k, n);                   // colk[i - k] = A(i, k), i >= k
        const R dkk = colk[0].x;
        if (!(dkk > R(0))) return k + 1;          // uniform: every lane reads the same word
        const R dsq = sqrt(dkk);
        const R inv = rsqrt(dkk);                 // in parallel with the square root, not after it
        const int m0 = n - k - 1;
        __syncwarp();
        if (lane == 0) { colk[0] = mk<R>(dsq, R(0)); invd[k] = inv; }
        for (int i = 1 + lane; i <= m0; i += 32) colk[i] = cscale(colk[i], inv);
        __syncwarp();
        if (m0 == 0) break;
        // column k+1 takes column k's rank-1 term: A(k+1+i, k+1) -= l(k+1+i) conj(l(k+1))
        C* colk1 = P + pk(k + 1, n);              // colk1[i] = A(k+1+i, k+1)
        const C lk1 = colk[1];
        for (int i = lane; i < m0; i += 32) colk1[i] = cfmsc(colk[1 + i], lk1, colk1[i]);
        __syncwarp();
        const R d1 = colk1[0].x;
        if (!(d1 > R(0))) return k + 2;
        const R dsq1 = sqrt(d1);
        const R inv1 = rsqrt(d1);
        const int m = m0 - 1;                     // trailing order (rows / columns >= k + 2)
        __syncwarp();
        if (lane == 0) { colk1[0] = mk<R>(dsq1, R(0)); invd[k + 1] = inv1; }
        for (int i = 1 + lane; i <= m; i += 32) colk1[i] = cscale(colk1[i], inv1);
        __syncwarp();
        if (m == 0) break;
        // trailing A22(r, j) -= l0_r conj(l0_j) + l1_r conj(l1_j), j <= r, l0 = colk[2..], l1 = colk1[1..]
        const int base = k + 2;
        const int h = (m + 1) >> 1;
        const int r1 = lane, r2 = m - 1 - lane;
        // A22(r, j) at P + pk(base) + r - j + sum_{t<j} (m - t): advances by m - j - 1 per column
        // rows r1 (r1 + 1 terms) then r2 (r2 + 1 terms) in one loop of uniform length m + 1
        if (lane < h) {
            const int tot = (r2 != r1) ? r1 + r2 + 2 : r1 + 1;
            C* a = P + pk(base, n) + r1;
            C l0 = colk[2 + r1], l1 = colk1[1 + r1];
            int jj = 0;
            for (int t = 0; t < tot; ++t) {
                if (t == r1 + 1) { a = P + pk(base, n) + r2; l0 = colk[2 + r2]; l1 = colk1[1 + r2]; jj = 0; }
                C v = cfmsc(l0, colk[2 + jj], *a);
                *a = cfmsc(l1, colk1[1 + jj], v);
                a += m - jj - 1;
                ++jj;
            }
        }
        __syncwarp();
    }
    return 0;
}

// ---------------------------------------------------------------- forward substitution
// y <- L^{-1} y for the thread's column; L packed (Lp) in shared memory.  Each solved
// entry w_k is stored through out(k, w_k) as soon as it is final.
template <int NMAX, typename R, typename Out>
__device__ __forceinline__ void col_trsm_lower(const cplx<R>* Lp, const R* invd, cplx<R> (&y)[NMAX], int n,
                                               Out&& out) {
    using C = cplx<R>;
    for (int k = 0; k < n; ++k) {
        C piv = y[0];
#define SBG_SEL(I) case I: if constexpr ((I) < NMAX) piv = y[I]; break;
        switch (k) { SBG_DESC64(SBG_SEL) default: break; }
#undef SBG_SEL
        const C wk = cscale(piv, invd[k]);
        out(k, wk);
        const C* lk = Lp + pk(k, n) - k;          // lk[i] = L(i, k)
        // rows n-1 .. k+1, by blocks of 8 from the block of n-1 down to the block of k+1
#define SBG_S(I) if constexpr ((I) < NMAX) { if ((I) > k && (I) < n) y[I] = cfms(lk[I], wk, y[I]); }
#define SBG_K(B) case B: if ((B) * 8 + 7 <= k) break; SBG_ROWS8(SBG_S, B)
        switch ((n - 1) >> 3) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
    }
}

// col_trsm_lower two steps per sweep: the pivots of k and k+1 are selected together, w_k formed,
// row k+1 updated by it alone and w_{k+1} formed, then ONE sweep over the rows below subtracts
// L(i, k) w_k and L(i, k+1) w_{k+1}, in that order (every y[i] takes the same operations as in
// the one-step sweep).  Since the descending sweep reaches row k+1 last, the next pivot no longer
// waits for a whole sweep per step.
template <int NMAX, typename R, typename Out>
__device__ __forceinline__ void col_trsm_lower2(const cplx<R>* Lp, const R* invd, cplx<R> (&y)[NMAX], int n,
                                                Out&& out) {
    using C = cplx<R>;
    int k = 0;
    for (; k + 1 < n; k += 2) {
        C piv = y[0], piv1 = y[0];
#define SBG_SEL(I) case I: if constexpr ((I) < NMAX) { piv = y[I]; if constexpr ((I) + 1 < NMAX) piv1 = y[(I) + 1]; } break;
        switch (k) { SBG_DESC64(SBG_SEL) default: break; }
#undef SBG_SEL
        const C* lk = Lp + pk(k, n) - k;           // lk[i] = L(i, k)
        const C* lk1 = Lp + pk(k + 1, n) - (k + 1); // lk1[i] = L(i, k + 1)
        const C wk = cscale(piv, invd[k]);
        out(k, wk);
        const C wk1 = cscale(cfms(lk[k + 1], wk, piv1), invd[k + 1]);
        out(k + 1, wk1);
#define SBG_S(I) if constexpr ((I) < NMAX) { if ((I) > k + 1 && (I) < n) y[I] = cfms(lk1[I], wk1, cfms(lk[I], wk, y[I])); }
#define SBG_K(B) case B: if ((B) * 8 + 7 <= k + 1) break; SBG_ROWS8(SBG_S, B)
        switch ((n - 1) >> 3) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
    }
    if (k < n) {                                  // an odd n: the last row alone
        C piv = y[0];
#define SBG_SEL(I) case I: if constexpr ((I) < NMAX) piv = y[I]; break;
        switch (k) { SBG_DESC64(SBG_SEL) default: break; }
#undef SBG_SEL
        out(k, cscale(piv, invd[k]));
    }
}

// row_trsm_right_lowerH two steps per sweep, as col_trsm_lower2: c_k, then row k+1's value takes
// c_k's term alone and gives c_{k+1}, then one sweep subtracts both from the columns above.
template <int NMAX, typename R, typename Out>
__device__ __forceinline__ void row_trsm_right_lowerH2(const cplx<R>* Lp, const R* invd, cplx<R> (&y)[NMAX], int n,
                                                       int i, int kmax, Out&& out) {
    using C = cplx<R>;
    int k = 0;
    for (; k + 1 <= kmax; k += 2) {              // kmax: the largest row of the warp (uniform loop)
        C piv = y[0], piv1 = y[0];
#define SBG_SEL(I) case I: if constexpr ((I) < NMAX) { piv = y[I]; if constexpr ((I) + 1 < NMAX) piv1 = y[(I) + 1]; } break;
        switch (k) { SBG_DESC64(SBG_SEL) default: break; }
#undef SBG_SEL
        const C* lk = Lp + pk(k, n) - k;          // lk[kk] = L(kk, k)
        const C* lk1 = Lp + pk(k + 1, n) - (k + 1);
        const C ck = cscale(piv, invd[k]);
        if (k <= i) out(k, ck);
        const C ck1 = cscale(cfmsc(ck, lk[k + 1], piv1), invd[k + 1]);
        if (k + 1 <= i) out(k + 1, ck1);
#define SBG_S(I) if constexpr ((I) < NMAX) { if ((I) > k + 1 && (I) <= i) y[I] = cfmsc(ck1, lk1[I], cfmsc(ck, lk[I], y[I])); }
#define SBG_K(B) case B: if ((B) * 8 + 7 <= k + 1) break; SBG_ROWS8(SBG_S, B)
        switch (kmax >> 3) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
    }
    if (k <= kmax) {                              // one step left
        C piv = y[0];
#define SBG_SEL(I) case I: if constexpr ((I) < NMAX) piv = y[I]; break;
        switch (k) { SBG_DESC64(SBG_SEL) default: break; }
#undef SBG_SEL
        const C ck = cscale(piv, invd[k]);
        if (k <= i) out(k, ck);
    }
}

// Row i of C = W L^{-H}, columns kk <= i (the rest is not needed: C is Hermitian).
// y holds W(i, 0..i); the solved C(i, k) go through out(k, c).
template <int NMAX, typename R, typename Out>
__device__ __forceinline__ void row_trsm_right_lowerH(const cplx<R>* Lp, const R* invd, cplx<R> (&y)[NMAX], int n,
                                                      int i, int kmax, Out&& out) {
    using C = cplx<R>;
    for (int k = 0; k <= kmax; ++k) {            // kmax: the largest row of the warp (uniform loop)
        C piv = y[0];
#define SBG_SEL(I) case I: if constexpr ((I) < NMAX) piv = y[I]; break;
        switch (k) { SBG_DESC64(SBG_SEL) default: break; }
#undef SBG_SEL
        const C ck = cscale(piv, invd[k]);
        if (k <= i) out(k, ck);
        const C* lk = Lp + pk(k, n) - k;          // lk[kk] = L(kk, k)
#define SBG_S(I) if constexpr ((I) < NMAX) { if ((I) > k && (I) <= i) y[I] = cfmsc(ck, lk[I], y[I]); }
#define SBG_K(B) case B: if ((B) * 8 + 7 <= k) break; SBG_ROWS8(SBG_S, B)
        switch (kmax >> 3) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
    }
}

// ---------------------------------------------------------------- G lanes per column
// The sweeps with a column's rows spread over G adjacent lanes (G a power of two): lane g of
// the group holds rows i = G r + g in y[r], r < RM.  Control flow is uniform over the group
// (the sweep's block range is taken for the whole group, rows are predicated), so the
// group's partial dot products combine with one shuffle; every lane of the warp must call.

// y <- Q y, Q = H_0 ... H_{n-2}, reflectors along the rows of the LV tile (ld): v_k(i) = LV(k, i)
// for i >= k + 1, the superdiagonal entry LV(k, k+1) holding v_k(k+1) = 1.
template <int G, int RM, typename R>
__device__ __forceinline__ void grp_apply_q(const cplx<R>* LV, int ld, const cplx<R>* tau, cplx<R> (&y)[RM], int n,
                                            int g) {
    using C = cplx<R>;
    const int nb = ((n - 1) / G) >> 3;               // block of the highest slot any lane holds
    for (int k = n - 2; k >= 0; --k) {
        const C tk = tau[k];
        if (tk.x == R(0) && tk.y == R(0)) continue;
        const C* vrow = LV + k;                      // v_k(i) = vrow[i * ld], i >= k + 1
        const int kb = (k + 1) / G - 1;              // slots <= kb are inactive on every lane
        C s0 = mk<R>(R(0), R(0)), s1 = s0, s2 = s0, s3 = s0;    // four chains: the dot's FMAs overlap
#define SBG_S(I) if constexpr ((I) < RM) { const int i = G * (I) + g; if (i > k && i < n) { \
        if (((I) & 3) == 0) s0 = cfmac(vrow[i * ld], y[I], s0); \
        else if (((I) & 3) == 1) s1 = cfmac(vrow[i * ld], y[I], s1); \
        else if (((I) & 3) == 2) s2 = cfmac(vrow[i * ld], y[I], s2); \
        else s3 = cfmac(vrow[i * ld], y[I], s3); } }
#define SBG_K(B) case B: if ((B) * 8 + 7 <= kb) break; SBG_ROWS8(SBG_S, B)
        switch (nb) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
        C s = cadd(cadd(s0, s1), cadd(s2, s3));
        if constexpr (G > 1) {
#pragma unroll
            for (int m = 1; m < G; m <<= 1) { s.x += shfl_xor(s.x, m); s.y += shfl_xor(s.y, m); }
        }
        s = cmul(tk, s);
        asm volatile("" ::: "memory");               // reload v_k below rather than hold it in registers
#define SBG_S(I) if constexpr ((I) < RM) { const int i = G * (I) + g; if (i > k && i < n) y[I] = cfms(vrow[i * ld], s, y[I]); }
#define SBG_K(B) case B: if ((B) * 8 + 7 <= kb) break; SBG_ROWS8(SBG_S, B)
        switch (nb) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
    }
}

// y <- Q y as grp_apply_q, two reflectors per pass.  For the pair (a, b = a - 1), H_a applied
// first: one pass over the rows forms both dot products s_a = v_a^H y (rows > a) and
// s_b = v_b^H y (rows >= a), then t_a = tau_a s_a and t_b = tau_b (s_b - c_a t_a) with
// c_a = v_b^H v_a (cpair[a], formed once per pair of the batch), and one pass subtracts
// v_a t_a, then v_b t_b, from every row -- the same two reflections, in the same order, with half
// as many dependent dot-product / update rounds for the column to wait on.  A reflector with
// tau = 0 contributes t = 0.  The compiler barrier after each block of 8 rows keeps the two
// vectors' loads from being hoisted ahead en bloc (which spilled the column's registers).
template <int G, int RM, typename R>
__device__ __forceinline__ void grp_apply_q2(const cplx<R>* LV, int ld, const cplx<R>* tau, const cplx<R>* cpair,
                                             cplx<R> (&y)[RM], int n, int g) {
    using C = cplx<R>;
    const int nb = ((n - 1) / G) >> 3;               // block of the highest slot any lane holds
    int k = n - 2;
#pragma unroll 1
    for (; k >= 1; k -= 2) {
        const int a = k;
        const C* va = LV + a;                        // v_a(i) = va[i * ld], i >= a + 1
        // v_b(i) = va[i * ld - 1] (row b = a - 1 of the tile), i >= a, v_b(a) = 1: one base pointer,
        // so every row's two loads are immediate offsets from it
        const int kb = a / G - 1;                    // slots <= kb hold only rows < a on every lane
        C sa0 = mk<R>(R(0), R(0)), sa1 = sa0, sb0 = sa0, sb1 = sa0;
#define SBG_S(I) if constexpr ((I) < RM) { const int i = G * (I) + g; if (i >= a && i < n) { \
        const C vai = (i > a) ? va[i * ld] : mk<R>(R(0), R(0)); \
        if (((I) & 1) == 0) { sb0 = cfmac(va[i * ld - 1], y[I], sb0); sa0 = cfmac(vai, y[I], sa0); } \
        else { sb1 = cfmac(va[i * ld - 1], y[I], sb1); sa1 = cfmac(vai, y[I], sa1); } } }
#define SBG_K(B) case B: if ((B) * 8 + 7 <= kb) break; SBG_ROWS8(SBG_S, B) asm volatile("" ::: "memory");
        switch (nb) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
        C sa = cadd(sa0, sa1), sb = cadd(sb0, sb1);
        if constexpr (G > 1) {
#pragma unroll
            for (int m = 1; m < G; m <<= 1) {
                sa.x += shfl_xor(sa.x, m); sa.y += shfl_xor(sa.y, m);
                sb.x += shfl_xor(sb.x, m); sb.y += shfl_xor(sb.y, m);
            }
        }
        const C ta = cmul(tau[a], sa);
        const C tb = cmul(tau[a - 1], cfms(cpair[a], ta, sb));
        asm volatile("" ::: "memory");               // reload v below rather than hold it in registers
#define SBG_S(I) if constexpr ((I) < RM) { const int i = G * (I) + g; if (i >= a && i < n) { \
        const C vai = (i > a) ? va[i * ld] : mk<R>(R(0), R(0)); \
        y[I] = cfms(va[i * ld - 1], tb, cfms(vai, ta, y[I])); } }
#define SBG_K(B) case B: if ((B) * 8 + 7 <= kb) break; SBG_ROWS8(SBG_S, B) asm volatile("" ::: "memory");
        switch (nb) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
    }
    if (k == 0) {                                    // an odd count: H_0 alone
        const C tk = tau[0];
        C s0 = mk<R>(R(0), R(0)), s1 = s0;
#define SBG_S(I) if constexpr ((I) < RM) { const int i = G * (I) + g; if (i > 0 && i < n) { \
        if (((I) & 1) == 0) s0 = cfmac(LV[i * ld], y[I], s0); else s1 = cfmac(LV[i * ld], y[I], s1); } }
#define SBG_K(B) case B: SBG_ROWS8(SBG_S, B)
        switch (nb) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
        C s = cadd(s0, s1);
        if constexpr (G > 1) {
#pragma unroll
            for (int m = 1; m < G; m <<= 1) { s.x += shfl_xor(s.x, m); s.y += shfl_xor(s.y, m); }
        }
        s = cmul(tk, s);
#define SBG_S(I) if constexpr ((I) < RM) { const int i = G * (I) + g; if (i > 0 && i < n) y[I] = cfms(LV[i * ld], s, y[I]); }
#define SBG_K(B) case B: SBG_ROWS8(SBG_S, B)
        switch (nb) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
    }
}

// c_a = v_{a-1}^H v_a for a = 1 .. n-2 into cpair[a] (the coupling grp_apply_q2 needs), reflectors
// along the rows of the LV tile as there; every thread of the CTA calls (T threads).
template <typename R>
__device__ __forceinline__ void reflector_couplings(const cplx<R>* LV, int ld, int n, cplx<R>* cpair, int T) {
    for (int a = 1 + static_cast<int>(threadIdx.x); a + 1 < n; a += T) {
        cplx<R> c = mk<R>(R(0), R(0));
        for (int i = a + 1; i < n; ++i) c = cfmac(LV[(a - 1) + i * ld], LV[a + i * ld], c);
        cpair[a] = c;
    }
}

// y <- L^{-1} y (forward substitution) with L packed by columns (Lp, order n): lane g of the
// group holds rows G r + g.  Each solved w_k stays in its slot of the owning lane.
template <int G, int RM, typename R>
__device__ __forceinline__ void grp_trsm_lower_packed(const cplx<R>* Lp, const R* invd, cplx<R> (&y)[RM], int n,
                                                      int g) {
    using C = cplx<R>;
    const int lane = threadIdx.x & 31;
    const int nb = ((n - 1) / G) >> 3;
    for (int k = 0; k < n; ++k) {
        const int rk = k / G, gk = k - rk * G;
        C piv = y[0];
#define SBG_SEL(I) case I: if constexpr ((I) < RM) piv = y[I]; break;
        switch (rk) { SBG_DESC64(SBG_SEL) default: break; }
#undef SBG_SEL
        if constexpr (G > 1) piv = cshfl(piv, (lane & ~(G - 1)) | gk);
        const C wk = cscale(piv, invd[k]);
        if (g == gk) {
#define SBG_SET(I) case I: if constexpr ((I) < RM) y[I] = wk; break;
            switch (rk) { SBG_DESC64(SBG_SET) default: break; }
#undef SBG_SET
        }
        const C* lk = Lp + pk(k, n) - k;             // lk[i] = L(i, k)
        const int kb = (k + 1) / G - 1;              // slots <= kb are inactive on every lane
#define SBG_S(I) if constexpr ((I) < RM) { const int i = G * (I) + g; if (i > k && i < n) y[I] = cfms(lk[i], wk, y[I]); }
#define SBG_K(B) case B: if ((B) * 8 + 7 <= kb) break; SBG_ROWS8(SBG_S, B)
        switch (nb) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
    }
}

// x = L^{-H} y (backward substitution), L full lower in the LV tile (ld); each x_k goes through
// out(k, x_k), on the lane that holds row k, as soon as it is final.
template <int G, int RM, typename R, typename Out>
__device__ __forceinline__ void grp_trsm_lowerH(const cplx<R>* LV, int ld, const R* invd, cplx<R> (&y)[RM], int n,
                                                int g, Out&& out) {
    using C = cplx<R>;
    const int lane = threadIdx.x & 31;
    for (int k = n - 1; k >= 0; --k) {
        const int rk = k / G, gk = k - rk * G;       // row k: slot rk of lane gk
        C piv = y[0];
#define SBG_SEL(I) case I: if constexpr ((I) < RM) piv = y[I]; break;
        switch (rk) { SBG_DESC64(SBG_SEL) default: break; }
#undef SBG_SEL
        if constexpr (G > 1) piv = cshfl(piv, (lane & ~(G - 1)) | gk);
        const C xk = cscale(piv, invd[k]);
        if (g == gk) out(k, xk);
        if (k == 0) break;
        const C* lrow = LV + k;                      // L(k, i) = lrow[i * ld], i < k
#define SBG_S(I) if constexpr ((I) < RM) { const int i = G * (I) + g; if (i < k) y[I] = cfms(cconj(lrow[i * ld]), xk, y[I]); }
#define SBG_K(B) case B: SBG_ROWS8(SBG_S, B)
        switch (((k - 1) / G) >> 3) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
    }
}

// grp_trsm_lowerH two steps per sweep: rows k and k-1 are selected together, x_k formed, row k-1
// takes x_k's term alone and gives x_{k-1}, then one sweep over the rows above subtracts
// conj(L(k, i)) x_k and conj(L(k-1, i)) x_{k-1}, in that order (the same operations per entry as
// the one-step sweeps, half as many sweeps).
template <int G, int RM, typename R, typename Out>
__device__ __forceinline__ void grp_trsm_lowerH2(const cplx<R>* LV, int ld, const R* invd, cplx<R> (&y)[RM], int n,
                                                 int g, Out&& out) {
    using C = cplx<R>;
    const int lane = threadIdx.x & 31;
    int k = n - 1;
    for (; k >= 1; k -= 2) {
        const int rk = k / G, gk = k - rk * G;       // row k: slot rk of lane gk
        const int rk1 = (k - 1) / G, gk1 = (k - 1) - rk1 * G;
        C piv = y[0], piv1 = y[0];
#define SBG_SEL(I) case I: if constexpr ((I) < RM) piv = y[I]; break;
        switch (rk) { SBG_DESC64(SBG_SEL) default: break; }
#undef SBG_SEL
#define SBG_SEL(I) case I: if constexpr ((I) < RM) piv1 = y[I]; break;
        switch (rk1) { SBG_DESC64(SBG_SEL) default: break; }
#undef SBG_SEL
        if constexpr (G > 1) {
            piv = cshfl(piv, (lane & ~(G - 1)) | gk);
            piv1 = cshfl(piv1, (lane & ~(G - 1)) | gk1);
        }
        const C* lrow = LV + k;                      // L(k, i) = lrow[i * ld], i < k
        const C* lrow1 = LV + k - 1;                 // L(k-1, i) = lrow1[i * ld], i < k - 1
        const C xk = cscale(piv, invd[k]);
        if (g == gk) out(k, xk);
        const C xk1 = cscale(cfms(cconj(lrow[(k - 1) * ld]), xk, piv1), invd[k - 1]);
        if (g == gk1) out(k - 1, xk1);
        if (k == 1) { k = -1; break; }
#define SBG_S(I) if constexpr ((I) < RM) { const int i = G * (I) + g; if (i < k - 1) \
        y[I] = cfms(cconj(lrow1[i * ld]), xk1, cfms(cconj(lrow[i * ld]), xk, y[I])); }
#define SBG_K(B) case B: SBG_ROWS8(SBG_S, B)
        switch (((k - 2) / G) >> 3) { SBG_BLOCKS(SBG_K) default: break; }
#undef SBG_K
#undef SBG_S
    }
    if (k == 0) {                                    // an odd n: row 0 alone
        C piv = y[0];
        if constexpr (G > 1) piv = cshfl(piv, lane & ~(G - 1));
        const C x0 = cscale(piv, invd[0]);
        if (g == 0) out(0, x0);
    }
}

}  // namespace sbg
