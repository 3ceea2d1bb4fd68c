// Complex FP64 tile products on the FP64 tensor cores (mma.sync.m8n8k4.f64), one CTA of 4 warps
// per product of 32 x 32 output tiles, operands read from global memory (L2) through 16-deep
// shared-memory panels.  Used by the mixed form's refinement (mixed_big.cu) and the blocked FP64
// Cholesky and reduction (reduce_tc.cu).
//
// Operands are views of column-major matrices: element (i, j) at p[i + j * ld] for i < rows,
// j < cols, zero outside.  op(M)(i, j) is M(i, j) (kOpN) or conj(M(j, i)) (kOpC).  A warp holds a
// 16 x 16 quarter of the tile as 2 x 2 blocks of 8 x 8 in the MMA accumulator layout; a complex
// product is four real MMAs.
#pragma once

#include "common.cuh"

namespace sbg {

constexpr int kTileThreads = 128;        // 4 warps, 2 x 2 over a 32 x 32 output tile
constexpr int kTile = 32;
constexpr int kTileKP = 16;              // k values per staged panel
constexpr int kTileLDA = kTile + 2;      // As: A(r, k) at k * kTileLDA + r (16-byte entries)
constexpr int kTileLDB = kTileKP + 4;    // Bs: B(k, c) at c * kTileLDB + k
constexpr int kTileWarps = kTileThreads / 32;

// The strides keep the fragment loads free of bank conflicts: a quarter-warp phase of 16-byte
// loads covers lanes (g, t), g in {0, 1}, t in 0..3, at entries t * kTileLDA + g (A: 2t + g mod 8
// distinct) and g * kTileLDB + t (B: 4g + t mod 8 distinct).
static_assert(kTileLDA % 8 == 2 && kTileLDB % 8 == 4, "fragment strides");

enum TileOp : int { kOpN = 0, kOpC = 1 };

struct MatView {
    const double2* p;
    int ld, rows, cols;
};

struct TileSmem {
    double2 As[kTileKP * kTileLDA];
    double2 Bs[2][kTile * kTileLDB];
};

// D(8x8) += A(8x4) B(4x8), FP64, one warp: lane (g, t) = (lane / 4, lane % 4) holds a = A(g, t),
// b = B(t, g) and d0, d1 = D(g, 2t), D(g, 2t + 1).
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

__device__ __forceinline__ double2 ldcg2(const double2* p) { return __ldcg(p); }

// op(M)(i, j), zero outside the view.
template <int OP>
__device__ __forceinline__ double2 view_at(const MatView& m, int i, int j) {
    if (OP == kOpN)
        return (i < m.rows && j < m.cols) ? ldcg2(m.p + i + static_cast<size_t>(j) * m.ld) : make_double2(0.0, 0.0);
    const double2 v = (j < m.rows && i < m.cols) ? ldcg2(m.p + j + static_cast<size_t>(i) * m.ld)
                                                 : make_double2(0.0, 0.0);
    return make_double2(v.x, -v.y);
}

// A warp's 16 x 16 quarter of a 32 x 32 complex tile.  Block (br, bc) holds rows
// 16 wr + 8 br + g, columns 16 wc + 8 bc + 2t + q (w = 2 wr + wc).
struct Quarter {
    double re[2][2][2], im[2][2][2];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int br = 0; br < 2; ++br)
#pragma unroll
            for (int bc = 0; bc < 2; ++bc)
#pragma unroll
                for (int q = 0; q < 2; ++q) re[br][bc][q] = im[br][bc][q] = 0.0;
    }
};

// Position (tile-local) of this lane's accumulator entry (br, bc, q).
__device__ __forceinline__ void quarter_pos(int br, int bc, int q, int& row, int& col) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    row = 16 * (w >> 1) + 8 * br + g;
    col = 16 * (w & 1) + 8 * bc + 2 * t + q;
}

// acc = op(M) on the tile.
template <int OP>
__device__ __forceinline__ void quarter_load(Quarter& acc, const MatView& m) {
#pragma unroll
    for (int br = 0; br < 2; ++br)
#pragma unroll
        for (int bc = 0; bc < 2; ++bc)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                int row, col;
                quarter_pos(br, bc, q, row, col);
                const double2 v = view_at<OP>(m, row, col);
                acc.re[br][bc][q] = v.x;
                acc.im[br][bc][q] = v.y;
            }
}

// Stores the tile into M (column-major, ld) at rows < rows, columns < cols; with lower, only the
// entries whose global row (row0 + row) is >= global column (col0 + col).
__device__ __forceinline__ void quarter_store(const Quarter& acc, double2* p, int ld, int rows, int cols,
                                              bool lower = false, int row0 = 0, int col0 = 0) {
#pragma unroll
    for (int br = 0; br < 2; ++br)
#pragma unroll
        for (int bc = 0; bc < 2; ++bc)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                int row, col;
                quarter_pos(br, bc, q, row, col);
                if (row < rows && col < cols && (!lower || row0 + row >= col0 + col))
                    __stcg(p + row + static_cast<size_t>(col) * ld, make_double2(acc.re[br][bc][q], acc.im[br][bc][q]));
            }
}

// acc[o] += op(A)(0..31, k) op(B_o)(k, 0..31) summed over k < kn, o < NOUT (B1 is read only when
// NOUT == 2); with negA, op(A) is negated.  All threads of the CTA take part (the panel staging is
// shared); the caller synchronises before it reuses anything the product read.  The next panel is
// fetched into registers while the current one is multiplied.
template <int OPA, int OPB, int NOUT>
__device__ void tile_mm(Quarter (&acc)[NOUT], const MatView& A, const MatView& B0, const MatView& B1, int kn,
                        TileSmem& sm, bool negA = false) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = lane >> 2, t = lane & 3;
    const int wr = w >> 1, wc = w & 1;
    constexpr int kPer = kTileKP * kTile / kTileThreads;     // entries per thread per operand panel
    double2 ra[kPer], rb[NOUT][kPer];
    // entry e of a panel: for op N of A / op C of B the 32-long index runs fastest (a column run in
    // memory), for op C of A / op N of B the 16-long k index does
    auto fetch = [&](int kb) {
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int e = tid + kTileThreads * u;
            const int ar = OPA == kOpN ? e % kTile : e / kTileKP, ak = OPA == kOpN ? e / kTile : e % kTileKP;
            double2 v = ak + kb < kn ? view_at<OPA>(A, ar, kb + ak) : make_double2(0.0, 0.0);
            if (negA) { v.x = -v.x; v.y = -v.y; }
            ra[u] = v;
            const int bc = OPB == kOpN ? e / kTileKP : e % kTile, bk = OPB == kOpN ? e % kTileKP : e / kTile;
#pragma unroll
            for (int o = 0; o < NOUT; ++o)
                rb[o][u] = bk + kb < kn ? view_at<OPB>(o == 0 ? B0 : B1, kb + bk, bc) : make_double2(0.0, 0.0);
        }
    };
    auto stash = [&]() {
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int e = tid + kTileThreads * u;
            const int ar = OPA == kOpN ? e % kTile : e / kTileKP, ak = OPA == kOpN ? e / kTile : e % kTileKP;
            sm.As[ak * kTileLDA + ar] = ra[u];
            const int bc = OPB == kOpN ? e / kTileKP : e % kTile, bk = OPB == kOpN ? e % kTileKP : e / kTile;
#pragma unroll
            for (int o = 0; o < NOUT; ++o) sm.Bs[o][bc * kTileLDB + bk] = rb[o][u];
        }
    };
    if (kn <= 0) return;
    fetch(0);
    for (int kb = 0; kb < kn; kb += kTileKP) {
        __syncthreads();                                     // the previous panel is consumed
        stash();
        __syncthreads();
        if (kb + kTileKP < kn) fetch(kb + kTileKP);          // in flight while this panel is multiplied
#pragma unroll
        for (int k0 = 0; k0 < kTileKP; k0 += 4) {
            double2 a[2], bf[NOUT][2];
#pragma unroll
            for (int br = 0; br < 2; ++br) a[br] = sm.As[(k0 + t) * kTileLDA + 16 * wr + 8 * br + g];
#pragma unroll
            for (int o = 0; o < NOUT; ++o)
#pragma unroll
                for (int bc = 0; bc < 2; ++bc) bf[o][bc] = sm.Bs[o][(16 * wc + 8 * bc + g) * kTileLDB + k0 + t];
#pragma unroll
            for (int o = 0; o < NOUT; ++o)
#pragma unroll
                for (int br = 0; br < 2; ++br)
#pragma unroll
                    for (int bc = 0; bc < 2; ++bc) {
                        double* dr = acc[o].re[br][bc];
                        double* di = acc[o].im[br][bc];
                        dmma(dr[0], dr[1], a[br].x, bf[o][bc].x);
                        dmma(dr[0], dr[1], -a[br].y, bf[o][bc].y);
                        dmma(di[0], di[1], a[br].x, bf[o][bc].y);
                        dmma(di[0], di[1], a[br].y, bf[o][bc].x);
                    }
        }
    }
}

// The view of a rows x cols column-major matrix M (leading dimension ld) from element (r0, c0) on:
// its (i, j) is M(r0 + i, c0 + j).  An op-C operand whose op(M)(i, j) is conj(M(a + j, b + i)) is
// the view from (a, b).  Every load a tile product issues is a read of the caller's workspace or
// inputs; the caller synchronises the CTA between a tile store and a product that reads it (a
// product fetches its first panel before its first barrier).
__device__ __forceinline__ MatView sub_view(const double2* M, int ld, int rows, int cols, int r0, int c0) {
    return MatView{M + r0 + static_cast<size_t>(c0) * ld, ld, rows - r0, cols - c0};
}

}  // namespace sbg
