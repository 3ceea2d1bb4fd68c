// Oracle for the batched Hermitian-definite generalized eigensolve A x = lambda B x.
//
// TEST INFRASTRUCTURE ONLY.  This library is the CPU checker: tests, the smoke
// check and the bench's cpu_baseline / reference arm may call it; the product
// path (the CUDA library under sunny-batched-geneig_b200/) never does.
//
// What it restates from the reference (riteshbhirud/sunny-batched-geneig):
//   * the fixture generator of tests/lapack_reference.cpp:86-150 and :167-175
//     (std::mt19937_64 seeded with --seed, a fresh std::normal_distribution(0,1)
//     per helper call, column-major fill, H = A + A^H, S = A A^H + n I or
//     S = (1 + n/2) I + 0.1 (B + B^H)), so that the twelve GEIG v1 fixtures in
//     tests/data/ regenerate bit-identically here and on machines without the
//     reference tree;
//   * the reference's CPU solve, LAPACKE_zhegv(itype=1,'V','L') per pair
//     (tests/test_full_batched_n54.cpp:238-256), and LAPACKE_zhegvd, which made
//     the fixtures (tests/lapack_reference.cpp:186-194);
//   * the per-stage LAPACK twins the reference's staged tests check against:
//     zpotrf 'L' with the strict upper triangle zeroed (tests/test_chol_n54.cpp),
//     zpotrf+zhegst itype 1 'L' with the strict upper zeroed
//     (tests/test_reduce_n54.cpp:134-163), zpotrf+zhegst+zheev 'V','L'
//     (tests/test_reduce_eig_n54.cpp:143-155), and the finish stage
//     heev(M) then U = L^{-H} V (src/geneig_fixed.cu:516-567).
// LAPACK itself comes from the OpenBLAS 0.3.15 shipped in this image.
//
// Every batch routine partitions the pairs over `nthreads` host threads, one pair
// per task, with OpenBLAS forced to one thread (the reference's own CPU loop,
// tests/test_full_batched_n54.cpp:238-256, solves one pair per LAPACKE call; the
// threads run such calls side by side without oversubscribing the cores).

#include <lapacke.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

using cdouble = std::complex<double>;

extern "C" {
void openblas_set_num_threads(int);
void ztrsm_(const char* side, const char* uplo, const char* transa, const char* diag,
            const int* m, const int* n, const cdouble* alpha, const cdouble* a, const int* lda,
            cdouble* b, const int* ldb, size_t, size_t, size_t, size_t);
}

namespace {

// Runs body(b) for b in [0, batch) on nthreads threads with dynamic hand-out.
template <class F>
void parallel_pairs(int batch, int nthreads, F&& body) {
    if (batch <= 0) return;
    openblas_set_num_threads(1);
    if (nthreads <= 1 || batch == 1) {
        for (int b = 0; b < batch; ++b) body(b);
        return;
    }
    nthreads = std::min(nthreads, batch);
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    pool.reserve(nthreads);
    for (int t = 0; t < nthreads; ++t) {
        pool.emplace_back([&]() {
            for (;;) {
                int b = next.fetch_add(1);
                if (b >= batch) break;
                body(b);
            }
        });
    }
    for (auto& th : pool) th.join();
}

// tests/lapack_reference.cpp:86-101 — H = G + G^H, G complex normal(0,1) entries.
void gen_hermitian(int n, std::mt19937_64& rng, cdouble* H) {
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<cdouble> G(static_cast<size_t>(n) * n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) G[static_cast<size_t>(j) * n + i] = cdouble(nd(rng), nd(rng));
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            H[static_cast<size_t>(j) * n + i] =
                G[static_cast<size_t>(j) * n + i] + std::conj(G[static_cast<size_t>(i) * n + j]);
}

// tests/lapack_reference.cpp:105-127 — S = G G^H + n I.
void gen_hpd_wide(int n, std::mt19937_64& rng, cdouble* S) {
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<cdouble> G(static_cast<size_t>(n) * n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) G[static_cast<size_t>(j) * n + i] = cdouble(nd(rng), nd(rng));
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            cdouble acc(0.0, 0.0);
            for (int k = 0; k < n; ++k)
                acc += G[static_cast<size_t>(k) * n + i] * std::conj(G[static_cast<size_t>(k) * n + j]);
            S[static_cast<size_t>(j) * n + i] = acc;
        }
    for (int i = 0; i < n; ++i) S[static_cast<size_t>(i) * n + i] += cdouble(static_cast<double>(n), 0.0);
}

// tests/lapack_reference.cpp:132-150 — S = (1 + n/2) I + 0.1 (G + G^H).
void gen_hpd_near_identity(int n, std::mt19937_64& rng, cdouble* S) {
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<cdouble> G(static_cast<size_t>(n) * n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) G[static_cast<size_t>(j) * n + i] = cdouble(nd(rng), nd(rng));
    const double shift = 1.0 + 0.5 * static_cast<double>(n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            cdouble v = 0.1 * (G[static_cast<size_t>(j) * n + i] + std::conj(G[static_cast<size_t>(i) * n + j]));
            if (i == j) v += cdouble(shift, 0.0);
            S[static_cast<size_t>(j) * n + i] = v;
        }
}

void zero_strict_upper(int n, cdouble* M) {
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < j; ++i) M[static_cast<size_t>(j) * n + i] = cdouble(0.0, 0.0);
}

// U = L^{-H} V  (ztrsm side 'L', uplo 'L', trans 'C', diag 'N').
void back_transform(int n, const cdouble* L, cdouble* V) {
    const cdouble one(1.0, 0.0);
    ztrsm_("L", "L", "C", "N", &n, &n, &one, L, &n, V, &n, 1, 1, 1, 1);
}

}  // namespace

extern "C" {

// Regenerates a GEIG v1 fixture's inputs (H then S per pair, column-major).
// s_mode: 0 = random (wide-spectrum HPD), 1 = near-identity.
void sbo_gen_fixture_pairs(int n, int batch, int seed, int s_mode, cdouble* H, cdouble* S) {
    std::mt19937_64 rng(static_cast<std::uint64_t>(seed));
    const size_t mat = static_cast<size_t>(n) * n;
    for (int b = 0; b < batch; ++b) {
        gen_hermitian(n, rng, H + mat * b);
        if (s_mode == 0) gen_hpd_wide(n, rng, S + mat * b);
        else             gen_hpd_near_identity(n, rng, S + mat * b);
    }
}

// Full solve per pair with LAPACKE_zhegv (use_dc = 0) or LAPACKE_zhegvd (use_dc = 1).
// W[b*n + i] ascending, U column-major B-orthonormal eigenvectors, info per pair.
void sbo_hegv_batch(int n, int batch, const cdouble* H, const cdouble* S, double* W, cdouble* U,
                    int* info, int use_dc, int nthreads) {
    const size_t mat = static_cast<size_t>(n) * n;
    parallel_pairs(batch, nthreads, [&](int b) {
        std::vector<cdouble> Bw(S + mat * b, S + mat * (b + 1));
        cdouble* Aw = U + mat * b;
        std::memcpy(Aw, H + mat * b, sizeof(cdouble) * mat);
        lapack_int r = use_dc ? LAPACKE_zhegvd(LAPACK_COL_MAJOR, 1, 'V', 'L', n, Aw, n, Bw.data(), n,
                                               W + static_cast<size_t>(n) * b)
                              : LAPACKE_zhegv(LAPACK_COL_MAJOR, 1, 'V', 'L', n, Aw, n, Bw.data(), n,
                                              W + static_cast<size_t>(n) * b);
        info[b] = static_cast<int>(r);
    });
}

// Eigenvalues only (jobz 'N'), for the throughput baseline's lighter variant.
void sbo_hegv_values_batch(int n, int batch, const cdouble* H, const cdouble* S, double* W,
                           int* info, int nthreads) {
    const size_t mat = static_cast<size_t>(n) * n;
    parallel_pairs(batch, nthreads, [&](int b) {
        std::vector<cdouble> Aw(H + mat * b, H + mat * (b + 1));
        std::vector<cdouble> Bw(S + mat * b, S + mat * (b + 1));
        info[b] = static_cast<int>(LAPACKE_zhegv(LAPACK_COL_MAJOR, 1, 'N', 'L', n, Aw.data(), n,
                                                 Bw.data(), n, W + static_cast<size_t>(n) * b));
    });
}

// Stage twin of the Cholesky kernel: L (lower, strict upper zeroed).
void sbo_potrf_batch(int n, int batch, const cdouble* S, cdouble* L, int* info, int nthreads) {
    const size_t mat = static_cast<size_t>(n) * n;
    parallel_pairs(batch, nthreads, [&](int b) {
        cdouble* Lb = L + mat * b;
        std::memcpy(Lb, S + mat * b, sizeof(cdouble) * mat);
        info[b] = static_cast<int>(LAPACKE_zpotrf(LAPACK_COL_MAJOR, 'L', n, Lb, n));
        zero_strict_upper(n, Lb);
    });
}

// Stage twin of the reduction kernel: M = L^{-1} H L^{-H}, lower, strict upper zeroed.
// Also returns L (lower, strict upper zeroed) when L_out is non-null.
void sbo_reduce_batch(int n, int batch, const cdouble* H, const cdouble* S, cdouble* M,
                      cdouble* L_out, int* info, int nthreads) {
    const size_t mat = static_cast<size_t>(n) * n;
    parallel_pairs(batch, nthreads, [&](int b) {
        std::vector<cdouble> Lw(S + mat * b, S + mat * (b + 1));
        cdouble* Mb = M + mat * b;
        std::memcpy(Mb, H + mat * b, sizeof(cdouble) * mat);
        lapack_int r = LAPACKE_zpotrf(LAPACK_COL_MAJOR, 'L', n, Lw.data(), n);
        if (r == 0) r = LAPACKE_zhegst(LAPACK_COL_MAJOR, 1, 'L', n, Mb, n, Lw.data(), n);
        info[b] = static_cast<int>(r);
        zero_strict_upper(n, Mb);
        if (L_out) {
            zero_strict_upper(n, Lw.data());
            std::memcpy(L_out + mat * b, Lw.data(), sizeof(cdouble) * mat);
        }
    });
}

// Stage twin of reduce+eig: zpotrf -> zhegst -> zheev; W ascending, V eigenvectors of M.
void sbo_reduce_eig_batch(int n, int batch, const cdouble* H, const cdouble* S, double* W,
                          cdouble* V, int* info, int nthreads) {
    const size_t mat = static_cast<size_t>(n) * n;
    parallel_pairs(batch, nthreads, [&](int b) {
        std::vector<cdouble> Lw(S + mat * b, S + mat * (b + 1));
        cdouble* Vb = V + mat * b;
        std::memcpy(Vb, H + mat * b, sizeof(cdouble) * mat);
        lapack_int r = LAPACKE_zpotrf(LAPACK_COL_MAJOR, 'L', n, Lw.data(), n);
        if (r == 0) r = LAPACKE_zhegst(LAPACK_COL_MAJOR, 1, 'L', n, Vb, n, Lw.data(), n);
        if (r == 0) r = LAPACKE_zheev(LAPACK_COL_MAJOR, 'V', 'L', n, Vb, n, W + static_cast<size_t>(n) * b);
        info[b] = static_cast<int>(r);
    });
}

// Stage twin of the finish kernel: given L and M (lower read), W/V = heev(M), U = L^{-H} V.
void sbo_finish_batch(int n, int batch, const cdouble* L, const cdouble* M, double* W, cdouble* U,
                      int* info, int nthreads) {
    const size_t mat = static_cast<size_t>(n) * n;
    parallel_pairs(batch, nthreads, [&](int b) {
        cdouble* Ub = U + mat * b;
        std::memcpy(Ub, M + mat * b, sizeof(cdouble) * mat);
        lapack_int r = LAPACKE_zheev(LAPACK_COL_MAJOR, 'V', 'L', n, Ub, n, W + static_cast<size_t>(n) * b);
        if (r == 0) back_transform(n, L + mat * b, Ub);
        info[b] = static_cast<int>(r);
    });
}

// The same chain as sbo_finish_batch but from (H, S): potrf -> hegst -> heev -> trsm.
// This is the reference kernel's stage order (src/geneig_fixed.cu:455-464) in LAPACK.
void sbo_staged_full_batch(int n, int batch, const cdouble* H, const cdouble* S, double* W,
                           cdouble* U, int* info, int nthreads) {
    const size_t mat = static_cast<size_t>(n) * n;
    parallel_pairs(batch, nthreads, [&](int b) {
        std::vector<cdouble> Lw(S + mat * b, S + mat * (b + 1));
        cdouble* Ub = U + mat * b;
        std::memcpy(Ub, H + mat * b, sizeof(cdouble) * mat);
        lapack_int r = LAPACKE_zpotrf(LAPACK_COL_MAJOR, 'L', n, Lw.data(), n);
        if (r == 0) r = LAPACKE_zhegst(LAPACK_COL_MAJOR, 1, 'L', n, Ub, n, Lw.data(), n);
        if (r == 0) r = LAPACKE_zheev(LAPACK_COL_MAJOR, 'V', 'L', n, Ub, n, W + static_cast<size_t>(n) * b);
        if (r == 0) back_transform(n, Lw.data(), Ub);
        info[b] = static_cast<int>(r);
    });
}

// Standard Hermitian eigenvalues (jobz 'N'), used by the workload generators to
// place the smallest eigenvalue of B.
void sbo_heev_values_batch(int n, int batch, const cdouble* M, double* W, int* info, int nthreads) {
    const size_t mat = static_cast<size_t>(n) * n;
    parallel_pairs(batch, nthreads, [&](int b) {
        std::vector<cdouble> Mw(M + mat * b, M + mat * (b + 1));
        info[b] = static_cast<int>(
            LAPACKE_zheev(LAPACK_COL_MAJOR, 'N', 'L', n, Mw.data(), n, W + static_cast<size_t>(n) * b));
    });
}

int sbo_hardware_threads() { return static_cast<int>(std::thread::hardware_concurrency()); }

}  // extern "C"
