/* Minimal LAPACKE declarations for building the reference's CPU oracle and the
 * C++ restatement against the OpenBLAS shipped in this image (which exports the
 * LAPACKE_* symbols but installs no lapacke.h).  Only the entry points the
 * reference's tests call are declared: tests/lapack_reference.cpp:186-194
 * (zhegvd), tests/test_full_batched_n54.cpp:244-251 (zhegv),
 * tests/test_reduce_eig_n54.cpp:143-155 (zpotrf, zhegst, zheev). */
#ifndef SBG_LAPACKE_SHIM_H
#define SBG_LAPACKE_SHIM_H

#ifdef __cplusplus
#include <complex>
typedef std::complex<double> lapack_complex_double;
extern "C" {
#else
#include <complex.h>
typedef double _Complex lapack_complex_double;
#endif

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

lapack_int LAPACKE_zhegv(int layout, lapack_int itype, char jobz, char uplo, lapack_int n,
                         lapack_complex_double* a, lapack_int lda,
                         lapack_complex_double* b, lapack_int ldb, double* w);
lapack_int LAPACKE_zhegvd(int layout, lapack_int itype, char jobz, char uplo, lapack_int n,
                          lapack_complex_double* a, lapack_int lda,
                          lapack_complex_double* b, lapack_int ldb, double* w);
lapack_int LAPACKE_zpotrf(int layout, char uplo, lapack_int n,
                          lapack_complex_double* a, lapack_int lda);
lapack_int LAPACKE_zhegst(int layout, lapack_int itype, char uplo, lapack_int n,
                          lapack_complex_double* a, lapack_int lda,
                          const lapack_complex_double* b, lapack_int ldb);
lapack_int LAPACKE_zheev(int layout, char jobz, char uplo, lapack_int n,
                         lapack_complex_double* a, lapack_int lda, double* w);

#ifdef __cplusplus
}
#endif
#endif
