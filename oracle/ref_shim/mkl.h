/*
 * Minimal stand-in for the two Intel MKL CBLAS entry points the reference's CPU library
 * uses (cpp_src/mkl_linalg.cpp:7-22).  MKL is not installed here; these declarations let
 * oracle/build_ref.sh compile the reference sources unmodified.  The implementations are
 * plain loops in ref_shim.cpp (unconjugated complex dot, row-major complex gemv).
 * Test infrastructure only.
 */
#ifndef ORACLE_REF_SHIM_MKL_H
#define ORACLE_REF_SHIM_MKL_H
#ifdef __cplusplus
extern "C" {
#endif
typedef long long MKL_INT;
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
void cblas_cdotu_sub(const MKL_INT n, const void *x, const MKL_INT incx, const void *y,
                     const MKL_INT incy, void *dotu);
void cblas_cgemv(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE trans, const MKL_INT m,
                 const MKL_INT n, const void *alpha, const void *a, const MKL_INT lda,
                 const void *x, const MKL_INT incx, const void *beta, void *y,
                 const MKL_INT incy);
#ifdef __cplusplus
}
#endif
#endif
