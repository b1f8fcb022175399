/*
 * ORACLE — test infrastructure only.
 *
 * Stand-in for Intel MKL's <mkl.h> so the reference's CPU sources compile with
 * gcc. It declares exactly the CBLAS/LAPACKE entry points the reference calls
 * (DIIS.c, TinySCF.c, build_DF_tensor.c, build_Fock.c, build_density.c) and
 * routes them to the OpenBLAS build that ships with scipy (exported with a
 * "scipy_" prefix). mkl_domatadd and cblas_dgemm_batch (MKL's group API) are
 * implemented in mkl_shim.c.
 */
#ifndef ORACLE_MKL_SHIM_H
#define ORACLE_MKL_SHIM_H

#include <stddef.h>
#include "guard_malloc.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef int MKL_INT;
typedef int lapack_int;

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef CBLAS_LAYOUT CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

void   scipy_cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                         int m, int n, int k, double alpha, const double *a, int lda,
                         const double *b, int ldb, double beta, double *c, int ldc);
double scipy_cblas_ddot(int n, const double *x, int incx, const double *y, int incy);
void   scipy_cblas_daxpy(int n, double alpha, const double *x, int incx, double *y, int incy);
lapack_int scipy_LAPACKE_dsyev(int layout, char jobz, char uplo, lapack_int n, double *a,
                               lapack_int lda, double *w);
lapack_int scipy_LAPACKE_dpstrf(int layout, char uplo, lapack_int n, double *a, lapack_int lda,
                                lapack_int *piv, lapack_int *rank, double tol);
lapack_int scipy_LAPACKE_dgesv(int layout, lapack_int n, lapack_int nrhs, double *a, lapack_int lda,
                               lapack_int *ipiv, double *b, lapack_int ldb);
void scipy_openblas_set_num_threads(int n);
int  scipy_openblas_get_num_threads(void);

#define cblas_dgemm     scipy_cblas_dgemm
#define cblas_ddot      scipy_cblas_ddot
#define cblas_daxpy     scipy_cblas_daxpy
#define LAPACKE_dsyev   scipy_LAPACKE_dsyev
#define LAPACKE_dpstrf  scipy_LAPACKE_dpstrf
#define LAPACKE_dgesv   scipy_LAPACKE_dgesv

/* MKL group-batched GEMM: group g has group_size[g] products sharing the
 * g-th entry of every parameter array; pointer arrays run over all products. */
void cblas_dgemm_batch(CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE *transa, const CBLAS_TRANSPOSE *transb,
                       const MKL_INT *m, const MKL_INT *n, const MKL_INT *k, const double *alpha,
                       const double **a, const MKL_INT *lda, const double **b, const MKL_INT *ldb,
                       const double *beta, double **c, const MKL_INT *ldc,
                       MKL_INT group_count, const MKL_INT *group_size);

/* C = alpha * op(A) + beta * op(B), row-major ('R') only. */
void mkl_domatadd(char ordering, char transa, char transb, size_t rows, size_t cols,
                  double alpha, const double *A, size_t lda, double beta, const double *B, size_t ldb,
                  double *C, size_t ldc);

#ifdef __cplusplus
}
#endif

#endif
