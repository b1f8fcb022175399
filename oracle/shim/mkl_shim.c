/*
 * ORACLE — test infrastructure only. The two MKL extensions the reference
 * uses that OpenBLAS does not provide under MKL's calling convention.
 */
#include <stdlib.h>
#include <omp.h>
#include "mkl.h"

void *oracle_guard_tab[ORACLE_GUARD_SLOTS];

void cblas_dgemm_batch(CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE *transa, const CBLAS_TRANSPOSE *transb,
                       const MKL_INT *m, const MKL_INT *n, const MKL_INT *k, const double *alpha,
                       const double **a, const MKL_INT *lda, const double **b, const MKL_INT *ldb,
                       const double *beta, double **c, const MKL_INT *ldc,
                       MKL_INT group_count, const MKL_INT *group_size)
{
    int total = 0;
    for (int g = 0; g < group_count; g++) total += group_size[g];
    int *gid = (int *) malloc(sizeof(int) * (total > 0 ? total : 1));
    for (int g = 0, p = 0; g < group_count; g++)
        for (int i = 0; i < group_size[g]; i++) gid[p++] = g;
    /* Like MKL, spread independent products over the threads, one BLAS thread each. */
    int nt = scipy_openblas_get_num_threads();
    scipy_openblas_set_num_threads(1);
    #pragma omp parallel for schedule(dynamic)
    for (int p = 0; p < total; p++)
    {
        int g = gid[p];
        scipy_cblas_dgemm(layout, transa[g], transb[g], m[g], n[g], k[g], alpha[g],
                          a[p], lda[g], b[p], ldb[g], beta[g], c[p], ldc[g]);
    }
    scipy_openblas_set_num_threads(nt);
    free(gid);
}

void mkl_domatadd(char ordering, char transa, char transb, size_t rows, size_t cols,
                  double alpha, const double *A, size_t lda, double beta, const double *B, size_t ldb,
                  double *C, size_t ldc)
{
    (void) ordering;
    #pragma omp parallel for
    for (size_t i = 0; i < rows; i++)
        for (size_t j = 0; j < cols; j++)
        {
            double av = (transa == 'T' || transa == 't') ? A[j * lda + i] : A[i * lda + j];
            double bv = (transb == 'T' || transb == 't') ? B[j * ldb + i] : B[i * ldb + j];
            C[i * ldc + j] = alpha * av + beta * bv;
        }
}
