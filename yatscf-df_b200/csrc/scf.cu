// Per-iteration SCF pieces besides J/K: energy reduction, commutator DIIS with
// the reference's replacement policy (DIIS.c:12-123) kept entirely on the
// device, and the density from the orthogonalised Fock eigenvectors
// (build_density.c:37-69).
#include <cfloat>
#include <cmath>
#include <cstdio>

#include "tscf_internal.h"

namespace tscf {

__global__ void k_energy_reduce(const double *part, double *E)
{
    // fixed-order two-level sum: deterministic
    __shared__ double sh[ENERGY_BLOCKS];
    for (int i = threadIdx.x; i < ENERGY_BLOCKS; i += blockDim.x) sh[i] = part[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < ENERGY_BLOCKS; i++) s += sh[i];
        *E = s;
    }
}

void energy_reduce(const double *d_epart, double *d_E, cudaStream_t s)
{
    g_launches++;
    k_energy_reduce<<<1, 256, 0, s>>>(d_epart, d_E);
}

void xtfx(const double *d_X, const double *d_F, double *d_out, double *d_tmp, int n, cudaStream_t s)
{
    dgemm(true, false, n, n, n, 1.0, d_X, n, d_F, n, 0.0, d_tmp, n, s);    // X^T F
    dgemm(false, false, n, n, n, 1.0, d_tmp, n, d_X, n, 0.0, d_out, n, s);  // (X^T F) X
}

// ------------------------------------------------------------------ DIIS
__global__ void k_diis_init(DiisState *st)
{
    st->len = 0;
    st->bmax_id = 0;
    st->idx = 0;
    st->bmax = -DBL_MAX;
    for (int i = 0; i < MAXDIIS + 1; i++)
        for (int j = 0; j < MAXDIIS + 1; j++) st->B[i * (MAXDIIS + 1) + j] = (i == j) ? 0.0 : -1.0;
    for (int i = 0; i < MAXDIIS + 1; i++) st->coef[i] = 0.0;
}

void diis_init(DiisState *d_st, cudaStream_t s)
{
    g_launches++;
    k_diis_init<<<1, 1, 0, s>>>(d_st);
}

// DIIS.c:30-37: pick the slot to (re)place.
__global__ void k_diis_select(DiisState *st, int max_diis)
{
    if (st->len < max_diis) {
        st->idx = st->len;
        st->len++;
    } else {
        st->idx = st->bmax_id;
    }
}

__global__ void k_antisym(const double *A, double *out, int n)
{
    size_t idx = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t) n * n) return;
    int i = (int) (idx / n), j = (int) (idx % n);
    out[idx] = A[idx] - A[(size_t) j * n + i];
}

__global__ void k_copy_to_slot(const double *src, double *slots, const DiisState *st, size_t nn)
{
    size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nn) slots[(size_t) st->idx * nn + i] = src[i];
}

// dots[j] = <R_idx, R_j> for j < len; one block per j.
__global__ void k_diis_dots(const double *R, DiisState *st, size_t nn)
{
    const int j = blockIdx.x;
    if (j >= st->len) return;
    const double *a = R + (size_t) st->idx * nn, *b = R + (size_t) j * nn;
    double s = 0.0;
    for (size_t i = threadIdx.x; i < nn; i += blockDim.x) s = fma(a[i], b[i], s);
    __shared__ double sh[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffff, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffff, s, o);
        if (threadIdx.x == 0) st->dots[j] = s;
    }
}

// DIIS.c:76-110: update B, track the historically largest residual, and
// solve the (len+1) bordered system by Gaussian elimination with partial
// pivoting (first maximum, as LAPACK dgesv/idamax).
__global__ void k_diis_solve(DiisState *st)
{
    const int ld = MAXDIIS + 1;
    const int len = st->len, idx = st->idx;
    for (int i = 0; i < len; i++) {
        st->B[idx * ld + i] = st->dots[i];
        st->B[i * ld + idx] = st->dots[i];
    }
    for (int i = 0; i < len; i++)
        if (st->B[i * ld + i] > st->bmax) {
            st->bmax = st->B[i * ld + i];
            st->bmax_id = i;
        }
    const int n = len + 1;
    double a[(MAXDIIS + 1) * (MAXDIIS + 1)], b[MAXDIIS + 1];
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < n; j++) a[i * n + j] = st->B[i * ld + j];
        b[i] = (i == len) ? -1.0 : 0.0;
    }
    for (int k = 0; k < n; k++) {
        int p = k;
        double mx = fabs(a[k * n + k]);
        for (int i = k + 1; i < n; i++)
            if (fabs(a[i * n + k]) > mx) {
                mx = fabs(a[i * n + k]);
                p = i;
            }
        if (p != k) {
            for (int j = 0; j < n; j++) {
                double t = a[k * n + j]; a[k * n + j] = a[p * n + j]; a[p * n + j] = t;
            }
            double t = b[k]; b[k] = b[p]; b[p] = t;
        }
        double piv = a[k * n + k];
        if (piv == 0.0) continue;
        for (int i = k + 1; i < n; i++) {
            double f = a[i * n + k] / piv;
            a[i * n + k] = f;
            for (int j = k + 1; j < n; j++) a[i * n + j] -= f * a[k * n + j];
            b[i] -= f * b[k];
        }
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = b[i];
        for (int j = i + 1; j < n; j++) s -= a[i * n + j] * b[j];
        b[i] = s / a[i * n + i];
    }
    for (int i = 0; i < n; i++) st->coef[i] = b[i];
}

// F = sum_{i<len} coef_i F0_i (DIIS.c:112-122)
__global__ void k_diis_combine(const double *F0, const DiisState *st, double *F, size_t nn)
{
    size_t e = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nn) return;
    const int len = st->len;
    double s = 0.0;
    for (int i = 0; i < len; i++) s += st->coef[i] * F0[(size_t) i * nn + e];
    F[e] = s;
}

void diis_step(DiisState *st, int max_diis, const double *d_F, const double *d_D, const double *d_S,
               const double *d_X, double *d_Fout, double *d_F0, double *d_R, double *d_tmp, double *d_tmp2, int n,
               cudaStream_t s)
{
    const size_t nn = (size_t) n * n;
    const unsigned nb = (unsigned) ((nn + 255) / 256);
    g_launches += 7;
    k_diis_select<<<1, 1, 0, s>>>(st, max_diis);
    dgemm(false, false, n, n, n, 1.0, d_F, n, d_D, n, 0.0, d_tmp, n, s);     // F D
    dgemm(false, false, n, n, n, 1.0, d_tmp, n, d_S, n, 0.0, d_tmp2, n, s);  // F D S
    k_antisym<<<nb, 256, 0, s>>>(d_tmp2, d_tmp, n);                          // FDS - (FDS)^T
    dgemm(true, false, n, n, n, 1.0, d_X, n, d_tmp, n, 0.0, d_tmp2, n, s);   // X^T (.)
    dgemm(false, false, n, n, n, 1.0, d_tmp2, n, d_X, n, 0.0, d_tmp, n, s);  // (.) X
    k_copy_to_slot<<<nb, 256, 0, s>>>(d_tmp, d_R, st, nn);
    k_diis_dots<<<MAXDIIS, 1024, 0, s>>>(d_R, st, nn);
    xtfx(d_X, d_F, d_tmp2, d_tmp, n, s);                                     // X^T F X
    k_copy_to_slot<<<nb, 256, 0, s>>>(d_tmp2, d_F0, st, nn);
    k_diis_solve<<<1, 1, 0, s>>>(st);
    k_diis_combine<<<nb, 256, 0, s>>>(d_F0, st, d_Fout, nn);
}

// ------------------------------------------------------------------ density
void density_from_eig(const double *d_X, const double *d_V, double *d_Cocc, double *d_D, int n, int nocc,
                      cudaStream_t s)
{
    // Cocc = X * C0(:, 0:nocc) with C0's columns = rows of V
    dgemm(false, true, n, nocc, n, 1.0, d_X, n, d_V, n, 0.0, d_Cocc, nocc, s);
    // D = Cocc Cocc^T
    dgemm(false, true, n, n, nocc, 1.0, d_Cocc, nocc, d_Cocc, nocc, 0.0, d_D, n, s);
}

}  // namespace tscf
