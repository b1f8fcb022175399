// Per-iteration SCF pieces besides J/K: energy reduction, commutator DIIS with
// the reference's replacement policy (DIIS.c:12-123) kept entirely on the
// device, and the density from the orthogonalised Fock eigenvectors
// (build_density.c:37-69).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>

#include "batch.h"
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

// DIIS.c:75-81: store the new residual in slot idx and form
// dots[j] = <R_idx, R_j> for j < len, over the whole grid: block b takes the
// elements b * 256 + t + k * 256 * gridDim, reads the new residual once for
// every j and writes its sums to part[b][j]; k_diis_dots_sum adds the parts in
// block order, so the dots do not depend on timing.
constexpr int DOT_THREADS = 256;

__global__ void __launch_bounds__(DOT_THREADS) k_diis_slot_dots(const double *src, double *R, DiisState *st, size_t nn)
{
    const int len = st->len, idx = st->idx;
    double *slot = R + (size_t) idx * nn;
    double s[MAXDIIS];
#pragma unroll
    for (int j = 0; j < MAXDIIS; j++) s[j] = 0.0;
    const size_t step = (size_t) gridDim.x * DOT_THREADS;
    for (size_t i = (size_t) blockIdx.x * DOT_THREADS + threadIdx.x; i < nn; i += step) {
        const double a = src[i];
        slot[i] = a;
#pragma unroll
        for (int j = 0; j < MAXDIIS; j++)
            if (j < len) s[j] = fma(a, j == idx ? a : R[(size_t) j * nn + i], s[j]);
    }
    __shared__ double sh[MAXDIIS][DOT_THREADS / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < MAXDIIS; j++) {
        double v = s[j];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffff, v, o);
        if (lane == 0) sh[j][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < MAXDIIS) {
        double v = 0.0;
        for (int w = 0; w < DOT_THREADS / 32; w++) v += sh[threadIdx.x][w];
        st->part[blockIdx.x * MAXDIIS + threadIdx.x] = v;
    }
}

// One warp per j: dots[j] = sum over the blocks' parts, in a fixed order.
__global__ void __launch_bounds__(32 * MAXDIIS) k_diis_dots_sum(DiisState *st, int nblocks)
{
    const int j = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (j >= st->len) return;   // uniform per warp
    double v = 0.0;
    for (int b = lane; b < nblocks; b += 32) v += st->part[b * MAXDIIS + j];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffff, v, o);
    if (lane == 0) st->dots[j] = v;
}

// The residual's slot and dots: two launches.
void diis_slot_dots(const double *src, double *R, DiisState *st, size_t nn, cudaStream_t s)
{
    const size_t need = (nn + DOT_THREADS - 1) / DOT_THREADS;
    const int nblk = (int) std::max<size_t>(1, std::min<size_t>(need, std::min(2 * num_sms(), DIIS_DOT_BLOCKS)));
    k_diis_slot_dots<<<nblk, DOT_THREADS, 0, s>>>(src, R, st, nn);
    k_diis_dots_sum<<<1, 32 * MAXDIIS, 0, s>>>(st, nblk);
}

// DIIS.c:76-110: update B, track the historically largest residual, and
// solve the (len+1) bordered system by Gaussian elimination with partial
// pivoting (first maximum, as LAPACK dgesv/idamax).
__device__ void diis_solve_body(DiisState *st)
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

// The same update and elimination with one warp: lane i holds row i of the
// bordered system (n <= MAXDIIS + 1 <= 32), the pivot search is a first-maximum
// reduction over the lanes, and each lane eliminates its own row with the
// pivot row broadcast by shuffles; the arithmetic of every element is that
// of diis_solve_body.
__global__ void __launch_bounds__(32) k_diis_solve(DiisState *st)
{
    constexpr int ld = MAXDIIS + 1;
    const int lane = threadIdx.x;
    const int len = st->len, idx = st->idx, n = len + 1;
    if (lane < len) {
        st->B[idx * ld + lane] = st->dots[lane];
        st->B[lane * ld + idx] = st->dots[lane];
    }
    __syncwarp();
    if (lane == 0)
        for (int i = 0; i < len; i++)
            if (st->B[i * ld + i] > st->bmax) {
                st->bmax = st->B[i * ld + i];
                st->bmax_id = i;
            }
    double a[ld], b;
#pragma unroll
    for (int j = 0; j < ld; j++) a[j] = (lane < n && j < n) ? st->B[lane * ld + j] : 0.0;
    b = (lane == len) ? -1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < ld; k++) {
        if (k >= n) break;
        // first maximum of |a(i, k)| over rows i >= k
        double mx = (lane >= k && lane < n) ? fabs(a[k]) : -1.0;
        int p = lane;
        for (int o = 16; o > 0; o >>= 1) {
            const double m2 = __shfl_xor_sync(0xffffffff, mx, o);
            const int p2 = __shfl_xor_sync(0xffffffff, p, o);
            if (m2 > mx || (m2 == mx && p2 < p)) {
                mx = m2;
                p = p2;
            }
        }
        p = __shfl_sync(0xffffffff, p, 0);   // one pivot for the whole warp (even with NaN entries)
        if (p != k) {   // swap rows k and p
#pragma unroll
            for (int j = 0; j < ld; j++) {
                const double vk = __shfl_sync(0xffffffff, a[j], k), vp = __shfl_sync(0xffffffff, a[j], p);
                if (lane == k) a[j] = vp;
                if (lane == p) a[j] = vk;
            }
            const double bk = __shfl_sync(0xffffffff, b, k), bp = __shfl_sync(0xffffffff, b, p);
            if (lane == k) b = bp;
            if (lane == p) b = bk;
        }
        double prow[ld];
#pragma unroll
        for (int j = 0; j < ld; j++) prow[j] = __shfl_sync(0xffffffff, a[j], k);
        const double bkk = __shfl_sync(0xffffffff, b, k);
        const double piv = prow[k];
        if (piv == 0.0) continue;
        if (lane > k && lane < n) {
            const double f = a[k] / piv;
            a[k] = f;
#pragma unroll
            for (int j = 0; j < ld; j++)
                if (j > k && j < n) a[j] -= f * prow[j];
            b -= f * bkk;
        }
    }
    // back substitution from the last row; each solved entry is broadcast
    double sol[ld];
#pragma unroll
    for (int j = 0; j < ld; j++) sol[j] = 0.0;
    for (int i = n - 1; i >= 0; i--) {
        double v = 0.0;
        if (lane == i) {
            double s2 = b;
#pragma unroll
            for (int j = 0; j < ld; j++)
                if (j > i && j < n) s2 -= a[j] * sol[j];
            v = s2 / a[i];
        }
        v = __shfl_sync(0xffffffff, v, i);
#pragma unroll
        for (int j = 0; j < ld; j++)
            if (j == i) sol[j] = v;
    }
    if (lane < n) {
#pragma unroll
        for (int j = 0; j < ld; j++)
            if (j == lane) st->coef[lane] = sol[j];
    }
}

// one thread per molecule of a batch
__global__ void k_diis_solve_batched(const MolDev *mols, const int *active, int nmol)
{
    const int mol = blockIdx.x * blockDim.x + threadIdx.x;
    if (mol < nmol && active[mol]) diis_solve_body(mols[mol].diis);
}

void diis_solve_batched(const MolDev *d_mols, const int *d_active, int nmol, cudaStream_t s)
{
    g_launches++;
    k_diis_solve_batched<<<(nmol + 63) / 64, 64, 0, s>>>(d_mols, d_active, nmol);
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
    diis_slot_dots(d_tmp, d_R, st, nn, s);
    xtfx(d_X, d_F, d_tmp2, d_tmp, n, s);                                     // X^T F X
    k_copy_to_slot<<<nb, 256, 0, s>>>(d_tmp2, d_F0, st, nn);
    k_diis_solve<<<1, 32, 0, s>>>(st);
    k_diis_combine<<<nb, 256, 0, s>>>(d_F0, st, d_Fout, nn);
}

// [B | -A] from [A | B] (both n x 2o, row-major)
__global__ void k_swap_neg(const double *AB, double *BA, int n, int o)
{
    const size_t idx = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    const int o2 = 2 * o;
    if (idx >= (size_t) n * o2) return;
    const size_t i = idx / o2;
    const int c = (int) (idx % o2);
    BA[idx] = c < o ? AB[i * o2 + o + c] : -AB[i * o2 + c - o];
}

// The same step when D = Cocc Cocc^T (the engine's own density builds):
// FDS = P Q^T with P = F Cocc, Q = S Cocc, so the commutator
// X^T (FDS - (FDS)^T) X = A B^T - B A^T, A = X^T P, B = X^T Q: 12 n^2 n_occ
// flops instead of the four n^3 products of FD, FDS, X^T (.) and (.) X.
void diis_step_cocc(DiisState *st, int max_diis, const double *d_F, const double *d_Cocc, int o, const double *d_S,
                    const double *d_X, double *d_Fout, double *d_F0, double *d_R, double *d_tmp, double *d_tmp2, int n,
                    cudaStream_t s)
{
    const size_t nn = (size_t) n * n;
    const unsigned nb = (unsigned) ((nn + 255) / 256);
    const int o2 = 2 * o;
    g_launches += 7;
    k_diis_select<<<1, 1, 0, s>>>(st, max_diis);
    dgemm(false, false, n, o, n, 1.0, d_F, n, d_Cocc, o, 0.0, d_tmp, o2, s);       // P = F C
    dgemm(false, false, n, o, n, 1.0, d_S, n, d_Cocc, o, 0.0, d_tmp + o, o2, s);   // Q = S C
    dgemm(true, false, n, o2, n, 1.0, d_X, n, d_tmp, o2, 0.0, d_tmp2, o2, s);     // [A | B] = X^T [P | Q]
    k_swap_neg<<<(unsigned) (((size_t) n * o2 + 255) / 256), 256, 0, s>>>(d_tmp2, d_tmp, n, o);   // [B | -A]
    dgemm(false, true, n, n, o2, 1.0, d_tmp2, o2, d_tmp, o2, 0.0, d_Fout, n, s);  // A B^T - B A^T
    diis_slot_dots(d_Fout, d_R, st, nn, s);
    xtfx(d_X, d_F, d_tmp2, d_tmp, n, s);                                           // X^T F X
    k_copy_to_slot<<<nb, 256, 0, s>>>(d_tmp2, d_F0, st, nn);
    k_diis_solve<<<1, 32, 0, s>>>(st);
    k_diis_combine<<<nb, 256, 0, s>>>(d_F0, st, d_Fout, nn);
}

// ------------------------------------------------------------------ occupied-subspace refinement
// Between full eigensolves the occupied subspace of F' is refined from the
// previous one: U (o x n, orthonormal rows in the orthogonal basis) moves along
// the residual R = (I - U^T U) F' U^T, preconditioned with the last full
// eigenbasis (virtual rows Vv, eigenvalues wv):
//   U_i += sum_a Vv_a (Vv_a . R_i) / (eps_i - wv_a),   eps_i = (U F' U^T)_ii,
// then Loewdin re-orthonormalisation. The fixed point is the invariant
// subspace continuously connected to the previous occupied one, i.e. the
// aufbau occupied space of build_density.c:37-69 as long as no level crosses
// the gap.
__global__ void k_sub(const double *A, double *R, size_t n)   // R = A - R
{
    size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) R[i] = A[i] - R[i];
}

__global__ void k_precond(double *Cv, const double *UA, const double *wv, int v, int o)
{
    size_t idx = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t) v * o) return;
    int a = (int) (idx / o), i = (int) (idx % o);
    double d = UA[(size_t) i * o + i] - wv[a];
    Cv[idx] = (fabs(d) > 1e-6) ? Cv[idx] / d : 0.0;
}

__global__ void k_add_transposed(double *U, const double *DT, int o, int n)   // U (o x n) += DT^T (DT: n x o)
{
    size_t idx = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t) o * n) return;
    int i = (int) (idx / n), k = (int) (idx % n);
    U[idx] += DT[(size_t) k * o + i];
}

__global__ void k_absmax(const double *x, size_t n, double *out)
{
    __shared__ double sh[32];
    double m = 0.0;
    for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
        m = fmax(m, fabs(x[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffff, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffff, m, o));
        if (threadIdx.x == 0) {
            unsigned long long *p = (unsigned long long *) out;
            atomicMax(p, __double_as_longlong(m));   // m >= 0: integer order = float order
        }
    }
}

__global__ void k_ns_step(double *T, int n)   // T <- 1.5 I - 0.5 T
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * n) return;
    T[idx] = (idx / n == idx % n ? 1.5 : 0.0) - 0.5 * T[idx];
}

__global__ void k_eye(double *A, int n)
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < n * n) A[idx] = (idx / n == idx % n) ? 1.0 : 0.0;
}

// M^-1/2 of an SPD matrix close to I (coupled Newton-Schulz), result in Z.
static void inv_sqrt_ns(const double *M, double *Y, double *Z, double *T, double *W, int o, int iters, cudaStream_t s)
{
    const unsigned nb = (unsigned) ((o * o + 255) / 256);
    cudaMemcpyAsync(Y, M, sizeof(double) * o * o, cudaMemcpyDeviceToDevice, s);
    k_eye<<<nb, 256, 0, s>>>(Z, o);
    g_launches++;
    for (int it = 0; it < iters; it++) {
        dgemm(false, false, o, o, o, 1.0, Z, o, Y, o, 0.0, T, o, s);        // T = Z Y
        k_ns_step<<<nb, 256, 0, s>>>(T, o);                                  // T = 1.5 I - 0.5 Z Y
        dgemm(false, false, o, o, o, 1.0, Y, o, T, o, 0.0, W, o, s);        // Y <- Y T
        cudaMemcpyAsync(Y, W, sizeof(double) * o * o, cudaMemcpyDeviceToDevice, s);
        dgemm(false, false, o, o, o, 1.0, T, o, Z, o, 0.0, W, o, s);        // Z <- T Z
        cudaMemcpyAsync(Z, W, sizeof(double) * o * o, cudaMemcpyDeviceToDevice, s);
        g_launches++;
    }
}

// res = max|R|, R = (I - U^T U) F' U^T; UA = U F' U^T
static void refine_residual(const double *d_Fp, const double *d_U, int n, int o, SubspaceWork &w, cudaStream_t s)
{
    dgemm(false, true, n, o, n, 1.0, d_Fp, n, d_U, n, 0.0, w.A, o, s);          // A = F' U^T (n x o)
    dgemm(false, false, o, o, n, 1.0, d_U, n, w.A, o, 0.0, w.UA, o, s);        // UA = U F' U^T
    dgemm(true, false, n, o, o, 1.0, d_U, n, w.UA, o, 0.0, w.R, o, s);         // R = U^T UA
    k_sub<<<(unsigned) (((size_t) n * o + 255) / 256), 256, 0, s>>>(w.A, w.R, (size_t) n * o);   // R = A - R
    cudaMemsetAsync(w.res, 0, sizeof(double), s);
    k_absmax<<<num_sms(), 256, 0, s>>>(w.R, (size_t) n * o, w.res);
    g_launches += 2;
}

// one preconditioned step on U followed by Loewdin re-orthonormalisation
static void refine_update(const double *d_Vstale, const double *d_wstale, double *d_U, int n, int o, SubspaceWork &w,
                          cudaStream_t s)
{
    const int v = n - o;
    const double *Vv = d_Vstale + (size_t) o * n;
    const double *wv = d_wstale + o;
    dgemm(false, false, v, o, n, 1.0, Vv, n, w.R, o, 0.0, w.Cv, o, s);        // Cv = Vv R
    k_precond<<<(unsigned) (((size_t) v * o + 255) / 256), 256, 0, s>>>(w.Cv, w.UA, wv, v, o);
    dgemm(true, false, n, o, v, 1.0, Vv, n, w.Cv, o, 0.0, w.A, o, s);         // A = Vv^T Cv (n x o)
    k_add_transposed<<<(unsigned) (((size_t) o * n + 255) / 256), 256, 0, s>>>(d_U, w.A, o, n);
    dgemm(false, true, o, o, n, 1.0, d_U, n, d_U, n, 0.0, w.M, o, s);         // M = U U^T
    inv_sqrt_ns(w.M, w.Y, w.Z, w.T, w.W, o, 5, s);                              // Z = M^-1/2
    dgemm(false, false, o, n, o, 1.0, w.Z, o, d_U, n, 0.0, w.A, n, s);        // U = Z U
    cudaMemcpyAsync(d_U, w.A, sizeof(double) * (size_t) o * n, cudaMemcpyDeviceToDevice, s);
    g_launches += 2;
}

// Stop rule shared by the host loop and the graph's device-side loop: stop when
// converged, when the first residual shows F' far from the last subspace, or
// when the observed contraction cannot reach tol within the steps left.
__host__ __device__ inline bool refine_continue(double res, double prev, int step, int max_steps, double tol)
{
    if (res < tol || step >= max_steps) return false;
    if (step == 0) return res <= 5e-2;
    return res * pow(res / prev, max_steps - step) <= tol;
}

int subspace_refine(const double *d_Fp, const double *d_Vstale, const double *d_wstale, double *d_U, int n, int o,
                    SubspaceWork &w, double tol, int max_steps, int *steps_out, double *res_out, cudaStream_t s)
{
    double res = 1e300, prev = 1e300;
    int step = 0;
    for (;; step++) {
        refine_residual(d_Fp, d_U, n, o, w, s);
        cudaMemcpyAsync(&res, w.res, sizeof(double), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) return ERR_CUDA;
        if (!refine_continue(res, prev, step, max_steps, tol)) break;
        prev = res;
        refine_update(d_Vstale, d_wstale, d_U, n, o, w, s);
    }
    *steps_out = step;
    *res_out = res;
    return OK;
}

// Device-side loop control for the captured iteration: reads the residual the
// preceding kernels produced and sets the WHILE node's condition.
__global__ void k_refine_decide(RefineCtl *c, const double *res, cudaGraphConditionalHandle h, int first)
{
    const double r = *res;
    if (first) {
        c->step = 0;
        c->prev = 1e300;
    } else {
        c->step++;
    }
    c->res = r;
    c->converged = r < c->tol;
    const bool cont = refine_continue(r, c->prev, c->step, c->max_steps, c->tol);
    c->prev = r;
    cudaGraphSetConditional(h, cont ? 1u : 0u);
}

int subspace_refine_capture(const double *d_Fp, const double *d_Vstale, const double *d_wstale, double *d_U, int n,
                            int o, SubspaceWork &w, RefineCtl *d_ctl, cudaStream_t s, cudaStream_t s_body,
                            long long *body_launches)
{
    refine_residual(d_Fp, d_U, n, o, w, s);
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    if (cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &ndeps) != cudaSuccess || st != cudaStreamCaptureStatusActive)
        return ERR_CUDA;
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) return ERR_CUDA;
    k_refine_decide<<<1, 1, 0, s>>>(d_ctl, w.res, h, 1);
    g_launches++;
    if (cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &ndeps) != cudaSuccess) return ERR_CUDA;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, g, deps, ndeps, &cp) != cudaSuccess) return ERR_CUDA;
    if (cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
        return ERR_CUDA;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(s_body, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
        return ERR_CUDA;
    const long long l0 = g_launches;
    refine_update(d_Vstale, d_wstale, d_U, n, o, w, s_body);
    refine_residual(d_Fp, d_U, n, o, w, s_body);
    k_refine_decide<<<1, 1, 0, s_body>>>(d_ctl, w.res, h, 0);
    g_launches++;
    *body_launches = g_launches - l0;
    g_launches = l0;
    cudaGraph_t out = nullptr;
    if (cudaStreamEndCapture(s_body, &out) != cudaSuccess) return ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? OK : ERR_CUDA;
}

// Cocc = X U^T (U: occupied rows in the orthogonal basis), D = Cocc Cocc^T
void density_from_rows(const double *d_X, const double *d_U, double *d_Cocc, double *d_D, int n, int nocc,
                       cudaStream_t s)
{
    dgemm(false, true, n, nocc, n, 1.0, d_X, n, d_U, n, 0.0, d_Cocc, nocc, s);
    dgemm(false, true, n, n, nocc, 1.0, d_Cocc, nocc, d_Cocc, nocc, 0.0, d_D, n, s);
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
