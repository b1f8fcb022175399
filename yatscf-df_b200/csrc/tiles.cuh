// Tile bodies shared by the single-molecule kernels and the batched
// (many-molecule) kernels: the same arithmetic in the same order, so a batched
// SCF reproduces the single-molecule one.
#pragma once
#include "tscf_internal.h"

namespace tscf {

// ---- FP64 GEMM tile: BM x BN outputs per 256 threads (a 16 x 16 thread grid,
// BM/16 x BN/16 outputs per thread), K step 16. op(A) is m x k, op(B) is
// k x n, row-major; C = alpha op(A) op(B) + beta C. Every tile shape sums
// over k in the same order, so all shapes give identical results.
constexpr int GB_M = 64, GB_N = 64, GB_K = 16;

template <bool TA, bool TB, int BM = 64, int BN = 64>
__device__ __forceinline__ void dgemm_tile(int m, int n, int k, double alpha, const double *__restrict__ A, int lda,
                                           const double *__restrict__ B, int ldb, double beta, double *C, int ldc,
                                           int m0, int n0)
{
    constexpr int TM = BM / 16, TN = BN / 16;
    __shared__ double As[GB_K][BM + 1];
    __shared__ double Bs[GB_K][BN + 1];
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    double acc[TM][TN] = {};
    for (int k0 = 0; k0 < k; k0 += GB_K) {
#pragma unroll
        for (int r = 0; r < BM / 16; r++) {
            const int l = tid + 256 * r;
            int row, kk;
            if (!TA) { row = l / GB_K; kk = l % GB_K; } else { kk = l / BM; row = l % BM; }
            const int gi = m0 + row, gk = k0 + kk;
            double v = 0.0;
            if (gi < m && gk < k) v = TA ? A[(size_t) gk * lda + gi] : A[(size_t) gi * lda + gk];
            As[kk][row] = v;
        }
#pragma unroll
        for (int r = 0; r < BN / 16; r++) {
            const int l = tid + 256 * r;
            int col, kk;
            if (!TB) { kk = l / BN; col = l % BN; } else { col = l / GB_K; kk = l % GB_K; }
            const int gj = n0 + col, gk = k0 + kk;
            double w = 0.0;
            if (gj < n && gk < k) w = TB ? B[(size_t) gj * ldb + gk] : B[(size_t) gk * ldb + gj];
            Bs[kk][col] = w;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GB_K; kk++) {
            double a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < TN; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int j = 0; j < TN; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const int gi = m0 + ty + 16 * i;
        if (gi >= m) continue;
#pragma unroll
        for (int j = 0; j < TN; j++) {
            const int gj = n0 + tx + 16 * j;
            if (gj >= n) continue;
            double *c = C + (size_t) gi * ldc + gj;
            *c = (beta == 0.0) ? alpha * acc[i][j] : alpha * acc[i][j] + beta * *c;
        }
    }
}

// FP64 tensor-core MMA: D(8x8) += A(8x4, row-major) B(4x8, column-major); lane
// l holds A(l/4, l%4), B(l%4, l/4) and D(l/4, 2(l%4)..2(l%4)+1).
__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// ---- FP64 GEMM tile on the FP64 tensor cores: 128 x 128 outputs per 256
// threads, 8 warps of 64 x 32 (8 x 4 DMMA tiles). Same operand conventions as
// dgemm_tile.
template <bool TA, bool TB>
__device__ __forceinline__ void dgemm_tile_dmma(int m, int n, int k, double alpha, const double *__restrict__ A,
                                                int lda, const double *__restrict__ B, int ldb, double beta, double *C,
                                                int ldc, int m0, int n0)
{
    constexpr int BT = 128;
    __shared__ double As[BT][GB_K + 4];   // row-major in M / N: conflict-free fragment reads
    __shared__ double Bs[BT][GB_K + 4];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;
    const int fr = lane >> 2, fc = lane & 3;
    double acc[8][4][2];
#pragma unroll
    for (int x = 0; x < 8; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y][0] = acc[x][y][1] = 0.0;
    // the next K step's operands are fetched into registers while the DMMAs
    // of the current one run
    double pa[BT / 16], pb[BT / 16];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int r = 0; r < BT / 16; r++) {
            const int l = tid + 256 * r;
            int row, kk;
            if (!TA) { row = l / GB_K; kk = l % GB_K; } else { kk = l / BT; row = l % BT; }
            const int gi = m0 + row, gk = k0 + kk;
            pa[r] = (gi < m && gk < k) ? (TA ? A[(size_t) gk * lda + gi] : A[(size_t) gi * lda + gk]) : 0.0;
            int col;
            if (!TB) { kk = l / BT; col = l % BT; } else { col = l / GB_K; kk = l % GB_K; }
            const int gj = n0 + col, gk2 = k0 + kk;
            pb[r] = (gj < n && gk2 < k) ? (TB ? B[(size_t) gj * ldb + gk2] : B[(size_t) gk2 * ldb + gj]) : 0.0;
        }
    };
    if (k > 0) fetch(0);
    for (int k0 = 0; k0 < k; k0 += GB_K) {
#pragma unroll
        for (int r = 0; r < BT / 16; r++) {
            const int l = tid + 256 * r;
            int row, kk;
            if (!TA) { row = l / GB_K; kk = l % GB_K; } else { kk = l / BT; row = l % BT; }
            As[row][kk] = pa[r];
            int col;
            if (!TB) { kk = l / BT; col = l % BT; } else { col = l / GB_K; kk = l % GB_K; }
            Bs[col][kk] = pb[r];
        }
        __syncthreads();
        if (k0 + GB_K < k) fetch(k0 + GB_K);
#pragma unroll
        for (int k4 = 0; k4 < GB_K; k4 += 4) {
            double a[8], b[4];
#pragma unroll
            for (int x = 0; x < 8; x++) a[x] = As[wm + 8 * x + fr][k4 + fc];
#pragma unroll
            for (int y = 0; y < 4; y++) b[y] = Bs[wn + 8 * y + fr][k4 + fc];
#pragma unroll
            for (int x = 0; x < 8; x++)
#pragma unroll
                for (int y = 0; y < 4; y++) dmma_8x8x4(acc[x][y][0], acc[x][y][1], a[x], b[y]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int x = 0; x < 8; x++) {
        const int gi = m0 + wm + 8 * x + fr;
        if (gi >= m) continue;
#pragma unroll
        for (int y = 0; y < 4; y++) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int gj = n0 + wn + 8 * y + 2 * fc + h;
                if (gj >= n) continue;
                double *c = C + (size_t) gi * ldc + gj;
                *c = (beta == 0.0) ? alpha * acc[x][y][h] : alpha * acc[x][y][h] + beta * *c;
            }
        }
    }
}

// ---- FP64 GEMM tile on the FP64 tensor cores, 64 x 64 outputs per 128
// threads (4 warps of 32 x 32 = 4 x 4 DMMA tiles): four times the CTAs of the
// 128 x 128 tile for the nbf-sized matrices of DIIS and the density.
template <bool TA, bool TB>
__device__ __forceinline__ void dgemm_tile_dmma64(int m, int n, int k, double alpha, const double *__restrict__ A,
                                                  int lda, const double *__restrict__ B, int ldb, double beta,
                                                  double *C, int ldc, int m0, int n0)
{
    constexpr int BT = 64;
    __shared__ double As[BT][GB_K + 4];
    __shared__ double Bs[BT][GB_K + 4];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int fr = lane >> 2, fc = lane & 3;
    double acc[4][4][2];
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y][0] = acc[x][y][1] = 0.0;
    for (int k0 = 0; k0 < k; k0 += GB_K) {
#pragma unroll
        for (int r = 0; r < BT * GB_K / 128; r++) {
            const int l = tid + 128 * r;
            int row, kk;
            if (!TA) { row = l / GB_K; kk = l % GB_K; } else { kk = l / BT; row = l % BT; }
            const int gi = m0 + row, gk = k0 + kk;
            As[row][kk] = (gi < m && gk < k) ? (TA ? A[(size_t) gk * lda + gi] : A[(size_t) gi * lda + gk]) : 0.0;
            int col;
            if (!TB) { kk = l / BT; col = l % BT; } else { col = l / GB_K; kk = l % GB_K; }
            const int gj = n0 + col, gk2 = k0 + kk;
            Bs[col][kk] = (gj < n && gk2 < k) ? (TB ? B[(size_t) gj * ldb + gk2] : B[(size_t) gk2 * ldb + gj]) : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int k4 = 0; k4 < GB_K; k4 += 4) {
            double a[4], b[4];
#pragma unroll
            for (int x = 0; x < 4; x++) a[x] = As[wm + 8 * x + fr][k4 + fc];
#pragma unroll
            for (int y = 0; y < 4; y++) b[y] = Bs[wn + 8 * y + fr][k4 + fc];
#pragma unroll
            for (int x = 0; x < 4; x++)
#pragma unroll
                for (int y = 0; y < 4; y++) dmma_8x8x4(acc[x][y][0], acc[x][y][1], a[x], b[y]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int x = 0; x < 4; x++) {
        const int gi = m0 + wm + 8 * x + fr;
        if (gi >= m) continue;
#pragma unroll
        for (int y = 0; y < 4; y++) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int gj = n0 + wn + 8 * y + 2 * fc + h;
                if (gj >= n) continue;
                double *c = C + (size_t) gi * ldc + gj;
                *c = (beta == 0.0) ? alpha * acc[x][y][h] : alpha * acc[x][y][h] + beta * *c;
            }
        }
    }
}

// ---- K half-transform tile: T[i][s0:s0+64][p0:p0+64] = sum_{r in CSR row i} C[j_r][s] B[u_r][p]
constexpr int KT_M = 64, KT_N = 64, KT_K = 16;

__device__ __forceinline__ void half_tile(const double *__restrict__ B, const double *__restrict__ C,
                                          const int *__restrict__ csr_j, const int *__restrict__ csr_u,
                                          const int *__restrict__ displs, int nocc, int naux, double *__restrict__ T,
                                          int i, int s0, int p0)
{
    __shared__ double As[KT_K][KT_M + 1];
    __shared__ double Bs[KT_K][KT_N + 1];
    __shared__ int rj[KT_K], ru[KT_K];
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    const int r_beg = displs[i], r_end = displs[i + 1];
    double acc[4][4] = {};
    for (int r0 = r_beg; r0 < r_end; r0 += KT_K) {
        if (tid < KT_K) {
            int r = r0 + tid;
            rj[tid] = (r < r_end) ? csr_j[r] : -1;
            ru[tid] = (r < r_end) ? csr_u[r] : -1;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; q++) {
            int l = tid + 256 * q;
            int kk = l / KT_M, c = l % KT_M;
            int j = rj[kk], u = ru[kk];
            int sg = s0 + c, pg = p0 + c;
            As[kk][c] = (j >= 0 && sg < nocc) ? C[(size_t) j * nocc + sg] : 0.0;
            Bs[kk][c] = (u >= 0 && pg < naux) ? B[(size_t) u * naux + pg] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KT_K; kk++) {
            double a[4], b[4];
#pragma unroll
            for (int x = 0; x < 4; x++) a[x] = As[kk][ty + 16 * x];
#pragma unroll
            for (int y = 0; y < 4; y++) b[y] = Bs[kk][tx + 16 * y];
#pragma unroll
            for (int x = 0; x < 4; x++)
#pragma unroll
                for (int y = 0; y < 4; y++) acc[x][y] = fma(a[x], b[y], acc[x][y]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int x = 0; x < 4; x++) {
        int sg = s0 + ty + 16 * x;
        if (sg >= nocc) continue;
#pragma unroll
        for (int y = 0; y < 4; y++) {
            int pg = p0 + tx + 16 * y;
            if (pg < naux) T[((size_t) i * nocc + sg) * naux + pg] = acc[x][y];
        }
    }
}

// ---- K half-transform tile, 64 (s) x 256 (P) outputs per 256 threads (4 x 16
// per thread, fewer shared-memory reads per FMA than the 64 x 64 tile), next
// CSR chunk prefetched into registers. Same summation order as half_tile.
constexpr int KH_S = 64, KH_P = 256;

__device__ __forceinline__ void half_tile_wide(const double *__restrict__ B, const double *__restrict__ C,
                                               const int *__restrict__ csr_j, const int *__restrict__ csr_u,
                                               const int *__restrict__ displs, int nocc, int naux,
                                               double *__restrict__ T, int i, int s0, int p0)
{
    __shared__ double As[KT_K][KH_S + 1];
    __shared__ double Bs[KT_K][KH_P + 1];
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    const int r_beg = displs[i], r_end = displs[i + 1];
    double acc[4][16];
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 16; y++) acc[x][y] = 0.0;
    double pa[4], pb[16];
    auto fetch = [&](int r0) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int l = tid + 256 * q, kk = l / KH_S, c = l % KH_S, r = r0 + kk, sg = s0 + c;
            pa[q] = (r < r_end && sg < nocc) ? C[(size_t) csr_j[r] * nocc + sg] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int l = tid + 256 * q, kk = l / KH_P, c = l % KH_P, r = r0 + kk, pg = p0 + c;
            pb[q] = (r < r_end && pg < naux) ? B[(size_t) csr_u[r] * naux + pg] : 0.0;
        }
    };
    if (r_beg < r_end) fetch(r_beg);
    for (int r0 = r_beg; r0 < r_end; r0 += KT_K) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int l = tid + 256 * q;
            As[l / KH_S][l % KH_S] = pa[q];
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int l = tid + 256 * q;
            Bs[l / KH_P][l % KH_P] = pb[q];
        }
        __syncthreads();
        if (r0 + KT_K < r_end) fetch(r0 + KT_K);
#pragma unroll
        for (int kk = 0; kk < KT_K; kk++) {
            double a[4];
#pragma unroll
            for (int x = 0; x < 4; x++) a[x] = As[kk][ty + 16 * x];
#pragma unroll
            for (int y = 0; y < 16; y++) {
                const double b = Bs[kk][tx + 16 * y];
#pragma unroll
                for (int x = 0; x < 4; x++) acc[x][y] = fma(a[x], b, acc[x][y]);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int x = 0; x < 4; x++) {
        const int sg = s0 + ty + 16 * x;
        if (sg >= nocc) continue;
#pragma unroll
        for (int y = 0; y < 16; y++) {
            const int pg = p0 + tx + 16 * y;
            if (pg < naux) T[((size_t) i * nocc + sg) * naux + pg] = acc[x][y];
        }
    }
}

// ---- K = T T^T partial tile over q in [q_beg, q_end) of the flattened (s,P) index
__device__ __forceinline__ void syrk_tile(const double *__restrict__ T, int nbf, long long Q, long long q_beg,
                                          long long q_end, int i0, int j0, double *__restrict__ out)
{
    __shared__ double As[KT_K][KT_M + 1];
    __shared__ double Bs[KT_K][KT_N + 1];
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    double acc[4][4] = {};
    for (long long q0 = q_beg; q0 < q_end; q0 += KT_K) {
#pragma unroll
        for (int r = 0; r < 4; r++) {
            int l = tid + 256 * r;
            int row = l / KT_K, kk = l % KT_K;
            long long q = q0 + kk;
            int gi = i0 + row, gj = j0 + row;
            As[kk][row] = (gi < nbf && q < q_end) ? T[(size_t) gi * Q + q] : 0.0;
            Bs[kk][row] = (gj < nbf && q < q_end) ? T[(size_t) gj * Q + q] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KT_K; kk++) {
            double a[4], b[4];
#pragma unroll
            for (int x = 0; x < 4; x++) a[x] = As[kk][ty + 16 * x];
#pragma unroll
            for (int y = 0; y < 4; y++) b[y] = Bs[kk][tx + 16 * y];
#pragma unroll
            for (int x = 0; x < 4; x++)
#pragma unroll
                for (int y = 0; y < 4; y++) acc[x][y] = fma(a[x], b[y], acc[x][y]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int x = 0; x < 4; x++) {
        int gi = i0 + ty + 16 * x;
        if (gi >= nbf) continue;
#pragma unroll
        for (int y = 0; y < 4; y++) {
            int gj = j0 + tx + 16 * y;
            if (gj < nbf) out[(size_t) gi * nbf + gj] = acc[x][y];
        }
    }
}

// ---- K = T T^T partial tile, 128 x 128 outputs per 256 threads (8 x 8 per
// thread, half the shared-memory reads per FMA of the 64 x 64 tile); the next
// K-step's operands are prefetched into registers while the current one runs.
// Same summation order over q as syrk_tile.
constexpr int KB_T = 128;

__device__ __forceinline__ void syrk_tile128(const double *__restrict__ T, int nbf, long long Q, long long q_beg,
                                             long long q_end, int i0, int j0, double *__restrict__ out)
{
    __shared__ double As[KT_K][KB_T + 1];
    __shared__ double Bs[KT_K][KB_T + 1];
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    double acc[8][8];
#pragma unroll
    for (int x = 0; x < 8; x++)
#pragma unroll
        for (int y = 0; y < 8; y++) acc[x][y] = 0.0;
    double pa[8], pb[8];
    auto fetch = [&](long long q0) {
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int l = tid + 256 * r;
            const int row = l / KT_K, kk = l % KT_K;
            const long long q = q0 + kk;
            const int gi = i0 + row, gj = j0 + row;
            pa[r] = (gi < nbf && q < q_end) ? T[(size_t) gi * Q + q] : 0.0;
            pb[r] = (gj < nbf && q < q_end) ? T[(size_t) gj * Q + q] : 0.0;
        }
    };
    if (q_beg < q_end) fetch(q_beg);
    for (long long q0 = q_beg; q0 < q_end; q0 += KT_K) {
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int l = tid + 256 * r;
            As[l % KT_K][l / KT_K] = pa[r];
            Bs[l % KT_K][l / KT_K] = pb[r];
        }
        __syncthreads();
        if (q0 + KT_K < q_end) fetch(q0 + KT_K);
#pragma unroll
        for (int kk = 0; kk < KT_K; kk++) {
            double a[8], b[8];
#pragma unroll
            for (int x = 0; x < 8; x++) a[x] = As[kk][ty + 16 * x];
#pragma unroll
            for (int y = 0; y < 8; y++) b[y] = Bs[kk][tx + 16 * y];
#pragma unroll
            for (int x = 0; x < 8; x++)
#pragma unroll
                for (int y = 0; y < 8; y++) acc[x][y] = fma(a[x], b[y], acc[x][y]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int x = 0; x < 8; x++) {
        const int gi = i0 + ty + 16 * x;
        if (gi >= nbf) continue;
#pragma unroll
        for (int y = 0; y < 8; y++) {
            const int gj = j0 + tx + 16 * y;
            if (gj < nbf) out[(size_t) gi * nbf + gj] = acc[x][y];
        }
    }
}

// ---- K = T T^T partial tile on the FP64 tensor cores (DMMA, mma.sync
// m8n8k4): 128 x 128 outputs per 256 threads, 8 warps of 64 x 32 (8 x 4 DMMA
// tiles each). Per 4-wide K step a thread reads 12 doubles from shared memory
// for 32 DMMAs (8192 FMAs per warp), so the FP64 pipe, not shared memory, sets
// the pace. Operands staged as in syrk_tile128 (register prefetch of the next
// 16-wide K step).
__device__ __forceinline__ void syrk_tile_dmma(const double *__restrict__ T, int nbf, long long Q, long long q_beg,
                                               long long q_end, int i0, int j0, double *__restrict__ out)
{
    // operands stored row-major in M/N with rows of KT_K + 4 doubles: the
    // fragment reads (8 rows x 4 K per warp) then hit 32 distinct banks per wavefront
    __shared__ double As[KB_T][KT_K + 4];
    __shared__ double Bs[KB_T][KT_K + 4];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;   // warp tile origin inside the CTA tile
    const int fr = lane >> 2, fc = lane & 3;                 // fragment row / column of this lane
    double acc[8][4][2];
#pragma unroll
    for (int x = 0; x < 8; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y][0] = acc[x][y][1] = 0.0;
    double pa[8], pb[8];
    auto fetch = [&](long long q0) {
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int l = tid + 256 * r;
            const int row = l / KT_K, kk = l % KT_K;
            const long long q = q0 + kk;
            const int gi = i0 + row, gj = j0 + row;
            pa[r] = (gi < nbf && q < q_end) ? T[(size_t) gi * Q + q] : 0.0;
            pb[r] = (gj < nbf && q < q_end) ? T[(size_t) gj * Q + q] : 0.0;
        }
    };
    if (q_beg < q_end) fetch(q_beg);
    for (long long q0 = q_beg; q0 < q_end; q0 += KT_K) {
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int l = tid + 256 * r;
            As[l / KT_K][l % KT_K] = pa[r];
            Bs[l / KT_K][l % KT_K] = pb[r];
        }
        __syncthreads();
        if (q0 + KT_K < q_end) fetch(q0 + KT_K);
#pragma unroll
        for (int k4 = 0; k4 < KT_K; k4 += 4) {
            double a[8], b[4];
#pragma unroll
            for (int x = 0; x < 8; x++) a[x] = As[wm + 8 * x + fr][k4 + fc];   // A(row fr, k fc)
#pragma unroll
            for (int y = 0; y < 4; y++) b[y] = Bs[wn + 8 * y + fr][k4 + fc];   // B(k fc, col fr)
#pragma unroll
            for (int x = 0; x < 8; x++)
#pragma unroll
                for (int y = 0; y < 4; y++) dmma_8x8x4(acc[x][y][0], acc[x][y][1], a[x], b[y]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int x = 0; x < 8; x++) {
        const int gi = i0 + wm + 8 * x + fr;
        if (gi >= nbf) continue;
#pragma unroll
        for (int y = 0; y < 4; y++) {
            const int gj = j0 + wn + 8 * y + 2 * fc;   // C(row fr, cols 2 fc, 2 fc + 1)
            if (gj < nbf) out[(size_t) gi * nbf + gj] = acc[x][y][0];
            if (gj + 1 < nbf) out[(size_t) gi * nbf + gj + 1] = acc[x][y][1];
        }
    }
}

// ---- K half-transform tile on the FP64 tensor cores: 64 (s) x 256 (P)
// outputs per 256 threads, 8 warps of 32 x 64 (4 x 8 DMMA tiles each), CSR
// chunks of 16 prefetched into registers as in half_tile_wide.
__device__ __forceinline__ void half_tile_dmma(const double *__restrict__ B, const double *__restrict__ C,
                                               const int *__restrict__ csr_j, const int *__restrict__ csr_u,
                                               const int *__restrict__ displs, int nocc, int naux,
                                               double *__restrict__ T, int i, int s0, int p0)
{
    // K-major rows padded by 4 doubles (a row offset of 8 banks): the fragment
    // reads (4 K rows x 4 consecutive columns per 16-lane phase) and the
    // prefetch stores (consecutive columns) are both free of bank conflicts
    __shared__ double As[KT_K][KH_S + 4];
    __shared__ double Bs[KT_K][KH_P + 4];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ws = (warp >> 2) * 32, wp = (warp & 3) * 64;
    const int fr = lane >> 2, fc = lane & 3;
    const int r_beg = displs[i], r_end = displs[i + 1];
    double acc[4][8][2];
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 8; y++) acc[x][y][0] = acc[x][y][1] = 0.0;
    double pa[4], pb[16];
    auto fetch = [&](int r0) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int l = tid + 256 * q, kk = l / KH_S, c = l % KH_S, r = r0 + kk, sg = s0 + c;
            pa[q] = (r < r_end && sg < nocc) ? C[(size_t) csr_j[r] * nocc + sg] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int l = tid + 256 * q, kk = l / KH_P, c = l % KH_P, r = r0 + kk, pg = p0 + c;
            pb[q] = (r < r_end && pg < naux) ? B[(size_t) csr_u[r] * naux + pg] : 0.0;
        }
    };
    if (r_beg < r_end) fetch(r_beg);
    for (int r0 = r_beg; r0 < r_end; r0 += KT_K) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int l = tid + 256 * q;
            As[l / KH_S][l % KH_S] = pa[q];
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int l = tid + 256 * q;
            Bs[l / KH_P][l % KH_P] = pb[q];
        }
        __syncthreads();
        if (r0 + KT_K < r_end) fetch(r0 + KT_K);
#pragma unroll
        for (int k4 = 0; k4 < KT_K; k4 += 4) {
            double a[4], b[8];
#pragma unroll
            for (int x = 0; x < 4; x++) a[x] = As[k4 + fc][ws + 8 * x + fr];
#pragma unroll
            for (int y = 0; y < 8; y++) b[y] = Bs[k4 + fc][wp + 8 * y + fr];
#pragma unroll
            for (int x = 0; x < 4; x++)
#pragma unroll
                for (int y = 0; y < 8; y++) dmma_8x8x4(acc[x][y][0], acc[x][y][1], a[x], b[y]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int x = 0; x < 4; x++) {
        const int sg = s0 + ws + 8 * x + fr;
        if (sg >= nocc) continue;
        double *row = T + ((size_t) i * nocc + sg) * naux;
#pragma unroll
        for (int y = 0; y < 8; y++) {
            const int pg = p0 + wp + 8 * y + 2 * fc;
            if (pg < naux) row[pg] = acc[x][y][0];
            if (pg + 1 < naux) row[pg + 1] = acc[x][y][1];
        }
    }
}

// ---- J first pass: partial t(P) of upper rows [r0, r1), weights (2 - d_ij) D_ij.
// Thread x owns columns x, x + 512, ... (naux <= 8192).
constexpr int JT_THREADS = 512, JT_COLS = 16;

// BT = double, or float for the FP32 copy of the DF tensor (products and sums stay FP64)
// COLS columns per thread: naux <= COLS * JT_THREADS.
template <typename BT = double, int COLS = JT_COLS>
__device__ __forceinline__ void jt_rows(const BT *__restrict__ B, const int *__restrict__ up_u,
                                        const double *__restrict__ w, int naux, int r0, int r1,
                                        double *__restrict__ part_row)
{
    double acc[COLS];
#pragma unroll
    for (int c = 0; c < COLS; c++) acc[c] = 0.0;
    for (int r = r0; r < r1; r++) {
        const double wr = w[r];
        const BT *row = B + (size_t) up_u[r] * naux;
#pragma unroll
        for (int c = 0; c < COLS; c++) {
            int p = threadIdx.x + c * JT_THREADS;
            if (p < naux) acc[c] = fma(wr, (double) __ldg(row + p), acc[c]);
        }
    }
#pragma unroll
    for (int c = 0; c < COLS; c++) {
        int p = threadIdx.x + c * JT_THREADS;
        if (p < naux) part_row[p] = acc[c];
    }
}

// The FP32 copy with an even naux <= 8 * JT_THREADS and rows 8-byte aligned:
// each thread takes column pairs (float2 loads) and two rows per step, so as
// many bytes are in flight as with FP64 rows; every column is still summed
// row by row, so part_row equals jt_rows<float>'s bit for bit.
__device__ __forceinline__ void jt_rows_f2(const float *__restrict__ B, const int *__restrict__ up_u,
                                           const double *__restrict__ w, int naux, int r0, int r1,
                                           double *__restrict__ part_row)
{
    constexpr int PAIRS = 4;   // 4 * JT_THREADS column pairs
    const int npair = naux >> 1;
    double ax[PAIRS], ay[PAIRS];
#pragma unroll
    for (int c = 0; c < PAIRS; c++) ax[c] = ay[c] = 0.0;
    int r = r0;
    for (; r + 1 < r1; r += 2) {
        const double w0 = w[r], w1 = w[r + 1];
        const float2 *ra = (const float2 *) (B + (size_t) up_u[r] * naux);
        const float2 *rb = (const float2 *) (B + (size_t) up_u[r + 1] * naux);
        float2 va[PAIRS], vb[PAIRS];
#pragma unroll
        for (int c = 0; c < PAIRS; c++) {
            const int q = threadIdx.x + c * JT_THREADS;
            va[c] = q < npair ? __ldg(ra + q) : make_float2(0.f, 0.f);
            vb[c] = q < npair ? __ldg(rb + q) : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int c = 0; c < PAIRS; c++) {
            ax[c] = fma(w0, (double) va[c].x, ax[c]);
            ay[c] = fma(w0, (double) va[c].y, ay[c]);
            ax[c] = fma(w1, (double) vb[c].x, ax[c]);
            ay[c] = fma(w1, (double) vb[c].y, ay[c]);
        }
    }
    if (r < r1) {
        const double w0 = w[r];
        const float2 *ra = (const float2 *) (B + (size_t) up_u[r] * naux);
#pragma unroll
        for (int c = 0; c < PAIRS; c++) {
            const int q = threadIdx.x + c * JT_THREADS;
            if (q < npair) {
                const float2 v = __ldg(ra + q);
                ax[c] = fma(w0, (double) v.x, ax[c]);
                ay[c] = fma(w0, (double) v.y, ay[c]);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < PAIRS; c++) {
        const int q = threadIdx.x + c * JT_THREADS;
        if (q < npair) {
            part_row[2 * q] = ax[c];
            part_row[2 * q + 1] = ay[c];
        }
    }
}

// Whether jt_rows_f2 applies to an FP32 copy B with naux columns.
__host__ __device__ __forceinline__ bool jt_pairs_ok(const float *B, int naux)
{
    return B != nullptr && naux % 2 == 0 && naux <= 8 * JT_THREADS && ((uintptr_t) B & 7) == 0;
}

// t(P) = sum_b part[b][p] in block order for one column p; the loads of 16
// blocks are issued before their additions.
__device__ __forceinline__ double jt_reduce_col(const double *part, int nblk, int naux, int p)
{
    double s = 0.0;
    int b = 0;
    for (; b + 16 <= nblk; b += 16) {
        double v[16];
#pragma unroll
        for (int u = 0; u < 16; u++) v[u] = part[(size_t) (b + u) * naux + p];
#pragma unroll
        for (int u = 0; u < 16; u++) s += v[u];
    }
    for (; b < nblk; b++) s += part[(size_t) b * naux + p];
    return s;
}

// ---- F = H + 2J - K and the partial energy sum D (F + H) of one strided range
__device__ __forceinline__ double fock_energy_range(const double *H, const double *J, const double *K,
                                                    const double *D, double *F, size_t beg, size_t n, size_t stride)
{
    double e = 0.0;
    for (size_t i = beg; i < n; i += stride) {
        double h = H[i];
        double f = h + 2.0 * J[i] - K[i];
        F[i] = f;
        e += D[i] * (f + h);
    }
    return e;
}

__device__ __forceinline__ double block_sum(double e)
{
    __shared__ double sh[32];
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffff, e, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = e;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffff, r, o);
    }
    return r;   // valid in thread 0
}

}  // namespace tscf
