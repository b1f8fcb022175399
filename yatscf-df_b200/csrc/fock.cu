// Coulomb (J), exchange (K) and Fock assembly on sm_100a, FP64.
//
// J (build_Fock.c:37-130) is two bandwidth-bound passes over the DF tensor:
//   t(P)   = sum_{i<=j in CSR} (2 - d_ij) D_ij B(ij,P)        (row-streamed GEMV)
//   J_ij   = B(ij,:) . t                                       (one warp per pair)
// K (build_Fock.c:244-347) is the occupied half-transform
//   T(i,s,P) = sum_{j in row i} Cocc(j,s) B(ij,P)               (gather GEMM per row i)
// followed by K = T T^T over the flattened (s,P) index (upper tiles, split-K).
// The DF tensor is stored once per unordered pair (B_u); every ordered CSR
// entry of the reference (bf_pair_j / bf_mask_displs) maps to its row.
#include <cmath>
#include <cstdio>

#include "tscf_internal.h"

namespace tscf {

// ------------------------------------------------------------------ J
__global__ void k_j_weights(const int *up_i, const int *up_j, const double *D, double *w, int nup, int nbf)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nup) return;
    int i = up_i[k], j = up_j[k];
    w[k] = (i == j ? 1.0 : 2.0) * D[(size_t) i * nbf + j];
}

// Each block streams a contiguous range of upper rows and keeps its partial
// t(P) for every column in registers: thread x owns columns x, x+512, ...
constexpr int JT_THREADS = 512, JT_COLS = 16;   // naux <= 8192
__global__ void __launch_bounds__(JT_THREADS) k_j_tpart(const double *__restrict__ B, const int *__restrict__ up_u,
                                                        const double *__restrict__ w, int nup, int naux, int rows_per_blk,
                                                        double *__restrict__ part)
{
    double acc[JT_COLS];
#pragma unroll
    for (int c = 0; c < JT_COLS; c++) acc[c] = 0.0;
    const int r0 = blockIdx.x * rows_per_blk, r1 = min(nup, r0 + rows_per_blk);
    for (int r = r0; r < r1; r++) {
        const double wr = w[r];
        const double *row = B + (size_t) up_u[r] * naux;
#pragma unroll
        for (int c = 0; c < JT_COLS; c++) {
            int p = threadIdx.x + c * JT_THREADS;
            if (p < naux) acc[c] = fma(wr, __ldg(row + p), acc[c]);
        }
    }
#pragma unroll
    for (int c = 0; c < JT_COLS; c++) {
        int p = threadIdx.x + c * JT_THREADS;
        if (p < naux) part[(size_t) blockIdx.x * naux + p] = acc[c];
    }
}

__global__ void k_j_treduce(const double *part, int nblk, int naux, double *t)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= naux) return;
    double s = 0.0;
    for (int b = 0; b < nblk; b++) s += part[(size_t) b * naux + p];
    t[p] = s;
}

__global__ void __launch_bounds__(256) k_j_rows(const double *__restrict__ B, const int *up_i, const int *up_j,
                                                const int *up_u, const double *__restrict__ t, int nup, int naux,
                                                int nbf, double *J)
{
    extern __shared__ double ts[];
    for (int p = threadIdx.x; p < naux; p += blockDim.x) ts[p] = t[p];
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    for (int k = blockIdx.x * nw + wid; k < nup; k += gridDim.x * nw) {
        const double *row = B + (size_t) up_u[k] * naux;
        double s = 0.0;
        for (int p = lane; p < naux; p += 32) s = fma(__ldg(row + p), ts[p], s);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffff, s, o);
        if (lane == 0) {
            int i = up_i[k], j = up_j[k];
            J[(size_t) i * nbf + j] = s;
            J[(size_t) j * nbf + i] = s;
        }
    }
}

int build_J_part_blocks(const FockPlan &p)
{
    int nb = 2 * 148;
    if (p.nup < nb) nb = p.nup > 0 ? p.nup : 1;
    return nb;
}

void build_J(const FockPlan &p, const double *d_D, double *d_J, double *d_t, double *d_part, int nblk, double *d_w,
             cudaStream_t s)
{
    g_launches += 4;
    k_j_weights<<<(p.nup + 255) / 256, 256, 0, s>>>(p.up_i, p.up_j, d_D, d_w, p.nup, p.nbf);
    int rows_per_blk = (p.nup + nblk - 1) / nblk;
    k_j_tpart<<<nblk, JT_THREADS, 0, s>>>(p.B, p.up_u, d_w, p.nup, p.naux, rows_per_blk, d_part);
    k_j_treduce<<<(p.naux + 255) / 256, 256, 0, s>>>(d_part, nblk, p.naux, d_t);
    int blocks = 148 * 4;
    k_j_rows<<<blocks, 256, sizeof(double) * p.naux, s>>>(p.B, p.up_i, p.up_j, p.up_u, d_t, p.nup, p.naux, p.nbf, d_J);
}

// ------------------------------------------------------------------ K, FP64
// T[i][s][P]: block tile 64 (s) x 64 (P), K-step 16 rows of CSR row i.
constexpr int KT_M = 64, KT_N = 64, KT_K = 16;
__global__ void __launch_bounds__(256) k_halftransform(const double *__restrict__ B, const double *__restrict__ C,
                                                       const int *__restrict__ csr_j, const int *__restrict__ csr_u,
                                                       const int *__restrict__ displs, int nocc, int naux,
                                                       double *__restrict__ T)
{
    __shared__ double As[KT_K][KT_M + 1];
    __shared__ double Bs[KT_K][KT_N + 1];
    __shared__ int rj[KT_K], ru[KT_K];
    const int i = blockIdx.z;
    const int s0 = blockIdx.y * KT_M, p0 = blockIdx.x * KT_N;
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

// K partial tiles: upper tile pairs (bi <= bj) of 64x64, split over the
// flattened Q = nocc*naux index. Kpart[split][i][j].
__global__ void __launch_bounds__(256) k_syrk_part(const double *__restrict__ T, int nbf, long long Q, long long qchunk,
                                                   const int2 *__restrict__ tiles, double *__restrict__ Kpart)
{
    __shared__ double As[KT_K][KT_M + 1];
    __shared__ double Bs[KT_K][KT_N + 1];
    const int2 tl = tiles[blockIdx.x];
    const int split = blockIdx.y;
    const int i0 = tl.x * KT_M, j0 = tl.y * KT_N;
    const long long q_beg = (long long) split * qchunk, q_end = min(Q, q_beg + qchunk);
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
    double *out = Kpart + (size_t) split * nbf * nbf;
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

// K[i][j] = K[j][i] = sum_split Kpart[split][i][j] for i <= j (TinySCF keeps
// the upper triangle and mirrors it, build_Fock.c:369-379).
__global__ void k_syrk_reduce(const double *Kpart, int nsplit, int nbf, double *K)
{
    size_t idx = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t) nbf * nbf) return;
    int i = (int) (idx / nbf), j = (int) (idx % nbf);
    if (i > j) return;
    double s = 0.0;
    for (int k = 0; k < nsplit; k++) s += Kpart[(size_t) k * nbf * nbf + idx];
    K[idx] = s;
    K[(size_t) j * nbf + i] = s;
}

size_t build_K_part_elems(const FockPlan &p, int ksplit) { return (size_t) ksplit * p.nbf * p.nbf; }

void build_K_halftransform(const FockPlan &p, const double *d_Cocc, double *d_T, cudaStream_t s)
{
    dim3 g1((p.naux + KT_N - 1) / KT_N, (p.nocc + KT_M - 1) / KT_M, p.nbf);
    g_launches++;
    k_halftransform<<<g1, 256, 0, s>>>(p.B, d_Cocc, p.csr_j, p.csr_u, p.csr_displs, p.nocc, p.naux, d_T);
}

void build_K_syrk(const FockPlan &p, const double *d_T, double *d_K, double *d_Kpart, int ksplit, const int2 *d_tiles,
                  cudaStream_t s)
{
    const int nt = (p.nbf + KT_M - 1) / KT_M;
    const int ntiles = nt * (nt + 1) / 2;
    const long long Q = (long long) p.nocc * p.naux;
    long long qchunk = (Q + ksplit - 1) / ksplit;
    qchunk = (qchunk + KT_K - 1) / KT_K * KT_K;
    dim3 g2(ntiles, ksplit);
    g_launches += 2;
    k_syrk_part<<<g2, 256, 0, s>>>(d_T, p.nbf, Q, qchunk, d_tiles, d_Kpart);
    size_t nn = (size_t) p.nbf * p.nbf;
    k_syrk_reduce<<<(unsigned) ((nn + 255) / 256), 256, 0, s>>>(d_Kpart, ksplit, p.nbf, d_K);
}

// ------------------------------------------------------------------ F and energy
__global__ void k_fock_energy(const double *H, const double *J, const double *K, const double *D, double *F,
                              double *epart, size_t n)
{
    __shared__ double sh[32];
    double e = 0.0;
    for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x) {
        double h = H[i];
        double f = h + 2.0 * J[i] - K[i];
        F[i] = f;
        e += D[i] * (f + h);
    }
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffff, e, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x < 32) {
        e = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffff, e, o);
        if (threadIdx.x == 0) epart[blockIdx.x] = e;
    }
}

void build_F_energy(const double *d_H, const double *d_J, const double *d_K, const double *d_D, double *d_F,
                    double *d_epart, int n, cudaStream_t s)
{
    g_launches++;
    k_fock_energy<<<ENERGY_BLOCKS, 256, 0, s>>>(d_H, d_J, d_K, d_D, d_F, d_epart, (size_t) n * n);
}

}  // namespace tscf
