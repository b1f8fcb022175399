// Dense FP64 building blocks for the SCF: a tiled DGEMM, inverse square
// roots from eigenpairs (TinySCF.c:58-76, build_DF_tensor.c:205-237), and the
// pivoted Cholesky of the initial guess (TinySCF.c:282-322, LAPACK dpstf2
// semantics). The eigensolver itself is in eigh.cu.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <mutex>

#include <utility>
#include <vector>

#include "tiles.cuh"
#include "tune.h"
#include "tscf_internal.h"

namespace tscf {

std::atomic<long long> g_launches{0};

// ------------------------------------------------------------------ DGEMM
// Five tile shapes: FFMA 64x64 (default), 32x32 (more blocks for small
// matrices) and 128x64 (more reuse for large ones) (dgemm_tile), and 128x128
// and 64x64 on the FP64 tensor cores (dgemm_tile_dmma, dgemm_tile_dmma64). The
// autotuner picks one per call shape the first time the shape is met outside
// a stream capture.
template <bool TA, bool TB, int BM, int BN>
__global__ void __launch_bounds__(256) k_dgemm(int m, int n, int k, double alpha, const double *__restrict__ A, int lda,
                                               const double *__restrict__ B, int ldb, double beta, double *C, int ldc)
{
    dgemm_tile<TA, TB, BM, BN>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, blockIdx.y * BM, blockIdx.x * BN);
}

template <int BM, int BN>
static void dgemm_shape(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, int lda,
                        const double *B, int ldb, double beta, double *C, int ldc, cudaStream_t s)
{
    dim3 grid((n + BN - 1) / BN, (m + BM - 1) / BM);
    g_launches++;
    if (!ta && !tb) k_dgemm<false, false, BM, BN><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (!ta && tb) k_dgemm<false, true, BM, BN><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (ta && !tb) k_dgemm<true, false, BM, BN><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else k_dgemm<true, true, BM, BN><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(256, 1) k_dgemm_dmma(int m, int n, int k, double alpha, const double *__restrict__ A,
                                                       int lda, const double *__restrict__ B, int ldb, double beta,
                                                       double *C, int ldc)
{
    dgemm_tile_dmma<TA, TB>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, blockIdx.y * 128, blockIdx.x * 128);
}

static void dgemm_dmma(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, int lda, const double *B,
                       int ldb, double beta, double *C, int ldc, cudaStream_t s)
{
    dim3 grid((n + 127) / 128, (m + 127) / 128);
    g_launches++;
    if (!ta && !tb) k_dgemm_dmma<false, false><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (!ta && tb) k_dgemm_dmma<false, true><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (ta && !tb) k_dgemm_dmma<true, false><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else k_dgemm_dmma<true, true><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(128) k_dgemm_dmma64(int m, int n, int k, double alpha, const double *__restrict__ A,
                                                      int lda, const double *__restrict__ B, int ldb, double beta,
                                                      double *C, int ldc)
{
    dgemm_tile_dmma64<TA, TB>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, blockIdx.y * 64, blockIdx.x * 64);
}

static void dgemm_dmma64(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, int lda,
                         const double *B, int ldb, double beta, double *C, int ldc, cudaStream_t s)
{
    dim3 grid((n + 63) / 64, (m + 63) / 64);
    g_launches++;
    if (!ta && !tb) k_dgemm_dmma64<false, false><<<grid, 128, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (!ta && tb) k_dgemm_dmma64<false, true><<<grid, 128, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (ta && !tb) k_dgemm_dmma64<true, false><<<grid, 128, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else k_dgemm_dmma64<true, true><<<grid, 128, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

// ---- 32 x 32 output tile per 256 threads on the FP64 tensor cores, the K
// range split over the 8 warps: for the tall-skinny and small products of the
// density refinement, DIIS and orbital alignment (n x n_occ outputs, n_occ^2
// outputs with K = n), where the 64/128 tiles leave most SMs idle and a
// single warp per tile would run the whole K loop alone. Each 64-wide K chunk
// is prefetched into registers while the previous one is multiplied (warp w
// takes chunk rows 8w..8w+7); the eight partial tiles are summed through
// shared memory in a fixed order.
constexpr int KS_T = 32, KS_K = 64, KS_LD = KS_K + 4;

template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_dgemm_dmma32ks(int m, int n, int k, double alpha,
                                                        const double *__restrict__ A, int lda,
                                                        const double *__restrict__ B, int ldb, double beta,
                                                        double *C, int ldc)
{
    __shared__ double sm[2 * KS_T * KS_LD];   // As[32][68], Bs[32][68]; then the partial-tile slots
    double *As = sm, *Bs = sm + KS_T * KS_LD;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int fr = lane >> 2, fc = lane & 3;
    const int m0 = blockIdx.y * KS_T, n0 = blockIdx.x * KS_T;
    double acc[4][4][2];
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y][0] = acc[x][y][1] = 0.0;
    double pa[8], pb[8];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int l = tid + 256 * r;
            int row, kk;
            if (!TA) { row = l / KS_K; kk = l % KS_K; } else { kk = l / KS_T; row = l % KS_T; }
            const int gi = m0 + row, gk = k0 + kk;
            pa[r] = (gi < m && gk < k) ? (TA ? A[(size_t) gk * lda + gi] : A[(size_t) gi * lda + gk]) : 0.0;
            int col;
            if (!TB) { kk = l / KS_T; col = l % KS_T; } else { col = l / KS_K; kk = l % KS_K; }
            const int gj = n0 + col, gk2 = k0 + kk;
            pb[r] = (gj < n && gk2 < k) ? (TB ? B[(size_t) gj * ldb + gk2] : B[(size_t) gk2 * ldb + gj]) : 0.0;
        }
    };
    fetch(0);
    for (int k0 = 0; k0 < k; k0 += KS_K) {
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int l = tid + 256 * r;
            if (!TA) As[(l / KS_K) * KS_LD + l % KS_K] = pa[r];
            else As[(l % KS_T) * KS_LD + l / KS_T] = pa[r];
            if (!TB) Bs[(l % KS_T) * KS_LD + l / KS_T] = pb[r];
            else Bs[(l / KS_K) * KS_LD + l % KS_K] = pb[r];
        }
        __syncthreads();
        if (k0 + KS_K < k) fetch(k0 + KS_K);
#pragma unroll
        for (int k4 = 0; k4 < 8; k4 += 4) {
            const int kc = 8 * warp + k4 + fc;
            double a[4], b[4];
#pragma unroll
            for (int x = 0; x < 4; x++) a[x] = As[(8 * x + fr) * KS_LD + kc];
#pragma unroll
            for (int y = 0; y < 4; y++) b[y] = Bs[(8 * y + fr) * KS_LD + kc];
#pragma unroll
            for (int x = 0; x < 4; x++)
#pragma unroll
                for (int y = 0; y < 4; y++) dmma_8x8x4(acc[x][y][0], acc[x][y][1], a[x], b[y]);
        }
        __syncthreads();
    }
    // warps 4-7 into 0-3, then 2-3 into 0-1, then 1 into 0 (slots of 32 x 32 per warp)
    double *red = sm;
    for (int half = 4; half >= 1; half >>= 1) {
        if (warp >= half && warp < 2 * half) {
#pragma unroll
            for (int x = 0; x < 4; x++)
#pragma unroll
                for (int y = 0; y < 4; y++)
#pragma unroll
                    for (int h = 0; h < 2; h++) red[(warp - half) * 1024 + ((x * 4 + y) * 2 + h) * 32 + lane] = acc[x][y][h];
        }
        __syncthreads();
        if (warp < half) {
#pragma unroll
            for (int x = 0; x < 4; x++)
#pragma unroll
                for (int y = 0; y < 4; y++)
#pragma unroll
                    for (int h = 0; h < 2; h++) acc[x][y][h] += red[warp * 1024 + ((x * 4 + y) * 2 + h) * 32 + lane];
        }
        __syncthreads();
    }
    if (warp != 0) return;
#pragma unroll
    for (int x = 0; x < 4; x++) {
        const int gi = m0 + 8 * x + fr;
        if (gi >= m) continue;
#pragma unroll
        for (int y = 0; y < 4; y++) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int gj = n0 + 8 * y + 2 * fc + h;
                if (gj >= n) continue;
                double *c = C + (size_t) gi * ldc + gj;
                *c = (beta == 0.0) ? alpha * acc[x][y][h] : alpha * acc[x][y][h] + beta * *c;
            }
        }
    }
}

static void dgemm_dmma32ks(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, int lda,
                           const double *B, int ldb, double beta, double *C, int ldc, cudaStream_t s)
{
    dim3 grid((n + KS_T - 1) / KS_T, (m + KS_T - 1) / KS_T);
    g_launches++;
    if (!ta && !tb) k_dgemm_dmma32ks<false, false><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (!ta && tb) k_dgemm_dmma32ks<false, true><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (ta && !tb) k_dgemm_dmma32ks<true, false><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else k_dgemm_dmma32ks<true, true><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

static void dgemm_variant(int v, bool ta, bool tb, int m, int n, int k, double alpha, const double *A, int lda,
                          const double *B, int ldb, double beta, double *C, int ldc, cudaStream_t s)
{
    if (v == 5) dgemm_dmma32ks(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
    else if (v == 4) dgemm_dmma64(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
    else if (v == 3) dgemm_dmma(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
    else if (v == 1) dgemm_shape<32, 32>(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
    else if (v == 2) dgemm_shape<128, 64>(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
    else dgemm_shape<64, 64>(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
}

void dgemm(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, int lda, const double *B, int ldb,
           double beta, double *C, int ldc, cudaStream_t s)
{
    if (m <= 0 || n <= 0) return;
    char key[96];
    snprintf(key, sizeof(key), "dgemm:%d%d:%dx%dx%d", (int) ta, (int) tb, m, n, k);
    int v = tune_lookup(key);
    if (v < 0) {
        v = 0;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(s, &cs);
        // tune only where re-running is harmless: C overwritten (beta = 0) and
        // not read by the product
        const char *c0 = (const char *) C, *c1 = c0 + sizeof(double) * ((size_t) (m - 1) * ldc + n);
        auto disjoint = [&](const double *X, size_t elems) {
            const char *x0 = (const char *) X, *x1 = x0 + sizeof(double) * elems;
            return x1 <= c0 || c1 <= x0;
        };
        const size_t ea = ta ? (size_t) k * lda : (size_t) m * lda, eb = tb ? (size_t) n * ldb : (size_t) k * ldb;
        if (tune_enabled() && cs == cudaStreamCaptureStatusNone && beta == 0.0 && disjoint(A, ea) && disjoint(B, eb) &&
            (double) m * n * k >= 2e6) {
            v = tune_run(key, {0, 1, 2, 3, 4, 5}, [&](int c) { dgemm_variant(c, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s); }, s);
            return;
        }
    }
    dgemm_variant(v, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
}

// Tile shape from the call shape alone, for the many distinct shapes of the
// eigensolver's panel updates (tuning each one would cost more than it saves):
// the K-split tile for outputs of few 64 x 64 tiles with a long K, the 128 x 128 DMMA tile
// for large outputs, the 64 x 64 DMMA tile otherwise.
void dgemm_untuned(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, int lda, const double *B,
                   int ldb, double beta, double *C, int ldc, cudaStream_t s)
{
    if (m <= 0 || n <= 0) return;
    int v = 4;
    const double tiles64 = std::ceil(m / 64.0) * std::ceil(n / 64.0);
    const double nsm = num_sms();
    if (k >= 256 && tiles64 < 2.0 * nsm) v = 5;
    else if ((double) m * n >= 4.0 * nsm * 128 * 128) v = 3;
    dgemm_variant(v, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
}

// SM count of the current device (cached for the first 64 ordinals).
int num_sms()
{
    static std::atomic<int> cached[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    const bool cacheable = dev >= 0 && dev < 64;
    if (cacheable && cached[dev].load(std::memory_order_relaxed) > 0) return cached[dev].load(std::memory_order_relaxed);
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    if (v <= 0) v = 1;
    if (cacheable) cached[dev].store(v, std::memory_order_relaxed);
    return v;
}

int cuda_launch_rc(const char *what)
{
    const cudaError_t err = cudaPeekAtLastError();
    if (err == cudaSuccess) return OK;
    fprintf(stderr, "[tinyscf] CUDA error in %s: %s\n", what, cudaGetErrorString(err));
    return ERR_CUDA;
}

// ---------------------------------------------------------------- device memory
// The engine's large buffers come from the device's stream-ordered memory
// pool, kept reserved (release threshold: unlimited), so that freeing an
// engine hands its memory to the next one without unmapping and remapping;
// TINYSCF_MEMPOOL=0 uses cudaMalloc / cudaFree instead. The choice is made
// once per process. TinySCF_trim_memory returns the pool's unused memory.
static bool pool_mode()
{
    static const bool on = [] {
        const char *v = getenv("TINYSCF_MEMPOOL");
        return !(v && v[0] == '0');
    }();
    return on;
}

int dev_malloc(void **p, size_t bytes, cudaStream_t s)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    if (pool_mode()) {
        static std::mutex mu;
        static bool configured[64] = {};
        int dev = 0;
        cudaGetDevice(&dev);
        {
            std::lock_guard<std::mutex> lk(mu);
            if (dev >= 0 && dev < 64 && !configured[dev]) {
                cudaMemPool_t pool;
                if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
                    uint64_t thr = UINT64_MAX;
                    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
                }
                configured[dev] = true;
            }
        }
        if (cudaMallocAsync(p, bytes, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            return ERR_ALLOC;
        }
        return OK;
    }
    if (cudaMalloc(p, bytes) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return ERR_ALLOC;
    }
    return OK;
}

void dev_free(void *p, cudaStream_t s)
{
    if (!p) return;
    if (pool_mode()) cudaFreeAsync(p, s);
    else cudaFree(p);
}

int dev_trim(int device)
{
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) return ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return ERR_CUDA;
    return cudaMemPoolTrimTo(pool, 0) == cudaSuccess ? OK : ERR_CUDA;
}

__global__ void k_scale_rows_invsqrt(const double *w, const double *V, double *out, int n)
{
    size_t idx = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t) n * n) return;
    int k = (int) (idx / n);
    out[idx] = V[idx] / sqrt(w[k]);
}

void inv_sqrt_from_eig(const double *d_w, const double *d_V, double *d_X, double *d_tmp, int n, cudaStream_t s)
{
    size_t nn = (size_t) n * n;
    g_launches++;
    k_scale_rows_invsqrt<<<(unsigned) ((nn + 255) / 256), 256, 0, s>>>(d_w, d_V, d_tmp, n);
    // X = V^T diag(w^-1/2) V
    dgemm(true, false, n, n, n, 1.0, d_V, n, d_tmp, n, 0.0, d_X, n, s);
}

// ------------------------------------------------------------------ pivoted Cholesky
// One 1024-thread block runs LAPACK dpstf2 (UPLO = 'L') step for step on the
// logical matrix A(i,j) = A[i*n + j]: left-looking column updates, diagonal
// candidates A(i,i) - sum_k A(i,k)^2 accumulated in work[], first-maximum
// pivot, the same row/column swaps, stop when the pivot <= tol.
struct ValIdx {
    double v;
    int i;
};
__device__ __forceinline__ ValIdx better(ValIdx a, ValIdx b)
{
    if (b.v > a.v || (b.v == a.v && b.i < a.i)) return b;
    return a;
}

__device__ ValIdx block_argmax(ValIdx x, ValIdx *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        ValIdx y;
        y.v = __shfl_down_sync(0xffffffff, x.v, o);
        y.i = __shfl_down_sync(0xffffffff, x.i, o);
        x = better(x, y);
    }
    if (lane == 0) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        x = (lane < (int) (blockDim.x >> 5)) ? sh[lane] : ValIdx{-DBL_MAX, 0x7fffffff};
        for (int o = 16; o > 0; o >>= 1) {
            ValIdx y;
            y.v = __shfl_down_sync(0xffffffff, x.v, o);
            y.i = __shfl_down_sync(0xffffffff, x.i, o);
            x = better(x, y);
        }
        if (lane == 0) sh[0] = x;
    }
    __syncthreads();
    ValIdx r = sh[0];
    __syncthreads();
    return r;
}

// blkp (nullptr: one block): the block of every position, permuted with the
// pivots. A is block diagonal in these blocks (the SAD density: one block per
// atom), so column j of the factor is nonzero only in the rows of the pivot's
// block and every product with another block's entry is an exact zero: the
// rows of other blocks are skipped and their squared-norm sums left alone,
// which changes no bit of the result (adding +-0 is exact) but makes each
// step cost the pivot search instead of an (n - j) x j update.
__global__ void __launch_bounds__(1024) k_pstf2(double *A, int n, double tol, int *piv, int *rank_out, double *work,
                                                int *blkp)
{
    __shared__ ValIdx sh[32];
    __shared__ int s_stop;
    double *dot = work, *cand = work + n;
#define AA(i, j) A[(size_t) (i) * n + (j)]
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        dot[i] = 0.0;
        piv[i] = i;
    }
    __syncthreads();
    // j = 0: pivot on the largest diagonal element
    ValIdx best{-DBL_MAX, 0x7fffffff};
    for (int i = threadIdx.x; i < n; i += blockDim.x) best = better(best, ValIdx{AA(i, i), i});
    best = block_argmax(best, sh);
    double ajj = best.v;
    int pvt = best.i;
    if (threadIdx.x == 0) s_stop = (ajj <= 0.0 || isnan(ajj)) ? 1 : 0;
    __syncthreads();
    if (s_stop) {
        if (threadIdx.x == 0) *rank_out = 0;
        return;
    }
    int rank = n;
    for (int j = 0; j < n; j++) {
        if (j > 0) {
            ValIdx b{-DBL_MAX, 0x7fffffff};
            const int bprev = blkp ? blkp[j - 1] : 0;
            for (int i = j + threadIdx.x; i < n; i += blockDim.x) {
                if (!blkp || blkp[i] == bprev) {
                    double a = AA(i, j - 1);
                    dot[i] += a * a;
                }
                double c = AA(i, i) - dot[i];
                cand[i] = c;
                b = better(b, ValIdx{c, i});
            }
            b = block_argmax(b, sh);
            pvt = b.i;
            ajj = b.v;
            if (ajj <= tol || isnan(ajj)) {
                if (threadIdx.x == 0) AA(j, j) = ajj;
                rank = j;
                break;
            }
        }
        if (j != pvt) {
            __syncthreads();
            if (threadIdx.x == 0) {
                AA(pvt, pvt) = AA(j, j);
                double t = dot[j]; dot[j] = dot[pvt]; dot[pvt] = t;
                int p = piv[pvt]; piv[pvt] = piv[j]; piv[j] = p;
                if (blkp) {
                    const int q = blkp[pvt]; blkp[pvt] = blkp[j]; blkp[j] = q;
                }
            }
            for (int c = threadIdx.x; c < j; c += blockDim.x) {          // rows j and pvt, columns 0..j-1
                double t = AA(j, c); AA(j, c) = AA(pvt, c); AA(pvt, c) = t;
            }
            for (int r = pvt + 1 + threadIdx.x; r < n; r += blockDim.x) { // columns j and pvt below pvt
                double t = AA(r, j); AA(r, j) = AA(r, pvt); AA(r, pvt) = t;
            }
            for (int r = j + 1 + threadIdx.x; r < pvt; r += blockDim.x) { // column j (rows j+1..pvt-1) vs row pvt
                double t = AA(r, j); AA(r, j) = AA(pvt, r); AA(pvt, r) = t;
            }
            __syncthreads();
        }
        ajj = sqrt(ajj);
        if (threadIdx.x == 0) AA(j, j) = ajj;
        __syncthreads();
        // A(j+1:n, j) = (A(j+1:n, j) - A(j+1:n, 0:j) A(j, 0:j)^T) / ajj : one warp per row
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
        const double rinv = 1.0 / ajj;
        const int bj = blkp ? blkp[j] : 0;
        for (int r = j + 1 + wid; r < n; r += nw) {
            if (blkp && blkp[r] != bj) continue;   // zero column entry: (0 - 0) / ajj stays +0
            double s = 0.0;
            for (int c = lane; c < j; c += 32)
                if (!blkp || blkp[c] == bj) s += AA(r, c) * AA(j, c);
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffff, s, o);
            if (lane == 0) AA(r, j) = (AA(r, j) - s) * rinv;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *rank_out = rank;
#undef AA
}

void pivoted_cholesky(double *d_A, int n, double tol, int *d_piv, int *d_rank, double *d_work, cudaStream_t s,
                      const int *d_blk, int *d_blk_work)
{
    g_launches++;
    int *blkp = nullptr;
    if (d_blk && d_blk_work) {
        cudaMemcpyAsync(d_blk_work, d_blk, sizeof(int) * n, cudaMemcpyDeviceToDevice, s);
        blkp = d_blk_work;
    }
    k_pstf2<<<1, 1024, 0, s>>>(d_A, n, tol, d_piv, d_rank, d_work, blkp);
}

__global__ void k_d2cocc(const double *chol, const int *rank_p, double *C, int nbf, int nocc)
{
    size_t idx = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t) nbf * nocc) return;
    int i = (int) (idx / nocc), j = (int) (idx % nocc);
    int rank = *rank_p;
    double v = (j < nbf) ? chol[(size_t) i * nbf + j] : 0.0;
    if (rank < nocc && j >= rank) v = 0.0;
    if (i < nocc && j >= i) v = 0.0;
    C[idx] = v;
}

void d2cocc_copy(const double *d_chol, const int *d_rank, double *d_Cocc, int nbf, int nocc, cudaStream_t s)
{
    size_t n = (size_t) nbf * nocc;
    g_launches++;
    k_d2cocc<<<(unsigned) ((n + 255) / 256), 256, 0, s>>>(d_chol, d_rank, d_Cocc, nbf, nocc);
}

// ------------------------------------------------------------------ elementwise
__global__ void k_fill(double *d, double v, size_t n)
{
    size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = v;
}
void fill(double *d, double v, size_t n, cudaStream_t s)
{
    if (n) g_launches++;
    if (n) k_fill<<<(unsigned) ((n + 255) / 256), 256, 0, s>>>(d, v, n);
}
__global__ void k_scale_copy(const double *a, double *b, double f, size_t n)
{
    size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = f * a[i];
}
void scale_copy(const double *src, double *dst, double a, size_t n, cudaStream_t s)
{
    if (n) g_launches++;
    if (n) k_scale_copy<<<(unsigned) ((n + 255) / 256), 256, 0, s>>>(src, dst, a, n);
}

}  // namespace tscf
