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
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "tiles.cuh"
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
// t(P) for every column in registers (jt_rows).
template <typename BT, int COLS>
__global__ void __launch_bounds__(JT_THREADS) k_j_tpart(const BT *__restrict__ B, const int *__restrict__ up_u,
                                                        const double *__restrict__ w, int nup, int naux, int rows_per_blk,
                                                        double *__restrict__ part)
{
    const int r0 = blockIdx.x * rows_per_blk, r1 = min(nup, r0 + rows_per_blk);
    jt_rows<BT, COLS>(B, up_u, w, naux, r0, r1, part + (size_t) blockIdx.x * naux);
}

// The FP32 copy of B with an even naux (jt_rows_f2: float2 column pairs, two
// rows per step, the same sums as jt_rows<float> bit for bit).
__global__ void __launch_bounds__(JT_THREADS) k_j_tpart_f2(const float *__restrict__ B, const int *__restrict__ up_u,
                                                           const double *__restrict__ w, int nup, int naux,
                                                           int rows_per_blk, double *__restrict__ part)
{
    const int r0 = blockIdx.x * rows_per_blk, r1 = min(nup, r0 + rows_per_blk);
    jt_rows_f2(B, up_u, w, naux, r0, r1, part + (size_t) blockIdx.x * naux);
}

// t(P) = sum over the blocks' partial rows, in block order (jt_reduce_col).
__global__ void k_j_treduce(const double *part, int nblk, int naux, double *t)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= naux) return;
    t[p] = jt_reduce_col(part, nblk, naux, p);
}

template <typename BT>
__global__ void __launch_bounds__(256) k_j_rows(const BT *__restrict__ B, const int *up_i, const int *up_j,
                                                const int *up_u, const double *__restrict__ t, int nup, int naux,
                                                int nbf, double *J)
{
    extern __shared__ double ts[];
    for (int p = threadIdx.x; p < naux; p += blockDim.x) ts[p] = t[p];
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    for (int k = blockIdx.x * nw + wid; k < nup; k += gridDim.x * nw) {
        const BT *row = B + (size_t) up_u[k] * naux;
        double s = 0.0;
        for (int p = lane; p < naux; p += 32) s = fma((double) __ldg(row + p), ts[p], s);
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
    int nb = 2 * num_sms();
    if (p.nup < nb) nb = p.nup > 0 ? p.nup : 1;
    return nb;
}

template <typename BT>
static void build_J_t(const FockPlan &p, const BT *B, const double *d_D, double *d_J, double *d_t, double *d_part,
                      int nblk, double *d_w, cudaStream_t s)
{
    g_launches += 4;
    k_j_weights<<<(p.nup + 255) / 256, 256, 0, s>>>(p.up_i, p.up_j, d_D, d_w, p.nup, p.nbf);
    int rows_per_blk = (p.nup + nblk - 1) / nblk;
    if (sizeof(BT) == sizeof(float) && jt_pairs_ok((const float *) B, p.naux))
        k_j_tpart_f2<<<nblk, JT_THREADS, 0, s>>>((const float *) B, p.up_u, d_w, p.nup, p.naux, rows_per_blk,
                                                 d_part);
    else if (p.naux <= 8 * JT_THREADS)
        k_j_tpart<BT, 8><<<nblk, JT_THREADS, 0, s>>>(B, p.up_u, d_w, p.nup, p.naux, rows_per_blk, d_part);
    else
        k_j_tpart<BT, JT_COLS><<<nblk, JT_THREADS, 0, s>>>(B, p.up_u, d_w, p.nup, p.naux, rows_per_blk, d_part);
    k_j_treduce<<<(p.naux + 63) / 64, 64, 0, s>>>(d_part, nblk, p.naux, d_t);
    int blocks = num_sms() * 4;
    const size_t shm = sizeof(double) * p.naux;   // t(P) staged in shared memory
    if (shm > 48 * 1024) cudaFuncSetAttribute(k_j_rows<BT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) shm);
    k_j_rows<BT><<<blocks, 256, shm, s>>>(B, p.up_i, p.up_j, p.up_u, d_t, p.nup, p.naux, p.nbf, d_J);
}

void build_J(const FockPlan &p, const double *d_D, double *d_J, double *d_t, double *d_part, int nblk, double *d_w,
             cudaStream_t s)
{
    build_J_t<double>(p, p.B, d_D, d_J, d_t, d_part, nblk, d_w, s);
}

void build_J_f32(const FockPlan &p, const float *B32, const double *d_D, double *d_J, double *d_t, double *d_part,
                 int nblk, double *d_w, cudaStream_t s)
{
    build_J_t<float>(p, B32, d_D, d_J, d_t, d_part, nblk, d_w, s);
}

__global__ void k_to_f32(const double *in, float *out, size_t n)
{
    for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
        out[i] = (float) in[i];
}

void convert_f32(const double *in, float *out, size_t n, cudaStream_t s)
{
    g_launches++;
    k_to_f32<<<num_sms() * 8, 256, 0, s>>>(in, out, n);
}

// ------------------------------------------------------------------ K, FP64
// T[i][s][P]: block tile 64 (s) x 64 (P), K-step 16 rows of CSR row i.
__global__ void __launch_bounds__(256) k_halftransform(const double *__restrict__ B, const double *__restrict__ C,
                                                       const int *__restrict__ csr_j, const int *__restrict__ csr_u,
                                                       const int *__restrict__ displs, int nocc, int naux,
                                                       double *__restrict__ T)
{
    half_tile(B, C, csr_j, csr_u, displs, nocc, naux, T, blockIdx.z, blockIdx.y * KT_M, blockIdx.x * KT_N);
}

__global__ void __launch_bounds__(256, 1) k_halftransform_wide(const double *__restrict__ B, const double *__restrict__ C,
                                                               const int *__restrict__ csr_j,
                                                               const int *__restrict__ csr_u,
                                                               const int *__restrict__ displs, int nocc, int naux,
                                                               double *__restrict__ T)
{
    half_tile_wide(B, C, csr_j, csr_u, displs, nocc, naux, T, blockIdx.z, blockIdx.y * KH_S, blockIdx.x * KH_P);
}

__global__ void __launch_bounds__(256, 1) k_halftransform_dmma(const double *__restrict__ B, const double *__restrict__ C,
                                                               const int *__restrict__ csr_j,
                                                               const int *__restrict__ csr_u,
                                                               const int *__restrict__ displs, int nocc, int naux,
                                                               double *__restrict__ T)
{
    half_tile_dmma(B, C, csr_j, csr_u, displs, nocc, naux, T, blockIdx.z, blockIdx.y * KH_S, blockIdx.x * KH_P);
}

// ---- K half-transform on the FP64 tensor cores, persistent and pipelined.
// CTA b takes the items b, b + grid, ... (item = row i, 64 occupied columns
// s0.., 256 aux columns p0.., with the occupied tiles of one (i, p0) adjacent
// so the gathered DF rows are reused from L2). The CSR chunks of 16 partner
// rows (the K steps) of its items form one stream that cp.async copies
// KH_STAGES - 1 steps ahead of the DMMA tiles: the gathers of the next chunks,
// the tile math and the write-out of a finished item overlap. Each step's row
// indices are read one step earlier still, so no copy waits on an index load.
// Tiles and fragment layout are those of half_tile_dmma.
constexpr int KH_STAGES = 4;
constexpr int KH_AS = KH_S + 4, KH_BS = KH_P + 4;
constexpr int KH_STAGE_DOUBLES = KT_K * (KH_AS + KH_BS);
constexpr size_t KH_PIPE_SMEM = sizeof(double) * KH_STAGES * KH_STAGE_DOUBLES;

__device__ __forceinline__ void cp_async8(double *dst, const double *src, int bytes)
{
    const unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async16(double *dst, const double *src, int bytes)
{
    const unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

struct KhCursor {
    int item, i, s0, p0, r0, r_end, step, nsteps;
};

__device__ __forceinline__ void kh_set(KhCursor &c, int item, int n_items, int stiles, int ptiles,
                                       const int *__restrict__ displs)
{
    c.item = item;
    if (item >= n_items) return;
    const int per_row = stiles * ptiles;
    c.i = item / per_row;
    const int rem = item - c.i * per_row;
    c.p0 = (rem / stiles) * KH_P;
    c.s0 = (rem % stiles) * KH_S;
    c.r0 = displs[c.i];
    c.r_end = displs[c.i + 1];
    c.step = 0;
    c.nsteps = max(1, (c.r_end - c.r0 + KT_K - 1) / KT_K);   // a row without partners still writes its zeros
}

__device__ __forceinline__ void kh_next(KhCursor &c, int n_items, int stiles, int ptiles,
                                        const int *__restrict__ displs)
{
    if (c.item >= n_items) return;
    if (++c.step < c.nsteps) c.r0 += KT_K;
    else kh_set(c, c.item + gridDim.x, n_items, stiles, ptiles, displs);
}

// VEC: 16-byte copies of the DF rows (naux even, so every row starts 16-byte aligned)
template <bool VEC>
__global__ void __launch_bounds__(256, 1)
    k_halftransform_pipe(const double *__restrict__ B, const double *__restrict__ C, const int *__restrict__ csr_j,
                         const int *__restrict__ csr_u, const int *__restrict__ displs, int nocc, int naux,
                         double *__restrict__ T, int n_items, int stiles, int ptiles, unsigned long long *rowmax)
{
    extern __shared__ __align__(16) double khsm[];
    constexpr int NBR = VEC ? 8 : 16;   // DF rows whose copies this thread issues per step
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ws = (warp >> 2) * 32, wp = (warp & 3) * 64;
    const int fr = lane >> 2, fc = lane & 3;
    int iu[NBR], ij[4];
    KhCursor P, Q;   // P: the next step to copy; Q: the step the tiles consume
    kh_set(P, blockIdx.x, n_items, stiles, ptiles, displs);
    Q = P;
    auto load_idx = [&]() {   // row indices of P's step (-1: past the row, zero fill)
#pragma unroll
        for (int q = 0; q < NBR; q++) {
            const int r = P.r0 + (VEC ? 2 * q + (tid >> 7) : q);
            iu[q] = (P.item < n_items && r < P.r_end) ? csr_u[r] : -1;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int r = P.r0 + 4 * q + (tid >> 6);
            ij[q] = (P.item < n_items && r < P.r_end) ? csr_j[r] : -1;
        }
    };
    auto issue = [&](int buf) {   // copies of P's step into stage buffer buf, one commit group
        double *As = khsm + (size_t) buf * KH_STAGE_DOUBLES, *Bs = As + KT_K * KH_AS;
        if (P.item < n_items) {
#pragma unroll
            for (int q = 0; q < NBR; q++) {
                const int kk = VEC ? 2 * q + (tid >> 7) : q, cc = VEC ? (tid & 127) * 2 : tid;
                const int pg = P.p0 + cc;
                const bool ok = iu[q] >= 0 && pg < naux;
                const double *src = ok ? B + (size_t) iu[q] * naux + pg : B;
                if (VEC) cp_async16(&Bs[kk * KH_BS + cc], src, ok ? 16 : 0);
                else cp_async8(&Bs[kk * KH_BS + cc], src, ok ? 8 : 0);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int kk = 4 * q + (tid >> 6), cc = tid & 63, sg = P.s0 + cc;
                const bool ok = ij[q] >= 0 && sg < nocc;
                cp_async8(&As[kk * KH_AS + cc], ok ? C + (size_t) ij[q] * nocc + sg : C, ok ? 8 : 0);
            }
        }
        cp_async_commit();
    };
    for (int st = 0; st < KH_STAGES - 1; st++) {
        load_idx();
        issue(st);
        kh_next(P, n_items, stiles, ptiles, displs);
    }
    load_idx();
    double acc[4][8][2];
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 8; y++) acc[x][y][0] = acc[x][y][1] = 0.0;
    for (int g = 0; Q.item < n_items; g++) {
        cp_async_wait<KH_STAGES - 2>();   // this thread's copies of step g have landed
        __syncthreads();                  // everyone's have, and step g - 1's buffer is free
        issue((g + KH_STAGES - 1) % KH_STAGES);
        kh_next(P, n_items, stiles, ptiles, displs);
        load_idx();
        const double *As = khsm + (size_t) (g % KH_STAGES) * KH_STAGE_DOUBLES, *Bs = As + KT_K * KH_AS;
#pragma unroll
        for (int k4 = 0; k4 < KT_K; k4 += 4) {
            double a[4], b[8];
#pragma unroll
            for (int x = 0; x < 4; x++) a[x] = As[(k4 + fc) * KH_AS + ws + 8 * x + fr];
#pragma unroll
            for (int y = 0; y < 8; y++) b[y] = Bs[(k4 + fc) * KH_BS + wp + 8 * y + fr];
#pragma unroll
            for (int x = 0; x < 4; x++)
#pragma unroll
                for (int y = 0; y < 8; y++) dmma_8x8x4(acc[x][y][0], acc[x][y][1], a[x], b[y]);
        }
        if (++Q.step == Q.nsteps) {   // item done: write its tile, start the next
            double amax = 0.0;        // max |T| of the tile (padding entries are zero)
#pragma unroll
            for (int x = 0; x < 4; x++) {
                const int sg = Q.s0 + ws + 8 * x + fr;
                double *row = T + ((size_t) Q.i * nocc + (sg < nocc ? sg : 0)) * naux;
#pragma unroll
                for (int y = 0; y < 8; y++) {
                    const int pg = Q.p0 + wp + 8 * y + 2 * fc;
                    if (sg < nocc && pg < naux) row[pg] = acc[x][y][0];
                    if (sg < nocc && pg + 1 < naux) row[pg + 1] = acc[x][y][1];
                    amax = fmax(amax, fmax(fabs(acc[x][y][0]), fabs(acc[x][y][1])));
                    acc[x][y][0] = acc[x][y][1] = 0.0;
                }
            }
            if (rowmax) {   // row maxima for the integer-tensor-core K (non-negative: bit order = value order)
                for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffff, amax, o));
                if (lane == 0 && amax > 0.0) atomicMax(rowmax + Q.i, (unsigned long long) __double_as_longlong(amax));
            }
            kh_set(Q, Q.item + gridDim.x, n_items, stiles, ptiles, displs);
        }
    }
    cp_async_wait<0>();
}

// ---- the same half-transform with 168 x 128 tiles over 12 warps (3 x 4 warps
// of 56 x 32): n_occ up to 168 in one tile, so each CSR chunk of B is gathered
// once per (row, aux tile) instead of once per 64-wide occupied tile, and
// n_occ = 161 pads to 168 instead of 192.
constexpr int KH2_S = 168, KH2_P = 128, KH2_THREADS = 384;
constexpr int KH2_AS = KH2_S + 4, KH2_BS = KH2_P + 4;   // strides = 12 / 4 (mod 16) doubles: conflict-free fragments
constexpr int KH2_STAGE_DOUBLES = KT_K * (KH2_AS + KH2_BS);
constexpr size_t KH2_PIPE_SMEM = sizeof(double) * KH_STAGES * KH2_STAGE_DOUBLES;
constexpr int KH2_NA = KT_K * KH2_S / KH2_THREADS;   // 7 Cocc copies per thread per step

__device__ __forceinline__ void kh2_set(KhCursor &c, int item, int n_items, int stiles, int ptiles,
                                        const int *__restrict__ displs)
{
    c.item = item;
    if (item >= n_items) return;
    const int per_row = stiles * ptiles;
    c.i = item / per_row;
    const int rem = item - c.i * per_row;
    c.p0 = (rem / stiles) * KH2_P;
    c.s0 = (rem % stiles) * KH2_S;
    c.r0 = displs[c.i];
    c.r_end = displs[c.i + 1];
    c.step = 0;
    c.nsteps = max(1, (c.r_end - c.r0 + KT_K - 1) / KT_K);
}

__device__ __forceinline__ void kh2_next(KhCursor &c, int n_items, int stiles, int ptiles,
                                         const int *__restrict__ displs)
{
    if (c.item >= n_items) return;
    if (++c.step < c.nsteps) c.r0 += KT_K;
    else kh2_set(c, c.item + gridDim.x, n_items, stiles, ptiles, displs);
}

template <bool VEC>
__global__ void __launch_bounds__(KH2_THREADS, 1)
    k_halftransform_pipe2(const double *__restrict__ B, const double *__restrict__ C, const int *__restrict__ csr_j,
                          const int *__restrict__ csr_u, const int *__restrict__ displs, int nocc, int naux,
                          double *__restrict__ T, int n_items, int stiles, int ptiles, unsigned long long *rowmax)
{
    extern __shared__ __align__(16) double khsm[];
    constexpr int BCOPY = VEC ? 2 : 1;                                   // doubles per B copy
    constexpr int NBC = KT_K * KH2_P / BCOPY;                            // B copies per step
    constexpr int NB = (NBC + KH2_THREADS - 1) / KH2_THREADS;            // per thread
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ws = (warp >> 2) * 56, wp = (warp & 3) * 32;
    const int fr = lane >> 2, fc = lane & 3;
    int iu[NB], ij[KH2_NA];
    KhCursor P, Q;
    kh2_set(P, blockIdx.x, n_items, stiles, ptiles, displs);
    Q = P;
    auto load_idx = [&]() {
#pragma unroll
        for (int q = 0; q < NB; q++) {
            const int c = tid + KH2_THREADS * q;
            const int r = P.r0 + c / (KH2_P / BCOPY);
            iu[q] = (c < NBC && P.item < n_items && r < P.r_end) ? csr_u[r] : -1;
        }
#pragma unroll
        for (int q = 0; q < KH2_NA; q++) {
            const int r = P.r0 + (tid + KH2_THREADS * q) / KH2_S;
            ij[q] = (P.item < n_items && r < P.r_end) ? csr_j[r] : -1;
        }
    };
    auto issue = [&](int buf) {
        double *As = khsm + (size_t) buf * KH2_STAGE_DOUBLES, *Bs = As + KT_K * KH2_AS;
        if (P.item < n_items) {
#pragma unroll
            for (int q = 0; q < NB; q++) {
                const int c = tid + KH2_THREADS * q;
                if (c < NBC) {
                    const int kk = c / (KH2_P / BCOPY), cc = (c % (KH2_P / BCOPY)) * BCOPY;
                    const int pg = P.p0 + cc;
                    const bool ok = iu[q] >= 0 && pg < naux;
                    const double *src = ok ? B + (size_t) iu[q] * naux + pg : B;
                    if (VEC) cp_async16(&Bs[kk * KH2_BS + cc], src, ok ? 16 : 0);
                    else cp_async8(&Bs[kk * KH2_BS + cc], src, ok ? 8 : 0);
                }
            }
#pragma unroll
            for (int q = 0; q < KH2_NA; q++) {
                const int c = tid + KH2_THREADS * q;
                const int kk = c / KH2_S, cc = c % KH2_S, sg = P.s0 + cc;
                const bool ok = ij[q] >= 0 && sg < nocc;
                cp_async8(&As[kk * KH2_AS + cc], ok ? C + (size_t) ij[q] * nocc + sg : C, ok ? 8 : 0);
            }
        }
        cp_async_commit();
    };
    for (int st = 0; st < KH_STAGES - 1; st++) {
        load_idx();
        issue(st);
        kh2_next(P, n_items, stiles, ptiles, displs);
    }
    load_idx();
    double acc[7][4][2];
#pragma unroll
    for (int x = 0; x < 7; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y][0] = acc[x][y][1] = 0.0;
    for (int g = 0; Q.item < n_items; g++) {
        cp_async_wait<KH_STAGES - 2>();
        __syncthreads();
        issue((g + KH_STAGES - 1) % KH_STAGES);
        kh2_next(P, n_items, stiles, ptiles, displs);
        load_idx();
        const double *As = khsm + (size_t) (g % KH_STAGES) * KH2_STAGE_DOUBLES, *Bs = As + KT_K * KH2_AS;
#pragma unroll
        for (int k4 = 0; k4 < KT_K; k4 += 4) {
            double a[7], b[4];
#pragma unroll
            for (int x = 0; x < 7; x++) a[x] = As[(k4 + fc) * KH2_AS + ws + 8 * x + fr];
#pragma unroll
            for (int y = 0; y < 4; y++) b[y] = Bs[(k4 + fc) * KH2_BS + wp + 8 * y + fr];
#pragma unroll
            for (int x = 0; x < 7; x++)
#pragma unroll
                for (int y = 0; y < 4; y++) dmma_8x8x4(acc[x][y][0], acc[x][y][1], a[x], b[y]);
        }
        if (++Q.step == Q.nsteps) {
            double amax = 0.0;
#pragma unroll
            for (int x = 0; x < 7; x++) {
                const int sg = Q.s0 + ws + 8 * x + fr;
                double *row = T + ((size_t) Q.i * nocc + (sg < nocc ? sg : 0)) * naux;
#pragma unroll
                for (int y = 0; y < 4; y++) {
                    const int pg = Q.p0 + wp + 8 * y + 2 * fc;
                    if (sg < nocc && pg < naux) row[pg] = acc[x][y][0];
                    if (sg < nocc && pg + 1 < naux) row[pg + 1] = acc[x][y][1];
                    amax = fmax(amax, fmax(fabs(acc[x][y][0]), fabs(acc[x][y][1])));
                    acc[x][y][0] = acc[x][y][1] = 0.0;
                }
            }
            if (rowmax) {
                for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffff, amax, o));
                if (lane == 0 && amax > 0.0) atomicMax(rowmax + Q.i, (unsigned long long) __double_as_longlong(amax));
            }
            kh2_set(Q, Q.item + gridDim.x, n_items, stiles, ptiles, displs);
        }
    }
    cp_async_wait<0>();
}

// K partial tiles: upper tile pairs (bi <= bj) of 64x64, split over the
// flattened Q = nocc*naux index. Kpart[split][i][j].
__global__ void __launch_bounds__(256) k_syrk_part(const double *__restrict__ T, int nbf, long long Q, long long qchunk,
                                                   const int2 *__restrict__ tiles, double *__restrict__ Kpart)
{
    const int2 tl = tiles[blockIdx.x];
    const int split = blockIdx.y;
    const long long q_beg = (long long) split * qchunk, q_end = min(Q, q_beg + qchunk);
    syrk_tile(T, nbf, Q, q_beg, q_end, tl.x * KT_M, tl.y * KT_N, Kpart + (size_t) split * nbf * nbf);
}

__global__ void __launch_bounds__(256, 1) k_syrk_part128(const double *__restrict__ T, int nbf, long long Q,
                                                         long long qchunk, const int2 *__restrict__ tiles,
                                                         double *__restrict__ Kpart)
{
    const int2 tl = tiles[blockIdx.x];
    const int split = blockIdx.y;
    const long long q_beg = (long long) split * qchunk, q_end = min(Q, q_beg + qchunk);
    syrk_tile128(T, nbf, Q, q_beg, q_end, tl.x * KB_T, tl.y * KB_T, Kpart + (size_t) split * nbf * nbf);
}

__global__ void __launch_bounds__(256, 1) k_syrk_dmma(const double *__restrict__ T, int nbf, long long Q,
                                                      long long qchunk, const int2 *__restrict__ tiles,
                                                      double *__restrict__ Kpart)
{
    const int2 tl = tiles[blockIdx.x];
    const int split = blockIdx.y;
    const long long q_beg = (long long) split * qchunk, q_end = min(Q, q_beg + qchunk);
    syrk_tile_dmma(T, nbf, Q, q_beg, q_end, tl.x * KB_T, tl.y * KB_T, Kpart + (size_t) split * nbf * nbf);
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

void build_K_halftransform(const FockPlan &p, const double *d_Cocc, double *d_T, cudaStream_t s, int wide,
                           unsigned long long *d_rowmax)
{
    if (p.nbf <= 0 || p.nocc <= 0 || p.naux <= 0) return;   // T is empty: no grid to launch
    g_launches++;
    if (wide == 4) {
        if (d_rowmax) cudaMemsetAsync(d_rowmax, 0, sizeof(unsigned long long) * p.nbf, s);
        const int stiles = (p.nocc + KH2_S - 1) / KH2_S, ptiles = (p.naux + KH2_P - 1) / KH2_P;
        const long long items = (long long) p.nbf * stiles * ptiles;
        cudaFuncSetAttribute(k_halftransform_pipe2<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int) KH2_PIPE_SMEM);
        cudaFuncSetAttribute(k_halftransform_pipe2<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int) KH2_PIPE_SMEM);
        const int grid = (int) std::min<long long>(items, num_sms());
        if (p.naux % 2 == 0)
            k_halftransform_pipe2<true><<<grid, KH2_THREADS, KH2_PIPE_SMEM, s>>>(
                p.B, d_Cocc, p.csr_j, p.csr_u, p.csr_displs, p.nocc, p.naux, d_T, (int) items, stiles, ptiles, d_rowmax);
        else
            k_halftransform_pipe2<false><<<grid, KH2_THREADS, KH2_PIPE_SMEM, s>>>(
                p.B, d_Cocc, p.csr_j, p.csr_u, p.csr_displs, p.nocc, p.naux, d_T, (int) items, stiles, ptiles, d_rowmax);
    } else if (wide == 3) {
        if (d_rowmax) cudaMemsetAsync(d_rowmax, 0, sizeof(unsigned long long) * p.nbf, s);
        const int stiles = (p.nocc + KH_S - 1) / KH_S, ptiles = (p.naux + KH_P - 1) / KH_P;
        const long long items = (long long) p.nbf * stiles * ptiles;
        const int sms = num_sms();
        cudaFuncSetAttribute(k_halftransform_pipe<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int) KH_PIPE_SMEM);
        cudaFuncSetAttribute(k_halftransform_pipe<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int) KH_PIPE_SMEM);
        const int grid = (int) std::min<long long>(items, sms);
        if (p.naux % 2 == 0)
            k_halftransform_pipe<true><<<grid, 256, KH_PIPE_SMEM, s>>>(p.B, d_Cocc, p.csr_j, p.csr_u, p.csr_displs,
                                                                       p.nocc, p.naux, d_T, (int) items, stiles,
                                                                       ptiles, d_rowmax);
        else
            k_halftransform_pipe<false><<<grid, 256, KH_PIPE_SMEM, s>>>(p.B, d_Cocc, p.csr_j, p.csr_u,
                                                                        p.csr_displs, p.nocc, p.naux, d_T,
                                                                        (int) items, stiles, ptiles, d_rowmax);
    } else if (wide) {
        dim3 g1((p.naux + KH_P - 1) / KH_P, (p.nocc + KH_S - 1) / KH_S, p.nbf);
        if (wide == 2)
            k_halftransform_dmma<<<g1, 256, 0, s>>>(p.B, d_Cocc, p.csr_j, p.csr_u, p.csr_displs, p.nocc, p.naux, d_T);
        else
            k_halftransform_wide<<<g1, 256, 0, s>>>(p.B, d_Cocc, p.csr_j, p.csr_u, p.csr_displs, p.nocc, p.naux, d_T);
    } else {
        dim3 g1((p.naux + KT_N - 1) / KT_N, (p.nocc + KT_M - 1) / KT_M, p.nbf);
        k_halftransform<<<g1, 256, 0, s>>>(p.B, d_Cocc, p.csr_j, p.csr_u, p.csr_displs, p.nocc, p.naux, d_T);
    }
}

void build_K_syrk(const FockPlan &p, const double *d_T, double *d_K, double *d_Kpart, int ksplit, const int2 *d_tiles,
                  cudaStream_t s, int tile)
{
    const int tdim = tile == KSYRK_DMMA ? KB_T : tile;
    const int nt = (p.nbf + tdim - 1) / tdim;
    const int ntiles = nt * (nt + 1) / 2;
    const long long Q = (long long) p.nocc * p.naux;
    long long qchunk = (Q + ksplit - 1) / ksplit;
    qchunk = (qchunk + KT_K - 1) / KT_K * KT_K;
    dim3 g2(ntiles, ksplit);
    g_launches += 2;
    if (tile == KSYRK_DMMA) k_syrk_dmma<<<g2, 256, 0, s>>>(d_T, p.nbf, Q, qchunk, d_tiles, d_Kpart);
    else if (tile == KB_T) k_syrk_part128<<<g2, 256, 0, s>>>(d_T, p.nbf, Q, qchunk, d_tiles, d_Kpart);
    else k_syrk_part<<<g2, 256, 0, s>>>(d_T, p.nbf, Q, qchunk, d_tiles, d_Kpart);
    size_t nn = (size_t) p.nbf * p.nbf;
    k_syrk_reduce<<<(unsigned) ((nn + 255) / 256), 256, 0, s>>>(d_Kpart, ksplit, p.nbf, d_K);
}

// ------------------------------------------------------------------ F and energy
__global__ void k_fock_energy(const double *H, const double *J, const double *K, const double *D, double *F,
                              double *epart, size_t n)
{
    double e = fock_energy_range(H, J, K, D, F, (size_t) blockIdx.x * blockDim.x + threadIdx.x, n,
                                 (size_t) gridDim.x * blockDim.x);
    e = block_sum(e);
    if (threadIdx.x == 0) epart[blockIdx.x] = e;
}

void build_F_energy(const double *d_H, const double *d_J, const double *d_K, const double *d_D, double *d_F,
                    double *d_epart, int n, cudaStream_t s)
{
    g_launches++;
    k_fock_energy<<<ENERGY_BLOCKS, 256, 0, s>>>(d_H, d_J, d_K, d_D, d_F, d_epart, (size_t) n * n);
}

}  // namespace tscf
