// The exchange's rank-k product K = T T^T (build_Fock.c:317-341) in FP64
// accuracy on the integer tensor cores, by Ozaki scheme II (H. Ozaki,
// Y. Uchino, T. Imamura, "Ozaki Scheme II: A GEMM-oriented emulation of
// floating-point matrix multiplication using an integer modular technique",
// 2025):
//
//  1. row i of T is scaled by 2^(beta - e_i), max_q |T_iq| < 2^e_i, and
//     rounded to an integer X_iq with |X_iq| <= 2^beta (k_oz_rowexp,
//     k_oz_residues);
//  2. for each of the pairwise coprime moduli m_k <= 256 the signed residues
//     X mod m_k, in [-128, 127], are stored as int8 planes (k_oz_residues);
//  3. over K ranges of at most 130944 terms, sum_q (X_iq mod m_k)(X_jq mod m_k)
//     is exact in int32 (tcgen05.mma.kind::i8 into tensor memory) and is
//     reduced mod m_k to one byte per element (k_oz_gemm);
//  4. the Chinese remainder theorem gives each range's exact integer
//     sum_q X_iq X_jq (its magnitude is below M / 2, M = prod m_k), the ranges
//     are added in 128-bit integers and the total is rounded once to FP64 and
//     scaled by 2^(e_i + e_j - 2 beta) (k_oz_crt).
// With 15 moduli M ~ 2^117.8 and beta = 49: the only rounding before the final
// one is step 1's, 2^-50 of each row's largest element.
//
// k_oz_gemm: 256 x 256 output tiles over the upper triangle, one CTA pair
// (tcgen05 cta_group::2) per (tile, K range); in each CTA warp 0 issues the TMA
// loads of its halves of both residue tiles (128 B of K per stage), warp 1 of
// rank 0 the MMAs (M = 256, N = 256, K = 32 per instruction) of modulus k into
// TMEM buffer k & 1, warps 2-9 reduce the other buffer mod its modulus and
// store the bytes, so the drain overlaps the next modulus' MMAs. All mbarrier
// waits are bounded; a timeout sets an error flag instead of hanging.
#include <cuda.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <vector>

#include "tscf_internal.h"
#include "umma.cuh"

namespace tscf {

namespace {

using namespace umma;
typedef unsigned __int128 u128;

constexpr int OZ_MODULI[] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197};
constexpr int OZ_NMAX = 15;
constexpr int OM = 128;                 // tile rows per CTA (a CTA pair's MMA has M = 256)
constexpr int ON = 256;                 // tile columns (UMMA N); tiles are 256 x 256 per pair
constexpr int OKB = 128;                // K bytes per pipeline stage (one 128-byte swizzle row)
constexpr int OZ_MAX_CHUNKS = 1023;     // K range <= 1023 * 128 = 130944 terms: |sum| < 2^31
constexpr int OZ_STAGES = 6;
constexpr int OZ_EPI_WARPS = 8;         // two warps per TMEM lane quadrant, 128 columns each
constexpr int OZ_THREADS = 64 + 32 * OZ_EPI_WARPS;
constexpr int OZ_A_BYTES = OM * OKB, OZ_B_BYTES = (ON / 2) * OKB;   // per CTA of a pair: 128 rows each
constexpr int OZ_STAGE_BYTES = OZ_A_BYTES + OZ_B_BYTES;
constexpr int OZ_SMEM = OZ_STAGES * OZ_STAGE_BYTES + 1024 + 8 * (2 * OZ_STAGES + 4) + 16;
static_assert(OZ_SMEM <= 227 * 1024, "Ozaki GEMM stages exceed shared memory");
constexpr long long OZ_WAIT_CYCLES = 4000000000LL;   // ~2 s at 2 GHz
constexpr double MAGIC = 6755399441055744.0;        // 1.5 * 2^52: x + MAGIC rounds x to an integer

__device__ int g_oz_error;
__constant__ double c_m[OZ_NMAX], c_inv[OZ_NMAX];
__constant__ int c_mi[OZ_NMAX], c_y[OZ_NMAX];
__constant__ unsigned long long c_Mk[OZ_NMAX][2], c_M[2];

// kind::i8 instruction descriptor: S8 x S8 -> S32 (no saturation), K-major, M = m, N = n.
__host__ __device__ constexpr uint32_t idesc_s8(int m, int n)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (n >> 3) << 17) | ((uint32_t) (m >> 4) << 24);
}

__device__ __forceinline__ void umma_s8_pair(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

// e[i] with max_q |T_iq| < 2^e[i] (0 for a zero row).
__global__ void __launch_bounds__(1024) k_oz_rowexp(const double *__restrict__ T, long long Q, int *e)
{
    __shared__ double sh[32];
    const double *row = T + (size_t) blockIdx.x * Q;
    double m = 0.0;
    for (long long q = threadIdx.x; q < Q; q += blockDim.x) m = fmax(m, fabs(row[q]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffff, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffff, m, o));
        if (threadIdx.x == 0) {
            int ex = 0;
            if (m > 0.0) frexp(m, &ex);   // m = f 2^ex, 0.5 <= f < 1
            e[blockIdx.x] = ex;
        }
    }
}

// e[i] from row maxima given as double bits.
__global__ void k_oz_exp_from_max(const unsigned long long *__restrict__ rowmax, int nbf, int *e)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbf) return;
    const double m = __longlong_as_double((long long) rowmax[i]);
    int ex = 0;
    if (m > 0.0) frexp(m, &ex);
    e[i] = ex;
}

// Residue planes R[k][i][q] (pitch Qp, q >= Q zero) of X_iq = rint(T_iq 2^(beta - e_i)).
// One thread per 16 consecutive q of a row; q = fma(x, 1/m, MAGIC) - MAGIC is
// round(x / m) (|x / m| < 2^51; for odd m, x / m is at least 1/(2m) from a
// half-integer, far more than the 2^-53 relative error of 1/m), r = x - q m is
// exact, and the low byte of r + MAGIC is r as int8.
__global__ void __launch_bounds__(256) k_oz_residues(const double *__restrict__ T, int nbf, long long Q, long long Qp,
                                                     int rows_pad, const int *__restrict__ e, int beta, int nmod,
                                                     int8_t *__restrict__ R)
{
    const long long groups = Qp / 16, total = (long long) nbf * groups;
    const size_t plane = (size_t) rows_pad * Qp;
    for (long long g = (long long) blockIdx.x * blockDim.x + threadIdx.x; g < total;
         g += (long long) gridDim.x * blockDim.x) {
        const int i = (int) (g / groups);
        const long long q0 = (g % groups) * 16;
        const double scale = ldexp(1.0, beta - e[i]);
        const double *src = T + (size_t) i * Q + q0;
        double x[16];
        if (q0 + 16 <= Q && (((size_t) i * Q + q0) & 1) == 0) {
#pragma unroll
            for (int j = 0; j < 16; j += 2) {
                const double2 v = __ldcs((const double2 *) (src + j));
                x[j] = v.x;
                x[j + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 16; j++) x[j] = q0 + j < Q ? __ldcs(src + j) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] = __dadd_rn(__fma_rn(x[j], scale, MAGIC), -MAGIC);
        int8_t *dst = R + (size_t) i * Qp + q0;
        for (int k = 0; k < nmod; k++) {
            const double m = c_m[k], inv = c_inv[k];
            uint32_t w[4];
#pragma unroll
            for (int j4 = 0; j4 < 4; j4++) {
                uint32_t word = 0;
#pragma unroll
                for (int b = 0; b < 4; b++) {
                    const double xv = x[4 * j4 + b];
                    const double q = __dadd_rn(__fma_rn(xv, inv, MAGIC), -MAGIC);
                    const double r = __fma_rn(-q, m, xv);
                    const uint32_t byte = (uint32_t) __double2loint(__dadd_rn(r, MAGIC)) & 0xffu;
                    word |= byte << (8 * b);
                }
                w[j4] = word;
            }
            *(uint4 *) (dst + (size_t) k * plane) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

struct OzArgs {
    const int2 *tiles;       // upper tiles (row block, column block) of 256
    uint8_t *res;            // [ksplit][nmod][rows_pad][rows_pad] residues of the range sums
    int rows_pad, nmod, chunks_per_split, total_chunks;
    long long wait_cycles;
};

// One 256 x 256 tile per CTA pair (clusters of 2 along x): CTA r loads rows
// 128 r .. + 127 of the tile's row block (A) and of its column block (B) of
// residue plane k; rank 0 issues M = 256, N = 256 MMAs reading both CTAs'
// tiles, each CTA's tensor memory receives its 128 rows. Rank 0's stage-full
// barrier counts both CTAs' copies; its commits arrive at the stage-empty and
// accumulator-full barriers of both CTAs; both CTAs' epilogue warps arrive at
// rank 0's accumulator-empty barrier.
__global__ void __launch_bounds__(OZ_THREADS, 1)
k_oz_gemm(const __grid_constant__ CUtensorMap mR, OzArgs a)
{
    constexpr uint32_t TMEM_COLS = 512;
    constexpr uint32_t idesc = idesc_s8(2 * OM, ON);
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *) (((uintptr_t) smem_raw + 1023) & ~(uintptr_t) 1023);
    uint64_t *full = (uint64_t *) (smem + OZ_STAGES * OZ_STAGE_BYTES);
    uint64_t *empty = full + OZ_STAGES;
    uint64_t *tfull = empty + OZ_STAGES;   // [2] accumulator buffer ready (both CTAs)
    uint64_t *tempty = tfull + 2;          // [2] accumulator buffer drained (rank 0's counts both CTAs)
    uint32_t *tmem_slot = (uint32_t *) (tempty + 2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const int2 tile = a.tiles[blockIdx.x >> 1];
    const int m0 = tile.x * ON + (int) rank * OM, n0 = tile.y * ON, split = blockIdx.y;
    const int nb_own = n0 + (int) rank * OM;
    const int kc0 = split * a.chunks_per_split;
    const int nk = max(0, min(a.total_chunks, kc0 + a.chunks_per_split) - kc0);
    const int nit = nk * a.nmod;

    if (threadIdx.x == 0) {
        for (int s = 0; s < OZ_STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 2 * OZ_EPI_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc_pair(tmem_slot, TMEM_COLS);
    fence_before_sync();
    __syncthreads();
    cluster_sync();   // both CTAs' barriers exist before either signals the other's
    fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        const uint32_t full0 = mapa_shared(smem_u32(&full[0]), 0);   // rank 0's stage-full barriers
        bool ok = true;
        for (int it = 0; it < nit && ok; it++) {
            const int s = it % OZ_STAGES, k = it / nk, kb = it % nk;
            if (it >= OZ_STAGES) ok = mbar_wait_bounded(&empty[s], ((it / OZ_STAGES) - 1) & 1, &g_oz_error, 21,
                                                        a.wait_cycles);
            if (!ok) break;
            if (rank == 0) mbar_expect_tx(&full[s], 2 * OZ_STAGE_BYTES);
            unsigned char *st = smem + s * OZ_STAGE_BYTES;
            const int kx = (kc0 + kb) * OKB;
            const uint32_t bar = full0 + 8u * (uint32_t) s;
            tma_load_2d_pair(st, &mR, bar, kx, k * a.rows_pad + m0);
            tma_load_2d_pair(st + OZ_A_BYTES, &mR, bar, kx, k * a.rows_pad + nb_own);
        }
        // the pair's MMAs have consumed (so the copies have landed in) the last stages
        for (int it = (nit > OZ_STAGES ? nit - OZ_STAGES : 0); it < nit && ok; it++)
            mbar_wait_bounded(&empty[it % OZ_STAGES], (it / OZ_STAGES) & 1, &g_oz_error, 22, a.wait_cycles);
    } else if (warp == 1 && lane == 0 && rank == 0) {
        bool ok = true;
        int it = 0;
        for (int k = 0; k < a.nmod && ok && nk > 0; k++) {
            const int b = k & 1;
            if (k >= 2) ok = mbar_wait_bounded(&tempty[b], ((k >> 1) - 1) & 1, &g_oz_error, 23, a.wait_cycles);
            if (!ok) break;
            fence_after_sync();
            const uint32_t acc = tmem + b * ON;
            for (int kb = 0; kb < nk && ok; kb++, it++) {
                const int s = it % OZ_STAGES;
                ok = mbar_wait_bounded(&full[s], (it / OZ_STAGES) & 1, &g_oz_error, 24, a.wait_cycles);
                if (!ok) break;
                fence_after_sync();
                const uint32_t sa = smem_u32(smem + s * OZ_STAGE_BYTES), sb = sa + OZ_A_BYTES;
#pragma unroll
                for (int kk = 0; kk < OKB / 32; kk++)
                    umma_s8_pair(acc, desc_sw128(sa + kk * 32), desc_sw128(sb + kk * 32), idesc,
                                 (kb > 0 || kk > 0) ? 1u : 0u);
                umma_commit_pair(&empty[s], 0x3);
            }
            umma_commit_pair(&tfull[b], 0x3);
        }
    } else if (warp >= 2) {
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const int row = quad * 32 + lane;
        const uint32_t tq = tmem + ((uint32_t) (quad * 32) << 16) + half * 128;
        const uint32_t tempty0 = mapa_shared(smem_u32(&tempty[0]), 0);
        bool ok = true;
        for (int k = 0; k < a.nmod && ok && nk > 0; k++) {
            const int b = k & 1;
            ok = mbar_wait_bounded(&tfull[b], (k >> 1) & 1, &g_oz_error, 25, a.wait_cycles);
            if (!ok) break;
            fence_after_sync();
            const int m = c_mi[k];
            uint8_t *dst = a.res + (((size_t) split * a.nmod + k) * a.rows_pad + m0 + row) * a.rows_pad + n0 + half * 128;
#pragma unroll 1
            for (int c0 = 0; c0 < 128; c0 += 64) {
                uint32_t r0[32], r1[32];
                tmem_ld32_nowait(tq + b * ON + c0, r0);
                tmem_ld32_nowait(tq + b * ON + c0 + 32, r1);
                tmem_wait_ld();
                uint32_t w[16];
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    uint32_t word = 0;
#pragma unroll
                    for (int t = 0; t < 4; t++) {
                        const int c = 4 * q + t;
                        int v = (int) (c < 32 ? r0[c] : r1[c - 32]) % m;
                        v += v < 0 ? m : 0;
                        word |= (uint32_t) v << (8 * t);
                    }
                    w[q] = word;
                }
#pragma unroll
                for (int q = 0; q < 16; q += 4) *(uint4 *) (dst + c0 + 4 * q) = make_uint4(w[q], w[q + 1], w[q + 2], w[q + 3]);
            }
            fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(tempty0 + 8u * (uint32_t) b);
        }
    }
    fence_before_sync();
    __syncthreads();
    cluster_sync();   // the pair's MMAs, commits and remote arrivals are over
    if (warp == 1) {
        fence_after_sync();
        tmem_dealloc_pair(tmem, TMEM_COLS);
    }
}

__device__ __forceinline__ double u128_to_double(u128 x)
{
    return (double) (unsigned long long) (x >> 64) * 18446744073709551616.0 + (double) (unsigned long long) x;
}

// K[i][j] = K[j][i] for i <= j: per K range the CRT value of its residues in
// (-M/2, M/2), the ranges summed exactly in 128 bits, then one rounding.
__global__ void k_oz_crt(const uint8_t *__restrict__ res, int nsplit, int nmod, int rows_pad, int nbf,
                         const int *__restrict__ e, int beta, double *K)
{
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long) nbf * nbf) return;
    const int i = (int) (idx / nbf), j = (int) (idx % nbf);
    if (i > j) return;
    const u128 M = ((u128) c_M[1] << 64) | c_M[0];
    const u128 half = M >> 1;
    u128 pos = 0, neg = 0;   // total = pos - neg
    for (int r = 0; r < nsplit; r++) {
        u128 acc = 0;
        for (int k = 0; k < nmod; k++) {
            const uint32_t v = res[(((size_t) r * nmod + k) * rows_pad + i) * rows_pad + j];
            const uint32_t s = (v * (uint32_t) c_y[k]) % (uint32_t) c_mi[k];
            acc += (u128) s * (((u128) c_Mk[k][1] << 64) | c_Mk[k][0]);
            if (acc >= M) acc -= M;
        }
        if (acc > half) neg += M - acc;
        else pos += acc;
    }
    const double v = pos >= neg ? u128_to_double(pos - neg) : -u128_to_double(neg - pos);
    const double kv = ldexp(v, e[i] + e[j] - 2 * beta);
    K[(size_t) i * nbf + j] = kv;
    K[(size_t) j * nbf + i] = kv;
}

int oz_nmod_default()
{
    static const int n = [] {
        const char *v = getenv("TINYSCF_OZAKI_MODULI");
        const int c = v ? atoi(v) : OZ_NMAX;
        return (c >= 8 && c <= OZ_NMAX) ? c : OZ_NMAX;
    }();
    return n;
}

}  // namespace

struct OzSyrk {
    int nbf = 0, nmod = 0, beta = 0, rows_pad = 0, ntiles = 0, ksplit = 1, cps = 1, total_chunks = 0, nsm = 1;
    long long Q = 0, Qp = 0;
    int *e = nullptr;
    unsigned long long *rowmax = nullptr;
    int8_t *R = nullptr;
    uint8_t *res = nullptr;
    int2 *tiles = nullptr;
    CUtensorMap mR;
};

void oz_destroy(OzSyrk *o)
{
    if (!o) return;
    for (void *p : {(void *) o->e, (void *) o->rowmax, (void *) o->R, (void *) o->res, (void *) o->tiles})
        dev_free(p, 0);
    cudaStreamSynchronize(0);
    delete o;
}

// The exact product bound: each range sum is below Qr 2^(2 beta) with Qr < 2^17,
// so beta = floor((log2 M - 18) / 2) keeps it below M / 2.
static int oz_constants(int nmod, cudaStream_t s, int *log2M)
{
    u128 M = 1;
    for (int k = 0; k < nmod; k++) M *= (u128) OZ_MODULI[k];
    double hm[OZ_NMAX], hinv[OZ_NMAX];
    int hmi[OZ_NMAX], hy[OZ_NMAX];
    unsigned long long hMk[OZ_NMAX][2], hM[2] = {(unsigned long long) M, (unsigned long long) (M >> 64)};
    for (int k = 0; k < nmod; k++) {
        const int m = OZ_MODULI[k];
        const u128 Mk = M / (u128) m;
        const int r = (int) (Mk % (u128) m);
        int y = 0;
        for (int c = 1; c < m; c++)
            if ((r * c) % m == 1) {
                y = c;
                break;
            }
        if (!y) return ERR_UNSUPPORTED;
        hm[k] = m;
        hinv[k] = 1.0 / m;
        hmi[k] = m;
        hy[k] = y;
        hMk[k][0] = (unsigned long long) Mk;
        hMk[k][1] = (unsigned long long) (Mk >> 64);
    }
    TSCF_CUDA_CHECK(cudaMemcpyToSymbolAsync(c_m, hm, sizeof(double) * nmod, 0, cudaMemcpyHostToDevice, s));
    TSCF_CUDA_CHECK(cudaMemcpyToSymbolAsync(c_inv, hinv, sizeof(double) * nmod, 0, cudaMemcpyHostToDevice, s));
    TSCF_CUDA_CHECK(cudaMemcpyToSymbolAsync(c_mi, hmi, sizeof(int) * nmod, 0, cudaMemcpyHostToDevice, s));
    TSCF_CUDA_CHECK(cudaMemcpyToSymbolAsync(c_y, hy, sizeof(int) * nmod, 0, cudaMemcpyHostToDevice, s));
    TSCF_CUDA_CHECK(cudaMemcpyToSymbolAsync(c_Mk, hMk, sizeof(hMk[0]) * nmod, 0, cudaMemcpyHostToDevice, s));
    TSCF_CUDA_CHECK(cudaMemcpyToSymbolAsync(c_M, hM, sizeof(hM), 0, cudaMemcpyHostToDevice, s));
    int lg = 0;
    while (lg < 127 && (M >> (lg + 1)) != 0) lg++;   // floor(log2 M)
    *log2M = lg;
    return OK;
}

int oz_create(OzSyrk **out, int nbf, long long Q, cudaStream_t s)
{
    *out = nullptr;
    if (nbf <= 0 || Q <= 0) return ERR_INPUT;
    OzSyrk *o = new OzSyrk();
    o->nbf = nbf;
    o->Q = Q;
    o->nmod = oz_nmod_default();
    int lg = 0;
    const int crc = oz_constants(o->nmod, s, &lg);
    if (crc != OK) {
        oz_destroy(o);
        return crc;
    }
    o->beta = std::min(50, (lg - 18) / 2);   // q = round(x / m) stays exact for beta <= 50
    o->rows_pad = (nbf + ON - 1) / ON * ON;
    o->Qp = (Q + OKB - 1) / OKB * OKB;
    o->total_chunks = (int) (o->Qp / OKB);
    std::vector<int2> tl;
    for (int bj = 0; bj * ON < nbf; bj++)
        for (int bi = 0; bi <= bj; bi++) tl.push_back(make_int2(bi, bj));
    o->ntiles = (int) tl.size();
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 1;
    o->nsm = nsm;
    // K ranges: at most OZ_MAX_CHUNKS chunks each, and about one CTA per SM in total
    const int ks_min = (o->total_chunks + OZ_MAX_CHUNKS - 1) / OZ_MAX_CHUNKS;
    int ks = std::max(ks_min, nsm / (2 * o->ntiles));
    ks = std::max(1, std::min(ks, o->total_chunks));
    o->cps = (o->total_chunks + ks - 1) / ks;
    o->ksplit = (o->total_chunks + o->cps - 1) / o->cps;
    const size_t rbytes = (size_t) o->nmod * o->rows_pad * o->Qp;
    const size_t sbytes = (size_t) o->ksplit * o->nmod * o->rows_pad * o->rows_pad;
    if (dev_malloc((void **) &o->e, sizeof(int) * nbf, s) != OK ||
        dev_malloc((void **) &o->rowmax, sizeof(unsigned long long) * nbf, s) != OK ||
        dev_malloc((void **) &o->R, rbytes, s) != OK || dev_malloc((void **) &o->res, sbytes, s) != OK ||
        dev_malloc((void **) &o->tiles, sizeof(int2) * tl.size(), s) != OK) {
        oz_destroy(o);
        return ERR_ALLOC;
    }
    // rows nbf .. rows_pad-1 of every plane stay zero
    TSCF_CUDA_CHECK(cudaMemsetAsync(o->R, 0, rbytes, s));
    TSCF_CUDA_CHECK(cudaMemcpyAsync(o->tiles, tl.data(), sizeof(int2) * tl.size(), cudaMemcpyHostToDevice, s));
    const long long rows = (long long) o->nmod * o->rows_pad;
    if (!make_map_2d(&o->mR, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, o->R, rows, o->Qp, o->Qp, OKB, OM)) {
        oz_destroy(o);
        return ERR_CUDA;
    }
    if (cudaFuncSetAttribute(k_oz_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, OZ_SMEM) != cudaSuccess) {
        cudaGetLastError();
        oz_destroy(o);
        return ERR_CUDA;
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        oz_destroy(o);
        return ERR_CUDA;
    }
    *out = o;
    return OK;
}

unsigned long long *oz_rowmax(OzSyrk *o) { return o ? o->rowmax : nullptr; }

int oz_syrk(OzSyrk *o, const double *d_T, double *d_K, cudaStream_t s, const unsigned long long *d_rowmax)
{
    if (!o) return ERR_STATE;
    if (d_rowmax) k_oz_exp_from_max<<<(o->nbf + 255) / 256, 256, 0, s>>>(d_rowmax, o->nbf, o->e);
    else k_oz_rowexp<<<o->nbf, 1024, 0, s>>>(d_T, o->Q, o->e);
    k_oz_residues<<<o->nsm * 8, 256, 0, s>>>(d_T, o->nbf, o->Q, o->Qp, o->rows_pad, o->e, o->beta, o->nmod, o->R);
    OzArgs a{o->tiles, o->res, o->rows_pad, o->nmod, o->cps, o->total_chunks, OZ_WAIT_CYCLES};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * o->ntiles, o->ksplit);
    cfg.blockDim = dim3(OZ_THREADS);
    cfg.dynamicSmemBytes = OZ_SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, k_oz_gemm, o->mR, a) != cudaSuccess) return ERR_CUDA;
    const long long nn = (long long) o->nbf * o->nbf;
    k_oz_crt<<<(unsigned) ((nn + 255) / 256), 256, 0, s>>>(o->res, o->ksplit, o->nmod, o->rows_pad, o->nbf, o->e,
                                                          o->beta, d_K);
    g_launches += 4;
    return cuda_launch_rc("Ozaki rank-k product");
}

int oz_error_flag()
{
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_oz_error, sizeof(int));
    return v;
}

void oz_info(const OzSyrk *o, int info[6])
{
    info[0] = o->nmod;
    info[1] = o->beta;
    info[2] = o->ntiles;
    info[3] = o->ksplit;
    info[4] = o->cps;
    info[5] = o->rows_pad;
}

}  // namespace tscf
