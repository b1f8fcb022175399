// Mixed-precision exchange (K) on the 5th-generation tensor cores (tcgen05).
//
// Two warp-specialised UMMA kernels with K-major BF16 operands staged by TMA
// (128-byte swizzle) and FP32 accumulators in tensor memory. Every FP64/FP32
// operand x is split into x_hi = bf16(x), x_lo = bf16(x - x_hi); a product
// uses three MMAs (hi*hi + hi*lo + lo*hi; the half-transform adds lo*lo),
// which keeps ~16 significant bits per operand.
//
// The K build is incremental (build_Fock.c:244-347 restated on differences):
//   C'_n  = C_n R,  R = polar(C_n^T S C_{n-1})       (align the occupied orbitals)
//   dC    = C'_n - C_{n-1}
//   dT    = half-transform(dC)                         (k_half: persistent, per CSR row i)
//   T_n   = T_{n-1} + dT,  S_T = T_n + T_{n-1}
//   K_n   = K_{n-1} + sym(dT S_T^T)                    (k_gemm: split-K)
// so that T_n T_n^T - T_{n-1} T_{n-1}^T is formed from dT: the low-precision
// error of each increment scales with |dC| ~ |dD| and vanishes as the SCF
// converges. K_n is accumulated in FP64.
//
// Warp roles (320 threads): warp 0 issues TMA loads, warp 1 allocates tensor
// memory and issues the MMAs, warps 2-9 drain the accumulators (two warps per
// TMEM lane quadrant warp_id % 4, each taking half of the columns). All
// mbarrier waits are bounded; a timeout sets an error flag instead of hanging.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <vector>

#include "tscf_internal.h"
#include "umma.cuh"

namespace tscf {

namespace {

constexpr int UM = 128;          // UMMA M (rows of A per CTA)
constexpr int BK = 64;           // K per pipeline stage (one 128-byte swizzle row of BF16)
constexpr int UK = 16;           // K per tcgen05.mma.kind::f16
constexpr long long WAIT_CYCLES = 4000000000LL;   // ~2 s at 2 GHz

__device__ int g_umma_error;     // set to a nonzero code when a bounded wait times out

using namespace umma;

// Bounded wait on an mbarrier phase (at most `limit` clock cycles). Returns
// false (and records code in g_umma_error) on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t phase, int code, long long limit = WAIT_CYCLES)
{
    return mbar_wait_bounded(bar, phase, &g_umma_error, code, limit);
}

// kind::f16 instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_bf16(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (n >> 3) << 17) | ((uint32_t) (UM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16 &hi, __nv_bfloat16 &lo)
{
    hi = __float2bfloat16_rn(x);
    lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

struct HalfArgs {            // half-transform work items: (CSR row, 128-row block of P)
    const int *row_chunk0;   // [nbf+1] first 64-chunk of each padded CSR row
    float *Tm;               // T master [nbf][Qp] FP32
    __nv_bfloat16 *dTh, *dTl, *Sh, *Sl;   // [nbf][Qp]
    int nocc, naux;
    long long Qp;
    int n_items, ptiles;     // nbf * ptiles items, ptiles = ceil(naux / 128)
};
struct GArgs {               // split-K partial of dT S^T
    double *part;            // [ksplit][nbf][nbf]
    int nbf;
    int chunks_per_split;
    int total_chunks;
    // Bounded-wait check (kmix_wait_probe): probe != 0 issues no copies, so the
    // MMA and epilogue waits run out after wait_cycles with nothing in flight.
    int probe = 0;
    long long wait_cycles = WAIT_CYCLES;
};

constexpr int EPI_WARPS = 8;                  // two warps per TMEM lane quadrant
constexpr int THREADS = 64 + 32 * EPI_WARPS;  // TMA warp, MMA warp, epilogue warps
constexpr int SEG_CHUNKS = 4;                 // G: drain the accumulator every 256 K
constexpr int MAX_SEGS = 64;                  // G: at most 64 segment results summed in FP32 registers per split

// One k-chunk (64 K) of split-BF16 MMAs: hi*hi into acc_main, hi*lo + lo*hi
// into acc_corr. Keeping the small correction terms apart means the large
// accumulator takes one FP32 addition per 16 K instead of three.
template <bool LOLO>
__device__ __forceinline__ void mma_chunk(uint32_t a_hi, uint32_t a_lo, uint32_t b_hi, uint32_t b_lo, uint32_t acc_main,
                                          uint32_t acc_corr, uint32_t idesc, bool first)
{
#pragma unroll
    for (int kk = 0; kk < BK / UK; kk++) {
        const uint32_t off = kk * UK * 2;   // bytes along K inside the 128-byte row
        const uint64_t dah = desc_sw128(a_hi + off), dal = desc_sw128(a_lo + off);
        const uint64_t dbh = desc_sw128(b_hi + off), dbl = desc_sw128(b_lo + off);
        const uint32_t acc = (first && kk == 0) ? 0u : 1u;
        umma_bf16(acc_main, dah, dbh, idesc, acc);
        umma_bf16(acc_corr, dah, dbl, idesc, acc);
        umma_bf16(acc_corr, dal, dbh, idesc, 1u);
        if (LOLO) umma_bf16(acc_corr, dal, dbl, idesc, 1u);
    }
}

// ------------------------------------------------------------------ half-transform
// Persistent: CTA b takes work items b, b + gridDim.x, ...; item t covers aux
// rows P = 128 (t % ptiles) .. +127 of CSR row i = t / ptiles:
//   D[P][s] = sum_r BpT[P][r] CgT[s][r] over the padded CSR row i.
// The TMA warp runs ahead across items through the shared-memory stages; the
// MMA warp accumulates item t in TMEM buffer t & 1 while the epilogue warps
// update T and write the BF16 operands of the G GEMM from the other buffer,
// so the epilogue's global traffic overlaps the next item's loads and MMAs.
// All four split products go into one FP32 accumulator: a CSR row has at most
// a few hundred terms.
template <bool FIRST>
__device__ __forceinline__ void mma_chunk4(uint32_t a_hi, uint32_t a_lo, uint32_t b_hi, uint32_t b_lo, uint32_t acc,
                                           uint32_t idesc)
{
#pragma unroll
    for (int kk = 0; kk < BK / UK; kk++) {
        const uint32_t off = kk * UK * 2;
        const uint64_t dah = desc_sw128(a_hi + off), dal = desc_sw128(a_lo + off);
        const uint64_t dbh = desc_sw128(b_hi + off), dbl = desc_sw128(b_lo + off);
        umma_bf16(acc, dah, dbh, idesc, (FIRST && kk == 0) ? 0u : 1u);
        umma_bf16(acc, dah, dbl, idesc, 1u);
        umma_bf16(acc, dal, dbh, idesc, 1u);
        umma_bf16(acc, dal, dbl, idesc, 1u);
    }
}

template <int BN, int STAGES>
__global__ void __launch_bounds__(THREADS, 1)
k_half(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
       const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl, HalfArgs ha)
{
    constexpr int A_BYTES = UM * BK * 2;
    constexpr int B_BYTES = BN * BK * 2;
    constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    constexpr uint32_t ACC_COLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
    constexpr uint32_t TMEM_COLS = 2 * ACC_COLS;   // two accumulator buffers
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *) (((uintptr_t) smem_raw + 1023) & ~(uintptr_t) 1023);
    uint64_t *full = (uint64_t *) (smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;   // [2]
    uint64_t *tempty = tfull + 2;       // [2]
    uint32_t *tmem_slot = (uint32_t *) (tempty + 2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n_items = ha.n_items, ptiles = ha.ptiles;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], EPI_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc_warp(tmem_slot, TMEM_COLS);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        bool ok = true;
        long long g = 0;   // chunk counter across this CTA's items
        for (int t = blockIdx.x; t < n_items && ok; t += gridDim.x) {
            const int i = t / ptiles, m0 = (t % ptiles) * UM;
            const int kc0 = ha.row_chunk0[i], nk = ha.row_chunk0[i + 1] - kc0;
            for (int kb = 0; kb < nk && ok; kb++, g++) {
                const int s = (int) (g % STAGES);
                if (g >= STAGES) ok = mbar_wait(&empty[s], (uint32_t) (((g / STAGES) - 1) & 1), 1);
                if (!ok) break;
                unsigned char *st = smem + s * STAGE_BYTES;
                mbar_expect_tx(&full[s], STAGE_BYTES);
                const int kx = (kc0 + kb) * BK;
                tma_load_2d(st, &mAh, &full[s], kx, m0);
                tma_load_2d(st + A_BYTES, &mAl, &full[s], kx, m0);
                tma_load_2d(st + 2 * A_BYTES, &mBh, &full[s], kx, 0);
                tma_load_2d(st + 2 * A_BYTES + B_BYTES, &mBl, &full[s], kx, 0);
            }
        }
        // copies in flight finish before the CTA exits
        for (long long q = (g > STAGES ? g - STAGES : 0); q < g; q++)
            mbar_wait(&full[q % STAGES], (uint32_t) ((q / STAGES) & 1), 2);
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = idesc_bf16(BN);
        bool ok = true;
        long long g = 0;
        int li = 0;
        for (int t = blockIdx.x; t < n_items && ok; t += gridDim.x, li++) {
            const int i = t / ptiles;
            const int nk = ha.row_chunk0[i + 1] - ha.row_chunk0[i];
            const int b = li & 1;
            if (li >= 2) ok = mbar_wait(&tempty[b], (uint32_t) (((li >> 1) - 1) & 1), 5);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t acc = tmem + b * ACC_COLS;
            for (int kb = 0; kb < nk && ok; kb++, g++) {
                const int s = (int) (g % STAGES);
                ok = mbar_wait(&full[s], (uint32_t) ((g / STAGES) & 1), 3);
                if (!ok) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a_hi = smem_u32(smem + s * STAGE_BYTES);
                if (kb == 0) mma_chunk4<true>(a_hi, a_hi + A_BYTES, a_hi + 2 * A_BYTES, a_hi + 2 * A_BYTES + B_BYTES,
                                              acc, idesc);
                else mma_chunk4<false>(a_hi, a_hi + A_BYTES, a_hi + 2 * A_BYTES, a_hi + 2 * A_BYTES + B_BYTES, acc,
                                       idesc);
                umma_commit(&empty[s]);
            }
            umma_commit(&tfull[b]);
        }
    } else if (warp >= 2) {
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const int row = quad * 32 + lane;
        const uint32_t tq = tmem + ((uint32_t) (quad * 32) << 16);
        uint32_t rm[32];
        float dtv[32];
        bool ok = true;
        int li = 0;
        for (int t = blockIdx.x; t < n_items && ok; t += gridDim.x, li++) {
            const int i = t / ptiles, m0 = (t % ptiles) * UM;
            const int nk = ha.row_chunk0[i + 1] - ha.row_chunk0[i];
            const int b = li & 1;
            ok = mbar_wait(&tfull[b], (uint32_t) ((li >> 1) & 1), 4);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int P = m0 + row;
            const size_t base = (size_t) i * ha.Qp + P;
            for (int c0 = half * 32; c0 < BN; c0 += 64) {
                if (nk > 0) {
                    tmem_ld32(tq + b * ACC_COLS + c0, rm);
#pragma unroll
                    for (int q = 0; q < 32; q++) dtv[q] = __uint_as_float(rm[q]);
                } else {
#pragma unroll
                    for (int q = 0; q < 32; q++) dtv[q] = 0.f;
                }
                if (P >= ha.naux) continue;
#pragma unroll
                for (int h16 = 0; h16 < 32; h16 += 16) {
                    float told[16];
#pragma unroll
                    for (int q = h16; q < h16 + 16; q++) {   // loads first: 16 in flight per thread
                        const int s = c0 + q;
                        told[q - h16] = (s < ha.nocc) ? ha.Tm[base + (size_t) s * ha.naux] : 0.f;
                    }
#pragma unroll
                    for (int q = h16; q < h16 + 16; q++) {
                        const int s = c0 + q;
                        if (s < ha.nocc) {
                            const size_t idx = base + (size_t) s * ha.naux;
                            const float dt = dtv[q];
                            const float tnew = told[q - h16] + dt;
                            ha.Tm[idx] = tnew;
                            __nv_bfloat16 h, l;
                            split_bf16(dt, h, l);
                            ha.dTh[idx] = h;
                            ha.dTl[idx] = l;
                            split_bf16(told[q - h16] + tnew, h, l);
                            ha.Sh[idx] = h;
                            ha.Sl[idx] = l;
                        }
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tempty[b])) : "memory");
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// ------------------------------------------------------------------ G = dT S^T, split-K
// CTA (x, y, z): output tile rows 128x.., cols 128y.., K chunks of split z.
// The K range is cut into segments of SEG_CHUNKS chunks; each segment
// accumulates in one of two TMEM buffers (hi*hi in 128 columns, hi*lo + lo*hi
// in another 128) while the epilogue warps drain the other buffer into FP32
// registers, so no TMEM accumulation runs longer than 256 K. The register
// sums of a split (at most MAX_SEGS segments) are written once, as FP64.
template <int STAGES>
__global__ void __launch_bounds__(THREADS, 1)
k_gemm(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
       const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl, GArgs ga)
{
    constexpr int BN = 128;
    constexpr int A_BYTES = UM * BK * 2, B_BYTES = BN * BK * 2;
    constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    constexpr uint32_t TMEM_COLS = 512;
    constexpr int WC = BN / 2;                 // output columns per epilogue warp
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *) (((uintptr_t) smem_raw + 1023) & ~(uintptr_t) 1023);
    uint64_t *full = (uint64_t *) (smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;    // [2] accumulator buffer ready
    uint64_t *tempty = tfull + 2;        // [2] accumulator buffer drained
    uint32_t *tmem_slot = (uint32_t *) (tempty + 2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * UM, n0 = blockIdx.y * BN;
    const int kc0 = blockIdx.z * ga.chunks_per_split;
    const int nk = max(0, min(ga.total_chunks, kc0 + ga.chunks_per_split) - kc0);
    const int nseg = (nk + SEG_CHUNKS - 1) / SEG_CHUNKS;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], EPI_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc_warp(tmem_slot, TMEM_COLS);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0 && !ga.probe) {
        bool ok = true;
        for (int kb = 0; kb < nk && ok; kb++) {
            const int s = kb % STAGES;
            if (kb >= STAGES) ok = mbar_wait(&empty[s], ((kb / STAGES) - 1) & 1, 11, ga.wait_cycles);
            if (!ok) break;
            unsigned char *st = smem + s * STAGE_BYTES;
            mbar_expect_tx(&full[s], STAGE_BYTES);
            const int kx = (kc0 + kb) * BK;
            tma_load_2d(st, &mAh, &full[s], kx, m0);
            tma_load_2d(st + A_BYTES, &mAl, &full[s], kx, m0);
            tma_load_2d(st + 2 * A_BYTES, &mBh, &full[s], kx, n0);
            tma_load_2d(st + 2 * A_BYTES + B_BYTES, &mBl, &full[s], kx, n0);
        }
        for (int kb = (nk > STAGES ? nk - STAGES : 0); kb < nk; kb++)
            mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1, 12, ga.wait_cycles);
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = idesc_bf16(BN);
        bool ok = true;
        int kb = 0;
        for (int seg = 0; seg < nseg && ok; seg++) {
            const int b = seg & 1;
            if (seg >= 2) ok = mbar_wait(&tempty[b], ((seg >> 1) - 1) & 1, 13, ga.wait_cycles);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t acc_main = tmem + b * 256;
            const int kend = min(nk, (seg + 1) * SEG_CHUNKS);
            for (; kb < kend && ok; kb++) {
                const int s = kb % STAGES;
                ok = mbar_wait(&full[s], (kb / STAGES) & 1, 14, ga.wait_cycles);
                if (!ok) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a_hi = smem_u32(smem + s * STAGE_BYTES);
                const uint32_t a_lo = a_hi + A_BYTES, b_hi = a_hi + 2 * A_BYTES, b_lo = b_hi + B_BYTES;
                mma_chunk<false>(a_hi, a_lo, b_hi, b_lo, acc_main, acc_main + 128, idesc, kb == seg * SEG_CHUNKS);
                umma_commit(&empty[s]);
            }
            umma_commit(&tfull[b]);
        }
    } else if (warp >= 2) {
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const int row = quad * 32 + lane;
        const uint32_t tq = tmem + ((uint32_t) (quad * 32) << 16) + half * 64;
        const int gi = m0 + row;
        const int lim = ga.nbf - (n0 + half * WC);
        double *o = ga.part + (size_t) blockIdx.z * ga.nbf * ga.nbf + (size_t) gi * ga.nbf + n0 + half * WC;
        const bool own = gi < ga.nbf;
        // FP32 sums of the split's segment results (round-to-nearest adds),
        // written once into the split's FP64 partial, which this thread alone owns
        float acc[WC];
#pragma unroll
        for (int c = 0; c < WC; c++) acc[c] = 0.f;
        uint32_t r[32];
        bool ok = true;
        for (int seg = 0; seg < nseg && ok; seg++) {
            const int b = seg & 1;
            ok = mbar_wait(&tfull[b], (seg >> 1) & 1, 15, ga.wait_cycles);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int c0 = 0; c0 < WC; c0 += 32) {
                // main and correction columns in flight together, one wait
                uint32_t r2[32];
                tmem_ld32_nowait(tq + b * 256 + c0, r);
                tmem_ld32_nowait(tq + b * 256 + 128 + c0, r2);
                tmem_wait_ld();
#pragma unroll
                for (int q = 0; q < 32; q++) acc[c0 + q] += __uint_as_float(r[q]) + __uint_as_float(r2[q]);
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tempty[b])) : "memory");
        }
        if (own) {   // zero when the split is empty or a wait gave up
#pragma unroll
            for (int c = 0; c < WC; c++)
                if (c < lim) o[c] = ok ? (double) acc[c] : 0.0;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// ------------------------------------------------------------------ G = dT S^T on CTA pairs
// The product of k_gemm with 256 x 256 output tiles, each computed by a CTA
// pair (cta_group::2, clusters of 2 along x): CTA r of the pair loads rows
// m0 + 128 r .. + 127 of dT (hi, lo) and rows n0 + 128 r .. + 127 of S (hi, lo);
// rank 0 issues M = 256, N = 256 MMAs that read both CTAs' tiles, and the
// tensor memory of each CTA receives its 128 rows. Per byte staged in shared
// memory this is twice k_gemm's MMA work (k_gemm is bound by shared-memory and
// L2 bandwidth). The three split products share one FP32 accumulator, double
// buffered in 2 x 256 columns. Rank 0's stage-full barrier counts both CTAs'
// copies; its MMA commits arrive at the stage-empty and accumulator-full
// barriers of both CTAs; both CTAs' epilogue warps arrive at rank 0's
// accumulator-empty barrier.
__device__ __forceinline__ void umma_bf16_pair(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

constexpr int PAIR_N = 256;                 // output tile columns (and rows) per CTA pair
constexpr int PAIR_STAGES = 3;
__host__ __device__ constexpr int pair_stage_bytes() { return 2 * UM * BK * 2 + 2 * (PAIR_N / 2) * BK * 2; }
__host__ __device__ constexpr int pair_smem_bytes() { return PAIR_STAGES * pair_stage_bytes() + 1024 + 8 * (2 * PAIR_STAGES + 4) + 16; }
static_assert(pair_smem_bytes() <= 227 * 1024, "paired G GEMM stages exceed shared memory");

__device__ __forceinline__ void gemm2_body(const CUtensorMap *mAh, const CUtensorMap *mAl, const CUtensorMap *mBh,
                                           const CUtensorMap *mBl, const GArgs &ga, int tile_x, int tile_y, int split)
{
    constexpr int STAGES = PAIR_STAGES;
    constexpr int BH = PAIR_N / 2;                // rows of S per CTA
    constexpr int A_BYTES = UM * BK * 2, B_BYTES = BH * BK * 2;
    constexpr int STAGE_BYTES = pair_stage_bytes();
    constexpr uint32_t TMEM_COLS = 512;
    constexpr int WC = PAIR_N / 2;                // output columns per epilogue warp
    // kind::f16, BF16 x BF16 -> FP32, K-major, M = 256 (the pair), N = 256
    constexpr uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (PAIR_N >> 3) << 17) |
                               ((uint32_t) (256 >> 4) << 24);
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *) (((uintptr_t) smem_raw + 1023) & ~(uintptr_t) 1023);
    uint64_t *full = (uint64_t *) (smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;    // [2] accumulator buffer ready (both CTAs)
    uint64_t *tempty = tfull + 2;        // [2] accumulator buffer drained (rank 0's counts both CTAs)
    uint32_t *tmem_slot = (uint32_t *) (tempty + 2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const int m0 = tile_x * PAIR_N + (int) rank * UM;   // this CTA's rows of the tile
    const int n0 = tile_y * PAIR_N;                      // the tile's columns
    const int kc0 = split * ga.chunks_per_split;
    const int nk = max(0, min(ga.total_chunks, kc0 + ga.chunks_per_split) - kc0);
    const int nseg = (nk + SEG_CHUNKS - 1) / SEG_CHUNKS;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 2 * EPI_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc_pair(tmem_slot, TMEM_COLS);
    fence_before_sync();
    __syncthreads();
    cluster_sync();   // both CTAs' barriers exist before either signals the other's
    fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0 && !ga.probe) {
        const uint32_t full0 = mapa_shared(smem_u32(&full[0]), 0);   // rank 0's stage-full barriers
        bool ok = true;
        for (int kb = 0; kb < nk && ok; kb++) {
            const int s = kb % STAGES;
            if (kb >= STAGES) ok = mbar_wait(&empty[s], ((kb / STAGES) - 1) & 1, 31, ga.wait_cycles);
            if (!ok) break;
            if (rank == 0) mbar_expect_tx(&full[s], 2 * STAGE_BYTES);
            unsigned char *st = smem + s * STAGE_BYTES;
            const int kx = (kc0 + kb) * BK;
            const uint32_t bar = full0 + 8u * (uint32_t) s;
            tma_load_2d_pair(st, mAh, bar, kx, m0);
            tma_load_2d_pair(st + A_BYTES, mAl, bar, kx, m0);
            tma_load_2d_pair(st + 2 * A_BYTES, mBh, bar, kx, n0 + (int) rank * BH);
            tma_load_2d_pair(st + 2 * A_BYTES + B_BYTES, mBl, bar, kx, n0 + (int) rank * BH);
        }
        // the pair's MMAs have consumed (so the copies have landed in) the last stages
        for (int kb = (nk > STAGES ? nk - STAGES : 0); kb < nk && ok; kb++)
            mbar_wait(&empty[kb % STAGES], (kb / STAGES) & 1, 32, ga.wait_cycles);
    } else if (warp == 1 && lane == 0 && rank == 0) {
        bool ok = true;
        int kb = 0;
        for (int seg = 0; seg < nseg && ok; seg++) {
            const int b = seg & 1;
            if (seg >= 2) ok = mbar_wait(&tempty[b], ((seg >> 1) - 1) & 1, 33, ga.wait_cycles);
            if (!ok) break;
            fence_after_sync();
            const uint32_t acc = tmem + b * PAIR_N;
            const int kend = min(nk, (seg + 1) * SEG_CHUNKS);
            for (; kb < kend && ok; kb++) {
                const int s = kb % STAGES;
                ok = mbar_wait(&full[s], (kb / STAGES) & 1, 34, ga.wait_cycles);
                if (!ok) break;
                fence_after_sync();
                const uint32_t a_hi = smem_u32(smem + s * STAGE_BYTES);
                const uint32_t a_lo = a_hi + A_BYTES, b_hi = a_hi + 2 * A_BYTES, b_lo = b_hi + B_BYTES;
#pragma unroll
                for (int kk = 0; kk < BK / UK; kk++) {
                    const uint32_t off = kk * UK * 2;
                    const uint64_t dah = desc_sw128(a_hi + off), dal = desc_sw128(a_lo + off);
                    const uint64_t dbh = desc_sw128(b_hi + off), dbl = desc_sw128(b_lo + off);
                    umma_bf16_pair(acc, dah, dbh, idesc, (kb == seg * SEG_CHUNKS && kk == 0) ? 0u : 1u);
                    umma_bf16_pair(acc, dah, dbl, idesc, 1u);
                    umma_bf16_pair(acc, dal, dbh, idesc, 1u);
                }
                umma_commit_pair(&empty[s], 0x3);
            }
            umma_commit_pair(&tfull[b], 0x3);
        }
    } else if (warp >= 2) {
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const int row = quad * 32 + lane;
        const uint32_t tq = tmem + ((uint32_t) (quad * 32) << 16) + half * WC;
        const uint32_t tempty0 = mapa_shared(smem_u32(&tempty[0]), 0);
        const int gi = m0 + row;
        const int lim = ga.nbf - (n0 + half * WC);
        double *o = ga.part + (size_t) split * ga.nbf * ga.nbf + (size_t) gi * ga.nbf + n0 + half * WC;
        const bool own = gi < ga.nbf;
        float acc[WC];
#pragma unroll
        for (int c = 0; c < WC; c++) acc[c] = 0.f;
        uint32_t r[32];
        bool ok = true;
        for (int seg = 0; seg < nseg && ok; seg++) {
            const int b = seg & 1;
            ok = mbar_wait(&tfull[b], (seg >> 1) & 1, 35, ga.wait_cycles);
            if (!ok) break;
            fence_after_sync();
#pragma unroll
            for (int c0 = 0; c0 < WC; c0 += 32) {
                tmem_ld32(tq + b * PAIR_N + c0, r);
#pragma unroll
                for (int q = 0; q < 32; q++) acc[c0 + q] += __uint_as_float(r[q]);
            }
            fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(tempty0 + 8u * (uint32_t) b);
        }
        if (own) {   // zero when the split is empty or a wait gave up
#pragma unroll
            for (int c = 0; c < WC; c++)
                if (c < lim) o[c] = ok ? (double) acc[c] : 0.0;
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

__global__ void __launch_bounds__(THREADS, 1)
k_gemm2(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
        const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl, GArgs ga)
{
    gemm2_body(&mAh, &mAl, &mBh, &mBl, ga, blockIdx.x >> 1, blockIdx.y, blockIdx.z);
}

// ------------------------------------------------------------------ many molecules per launch
// The operands of one molecule of a batched tensor-core K (a device array;
// the TMA unit reads the tensor maps from global memory).
struct KMixDev {
    CUtensorMap mBh, mBl, mCh, mCl, mdTh, mdTl, mSh, mSl;
    HalfArgs ha;
    GArgs ga;
    int bn, mt, ksplit;
};

// The molecule of global item g: starts[m] <= g < starts[m + 1] (molecules
// without items have starts[m] == starts[m + 1]).
__device__ __forceinline__ int find_mol(const int *starts, int nmol, int g)
{
    int lo = 0, hi = nmol - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (starts[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

constexpr int KB_STAGES = 2;
constexpr int KB_BN = 256;   // shared-memory stages sized for the largest N
__host__ __device__ constexpr int kb_half_smem_bytes()
{
    return KB_STAGES * (2 * UM * BK * 2 + 2 * KB_BN * BK * 2) + 1024 + 8 * (2 * KB_STAGES + 4) + 16;
}
static_assert(kb_half_smem_bytes() <= 227 * 1024, "batched half-transform stages exceed shared memory");

// k_half over the items of many molecules: persistent CTAs take global items
// blockIdx.x, + gridDim.x, ...; each item is (molecule, CSR row, 128 aux rows)
// with the molecule's own N (padded n_occ), tensor maps and buffers.
__global__ void __launch_bounds__(THREADS, 1)
kb_half(const KMixDev *__restrict__ mols, const int *__restrict__ starts, int nmol)
{
    constexpr int STAGES = KB_STAGES;
    constexpr int A_BYTES = UM * BK * 2;
    constexpr int BMAX_BYTES = KB_BN * BK * 2;
    constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * BMAX_BYTES;
    constexpr uint32_t ACC_COLS = 256, TMEM_COLS = 512;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *) (((uintptr_t) smem_raw + 1023) & ~(uintptr_t) 1023);
    uint64_t *full = (uint64_t *) (smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;   // [2]
    uint64_t *tempty = tfull + 2;       // [2]
    uint32_t *tmem_slot = (uint32_t *) (tempty + 2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = starts[nmol];

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], EPI_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc_warp(tmem_slot, TMEM_COLS);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        bool ok = true;
        long long g = 0;   // chunk counter across this CTA's items
        for (int it = blockIdx.x; it < total && ok; it += gridDim.x) {
            const int m = find_mol(starts, nmol, it);
            const KMixDev &d = mols[m];
            const int t = it - starts[m];
            const int i = t / d.ha.ptiles, m0 = (t % d.ha.ptiles) * UM;
            const int kc0 = d.ha.row_chunk0[i], nk = d.ha.row_chunk0[i + 1] - kc0;
            const uint32_t bbytes = (uint32_t) d.bn * BK * 2;
            for (int kb = 0; kb < nk && ok; kb++, g++) {
                const int s = (int) (g % STAGES);
                if (g >= STAGES) ok = mbar_wait(&empty[s], (uint32_t) (((g / STAGES) - 1) & 1), 41);
                if (!ok) break;
                unsigned char *st = smem + s * STAGE_BYTES;
                mbar_expect_tx(&full[s], 2 * A_BYTES + 2 * bbytes);
                const int kx = (kc0 + kb) * BK;
                tma_load_2d(st, &d.mBh, &full[s], kx, m0);
                tma_load_2d(st + A_BYTES, &d.mBl, &full[s], kx, m0);
                tma_load_2d(st + 2 * A_BYTES, &d.mCh, &full[s], kx, 0);
                tma_load_2d(st + 2 * A_BYTES + BMAX_BYTES, &d.mCl, &full[s], kx, 0);
            }
        }
        for (long long q = (g > STAGES ? g - STAGES : 0); q < g; q++)
            mbar_wait(&full[q % STAGES], (uint32_t) ((q / STAGES) & 1), 42);
    } else if (warp == 1 && lane == 0) {
        bool ok = true;
        long long g = 0;
        int li = 0;
        for (int it = blockIdx.x; it < total && ok; it += gridDim.x, li++) {
            const int m = find_mol(starts, nmol, it);
            const KMixDev &d = mols[m];
            const int t = it - starts[m];
            const int i = t / d.ha.ptiles;
            const int nk = d.ha.row_chunk0[i + 1] - d.ha.row_chunk0[i];
            const uint32_t idesc = idesc_bf16(d.bn);
            const int b = li & 1;
            if (li >= 2) ok = mbar_wait(&tempty[b], (uint32_t) (((li >> 1) - 1) & 1), 43);
            if (!ok) break;
            fence_after_sync();
            const uint32_t acc = tmem + b * ACC_COLS;
            for (int kb = 0; kb < nk && ok; kb++, g++) {
                const int s = (int) (g % STAGES);
                ok = mbar_wait(&full[s], (uint32_t) ((g / STAGES) & 1), 44);
                if (!ok) break;
                fence_after_sync();
                const uint32_t a_hi = smem_u32(smem + s * STAGE_BYTES);
                if (kb == 0) mma_chunk4<true>(a_hi, a_hi + A_BYTES, a_hi + 2 * A_BYTES, a_hi + 2 * A_BYTES + BMAX_BYTES,
                                              acc, idesc);
                else mma_chunk4<false>(a_hi, a_hi + A_BYTES, a_hi + 2 * A_BYTES, a_hi + 2 * A_BYTES + BMAX_BYTES,
                                       acc, idesc);
                umma_commit(&empty[s]);
            }
            umma_commit(&tfull[b]);
        }
    } else if (warp >= 2) {
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const int row = quad * 32 + lane;
        const uint32_t tq = tmem + ((uint32_t) (quad * 32) << 16);
        uint32_t rm[32];
        float dtv[32];
        bool ok = true;
        int li = 0;
        for (int it = blockIdx.x; it < total && ok; it += gridDim.x, li++) {
            const int m = find_mol(starts, nmol, it);
            const KMixDev &d = mols[m];
            const HalfArgs &ha = d.ha;
            const int t = it - starts[m];
            const int i = t / ha.ptiles, m0 = (t % ha.ptiles) * UM;
            const int nk = ha.row_chunk0[i + 1] - ha.row_chunk0[i];
            const int b = li & 1;
            ok = mbar_wait(&tfull[b], (uint32_t) ((li >> 1) & 1), 45);
            if (!ok) break;
            fence_after_sync();
            const int P = m0 + row;
            const size_t base = (size_t) i * ha.Qp + P;
            for (int c0 = half * 32; c0 < d.bn; c0 += 64) {
                if (nk > 0) {
                    tmem_ld32(tq + b * ACC_COLS + c0, rm);
#pragma unroll
                    for (int q = 0; q < 32; q++) dtv[q] = __uint_as_float(rm[q]);
                } else {
#pragma unroll
                    for (int q = 0; q < 32; q++) dtv[q] = 0.f;
                }
                if (P >= ha.naux) continue;
#pragma unroll
                for (int h16 = 0; h16 < 32; h16 += 16) {
                    float told[16];
#pragma unroll
                    for (int q = h16; q < h16 + 16; q++) {
                        const int sq = c0 + q;
                        told[q - h16] = (sq < ha.nocc) ? ha.Tm[base + (size_t) sq * ha.naux] : 0.f;
                    }
#pragma unroll
                    for (int q = h16; q < h16 + 16; q++) {
                        const int sq = c0 + q;
                        if (sq < ha.nocc) {
                            const size_t idx = base + (size_t) sq * ha.naux;
                            const float dt = dtv[q];
                            const float tnew = told[q - h16] + dt;
                            ha.Tm[idx] = tnew;
                            __nv_bfloat16 h, l;
                            split_bf16(dt, h, l);
                            ha.dTh[idx] = h;
                            ha.dTl[idx] = l;
                            split_bf16(told[q - h16] + tnew, h, l);
                            ha.Sh[idx] = h;
                            ha.Sl[idx] = l;
                        }
                    }
                }
            }
            fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[b]);
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 1) {
        fence_after_sync();
        tmem_dealloc_warp(tmem, TMEM_COLS);
    }
}

// k_gemm2 over the tiles of many molecules: pair item p = blockIdx.x / 2 is
// (molecule, 256-row tile x, tile y, split) of that molecule's own G GEMM.
__global__ void __launch_bounds__(THREADS, 1)
kb_gemm2(const KMixDev *__restrict__ mols, const int *__restrict__ starts, int nmol)
{
    const int p = blockIdx.x >> 1;
    const int m = find_mol(starts, nmol, p);
    const KMixDev &d = mols[m];
    const int local = p - starts[m];
    const int tx = local % d.mt, ty = (local / d.mt) % d.mt, split = local / (d.mt * d.mt);
    gemm2_body(&d.mdTh, &d.mdTl, &d.mSh, &d.mSl, d.ga, tx, ty, split);
}

template <int BN, int STAGES>
constexpr int half_smem_bytes()
{
    return STAGES * (2 * UM * BK * 2 + 2 * BN * BK * 2) + 1024 + 8 * (2 * STAGES + 4) + 16;
}
template <int BN, int STAGES>
constexpr int gemm_smem_bytes()
{
    return STAGES * (2 * UM * BK * 2 + 2 * BN * BK * 2) + 1024 + 8 * (2 * STAGES + 4) + 16;
}

// ---------------------------------------------------------------- TMA descriptors
// 2D BF16 matrix rows x cols (cols contiguous, pitch in elements), box 64 cols x box_rows.
int make_map(CUtensorMap *m, const void *base, long long rows, long long cols, long long pitch, int box_rows)
{
    return make_map_2d(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, rows, cols, pitch, BK, box_rows) ? OK : ERR_CUDA;
}

}  // namespace

// N of the half-transform GEMM: the occupied orbitals padded to a multiple of 16.
int kmix_half_bn(int nocc) { return (nocc + 15) / 16 * 16; }

// ---------------------------------------------------------------- kernels around the GEMMs
// Transposed, row-padded copy of the DF tensor for the half-transform's A
// operand: BpT[P][r] = B(CSR entry of padded position r, P), zero in padding.
__global__ void k_build_bpt(const double *Bu, const int *pad_entry, const int *csr_u, int naux, long long rp,
                            __nv_bfloat16 *Bh, __nv_bfloat16 *Bl)
{
    __shared__ float tile[32][33];
    const long long r0 = (long long) blockIdx.x * 32;
    const int p0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8 threads
    for (int k = ty; k < 32; k += 8) {
        const long long r = r0 + k;
        const int e = (r < rp) ? pad_entry[r] : -1;
        const int p = p0 + tx;
        tile[k][tx] = (e >= 0 && p < naux) ? (float) Bu[(size_t) csr_u[e] * naux + p] : 0.f;
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int p = p0 + k;
        const long long r = r0 + tx;
        if (p < naux && r < rp) {
            __nv_bfloat16 h, l;
            split_bf16(tile[tx][k], h, l);
            Bh[(size_t) p * rp + r] = h;
            Bl[(size_t) p * rp + r] = l;
        }
    }
}

// CgT[s][r] = dC(j of padded position r, s): the half-transform's B operand.
__global__ void k_gather_dc(const double *dC, const int *pad_entry, const int *csr_j, int nocc, long long rp,
                            __nv_bfloat16 *Ch, __nv_bfloat16 *Cl)
{
    const long long r = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (r >= rp) return;
    const int e = pad_entry[r];
    const float v = (e >= 0 && s < nocc) ? (float) dC[(size_t) csr_j[e] * nocc + s] : 0.f;
    __nv_bfloat16 h, l;
    split_bf16(v, h, l);
    Ch[(size_t) s * rp + r] = h;
    Cl[(size_t) s * rp + r] = l;
}

// K[i][j] = (reset ? 0 : K[i][j]) + (G_ij + G_ji) / 2, G summed over splits in FP64.
__global__ void k_kmix_reduce(const double *part, int ksplit, int nbf, int reset, double *K)
{
    const size_t idx = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t) nbf * nbf) return;
    const int i = (int) (idx / nbf), j = (int) (idx % nbf);
    const size_t tdx = (size_t) j * nbf + i;
    const size_t nn = (size_t) nbf * nbf;
    double gij = 0.0, gji = 0.0;
    for (int k = 0; k < ksplit; k++) {
        gij += part[k * nn + idx];
        gji += part[k * nn + tdx];
    }
    const double d = 0.5 * (gij + gji);
    K[idx] = reset ? d : K[idx] + d;
}

// Newton-Schulz step helper: Z = 1.5 I - 0.5 Y
__global__ void k_ns_z(const double *Y, double *Z, int n)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * n) return;
    const int i = idx / n, j = idx % n;
    Z[idx] = (i == j ? 1.5 : 0.0) - 0.5 * Y[idx];
}

// R = X if max|X^T X - I| <= tol (Y holds X^T X) else I.
__global__ void k_select_r(const double *X, const double *Y, double *R, int n, double tol)
{
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int i = idx / n, j = idx % n;
        const double e = Y[idx] - (i == j ? 1.0 : 0.0);
        if (!(fabs(e) <= tol)) bad = 1;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int i = idx / n, j = idx % n;
        R[idx] = bad ? (i == j ? 1.0 : 0.0) : X[idx];
    }
}

// dC = C' - Cprev; Cprev = C'
__global__ void k_delta_c(const double *Cn, double *Cprev, double *dC, size_t n)
{
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double c = Cn[i];
    dC[i] = c - Cprev[i];
    Cprev[i] = c;
}

// ---------------------------------------------------------------- plan
struct KMix {
    int nbf = 0, naux = 0, nocc = 0, bn_half = 0, ksplit = 1, chunks_per_split = 1, total_chunks = 0;
    long long rp = 0, Qp = 0;
    int *row_chunk0 = nullptr, *pad_entry = nullptr;
    const int *csr_j = nullptr;
    __nv_bfloat16 *Bh = nullptr, *Bl = nullptr, *Ch = nullptr, *Cl = nullptr;
    float *Tm = nullptr;
    double *G = nullptr;
    __nv_bfloat16 *dTh = nullptr, *dTl = nullptr, *Sh = nullptr, *Sl = nullptr;
    double *Cprev = nullptr, *Cal = nullptr, *dC = nullptr, *SC = nullptr, *M = nullptr, *X = nullptr,
           *Y = nullptr, *Z = nullptr, *R = nullptr;
    CUtensorMap mBh, mBl, mCh, mCl, mdTh, mdTl, mSh, mSl;
    bool first = true;
    std::vector<void *> mem;
};

static int kalloc(KMix *k, void **p, size_t bytes)
{
    if (dev_malloc(p, bytes, 0) != OK) return ERR_ALLOC;
    k->mem.push_back(*p);
    return OK;
}

#define KRC(x)                  \
    do {                        \
        int rc__ = (x);         \
        if (rc__) return rc__;  \
    } while (0)

void kmix_destroy(KMix *k)
{
    if (!k) return;
    for (void *p : k->mem) dev_free(p, 0);
    cudaStreamSynchronize(0);
    delete k;
}

int kmix_create(KMix **out, const FockPlan &p, const int *h_displs, cudaStream_t s)
{
    *out = nullptr;
    if (p.nocc > 256) return ERR_UNSUPPORTED;
    KMix *k = new KMix();
    k->nbf = p.nbf;
    k->naux = p.naux;
    k->nocc = p.nocc;
    k->bn_half = kmix_half_bn(p.nocc);
    k->csr_j = p.csr_j;
    // padded CSR rows: each row starts at a multiple of 64 positions
    std::vector<int> chunk0(p.nbf + 1), pad;
    long long pos = 0;
    for (int i = 0; i < p.nbf; i++) {
        chunk0[i] = (int) (pos / BK);
        const int len = h_displs[i + 1] - h_displs[i];
        const int plen = (len + BK - 1) / BK * BK;
        for (int q = 0; q < plen; q++) pad.push_back(q < len ? h_displs[i] + q : -1);
        pos += plen;
    }
    chunk0[p.nbf] = (int) (pos / BK);
    k->rp = pos;
    k->Qp = ((long long) p.nocc * p.naux + BK - 1) / BK * BK;
    k->total_chunks = (int) (k->Qp / BK);
    // Split count: at least 4 CTAs per SM, at most MAX_SEGS segments per split
    // (their FP32 register sums are written once, as FP64, at the end), and
    // the CTA count rounded up to whole waves of the SM count when that costs little.
    const int mt = (p.nbf + UM - 1) / UM;
    const int tiles = mt * mt;
    const int nsm = num_sms();
    int ks = std::max((4 * nsm + tiles - 1) / tiles, (k->total_chunks + SEG_CHUNKS * MAX_SEGS - 1) / (SEG_CHUNKS * MAX_SEGS));
    {
        int best = ks;
        for (int c = ks; c <= ks + ks / 4 + 1; c++)
            if ((tiles * c) % nsm == 0) {
                best = c;
                break;
            }
        ks = best;
    }
    ks = std::max(1, std::min(ks, k->total_chunks / 4 > 0 ? k->total_chunks / 4 : 1));
    if (const char *ev = getenv("TINYSCF_KMIX_KSPLIT"))
        if (atoi(ev) > 0) ks = std::min(atoi(ev), k->total_chunks);
    k->chunks_per_split = (k->total_chunks + ks - 1) / ks;
    k->ksplit = (k->total_chunks + k->chunks_per_split - 1) / k->chunks_per_split;
    const size_t nbq = (size_t) p.nbf * k->Qp;
    const int nocc_pad = k->bn_half;
    int rc = OK;
    do {
        if ((rc = kalloc(k, (void **) &k->row_chunk0, sizeof(int) * chunk0.size()))) break;
        if ((rc = kalloc(k, (void **) &k->pad_entry, sizeof(int) * pad.size()))) break;
        if ((rc = kalloc(k, (void **) &k->Bh, 2 * (size_t) p.naux * k->rp))) break;
        if ((rc = kalloc(k, (void **) &k->Bl, 2 * (size_t) p.naux * k->rp))) break;
        if ((rc = kalloc(k, (void **) &k->Ch, 2 * (size_t) nocc_pad * k->rp))) break;
        if ((rc = kalloc(k, (void **) &k->Cl, 2 * (size_t) nocc_pad * k->rp))) break;
        if ((rc = kalloc(k, (void **) &k->Tm, 4 * nbq))) break;
        if ((rc = kalloc(k, (void **) &k->dTh, 2 * nbq))) break;
        if ((rc = kalloc(k, (void **) &k->dTl, 2 * nbq))) break;
        if ((rc = kalloc(k, (void **) &k->Sh, 2 * nbq))) break;
        if ((rc = kalloc(k, (void **) &k->Sl, 2 * nbq))) break;
        if ((rc = kalloc(k, (void **) &k->G, 8 * (size_t) k->ksplit * p.nbf * p.nbf))) break;
        const size_t nc = (size_t) p.nbf * p.nocc, oo = (size_t) p.nocc * p.nocc;
        if ((rc = kalloc(k, (void **) &k->Cprev, 8 * nc))) break;
        if ((rc = kalloc(k, (void **) &k->Cal, 8 * nc))) break;
        if ((rc = kalloc(k, (void **) &k->dC, 8 * nc))) break;
        if ((rc = kalloc(k, (void **) &k->SC, 8 * nc))) break;
        if ((rc = kalloc(k, (void **) &k->M, 8 * oo))) break;
        if ((rc = kalloc(k, (void **) &k->X, 8 * oo))) break;
        if ((rc = kalloc(k, (void **) &k->Y, 8 * oo))) break;
        if ((rc = kalloc(k, (void **) &k->Z, 8 * oo))) break;
        if ((rc = kalloc(k, (void **) &k->R, 8 * oo))) break;
    } while (0);
    if (rc) {
        kmix_destroy(k);
        return rc;
    }
    cudaMemcpyAsync(k->row_chunk0, chunk0.data(), sizeof(int) * chunk0.size(), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(k->pad_entry, pad.data(), sizeof(int) * pad.size(), cudaMemcpyHostToDevice, s);
    // padded tails of the K dimension stay zero forever
    cudaMemsetAsync(k->dTh, 0, 2 * nbq, s);
    cudaMemsetAsync(k->dTl, 0, 2 * nbq, s);
    cudaMemsetAsync(k->Sh, 0, 2 * nbq, s);
    cudaMemsetAsync(k->Sl, 0, 2 * nbq, s);
    dim3 gb((unsigned) ((k->rp + 31) / 32), (unsigned) ((p.naux + 31) / 32));
    k_build_bpt<<<gb, dim3(32, 8), 0, s>>>(p.B, k->pad_entry, p.csr_u, p.naux, k->rp, k->Bh, k->Bl);
    g_launches++;
    if (make_map(&k->mBh, k->Bh, p.naux, k->rp, k->rp, UM) || make_map(&k->mBl, k->Bl, p.naux, k->rp, k->rp, UM) ||
        make_map(&k->mCh, k->Ch, nocc_pad, k->rp, k->rp, nocc_pad) ||
        make_map(&k->mCl, k->Cl, nocc_pad, k->rp, k->rp, nocc_pad) ||
        make_map(&k->mdTh, k->dTh, p.nbf, k->Qp, k->Qp, UM) || make_map(&k->mdTl, k->dTl, p.nbf, k->Qp, k->Qp, UM) ||
        make_map(&k->mSh, k->Sh, p.nbf, k->Qp, k->Qp, UM) || make_map(&k->mSl, k->Sl, p.nbf, k->Qp, k->Qp, UM)) {
        kmix_destroy(k);
        return ERR_CUDA;
    }
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        kmix_destroy(k);
        return ERR_CUDA;
    }
    *out = k;
    return OK;
}

void kmix_reset(KMix *k, cudaStream_t s)
{
    cudaMemsetAsync(k->Tm, 0, 4 * (size_t) k->nbf * k->Qp, s);
    cudaMemsetAsync(k->Cprev, 0, 8 * (size_t) k->nbf * k->nocc, s);
    k->first = true;
}

template <int BN>
static int launch_half(const KMix *k, HalfArgs ha, cudaStream_t s)
{
    constexpr int STAGES = BN <= 112 ? 3 : 2;   // within 227 KB of shared memory
    constexpr int SMEM = half_smem_bytes<BN, STAGES>();
    static_assert(SMEM <= 227 * 1024, "half-transform stages exceed shared memory");
    static bool attr_set = false;
    if (!attr_set) {
        if (cudaFuncSetAttribute(k_half<BN, STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM) != cudaSuccess)
            return ERR_CUDA;
        attr_set = true;
    }
    ha.ptiles = (k->naux + UM - 1) / UM;
    ha.n_items = k->nbf * ha.ptiles;
    const int grid = std::max(1, std::min(ha.n_items, num_sms()));
    k_half<BN, STAGES><<<grid, THREADS, SMEM, s>>>(k->mBh, k->mBl, k->mCh, k->mCl, ha);
    g_launches++;
    return OK;
}

// The paired kernel (k_gemm2) unless TINYSCF_GEMM_PAIR=0.
static bool use_pair_gemm()
{
    const char *v = getenv("TINYSCF_GEMM_PAIR");
    return !(v && v[0] == '0');
}

static int launch_gemm2(const KMix *k, const GArgs &ga, cudaStream_t s)
{
    constexpr int SMEM = pair_smem_bytes();
    static bool attr_set = false;
    if (!attr_set) {
        if (cudaFuncSetAttribute(k_gemm2, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM) != cudaSuccess)
            return ERR_CUDA;
        attr_set = true;
    }
    const int mt = (k->nbf + PAIR_N - 1) / PAIR_N;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * mt, mt, k->ksplit);
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    g_launches++;
    if (cudaLaunchKernelEx(&cfg, k_gemm2, k->mdTh, k->mdTl, k->mSh, k->mSl, ga) != cudaSuccess) return ERR_CUDA;
    return OK;
}

static int launch_gemm(const KMix *k, const GArgs &ga, cudaStream_t s)
{
    if (use_pair_gemm()) return launch_gemm2(k, ga, s);
    constexpr int STAGES = 3;
    constexpr int SMEM = gemm_smem_bytes<128, STAGES>();
    static bool attr_set = false;
    if (!attr_set) {
        if (cudaFuncSetAttribute(k_gemm<STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM) != cudaSuccess)
            return ERR_CUDA;
        attr_set = true;
    }
    const int mt = (k->nbf + UM - 1) / UM;
    // Clusters of CTAs along the row tiles: the CTAs that read the same S tile
    // (and, cluster after cluster, the same dT tiles) run at the same time on
    // one GPC, so their TMA loads of the shared tiles meet in L2 instead of
    // each going to DRAM. No cluster feature is used inside the kernel.
    static const int cl_max = [] {
        const char *v = getenv("TINYSCF_GEMM_CLUSTER");
        const int c = v ? atoi(v) : 2;
        return (c == 1 || c == 2 || c == 4 || c == 8) ? c : 2;
    }();
    int cl = 1;
    for (int c = cl_max; c >= 2; c >>= 1)
        if (mt % c == 0) {
            cl = c;
            break;
        }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(mt, mt, k->ksplit);
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    g_launches++;
    if (cudaLaunchKernelEx(&cfg, k_gemm<STAGES>, k->mdTh, k->mdTl, k->mSh, k->mSl, ga) != cudaSuccess) return ERR_CUDA;
    return OK;
}

// One incremental K build from the new occupied factor Cocc (nbf x nocc).
// Alignment of the new occupied factor and the gathered dC operands of one
// molecule (everything of an incremental K build before the half-transform).
static void kmix_prepare(KMix *k, const double *Cocc, const double *S, cudaStream_t s)
{
    const int n = k->nbf, o = k->nocc;
    // align C_n to C_{n-1}: R = polar(C_n^T S C_{n-1}) by Newton-Schulz; R = I if it does not converge
    dgemm(false, false, n, o, n, 1.0, S, n, k->Cprev, o, 0.0, k->SC, o, s);
    dgemm(true, false, o, o, n, 1.0, Cocc, o, k->SC, o, 0.0, k->X, o, s);
    for (int it = 0; it < 12; it++) {
        dgemm(true, false, o, o, o, 1.0, k->X, o, k->X, o, 0.0, k->Y, o, s);
        k_ns_z<<<(o * o + 255) / 256, 256, 0, s>>>(k->Y, k->Z, o);
        dgemm(false, false, o, o, o, 1.0, k->X, o, k->Z, o, 0.0, k->M, o, s);
        std::swap(k->X, k->M);
        g_launches++;
    }
    dgemm(true, false, o, o, o, 1.0, k->X, o, k->X, o, 0.0, k->Y, o, s);
    k_select_r<<<1, 1024, 0, s>>>(k->X, k->Y, k->R, o, 1e-12);
    dgemm(false, false, n, o, o, 1.0, Cocc, o, k->R, o, 0.0, k->Cal, o, s);
    const size_t nc = (size_t) n * o;
    k_delta_c<<<(unsigned) ((nc + 255) / 256), 256, 0, s>>>(k->Cal, k->Cprev, k->dC, nc);
    dim3 gg((unsigned) ((k->rp + 255) / 256), k->bn_half);
    k_gather_dc<<<gg, 256, 0, s>>>(k->dC, k->pad_entry, k->csr_j, o, k->rp, k->Ch, k->Cl);
    g_launches += 3;
}

// K += sym(sum over the first nsplit splits of G) (the first build of a solve sets K).
static void kmix_finish(KMix *k, double *K, cudaStream_t s, int nsplit)
{
    const size_t nn = (size_t) k->nbf * k->nbf;
    k_kmix_reduce<<<(unsigned) ((nn + 255) / 256), 256, 0, s>>>(k->G, nsplit, k->nbf, k->first ? 1 : 0, K);
    g_launches++;
    k->first = false;
}

static HalfArgs half_args(const KMix *k)
{
    HalfArgs ha{k->row_chunk0, k->Tm, k->dTh, k->dTl, k->Sh, k->Sl, k->nocc, k->naux, k->Qp, 0, 0};
    ha.ptiles = (k->naux + UM - 1) / UM;
    ha.n_items = k->nbf * ha.ptiles;
    return ha;
}

int kmix_build(KMix *k, const double *Cocc, const double *S, double *K, cudaStream_t s,
               const std::function<void(int)> &mark)
{
    kmix_prepare(k, Cocc, S, s);
    HalfArgs ha = half_args(k);
    int rc;
    if (mark) mark(0);
    switch (k->bn_half) {
    case 16: rc = launch_half<16>(k, ha, s); break;
    case 32: rc = launch_half<32>(k, ha, s); break;
    case 48: rc = launch_half<48>(k, ha, s); break;
    case 64: rc = launch_half<64>(k, ha, s); break;
    case 80: rc = launch_half<80>(k, ha, s); break;
    case 96: rc = launch_half<96>(k, ha, s); break;
    case 112: rc = launch_half<112>(k, ha, s); break;
    case 128: rc = launch_half<128>(k, ha, s); break;
    case 144: rc = launch_half<144>(k, ha, s); break;
    case 160: rc = launch_half<160>(k, ha, s); break;
    case 176: rc = launch_half<176>(k, ha, s); break;
    case 192: rc = launch_half<192>(k, ha, s); break;
    case 208: rc = launch_half<208>(k, ha, s); break;
    case 224: rc = launch_half<224>(k, ha, s); break;
    case 240: rc = launch_half<240>(k, ha, s); break;
    case 256: rc = launch_half<256>(k, ha, s); break;
    default: rc = ERR_UNSUPPORTED;
    }
    if (rc) return rc;
    if (mark) mark(1);
    GArgs ga{k->G, k->nbf, k->chunks_per_split, k->total_chunks};
    rc = launch_gemm(k, ga, s);
    if (rc) return rc;
    if (mark) mark(2);
    kmix_finish(k, K, s, k->ksplit);
    return OK;
}

// ---------------------------------------------------------------- many molecules in one launch per kernel
struct KMixBatch {
    std::vector<KMix *> ks;
    std::vector<int> ksplit;           // the G GEMM's K splits of each molecule in the batch
    KMixDev *d_mols = nullptr;
    int *d_starts = nullptr;           // [2][nmol + 1]: half-transform items, G GEMM pair items
    std::vector<int> h_starts;
    int max_bn = 0;
};

void kmix_batch_destroy(KMixBatch *b)
{
    if (!b) return;
    cudaFree(b->d_mols);
    cudaFree(b->d_starts);
    delete b;
}

int kmix_batch_create(KMixBatch **out, KMix *const *ks, int n, cudaStream_t s)
{
    *out = nullptr;
    if (n <= 0) return ERR_INPUT;
    KMixBatch *b = new KMixBatch();
    b->ks.assign(ks, ks + n);
    std::vector<KMixDev> h(n);
    for (int m = 0; m < n; m++) {
        const KMix *k = ks[m];
        KMixDev &d = h[m];
        memset(&d, 0, sizeof(d));
        d.mBh = k->mBh;
        d.mBl = k->mBl;
        d.mCh = k->mCh;
        d.mCl = k->mCl;
        d.mdTh = k->mdTh;
        d.mdTl = k->mdTl;
        d.mSh = k->mSh;
        d.mSl = k->mSl;
        d.ha = half_args(k);
        d.ga.part = k->G;
        d.ga.nbf = k->nbf;
        // the molecule's own K splits: its G sums round exactly as in its builds one by one
        const int ksb = k->ksplit;
        d.ga.chunks_per_split = k->chunks_per_split;
        d.ga.total_chunks = k->total_chunks;
        d.ga.probe = 0;
        d.ga.wait_cycles = WAIT_CYCLES;
        d.bn = k->bn_half;
        d.mt = (k->nbf + PAIR_N - 1) / PAIR_N;
        d.ksplit = ksb;
        b->ksplit.push_back(ksb);
        b->max_bn = std::max(b->max_bn, d.bn);
    }
    b->h_starts.assign(2 * (n + 1), 0);
    if (cudaMalloc(&b->d_mols, sizeof(KMixDev) * n) != cudaSuccess ||
        cudaMalloc(&b->d_starts, sizeof(int) * 2 * (n + 1)) != cudaSuccess ||
        cudaMemcpyAsync(b->d_mols, h.data(), sizeof(KMixDev) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        kmix_batch_destroy(b);
        return ERR_ALLOC;
    }
    *out = b;
    return OK;
}

// One incremental K build of every molecule m with active[m] != 0: the
// alignments per molecule, then one half-transform launch and one G GEMM
// launch over all of them, then the per-molecule reductions into K[m].
int kmix_batch_build(KMixBatch *b, const int *active, const double *const *Cocc, const double *const *S,
                     double *const *K, cudaStream_t s)
{
    const int n = (int) b->ks.size();
    int *hh = b->h_starts.data(), *hg = hh + n + 1;
    hh[0] = hg[0] = 0;
    for (int m = 0; m < n; m++) {
        const KMix *k = b->ks[m];
        const int mt = (k->nbf + PAIR_N - 1) / PAIR_N;
        hh[m + 1] = hh[m] + (active[m] ? k->nbf * ((k->naux + UM - 1) / UM) : 0);
        hg[m + 1] = hg[m] + (active[m] ? mt * mt * b->ksplit[m] : 0);
    }
    if (hh[n] == 0) return OK;
    for (int m = 0; m < n; m++)
        if (active[m]) kmix_prepare(b->ks[m], Cocc[m], S[m], s);
    TSCF_CUDA_CHECK(cudaMemcpyAsync(b->d_starts, hh, sizeof(int) * 2 * (n + 1), cudaMemcpyHostToDevice, s));
    {
        constexpr int SMEM = kb_half_smem_bytes();
        static bool attr_set = false;
        if (!attr_set) {
            if (cudaFuncSetAttribute(kb_half, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM) != cudaSuccess)
                return ERR_CUDA;
            attr_set = true;
        }
        const int grid = std::max(1, std::min(hh[n], num_sms()));
        kb_half<<<grid, THREADS, SMEM, s>>>(b->d_mols, b->d_starts, n);
        g_launches++;
    }
    {
        constexpr int SMEM = pair_smem_bytes();
        static bool attr_set = false;
        if (!attr_set) {
            if (cudaFuncSetAttribute(kb_gemm2, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM) != cudaSuccess)
                return ERR_CUDA;
            attr_set = true;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2 * hg[n]);
        cfg.blockDim = dim3(THREADS);
        cfg.dynamicSmemBytes = SMEM;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        g_launches++;
        if (cudaLaunchKernelEx(&cfg, kb_gemm2, (const KMixDev *) b->d_mols, (const int *) (b->d_starts + n + 1), n) !=
            cudaSuccess)
            return ERR_CUDA;
    }
    for (int m = 0; m < n; m++)
        if (active[m]) kmix_finish(b->ks[m], K[m], s, b->ksplit[m]);
    return cuda_launch_rc("batched tensor-core exchange");
}

int kmix_error_flag()
{
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_umma_error, sizeof(int));
    return v;
}

// The bounded-wait path of the G GEMM kernel, run on purpose: one CTA with
// no copies issued, so its MMA warp waits on a stage that nothing fills and
// its epilogue on an accumulator that nothing completes. Both waits give up
// after wait_cycles, record their code, and the CTA frees its TMEM and
// returns; nothing is in flight. Returns the recorded code (0 if no wait gave
// up) and clears the flag again.
int kmix_wait_probe(KMix *k, long long wait_cycles, int *code, cudaStream_t s)
{
    if (!k || !code || wait_cycles < 0) return ERR_INPUT;
    const int zero = 0;
    TSCF_CUDA_CHECK(cudaMemcpyToSymbolAsync(g_umma_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s));
    GArgs ga{k->G, k->nbf, k->chunks_per_split, k->total_chunks};
    ga.probe = 1;
    ga.wait_cycles = wait_cycles;
    constexpr int STAGES = 3;
    constexpr int SMEM = gemm_smem_bytes<128, STAGES>();
    if (cudaFuncSetAttribute(k_gemm<STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM) != cudaSuccess)
        return ERR_CUDA;
    k_gemm<STAGES><<<dim3(1, 1, 1), THREADS, SMEM, s>>>(k->mdTh, k->mdTl, k->mSh, k->mSl, ga);
    g_launches++;
    TSCF_CUDA_CHECK(cudaGetLastError());
    TSCF_CUDA_CHECK(cudaStreamSynchronize(s));
    TSCF_CUDA_CHECK(cudaMemcpyFromSymbol(code, g_umma_error, sizeof(int)));
    TSCF_CUDA_CHECK(cudaMemcpyToSymbol(g_umma_error, &zero, sizeof(int)));
    return OK;
}

}  // namespace tscf
