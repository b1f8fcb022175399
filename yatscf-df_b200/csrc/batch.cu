// Batched SCF phases: one launch per phase for every molecule of a batch.
//
// Molecules of uneven size share each launch through a flattened work list:
// a phase's items are numbered molecule by molecule (prefix sums per phase),
// and a block finds its molecule by binary search over the prefix array. Each
// item runs the same tile body as the single-molecule kernel (tiles.cuh) with
// the same partition of the work, so every molecule's numbers are the ones
// its own SCF would produce. Molecules that have converged are skipped.
#include <cfloat>
#include <cmath>
#include <cstdio>

#include "batch.h"
#include "tiles.cuh"

namespace tscf {

namespace {

__device__ __forceinline__ int find_mol(const int *start, int nmol, int g)
{
    int lo = 0, hi = nmol - 1;
    while (lo < hi) {   // largest m with start[m] <= g
        int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

#define BATCH_ITEM(list)                                           \
    const int g__ = blockIdx.x;                                    \
    const int mol = find_mol((list).start, (list).nmol, g__);      \
    const int li = g__ - (list).start[mol];                        \
    const MolDev &m = mols[mol];                                   \
    if (!active[mol]) return;

// ---- J
__global__ void __launch_bounds__(JT_THREADS) kb_j_tpart(const MolDev *mols, const int *active, WorkList wl,
                                                         int use32)
{
    BATCH_ITEM(wl)
    const int nblk = wl.start[mol + 1] - wl.start[mol];
    const int rows = (m.nup + nblk - 1) / nblk;
    const int r0 = li * rows, r1 = min(m.nup, r0 + rows);
    if (use32 && jt_pairs_ok(m.B32, m.naux)) jt_rows_f2(m.B32, m.up_u, m.Jw, m.naux, r0, r1, m.Jpart + (size_t) li * m.naux);
    else if (use32 && m.B32) jt_rows<float>(m.B32, m.up_u, m.Jw, m.naux, r0, r1, m.Jpart + (size_t) li * m.naux);
    else jt_rows<double>(m.B, m.up_u, m.Jw, m.naux, r0, r1, m.Jpart + (size_t) li * m.naux);
}

__global__ void kb_j_weights(const MolDev *mols, const int *active, WorkList wl)
{
    BATCH_ITEM(wl)
    const int k = li * blockDim.x + threadIdx.x;
    if (k >= m.nup) return;
    const int i = m.up_i[k], j = m.up_j[k];
    m.Jw[k] = (i == j ? 1.0 : 2.0) * m.D[(size_t) i * m.nbf + j];
}

__global__ void kb_j_treduce(const MolDev *mols, const int *active, WorkList wl)
{
    BATCH_ITEM(wl)
    const int p = li * blockDim.x + threadIdx.x;
    if (p >= m.naux) return;
    m.Jt[p] = jt_reduce_col(m.Jpart, m.jblk, m.naux, p);
}

// 8 warps, 8 upper pairs per warp per item
template <typename BT>
__device__ __forceinline__ double row_dot(const BT *__restrict__ row, const double *ts, int naux, int lane)
{
    double s = 0.0;
    for (int p = lane; p < naux; p += 32) s = fma((double) __ldg(row + p), ts[p], s);
    return s;
}

__global__ void __launch_bounds__(256) kb_j_rows(const MolDev *mols, const int *active, WorkList wl, int use32)
{
    BATCH_ITEM(wl)
    extern __shared__ double ts[];
    for (int p = threadIdx.x; p < m.naux; p += blockDim.x) ts[p] = m.Jt[p];
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int q = 0; q < 8; q++) {
        const int k = li * 64 + wid * 8 + q;
        if (k >= m.nup) break;
        double s = (use32 && m.B32) ? row_dot<float>(m.B32 + (size_t) m.up_u[k] * m.naux, ts, m.naux, lane)
                                    : row_dot<double>(m.B + (size_t) m.up_u[k] * m.naux, ts, m.naux, lane);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffff, s, o);
        if (lane == 0) {
            const int i = m.up_i[k], j = m.up_j[k];
            m.J[(size_t) i * m.nbf + j] = s;
            m.J[(size_t) j * m.nbf + i] = s;
        }
    }
}

// ---- K (FP64)
__global__ void __launch_bounds__(256) kb_half(const MolDev *mols, const int *active, WorkList wl)
{
    BATCH_ITEM(wl)
    const int st = (m.nocc + KT_M - 1) / KT_M, pt = (m.naux + KT_N - 1) / KT_N;
    const int i = li / (st * pt), rem = li % (st * pt);
    half_tile(m.B, m.Cocc, m.csr_j, m.csr_u, m.displs, m.nocc, m.naux, m.T, i, (rem / pt) * KT_M, (rem % pt) * KT_N);
}

__global__ void __launch_bounds__(256) kb_syrk(const MolDev *mols, const int *active, WorkList wl)
{
    BATCH_ITEM(wl)
    const int tile = li / m.ksplit, split = li % m.ksplit;
    const long long Q = (long long) m.nocc * m.naux;
    long long qchunk = (Q + m.ksplit - 1) / m.ksplit;
    qchunk = (qchunk + KT_K - 1) / KT_K * KT_K;
    const long long q_beg = (long long) split * qchunk, q_end = min(Q, q_beg + qchunk);
    const int2 tl = m.tiles[tile];
    syrk_tile(m.T, m.nbf, Q, q_beg, q_end, tl.x * KT_M, tl.y * KT_N, m.Kpart + (size_t) split * m.nbf * m.nbf);
}

__global__ void __launch_bounds__(256, 1) kb_half_wide(const MolDev *mols, const int *active, WorkList wl)
{
    BATCH_ITEM(wl)
    const int st = (m.nocc + KH_S - 1) / KH_S, pt = (m.naux + KH_P - 1) / KH_P;
    const int i = li / (st * pt), rem = li % (st * pt);
    half_tile_wide(m.B, m.Cocc, m.csr_j, m.csr_u, m.displs, m.nocc, m.naux, m.T, i, (rem / pt) * KH_S,
                   (rem % pt) * KH_P);
}

__global__ void __launch_bounds__(256, 1) kb_half_dmma(const MolDev *mols, const int *active, WorkList wl)
{
    BATCH_ITEM(wl)
    const int st = (m.nocc + KH_S - 1) / KH_S, pt = (m.naux + KH_P - 1) / KH_P;
    const int i = li / (st * pt), rem = li % (st * pt);
    half_tile_dmma(m.B, m.Cocc, m.csr_j, m.csr_u, m.displs, m.nocc, m.naux, m.T, i, (rem / pt) * KH_S,
                   (rem % pt) * KH_P);
}

__global__ void __launch_bounds__(256, 1) kb_syrk128(const MolDev *mols, const int *active, WorkList wl)
{
    BATCH_ITEM(wl)
    const int tile = li / m.ksplit, split = li % m.ksplit;
    const long long Q = (long long) m.nocc * m.naux;
    long long qchunk = (Q + m.ksplit - 1) / m.ksplit;
    qchunk = (qchunk + KT_K - 1) / KT_K * KT_K;
    const long long q_beg = (long long) split * qchunk, q_end = min(Q, q_beg + qchunk);
    const int2 tl = m.tiles[tile];
    syrk_tile128(m.T, m.nbf, Q, q_beg, q_end, tl.x * KB_T, tl.y * KB_T, m.Kpart + (size_t) split * m.nbf * m.nbf);
}

__global__ void __launch_bounds__(256, 1) kb_syrk_dmma(const MolDev *mols, const int *active, WorkList wl)
{
    BATCH_ITEM(wl)
    const int tile = li / m.ksplit, split = li % m.ksplit;
    const long long Q = (long long) m.nocc * m.naux;
    long long qchunk = (Q + m.ksplit - 1) / m.ksplit;
    qchunk = (qchunk + KT_K - 1) / KT_K * KT_K;
    const long long q_beg = (long long) split * qchunk, q_end = min(Q, q_beg + qchunk);
    const int2 tl = m.tiles[tile];
    syrk_tile_dmma(m.T, m.nbf, Q, q_beg, q_end, tl.x * KB_T, tl.y * KB_T, m.Kpart + (size_t) split * m.nbf * m.nbf);
}

__global__ void kb_syrk_reduce(const MolDev *mols, const int *active, WorkList wl)
{
    BATCH_ITEM(wl)
    const size_t idx = (size_t) li * blockDim.x + threadIdx.x;
    const size_t nn = (size_t) m.nbf * m.nbf;
    if (idx >= nn) return;
    const int i = (int) (idx / m.nbf), j = (int) (idx % m.nbf);
    if (i > j) return;
    double s = 0.0;
    for (int k = 0; k < m.ksplit; k++) s += m.Kpart[(size_t) k * nn + idx];
    m.K[idx] = s;
    m.K[(size_t) j * m.nbf + i] = s;
}

// ---- Fock + energy: ENERGY_BLOCKS items per molecule with the single-molecule stride
__global__ void kb_fock(const MolDev *mols, const int *active, WorkList wl)
{
    BATCH_ITEM(wl)
    const size_t nn = (size_t) m.nbf * m.nbf;
    double e = fock_energy_range(m.H, m.J, m.K, m.D, m.F, (size_t) li * blockDim.x + threadIdx.x, nn,
                                 (size_t) ENERGY_BLOCKS * blockDim.x);
    e = block_sum(e);
    if (threadIdx.x == 0) m.epart[li] = e;
}

// one block per molecule: fixed-order sum of the partials, gathered into Eall
__global__ void kb_energy(const MolDev *mols, const int *active, double *Eall)
{
    const int mol = blockIdx.x;
    if (!active[mol]) return;
    if (threadIdx.x == 0) {
        const MolDev &m = mols[mol];
        double s = 0.0;
        for (int i = 0; i < ENERGY_BLOCKS; i++) s += m.epart[i];
        *m.E = s;
        Eall[mol] = s;
    }
}

// ---- batched DGEMM over per-molecule descriptors
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) kb_dgemm(const GemmDesc *descs, const int *active, WorkList wl)
{
    const int g = blockIdx.x;
    const int mol = find_mol(wl.start, wl.nmol, g);
    if (!active[mol]) return;
    const int li = g - wl.start[mol];
    const GemmDesc &d = descs[mol];
    const int nt = (d.n + GB_N - 1) / GB_N;
    dgemm_tile<TA, TB>(d.m, d.n, d.k, d.alpha, d.A, d.lda, d.B, d.ldb, d.beta, d.C, d.ldc, (li / nt) * GB_M,
                       (li % nt) * GB_N);
}

// ---- DIIS (DIIS.c:12-123), per-molecule state
__global__ void kb_diis_select(const MolDev *mols, const int *active, int nmol)
{
    const int mol = blockIdx.x * blockDim.x + threadIdx.x;
    if (mol >= nmol || !active[mol]) return;
    DiisState *st = mols[mol].diis;
    const int md = mols[mol].max_diis;
    if (st->len < md) {
        st->idx = st->len;
        st->len++;
    } else {
        st->idx = st->bmax_id;
    }
}

// out = A - A^T over the molecule's n x n (elementwise items of 256)
__global__ void kb_antisym(const MolDev *mols, const int *active, WorkList wl, int which)
{
    BATCH_ITEM(wl)
    const size_t idx = (size_t) li * blockDim.x + threadIdx.x;
    const int n = m.nbf;
    if (idx >= (size_t) n * n) return;
    const int i = (int) (idx / n), j = (int) (idx % n);
    const double *A = which ? m.tmp : m.tmp2;
    double *out = which ? m.tmp2 : m.tmp;
    out[idx] = A[idx] - A[(size_t) j * n + i];
}

// slots[idx] = src: which = 0 -> R slots from tmp, 1 -> F0 slots from tmp2
__global__ void kb_copy_to_slot(const MolDev *mols, const int *active, WorkList wl, int which)
{
    BATCH_ITEM(wl)
    const size_t nn = (size_t) m.nbf * m.nbf;
    const size_t i = (size_t) li * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    double *slots = which ? m.F0 : m.R;
    const double *src = which ? m.tmp2 : m.tmp;
    slots[(size_t) m.diis->idx * nn + i] = src[i];
}

__global__ void kb_diis_dots(const MolDev *mols, const int *active)
{
    const int mol = blockIdx.x / MAXDIIS, j = blockIdx.x % MAXDIIS;
    if (!active[mol]) return;
    const MolDev &m = mols[mol];
    DiisState *st = m.diis;
    if (j >= st->len) return;
    const size_t nn = (size_t) m.nbf * m.nbf;
    const double *a = m.R + (size_t) st->idx * nn, *b = m.R + (size_t) j * nn;
    double s = 0.0;
    for (size_t i = threadIdx.x; i < nn; i += blockDim.x) s = fma(a[i], b[i], s);
    s = block_sum(s);
    if (threadIdx.x == 0) st->dots[j] = s;
}

__global__ void kb_diis_combine(const MolDev *mols, const int *active, WorkList wl)
{
    BATCH_ITEM(wl)
    const size_t nn = (size_t) m.nbf * m.nbf;
    const size_t e = (size_t) li * blockDim.x + threadIdx.x;
    if (e >= nn) return;
    const DiisState *st = m.diis;
    double s = 0.0;
    for (int i = 0; i < st->len; i++) s += st->coef[i] * m.F0[(size_t) i * nn + e];
    m.Fp[e] = s;
}

// F' of every molecule into its slot of the eigensolver group buffer
__global__ void kb_copy_fp(const MolDev *mols, const int *active, WorkList wl)
{
    BATCH_ITEM(wl)
    const size_t nn = (size_t) m.nbf * m.nbf;
    const size_t i = (size_t) li * blockDim.x + threadIdx.x;
    if (i < nn) m.eigA[i] = m.Fp[i];
}

}  // namespace

void diis_solve_batched(const MolDev *d_mols, const int *d_active, int nmol, cudaStream_t s);

void batch_j(const BatchPlan &b, cudaStream_t s, int use32)
{
    const size_t shm = sizeof(double) * b.naux_max;
    if (shm > 48 * 1024) cudaFuncSetAttribute(kb_j_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) shm);
    kb_j_weights<<<b.nup256.total, 256, 0, s>>>(b.mols, b.active, b.nup256);
    kb_j_tpart<<<b.jblk.total, JT_THREADS, 0, s>>>(b.mols, b.active, b.jblk, use32);
    kb_j_treduce<<<b.naux256.total, 256, 0, s>>>(b.mols, b.active, b.naux256);
    kb_j_rows<<<b.nup64.total, 256, sizeof(double) * b.naux_max, s>>>(b.mols, b.active, b.nup64, use32);
    g_launches += 4;
}

void batch_k(const BatchPlan &b, const int *kact, cudaStream_t s)
{
    if (b.half.total) kb_half<<<b.half.total, 256, 0, s>>>(b.mols, kact, b.half);
    if (b.half_wide.total) kb_half_wide<<<b.half_wide.total, 256, 0, s>>>(b.mols, kact, b.half_wide);
    if (b.half_dmma.total) kb_half_dmma<<<b.half_dmma.total, 256, 0, s>>>(b.mols, kact, b.half_dmma);
    if (b.syrk.total) kb_syrk<<<b.syrk.total, 256, 0, s>>>(b.mols, kact, b.syrk);
    if (b.syrk128.total) kb_syrk128<<<b.syrk128.total, 256, 0, s>>>(b.mols, kact, b.syrk128);
    if (b.syrk_dmma.total) kb_syrk_dmma<<<b.syrk_dmma.total, 256, 0, s>>>(b.mols, kact, b.syrk_dmma);
    kb_syrk_reduce<<<b.nn256.total, 256, 0, s>>>(b.mols, kact, b.nn256);
    g_launches += 1 + (b.half.total > 0) + (b.half_wide.total > 0) + (b.half_dmma.total > 0) + (b.syrk.total > 0) +
                  (b.syrk128.total > 0) + (b.syrk_dmma.total > 0);
}

void batch_fock(const BatchPlan &b, double *d_Eall, cudaStream_t s)
{
    kb_fock<<<b.efb.total, 256, 0, s>>>(b.mols, b.active, b.efb);
    kb_energy<<<b.nmol, 32, 0, s>>>(b.mols, b.active, d_Eall);
    g_launches += 2;
}

void batch_gemm(const BatchGemm &g, const int *d_active, cudaStream_t s)
{
    if (g.wl.total <= 0) return;
    g_launches++;
    if (!g.ta && !g.tb) kb_dgemm<false, false><<<g.wl.total, 256, 0, s>>>(g.descs, d_active, g.wl);
    else if (!g.ta && g.tb) kb_dgemm<false, true><<<g.wl.total, 256, 0, s>>>(g.descs, d_active, g.wl);
    else if (g.ta && !g.tb) kb_dgemm<true, false><<<g.wl.total, 256, 0, s>>>(g.descs, d_active, g.wl);
    else kb_dgemm<true, true><<<g.wl.total, 256, 0, s>>>(g.descs, d_active, g.wl);
}

// X^T F X into Fp (iterations 0 and 1), or the full commutator DIIS step.
void batch_diis(const BatchPlan &b, bool full, cudaStream_t s)
{
    if (!full) {
        batch_gemm(b.g_xtf, b.active, s);     // tmp = X^T F
        batch_gemm(b.g_tx_fp, b.active, s);   // Fp = tmp X
        return;
    }
    kb_diis_select<<<(b.nmol + 127) / 128, 128, 0, s>>>(b.mols, b.active, b.nmol);
    batch_gemm(b.g_fd, b.active, s);          // tmp = F D
    batch_gemm(b.g_fds, b.active, s);         // tmp2 = tmp S
    kb_antisym<<<b.nn256.total, 256, 0, s>>>(b.mols, b.active, b.nn256, 0);   // tmp = tmp2 - tmp2^T
    batch_gemm(b.g_xtt, b.active, s);         // tmp2 = X^T tmp
    batch_gemm(b.g_t2x, b.active, s);         // tmp = tmp2 X
    kb_copy_to_slot<<<b.nn256.total, 256, 0, s>>>(b.mols, b.active, b.nn256, 0);
    kb_diis_dots<<<b.nmol * MAXDIIS, 1024, 0, s>>>(b.mols, b.active);
    batch_gemm(b.g_xtf, b.active, s);         // tmp = X^T F
    batch_gemm(b.g_tx_t2, b.active, s);       // tmp2 = tmp X
    kb_copy_to_slot<<<b.nn256.total, 256, 0, s>>>(b.mols, b.active, b.nn256, 1);
    diis_solve_batched(b.mols, b.active, b.nmol, s);
    kb_diis_combine<<<b.nn256.total, 256, 0, s>>>(b.mols, b.active, b.nn256);
    g_launches += 6;
}

void batch_copy_fp(const BatchPlan &b, const int *mask, cudaStream_t s)
{
    kb_copy_fp<<<b.nn256.total, 256, 0, s>>>(b.mols, mask, b.nn256);
    g_launches++;
}

}  // namespace tscf
