// FP64 symmetric eigensolver of the SCF: X = S^-1/2 (TinySCF.c:58-76), the
// DF metric's (P|Q)^-1/2 (build_DF_tensor.c:205-237) and the orthogonalised
// Fock eigensolve (build_density.c:37-69), where the reference calls
// LAPACKE_dsyev. Three stages, all on the device:
//
//  1. Householder tridiagonalisation Q^T A Q = T (LAPACK dsytrd/dlatrd's
//     recurrence). Panels of TRD_NB columns: one cooperative kernel per panel
//     runs the column steps -- update the column with the panel's earlier
//     reflectors, form the reflector, the symmetric matrix-vector product with
//     the trailing matrix (not yet updated for the panel), the panel
//     corrections -- separated by grid barriers; then two GEMMs apply the
//     rank-2*TRD_NB update to the trailing matrix.
//  2. Divide and conquer on T (Cuppen): T is torn by rank-one updates down to
//     1 x 1 pieces; each merge of two solved halves deflates small and close
//     components (LAPACK dlaed2's tests, Givens rotations for close pairs),
//     finds the roots of the secular equation by bisection on the offset from
//     the nearer pole, recomputes z from the roots (Gu-Eisenstat, so that the
//     eigenvectors come out orthogonal) and multiplies the halves' vectors by
//     the merge's vectors. All merges of one tree level run in the same launches.
//  3. Back-transformation with the compact WY form of each panel
//     (H_p..H_(p+nb-1) = I - V T V^T), three GEMMs per panel.
//
// Every grid barrier spins a bounded number of times; a barrier that runs out
// sets the object's error flag and every CTA returns (eig_error() reports it).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <vector>

#include "tiles.cuh"
#include "tscf_internal.h"

namespace tscf {

std::atomic<long long> g_eig_launches{0};

namespace {

constexpr int TRD_THREADS = 512;
constexpr int TRD_NB = 32;        // columns per panel
constexpr int TRD_SEG = 256;     // columns per item of the symmetric matrix-vector product
constexpr int GR_KS = 8;          // row slices of the reflector blocks' Gram matrices
constexpr int BT_NB = 128;        // reflectors per block of the back-transformation
constexpr int DC_CHUNK = 256;     // items per CTA of the thread-per-item D&C kernels
constexpr int DC_WCHUNK = 8;      // items per CTA of the warp-per-item D&C kernels (256 threads)
constexpr long long kBarrierSpins = 1LL << 22;   // acquire polls before a barrier gives up (~ 2 s)

__device__ __forceinline__ double warp_sum_bcast(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffff, v, o);
    return __shfl_sync(0xffffffff, v, 0);
}

__device__ __forceinline__ double warp_prod_bcast(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v *= __shfl_down_sync(0xffffffff, v, o);
    return __shfl_sync(0xffffffff, v, 0);
}

// Sum over the block in a fixed order (warp trees, then warp 0 over the
// warps); the result is returned to every thread.
template <int NT>
__device__ __forceinline__ double block_sum_all(double v, double *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffff, v, o);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (wid == 0) {
        double x = lane < NT / 32 ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffff, x, o);
        if (lane == 0) sh[32] = x;
    }
    __syncthreads();
    const double r = sh[32];
    __syncthreads();
    return r;
}

template <int NT>
__device__ __forceinline__ double block_max_all(double v, double *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffff, v, o));
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (wid == 0) {
        double x = lane < NT / 32 ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_down_sync(0xffffffff, x, o));
        if (lane == 0) sh[32] = x;
    }
    __syncthreads();
    const double r = sh[32];
    __syncthreads();
    return r;
}

// Grid barrier for a cooperative launch (all CTAs co-resident): a 64-bit
// ticket counter that only grows (zeroed before each solve). Thread 0 of each
// CTA arrives with a release add and spins with acquire loads until the
// counter reaches the end of its episode (the next multiple of nblk). The
// wait is bounded: a CTA whose wait runs out sets the error flag and returns
// false, and the caller returns; CTAs still waiting for it run out in turn.
__device__ __forceinline__ unsigned long long atom_add_release(unsigned long long *p, unsigned long long v)
{
    unsigned long long old;
    asm volatile("atom.add.release.gpu.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool grid_barrier(unsigned long long *bar, int *err, unsigned nblk)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long ticket = atom_add_release(bar, 1ull);
        const unsigned long long target = (ticket / nblk + 1) * nblk;
        long long spins = 0;
        bool ok = true;
        while (ld_acquire(bar) < target) {
            if (++spins > kBarrierSpins) {
                atomicExch(err, 1);
                ok = false;
                break;
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ------------------------------------------------------------------ tridiagonalisation
// Storage: reflector j is row j of VT (v_j[j+1] = 1, zero before); within a
// panel, PVW rows 0..NB-1 hold the panel's v and rows NB..2NB-1 its w, PWV the
// same two halves swapped, so that the trailing update A22 -= V W^T + W V^T is
// one GEMM PVW^T PWV with K = 2 NB, and every in-panel access to v or w runs
// along a row (coalesced).
struct TrdArgs {
    double *A;      // n x n work matrix (trailing part updated after each panel)
    double *VT;     // n x n reflectors as rows
    double *PVW, *PWV;   // 2 TRD_NB x n each
    double *d, *e, *tau;
    double *col;
    double *y;      // [segment][row] partial sums of A v
    double *part;   // [G] norms | [2 TRD_NB][G] panel dots | [G] w.v
    unsigned long long *bar;
    int *err;
    int n, p, cols, G;
};

__global__ void __launch_bounds__(TRD_THREADS, 1) k_sytrd_panel(TrdArgs a)
{
    extern __shared__ double sv[];   // v of the current column, by absolute row
    __shared__ double s_a2[TRD_NB], s_wv[TRD_NB], s_vv[TRD_NB], s_vj[TRD_NB], s_wj[TRD_NB];
    __shared__ double s_red[33];
    __shared__ double s_dot[TRD_THREADS / 32][2 * TRD_NB];
    __shared__ double s_tau, s_scal, s_beta;
    const int n = a.n, p = a.p, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int gtid = blockIdx.x * TRD_THREADS + tid, GT = a.G * TRD_THREADS;
    const int gw = blockIdx.x * (TRD_THREADS / 32) + wid, GW = a.G * (TRD_THREADS / 32);
    // Row r of the matrix belongs to the 8-lane group r for the whole panel
    // (G * TRD_THREADS / 8 >= n); lane l8 of the group keeps the row's entries
    // of panel columns l8, l8 + 8, l8 + 16, l8 + 24 of V and W in registers.
    const int l8 = lane & 7, r = gtid >> 3;
    const bool own = r < n;
    constexpr int NQ = TRD_NB / 8;
    double pv[NQ], pw[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) pv[q] = pw[q] = 0.0;
    const int nseg = (n + TRD_SEG - 1) / TRD_SEG;
    double *part_n = a.part, *part_d = a.part + a.G, *part_w = part_d + (size_t) a.G * 2 * TRD_NB;
    const double *A = a.A;
    // row p of the symmetric matrix: column p of the first step
    double arow = (own && r >= p && l8 == 0) ? A[(size_t) p * n + r] : 0.0;
    for (int c = 0; c < a.cols; c++) {
        const int j = p + c;
        // ---- phase 1: column j of the panel-corrected matrix, rows j..n-1 (s_vj, s_wj: row j's V and W)
        double v = 0.0;
        if (own && r >= j) {
            v = arow;
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                const int cc = l8 + 8 * q;
                if (cc < c) v -= pv[q] * s_wj[cc] + pw[q] * s_vj[cc];
            }
        }
        v += __shfl_xor_sync(0xffffffff, v, 1);
        v += __shfl_xor_sync(0xffffffff, v, 2);
        v += __shfl_xor_sync(0xffffffff, v, 4);
        double ss = 0.0;
        if (own && r >= j && l8 == 0) {
            a.col[r] = v;
            if (r >= j + 2) ss = v * v;
        }
        ss = block_sum_all<TRD_THREADS>(ss, s_red);
        if (tid == 0) part_n[blockIdx.x] = ss;
        if (!grid_barrier(a.bar, a.err, a.G)) return;
        if (j == n - 1) {
            if (gtid == 0) a.d[j] = a.col[j];
            break;
        }
        // ---- phase 2: reflector (every CTA forms the same one), v, y = A v by segments, panel dots
        for (int rr = j + 1 + tid; rr < n; rr += TRD_THREADS) sv[rr] = a.col[rr];   // issued with part_n's loads
        if (wid == 0) {
            double s = 0.0;
            for (int b = lane; b < a.G; b += 32) s += part_n[b];
            s = warp_sum_bcast(s);
            if (lane == 0) {
                const double alpha = a.col[j + 1];
                if (s == 0.0) {
                    s_tau = 0.0;
                    s_beta = alpha;
                    s_scal = 0.0;
                } else {
                    const double nrm = sqrt(alpha * alpha + s);
                    const double beta = alpha >= 0.0 ? -nrm : nrm;
                    s_tau = (beta - alpha) / beta;
                    s_beta = beta;
                    s_scal = 1.0 / (alpha - beta);
                }
            }
        }
        __syncthreads();
        const double tau = s_tau, scal = s_scal;
        for (int rr = j + 1 + tid; rr < n; rr += TRD_THREADS) sv[rr] = (rr == j + 1) ? 1.0 : sv[rr] * scal;
        __syncthreads();
        if (gtid == 0) {
            a.d[j] = a.col[j];
            a.e[j] = s_beta;
            a.tau[j] = tau;
        }
        for (int rr = j + 1 + gtid; rr < n; rr += GT) {
            const double vr = sv[rr];
            a.VT[(size_t) j * n + rr] = vr;
            a.PVW[(size_t) c * n + rr] = vr;
            a.PWV[(size_t) (TRD_NB + c) * n + rr] = vr;
        }
        const double vr_own = (own && r > j) ? sv[r] : 0.0;
        if (l8 == (c & 7)) {   // this row's entry of the new reflector (static register indexing)
#pragma unroll
            for (int q = 0; q < NQ; q++)
                if (q == (c >> 3)) pv[q] = vr_own;
        }
        {
            // items (row rr, segment sg) over rows j+1..n-1 and the segments holding columns j+1..n-1
            const int s0 = (j + 1) / TRD_SEG, ns = nseg - s0, m = n - j - 1;
            const long long nitems = (long long) m * ns;
            for (long long it = gw; it < nitems; it += GW) {
                const int rr = j + 1 + (int) (it / ns), sg = s0 + (int) (it % ns);
                const double *row = A + (size_t) rr * n;
                double acc[TRD_SEG / 32];
#pragma unroll
                for (int k = 0; k < TRD_SEG / 32; k++) {
                    const int c2 = sg * TRD_SEG + lane + 32 * k;
                    acc[k] = (c2 > j && c2 < n) ? row[c2] * sv[c2] : 0.0;
                }
                static_assert(TRD_SEG == 256, "the pairwise sum below is written for 8 values per lane");
                const double y = warp_sum_bcast(((acc[0] + acc[4]) + (acc[2] + acc[6])) +
                                                ((acc[1] + acc[5]) + (acc[3] + acc[7])));
                if (lane == 0) a.y[(size_t) sg * n + rr] = y;
            }
        }
        if (c > 0) {
            // panel dots W^T v and V^T v over this CTA's rows, from the registers: groups of a warp
            // (lanes with equal l8) summed by shuffles, then the warps in shared memory
            double dw[NQ], dv[NQ];
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                dw[q] = pw[q] * vr_own;
                dv[q] = pv[q] * vr_own;
                dw[q] += __shfl_xor_sync(0xffffffff, dw[q], 8);
                dw[q] += __shfl_xor_sync(0xffffffff, dw[q], 16);
                dv[q] += __shfl_xor_sync(0xffffffff, dv[q], 8);
                dv[q] += __shfl_xor_sync(0xffffffff, dv[q], 16);
            }
            if (lane < 8) {
#pragma unroll
                for (int q = 0; q < NQ; q++) {
                    s_dot[wid][lane + 8 * q] = dw[q];
                    s_dot[wid][TRD_NB + lane + 8 * q] = dv[q];
                }
            }
            __syncthreads();
            if (tid < 2 * TRD_NB) {
                double sacc = 0.0;
                for (int w = 0; w < TRD_THREADS / 32; w++) sacc += s_dot[w][tid];
                part_d[(size_t) tid * a.G + blockIdx.x] = sacc;
            }
        }
        if (!grid_barrier(a.bar, a.err, a.G)) return;
        // ---- phase 3: w = tau (y - V (W^T v) - W (V^T v)) for this row, partial w.v
        double ypart = 0.0;
        const int s0 = (j + 1) / TRD_SEG;
        if (own && r > j)
            for (int sg = s0 + l8; sg < nseg; sg += 8) ypart += a.y[(size_t) sg * n + r];
        for (int cc = wid; cc < c; cc += TRD_THREADS / 32) {
            double sw = 0.0, sx = 0.0;
            for (int b = lane; b < a.G; b += 32) {
                sw += part_d[(size_t) cc * a.G + b];
                sx += part_d[(size_t) (TRD_NB + cc) * a.G + b];
            }
            sw = warp_sum_bcast(sw);
            sx = warp_sum_bcast(sx);
            if (lane == 0) {
                s_wv[cc] = sw;
                s_vv[cc] = sx;
            }
        }
        // the next column's row of A (issued here, used after the next two barriers)
        const bool nxt = c + 1 < a.cols;
        arow = (nxt && own && r >= j + 1 && l8 == 0) ? A[(size_t) (j + 1) * n + r] : 0.0;
        __syncthreads();
        double t = ypart;
        if (own && r > j) {
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                const int cc = l8 + 8 * q;
                if (cc < c) t -= pv[q] * s_wv[cc] + pw[q] * s_vv[cc];
            }
        }
        t += __shfl_xor_sync(0xffffffff, t, 1);
        t += __shfl_xor_sync(0xffffffff, t, 2);
        t += __shfl_xor_sync(0xffffffff, t, 4);
        const double w = (own && r > j) ? tau * t : 0.0;
        if (l8 == (c & 7)) {
#pragma unroll
            for (int q = 0; q < NQ; q++)
                if (q == (c >> 3)) pw[q] = w;
        }
        double wd = 0.0;
        if (own && r > j && l8 == 0) {
            a.PWV[(size_t) c * n + r] = w;   // before its a2 v term; row j+1's entry is read by every CTA
            wd = w * vr_own;
        }
        wd = block_sum_all<TRD_THREADS>(wd, s_red);
        if (tid == 0) part_w[blockIdx.x] = wd;
        if (!grid_barrier(a.bar, a.err, a.G)) return;
        // ---- phase 4: a2 = -tau/2 (w.v), w += a2 v; row j+1's V and W for the next column
        if (wid == 0) {
            double s = 0.0;
            for (int b = lane; b < a.G; b += 32) s += part_w[b];
            s = warp_sum_bcast(s);
            if (lane == 0) s_a2[c] = -0.5 * tau * s;
        } else if (nxt && wid == 1 && lane <= c) {
            s_vj[lane] = a.PVW[(size_t) lane * n + j + 1];
            s_wj[lane] = a.PWV[(size_t) lane * n + j + 1];   // before a2 v; completed below
        }
        __syncthreads();
        if (l8 == (c & 7)) {
#pragma unroll
            for (int q = 0; q < NQ; q++)
                if (q == (c >> 3)) pw[q] += s_a2[c] * pv[q];
        }
        if (nxt && tid <= c) s_wj[tid] += s_a2[tid] * s_vj[tid];   // global W holds the values before a2 v
        __syncthreads();
    }
    // final W of this panel's rows, into both stacked panels for the trailing update
    if (own && r >= p + a.cols) {
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            const int cc = l8 + 8 * q;
            if (cc < a.cols) {
                a.PWV[(size_t) cc * n + r] = pw[q];
                a.PVW[(size_t) (TRD_NB + cc) * n + r] = pw[q];
            }
        }
    }
}

// Partial Gram matrices V_B^T V_B of the reflector blocks (the reflectors of
// block B are rows p0..p0+bb-1 of VT, zero before column p0 + 1): CTA (B,
// 32 x 32 tile, slice ks of the columns) writes its slice's sum to Gp[B][ks].
__global__ void __launch_bounds__(256) k_wy_gram(const double *VT, double *Gp, int n, int nref)
{
    __shared__ double As[32][65], Bs[32][65];
    const int B = blockIdx.x, tile = blockIdx.y, ks = blockIdx.z;
    const int p0 = B * BT_NB, bb = min(BT_NB, nref - p0);
    const int ta = tile / (BT_NB / 32), tb = tile % (BT_NB / 32);
    const int K0 = p0 + 1, K = n - K0, kper = (K + GR_KS - 1) / GR_KS;
    const int k0 = K0 + ks * kper, k1 = min(n, k0 + kper);
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double acc[2][2] = {};
    for (int kc = k0; kc < k1; kc += 64) {
        for (int l = threadIdx.x; l < 32 * 64; l += 256) {
            const int rr = l / 64, kk = l % 64, k = kc + kk;
            const int ra = ta * 32 + rr, rb = tb * 32 + rr;
            As[rr][kk] = (ra < bb && k < k1) ? VT[(size_t) (p0 + ra) * n + k] : 0.0;
            Bs[rr][kk] = (rb < bb && k < k1) ? VT[(size_t) (p0 + rb) * n + k] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < 64; kk++) {
            const double a0 = As[ty][kk], a1 = As[ty + 16][kk], b0 = Bs[tx][kk], b1 = Bs[tx + 16][kk];
            acc[0][0] += a0 * b0;
            acc[0][1] += a0 * b1;
            acc[1][0] += a1 * b0;
            acc[1][1] += a1 * b1;
        }
        __syncthreads();
    }
    double *G = Gp + (size_t) (B * GR_KS + ks) * BT_NB * BT_NB;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int jj = 0; jj < 2; jj++) G[(size_t) (ta * 32 + ty + 16 * i) * BT_NB + tb * 32 + tx + 16 * jj] = acc[i][jj];
}

// T of the compact WY form of each block of BT_NB reflectors:
// H_p0 ... H_(p0+bb-1) = I - V T V^T, T upper triangular (LAPACK dlarft,
// forward, columnwise), from the block's Gram matrix (the sum of its
// GR_KS slices). One CTA per block.
__global__ void __launch_bounds__(256) k_wy_tfactor(const double *Gp, const double *tau, double *Tf, int nref)
{
    extern __shared__ double tsm[];
    constexpr int LD = BT_NB + 1;
    double *T = tsm;                       // BT_NB x LD
    double *Gc = tsm + BT_NB * LD;         // column c of the Gram matrix
    const int B = blockIdx.x, p0 = B * BT_NB, bb = min(BT_NB, nref - p0), tid = threadIdx.x;
    const double *G = Gp + (size_t) B * GR_KS * BT_NB * BT_NB;
    for (int l = tid; l < BT_NB * LD; l += blockDim.x) T[l] = 0.0;
    __syncthreads();
    for (int c = 0; c < bb; c++) {
        const double tc = tau[p0 + c];
        if (tid < c) {
            double g = 0.0;
            for (int ks = 0; ks < GR_KS; ks++) g += G[(size_t) ks * BT_NB * BT_NB + (size_t) tid * BT_NB + c];
            Gc[tid] = g;
        }
        __syncthreads();
        if (tid < c) {
            double sacc = 0.0;
            for (int l = tid; l < c; l++) sacc += T[tid * LD + l] * Gc[l];
            T[tid * LD + c] = -tc * sacc;
        }
        if (tid == 0) T[c * LD + c] = tc;
        __syncthreads();
    }
    for (int l = tid; l < BT_NB * BT_NB; l += blockDim.x)
        Tf[(size_t) B * BT_NB * BT_NB + l] = T[(l / BT_NB) * LD + l % BT_NB];
}

// ------------------------------------------------------------------ divide and conquer
struct DcNodes {
    const int *lo, *mid, *hi;
    double *rho;      // per node, 2 |e[mid-1]|
    int *kcnt, *rcnt; // per node: non-deflated count, rotation count
};

struct DcPos {        // per position of the tridiagonal (node-local arrays start at lo)
    double *lam;      // eigenvalues of the solved pieces (ascending within each piece)
    double *ds;       // sorted, deflation-modified d
    double *dK, *zK;  // non-deflated d and z (compact)
    double *lamb, *tau;  // root j = lamb[j] + tau[j], lamb the nearer pole
    double *zh, *nrm;
    double *lamnew;
    int *perm;        // sorted position -> index into the concatenated children
    int *keep, *defl; // sorted positions kept / deflated (compact)
    int *rowinfo;     // sorted position -> kept index i, or -(deflated index + 1)
    int *colsrc;      // output column -> secular root j (< k) or k + deflated index
    int2 *rot;        // Givens rotations of the close pairs (rows pj, nj, sorted positions)
    double2 *rotcs;   // their (C, S)
};

// Both eigenvector buffers start as the identity: a piece of size one keeps
// its vector in both, so a merge finds it whichever buffer it reads.
__global__ void k_dc_init(const double *d, const double *e, double *lam, double *Qa, double *Qb, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // every boundary i|i+1 is the split point of exactly one merge: tear both sides
    double v = d[i];
    if (i + 1 < n) v -= fabs(e[i]);
    if (i > 0) v -= fabs(e[i - 1]);
    lam[i] = v;
    Qa[(size_t) i * n + i] = 1.0;
    Qb[(size_t) i * n + i] = 1.0;
}

// Sorting of the two halves, z, the tolerance and the deflation scan. One CTA per node.
__global__ void __launch_bounds__(512) k_dc_deflate(DcNodes nd, DcPos ps, const double *Q, const double *e, int n,
                                                    int node0)
{
    extern __shared__ double dsm[];
    __shared__ double s_red[33];
    const int node = node0 + blockIdx.x;
    const int lo = nd.lo[node], mid = nd.mid[node], hi = nd.hi[node];
    const int m = hi - lo, m1 = mid - lo, m2 = hi - mid;
    double *sd = dsm, *sz = dsm + m;
    int *sp = (int *) (dsm + 2 * m);
    const double rho_raw = e[mid - 1];
    const double rho = 2.0 * fabs(rho_raw), sg = rho_raw >= 0.0 ? 1.0 : -1.0;
    const double *L1 = ps.lam + lo, *L2 = ps.lam + mid;
    const double rs2 = 1.0 / sqrt(2.0);
    // every slot holds a valid index even if non-finite values make the merge below collide
    for (int idx = threadIdx.x; idx < m; idx += blockDim.x) {
        sd[idx] = 0.0;
        sz[idx] = 0.0;
        sp[idx] = idx;
    }
    __syncthreads();
    double dmax = 0.0, zmax = 0.0;
    for (int idx = threadIdx.x; idx < m; idx += blockDim.x) {
        double x, zz;
        int pos;
        if (idx < m1) {
            x = L1[idx];
            zz = Q[(size_t) (mid - 1) * n + lo + idx];
            int a = 0, b = m2;   // first L2 >= x
            while (a < b) {
                const int c = (a + b) >> 1;
                if (L2[c] < x) a = c + 1; else b = c;
            }
            pos = idx + a;
        } else {
            const int i2 = idx - m1;
            x = L2[i2];
            zz = sg * Q[(size_t) mid * n + mid + i2];
            int a = 0, b = m1;   // first L1 > x
            while (a < b) {
                const int c = (a + b) >> 1;
                if (L1[c] <= x) a = c + 1; else b = c;
            }
            pos = i2 + a;
        }
        pos = min(max(pos, 0), m - 1);
        zz *= rs2;
        sd[pos] = x;
        sz[pos] = zz;
        sp[pos] = idx;
        dmax = fmax(dmax, fabs(x));
        zmax = fmax(zmax, fabs(zz));
    }
    dmax = block_max_all<512>(dmax, s_red);
    zmax = block_max_all<512>(zmax, s_red);
    const double tol = 8.0 * DBL_EPSILON * fmax(dmax, zmax);
    int *keep = ps.keep + lo, *defl = ps.defl + lo, *rowinfo = ps.rowinfo + lo;
    if (threadIdx.x == 0) {
        int k = 0, nd_ = 0, nr = 0;
        if (rho * zmax <= tol) {
            for (int s = 0; s < m; s++) {
                rowinfo[s] = -(nd_ + 1);
                defl[nd_++] = s;
            }
        } else {
            int pj = -1;
            for (int s = 0; s < m; s++) {
                if (rho * fabs(sz[s]) <= tol) {
                    rowinfo[s] = -(nd_ + 1);
                    defl[nd_++] = s;
                    continue;
                }
                if (pj < 0) {
                    pj = s;
                    continue;
                }
                // close pair: |t C S| <= tol with C = z_s / h, S = -z_pj / h, h = hypot(z_s, z_pj)
                const double zp = sz[pj], zs = sz[s], t = sd[s] - sd[pj];
                if (fabs(t * zs * zp) <= tol * (zs * zs + zp * zp)) {
                    const double tt = hypot(zs, zp), C = zs / tt, S = -zp / tt;
                    sz[s] = tt;
                    sz[pj] = 0.0;
                    ps.rot[lo + nr] = make_int2(pj, s);
                    ps.rotcs[lo + nr] = make_double2(C, S);
                    nr++;
                    const double dp = sd[pj] * C * C + sd[s] * S * S;
                    sd[s] = sd[pj] * S * S + sd[s] * C * C;
                    sd[pj] = dp;
                    rowinfo[pj] = -(nd_ + 1);
                    defl[nd_++] = pj;
                    pj = s;
                } else {
                    rowinfo[pj] = k;
                    keep[k++] = pj;
                    pj = s;
                }
            }
            if (pj >= 0) {
                rowinfo[pj] = k;
                keep[k++] = pj;
            }
        }
        nd.kcnt[node] = k;
        nd.rcnt[node] = nr;
        nd.rho[node] = rho;
    }
    __syncthreads();
    const int k = nd.kcnt[node];
    for (int s = threadIdx.x; s < m; s += blockDim.x) {
        ps.ds[lo + s] = sd[s];
        ps.perm[lo + s] = sp[s];
    }
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const int s = keep[i];
        ps.dK[lo + i] = sd[s];
        ps.zK[lo + i] = sz[s];
    }
}

// Block tables: entry b = (node, first item) for the items [first, first + chunk) of that node.
__device__ __forceinline__ void secular_parts(const double *sd, const double *sz, int k, int j, double rho,
                                              double dorg, double t, int lane, double &p1, double &dp1, double &p2,
                                              double &dp2)
{
    double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
    for (int i = lane; i < k; i += 32) {
        const double q = sz[i] / ((sd[i] - dorg) - t);
        if (i <= j) {
            a += sz[i] * q;
            b += q * q;
        } else {
            c += sz[i] * q;
            d += q * q;
        }
    }
    p1 = rho * warp_sum_bcast(a);
    dp1 = rho * warp_sum_bcast(b);
    p2 = rho * warp_sum_bcast(c);
    dp2 = rho * warp_sum_bcast(d);
}

// Roots of f(l) = 1 + rho sum_i z_i^2 / (d_i - l) = 0, one warp per root:
// l_j = pole + tau, the pole the nearer of d_j, d_(j+1) (its position is the
// origin of tau, so tau keeps full relative accuracy), tau bracketed by the
// signs of f. Each step fits psi1 + psi2 on either side of the root by
// c + s / (pole - t) matched to value and slope at the current tau (the two
// poles around the root) and takes the model's root inside the bracket;
// a bisection step (geometric while the bracket spans more than a factor 4)
// when it falls outside. Stops when the step is below 2 eps |tau| or the
// bracket closes.
__global__ void __launch_bounds__(256) k_dc_secular(DcNodes nd, DcPos ps, const int2 *tab)
{
    extern __shared__ double dsm[];
    const int2 tb = tab[blockIdx.x];
    const int node = tb.x, lo = nd.lo[node], k = nd.kcnt[node];
    if (tb.y >= k) return;
    double *sd = dsm, *sz = dsm + k;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        sd[i] = ps.dK[lo + i];
        sz[i] = ps.zK[lo + i];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, j = tb.y + (threadIdx.x >> 5);
    if (j >= k) return;
    const double rho = nd.rho[node];
    int org;
    double tau;
    if (k == 1) {
        org = 0;
        tau = rho * sz[0] * sz[0];
    } else {
        const bool last = j == k - 1;
        double a, b;   // bracket in tau: f(a) < 0 < f(b)
        if (last) {
            double s = 0.0;
            for (int i = lane; i < k; i += 32) s += sz[i] * sz[i];
            org = j;
            a = 0.0;
            b = rho * warp_sum_bcast(s);
        } else {
            const double delta = sd[j + 1] - sd[j];
            double p1, dp1, p2, dp2;
            secular_parts(sd, sz, k, j, rho, sd[j], 0.5 * delta, lane, p1, dp1, p2, dp2);
            if (1.0 + p1 + p2 > 0.0) {
                org = j;
                a = 0.0;
                b = 0.5 * delta;
            } else {
                org = j + 1;
                a = -0.5 * delta;
                b = 0.0;
            }
        }
        const double dorg = sd[org];
        const double del1 = sd[j] - dorg;                       // lower pole, relative
        const double del2 = last ? 0.0 : sd[j + 1] - dorg;      // upper pole, relative
        tau = 0.5 * (a + b);
        for (int it = 0; it < 200; it++) {
            double p1, dp1, p2, dp2;
            secular_parts(sd, sz, k, j, rho, dorg, tau, lane, p1, dp1, p2, dp2);
            const double f = 1.0 + p1 + p2;
            if (f == 0.0) break;
            if (f < 0.0) a = tau; else b = tau;
            if (!(b - a > 4.0 * DBL_EPSILON * fmax(fabs(a), fabs(b)))) break;
            // two-pole model: C + s1 / (del1 - x) + s2 / (del2 - x) = 0
            const double e1 = del1 - tau, s1 = dp1 * e1 * e1, c1 = p1 - s1 / e1;
            double x = NAN;
            if (last) {
                const double C = 1.0 + c1 + p2;
                if (C > 0.0) x = del1 + s1 / C;
            } else {
                const double e2 = del2 - tau, s2 = dp2 * e2 * e2, c2 = p2 - s2 / e2;
                const double C = 1.0 + c1 + c2;
                const double qa = C, qb = -(C * (del1 + del2) + s1 + s2), qc = C * del1 * del2 + s1 * del2 + s2 * del1;
                const double disc = qb * qb - 4.0 * qa * qc;
                if (disc >= 0.0) {
                    const double q = -0.5 * (qb + copysign(sqrt(disc), qb));
                    const double r1 = q / qa, r2 = qc / q;
                    const bool in1 = r1 > a && r1 < b, in2 = r2 > a && r2 < b;
                    x = in1 && (!in2 || fabs(r1 - tau) < fabs(r2 - tau)) ? r1 : (in2 ? r2 : NAN);
                }
            }
            if (!(x > a && x < b)) {   // bisection, geometric on the side of the origin while the bracket is wide
                const double lo_ = fmin(fabs(a), fabs(b)), hi_ = fmax(fabs(a), fabs(b));
                const double sg = (a + b) >= 0.0 ? 1.0 : -1.0;
                x = (lo_ > 0.0 && hi_ > 4.0 * lo_ && a * b > 0.0) ? sg * sqrt(lo_ * hi_) : 0.5 * (a + b);
                if (x == 0.0) x = 0.5 * (a + b);
                if (!(x > a && x < b)) break;
            }
            const bool done = fabs(x - tau) <= 2.0 * DBL_EPSILON * fabs(x);
            tau = x;
            if (done) break;
        }
    }
    if (lane == 0) {
        ps.lamb[lo + j] = sd[org];
        ps.tau[lo + j] = tau;
    }
}

// z recomputed from the roots (Gu-Eisenstat): zh_i^2 = -(d_i - l_i) prod_(j != i) (d_i - l_j) / (d_i - d_j).
__global__ void __launch_bounds__(256) k_dc_zhat(DcNodes nd, DcPos ps, const int2 *tab)
{
    extern __shared__ double dsm[];
    const int2 tb = tab[blockIdx.x];
    const int node = tb.x, lo = nd.lo[node], k = nd.kcnt[node];
    if (tb.y >= k) return;
    double *sd = dsm, *sl = dsm + k, *st = dsm + 2 * k;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        sd[i] = ps.dK[lo + i];
        sl[i] = ps.lamb[lo + i];
        st[i] = ps.tau[lo + i];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, i = tb.y + (threadIdx.x >> 5);
    if (i >= k) return;
    const double di = sd[i];
    double pr = 1.0;
    for (int j = lane; j < k; j += 32) {
        const double del = (di - sl[j]) - st[j];
        pr *= (j == i) ? del : del / (di - sd[j]);
    }
    pr = warp_prod_bcast(pr);
    if (lane == 0) ps.zh[lo + i] = copysign(sqrt(fmax(-pr, 0.0)), ps.zK[lo + i]);
}

// Norm of each secular eigenvector u_j(i) = zh_i / (d_i - l_j).
__global__ void __launch_bounds__(256) k_dc_norms(DcNodes nd, DcPos ps, const int2 *tab)
{
    extern __shared__ double dsm[];
    const int2 tb = tab[blockIdx.x];
    const int node = tb.x, lo = nd.lo[node], k = nd.kcnt[node];
    if (tb.y >= k) return;
    double *sd = dsm, *sz = dsm + k;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        sd[i] = ps.dK[lo + i];
        sz[i] = ps.zh[lo + i];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, j = tb.y + (threadIdx.x >> 5);
    if (j >= k) return;
    const double lb = ps.lamb[lo + j], tj = ps.tau[lo + j];
    double s = 0.0;
    for (int i = lane; i < k; i += 32) {
        const double u = sz[i] / ((sd[i] - lb) - tj);
        s += u * u;
    }
    s = warp_sum_bcast(s);
    if (lane == 0) ps.nrm[lo + j] = sqrt(s);
}

// Output order of the node's eigenvalues (ascending; ties by source index) by rank counting.
__global__ void __launch_bounds__(DC_CHUNK) k_dc_order(DcNodes nd, DcPos ps, const int2 *tab)
{
    extern __shared__ double dsm[];
    const int2 tb = tab[blockIdx.x];
    const int node = tb.x, lo = nd.lo[node], m = nd.hi[node] - lo, k = nd.kcnt[node];
    double *sv = dsm;
    for (int a = threadIdx.x; a < m; a += blockDim.x)
        sv[a] = (a < k) ? ps.lamb[lo + a] + ps.tau[lo + a] : ps.ds[lo + ps.defl[lo + a - k]];
    __syncthreads();
    const int a = tb.y + threadIdx.x;
    if (a >= m) return;
    const double x = sv[a];
    int r = 0;
    for (int b = 0; b < m; b++) {
        const double y = sv[b];
        r += (y < x || (y == x && b < a)) ? 1 : 0;
    }
    r = min(r, m - 1);
    ps.lamnew[lo + r] = x;
    ps.colsrc[lo + r] = a;
}

// The merge's eigenvector matrix U, one warp per sorted position s (written to
// row perm[s], i.e. in the children's order): column c = secular vector j
// (normalised) or the unit vector of a deflated position.
__global__ void __launch_bounds__(256) k_dc_build(DcNodes nd, DcPos ps, const int2 *tab, double *Us, int n)
{
    const int2 tb = tab[blockIdx.x];
    const int node = tb.x, lo = nd.lo[node], m = nd.hi[node] - lo, k = nd.kcnt[node];
    const int lane = threadIdx.x & 31, s = tb.y + (threadIdx.x >> 5);
    if (s >= m) return;
    const int info = ps.rowinfo[lo + s];
    const double di = info >= 0 ? ps.dK[lo + info] : 0.0, zi = info >= 0 ? ps.zh[lo + info] : 0.0;
    double *row = Us + (size_t) (lo + ps.perm[lo + s]) * n + lo;   // row of the child-order basis
    for (int c = lane; c < m; c += 32) {
        const int src = ps.colsrc[lo + c];
        double v;
        if (src >= 0 && src < k) v = info >= 0 ? zi / ((di - ps.lamb[lo + src]) - ps.tau[lo + src]) / ps.nrm[lo + src] : 0.0;
        else v = (info < 0 && -(info + 1) == src - k) ? 1.0 : 0.0;
        row[c] = v;
    }
}

// Givens rotations of the deflation (on sorted positions, i.e. rows perm[.]
// of U), applied in reverse order; a thread per column.
__global__ void __launch_bounds__(DC_CHUNK) k_dc_rotate(DcNodes nd, DcPos ps, const int2 *tab, double *Us, int n)
{
    const int2 tb = tab[blockIdx.x];
    const int node = tb.x, lo = nd.lo[node], m = nd.hi[node] - lo, nr = nd.rcnt[node];
    const int c = tb.y + threadIdx.x;
    if (nr == 0 || c >= m) return;
    double *U = Us + (size_t) lo * n + lo + c;
    const int *perm = ps.perm + lo;
    for (int r = nr - 1; r >= 0; r--) {
        const int2 pr = ps.rot[lo + r];
        const double2 cs = ps.rotcs[lo + r];
        const size_t ix = (size_t) perm[pr.x] * n, iy = (size_t) perm[pr.y] * n;
        const double x = U[ix], y = U[iy];
        U[ix] = cs.x * x - cs.y * y;
        U[iy] = cs.y * x + cs.x * y;
    }
}

__global__ void k_dc_commit_lam(DcNodes nd, DcPos ps, const int2 *tab)
{
    const int2 tb = tab[blockIdx.x];
    const int node = tb.x, lo = nd.lo[node], m = nd.hi[node] - lo;
    const int a = tb.y + threadIdx.x;
    if (a < m) ps.lam[lo + a] = ps.lamnew[lo + a];
}

// New vectors of a node: [Q1 0; 0 Q2] U, one half at a time (rows of child
// 1 with child 1's block, rows of child 2 with child 2's), read from Qin and
// written to Qout; 64 x 64 tiles on the FP64 tensor cores. Tile entry:
// (node, half, tile row, tile column).
__global__ void __launch_bounds__(128) k_dc_gemm(DcNodes nd, const int4 *tiles, const double *Qin, const double *Us,
                                                 double *Qout, int n)
{
    const int4 t = tiles[blockIdx.x];
    const int node = t.x >> 1, half = t.x & 1;
    const int lo = nd.lo[node], mid = nd.mid[node], hi = nd.hi[node], m = hi - lo;
    const int r0 = half ? mid : lo, mh = half ? hi - mid : mid - lo;
    const double *Ab = Qin + (size_t) r0 * n + r0;
    const double *Bb = Us + (size_t) r0 * n + lo;
    double *Cb = Qout + (size_t) r0 * n + lo;
    dgemm_tile_dmma64<false, false>(mh, m, mh, 1.0, Ab, n, Bb, n, 0.0, Cb, n, t.y * 64, t.z * 64);
}

__global__ void k_transpose(const double *in, double *out, int n)
{
    __shared__ double tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int i = by + r, j = bx + threadIdx.x;
        if (i < n && j < n) tile[r][threadIdx.x] = in[(size_t) i * n + j];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int i = bx + r, j = by + threadIdx.x;
        if (i < n && j < n) out[(size_t) i * n + j] = tile[threadIdx.x][r];
    }
}

__global__ void k_copy_scalar_eig(const double *A, double *w, double *V)
{
    w[0] = A[0];
    V[0] = 1.0;
}

// ------------------------------------------------------------------ small Cholesky-QR helpers
// Lower Cholesky factor of a symmetric positive definite o x o matrix, in place
// (row-major, lower triangle), left-looking, one warp per row; a non-positive
// or non-finite pivot sets *fail.
__global__ void __launch_bounds__(1024) k_potrf_lower(double *G, int o, int *fail)
{
    __shared__ double s_piv;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j = 0; j < o; j++) {
        if (wid == 0) {
            double s = 0.0;
            for (int c = lane; c < j; c += 32) s += G[(size_t) j * o + c] * G[(size_t) j * o + c];
            s = warp_sum_bcast(s);
            if (lane == 0) {
                const double ajj = G[(size_t) j * o + j] - s;
                if (!(ajj > 0.0) || !isfinite(ajj)) *fail = 1;
                const double l = (ajj > 0.0 && isfinite(ajj)) ? sqrt(ajj) : 1.0;
                G[(size_t) j * o + j] = l;
                s_piv = l;
            }
        }
        __syncthreads();
        const double rinv = 1.0 / s_piv;
        for (int r = j + 1 + wid; r < o; r += nw) {
            double s = 0.0;
            for (int c = lane; c < j; c += 32) s += G[(size_t) r * o + c] * G[(size_t) j * o + c];
            s = warp_sum_bcast(s);
            if (lane == 0) G[(size_t) r * o + j] = (G[(size_t) r * o + j] - s) * rinv;
        }
        __syncthreads();
    }
}

// Xc = (L^-1)^T stored row-major (column j of L^-1 in row j of Xc), upper part
// of L^-1 zero; one thread per column of the inverse.
__global__ void k_trtri_lower(const double *L, double *Xc, int o)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= o) return;
    double *x = Xc + (size_t) j * o;
    for (int i = 0; i < j; i++) x[i] = 0.0;
    x[j] = 1.0 / L[(size_t) j * o + j];
    for (int i = j + 1; i < o; i++) {
        double s = 0.0;
        for (int kk = j; kk < i; kk++) s += L[(size_t) i * o + kk] * x[kk];
        x[i] = -s / L[(size_t) i * o + i];
    }
}

__global__ void k_hash_fill(double *A, size_t n)
{
    size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned long long h = (i + 1) * 0x9E3779B97F4A7C15ULL;
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ULL;
    h ^= h >> 29;
    A[i] = (double) (h >> 11) * (1.0 / 9007199254740992.0) - 0.5;
}

}  // namespace

// ------------------------------------------------------------------ host side
struct Eig {
    int n = 0, G = 1, npanels = 0, nblk = 0;
    // tridiagonalisation and back-transformation
    double *A = nullptr, *VT = nullptr, *PVW = nullptr, *PWV = nullptr, *d = nullptr, *e = nullptr, *tau = nullptr,
           *col = nullptr, *y = nullptr, *part = nullptr, *Gb = nullptr, *Tf = nullptr, *Y = nullptr, *Y2 = nullptr;
    unsigned long long *bar = nullptr;
    int *err = nullptr;
    // divide and conquer: eigenvector buffers of alternate tree levels (Qa reuses A) and the merge's U
    double *Qb = nullptr, *Us = nullptr;
    DcNodes nodes{};
    DcPos pos{};
    int *node_mem = nullptr;
    double *node_rho = nullptr;
    int2 *tab_c = nullptr, *tab_w = nullptr;
    int4 *tiles = nullptr;
    struct Level {
        int depth, node0, nnodes, maxm, c0, nc, w0, nw, t0, nt;
    };
    std::vector<Level> levels;
    // Cholesky-QR of dominant_subspace
    double *Gx = nullptr;
    int go = 0;
    int *acc = nullptr;
    std::vector<void *> allocs;
};

namespace {

template <typename T>
bool ealloc(Eig *e, T **p, size_t count)
{
    void *q = nullptr;
    if (dev_malloc(&q, sizeof(T) * (count ? count : 1), 0) != OK) return false;
    e->allocs.push_back(q);
    *p = (T *) q;
    return true;
}

bool dc_plan(Eig *E)
{
    const int n = E->n;
    struct Node {
        int dep, lo, mid, hi;
    };
    std::vector<Node> nodes;
    std::vector<Node> stack{{0, 0, 0, n}};
    while (!stack.empty()) {
        Node x = stack.back();
        stack.pop_back();
        if (x.hi - x.lo <= 1) continue;
        x.mid = x.lo + (x.hi - x.lo) / 2;
        nodes.push_back(x);
        stack.push_back({x.dep + 1, x.lo, 0, x.mid});
        stack.push_back({x.dep + 1, x.mid, 0, x.hi});
    }
    std::stable_sort(nodes.begin(), nodes.end(), [](const Node &a, const Node &b) { return a.dep > b.dep; });
    std::vector<int> lo, mid, hi;
    std::vector<int2> tc, tw;
    std::vector<int4> tt;
    E->levels.clear();
    size_t i = 0;
    while (i < nodes.size()) {
        Eig::Level L{};
        L.node0 = (int) i;
        L.c0 = (int) tc.size();
        L.w0 = (int) tw.size();
        L.t0 = (int) tt.size();
        const int dep = nodes[i].dep;
        L.depth = dep;
        for (; i < nodes.size() && nodes[i].dep == dep; i++) {
            const int id = (int) i, m = nodes[i].hi - nodes[i].lo;
            lo.push_back(nodes[i].lo);
            mid.push_back(nodes[i].mid);
            hi.push_back(nodes[i].hi);
            L.maxm = std::max(L.maxm, m);
            for (int f = 0; f < m; f += DC_CHUNK) tc.push_back(make_int2(id, f));
            for (int f = 0; f < m; f += DC_WCHUNK) tw.push_back(make_int2(id, f));
            const int ntc = (m + 63) / 64;
            for (int h = 0; h < 2; h++) {
                const int mh = h ? nodes[i].hi - nodes[i].mid : nodes[i].mid - nodes[i].lo;
                for (int a = 0; a < (mh + 63) / 64; a++)
                    for (int b = 0; b < ntc; b++) tt.push_back(make_int4(2 * id + h, a, b, 0));
            }
        }
        L.nnodes = (int) i - L.node0;
        L.nc = (int) tc.size() - L.c0;
        L.nw = (int) tw.size() - L.w0;
        L.nt = (int) tt.size() - L.t0;
        E->levels.push_back(L);
    }
    const size_t nn = nodes.size();
    if (!ealloc(E, &E->node_mem, 5 * nn) || !ealloc(E, &E->node_rho, nn)) return false;
    std::vector<int> packed(5 * nn, 0);
    std::copy(lo.begin(), lo.end(), packed.begin());
    std::copy(mid.begin(), mid.end(), packed.begin() + nn);
    std::copy(hi.begin(), hi.end(), packed.begin() + 2 * nn);
    if (nn && cudaMemcpy(E->node_mem, packed.data(), sizeof(int) * 5 * nn, cudaMemcpyHostToDevice) != cudaSuccess)
        return false;
    E->nodes.lo = E->node_mem;
    E->nodes.mid = E->node_mem + nn;
    E->nodes.hi = E->node_mem + 2 * nn;
    E->nodes.kcnt = E->node_mem + 3 * nn;
    E->nodes.rcnt = E->node_mem + 4 * nn;
    E->nodes.rho = E->node_rho;
    if (!ealloc(E, &E->tab_c, tc.size()) || !ealloc(E, &E->tab_w, tw.size()) || !ealloc(E, &E->tiles, tt.size()))
        return false;
    if (!tc.empty() && cudaMemcpy(E->tab_c, tc.data(), sizeof(int2) * tc.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return false;
    if (!tw.empty() && cudaMemcpy(E->tab_w, tw.data(), sizeof(int2) * tw.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return false;
    if (!tt.empty() && cudaMemcpy(E->tiles, tt.data(), sizeof(int4) * tt.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return false;
    return true;
}

// Opt in to the dynamic shared memory the kernels ask for: the device's
// per-block opt-in maximum less each kernel's static shared memory.
template <typename K>
bool optin_one(K kern, int optin)
{
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) return false;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                optin - (int) fa.sharedSizeBytes) == cudaSuccess;
}

bool smem_optin()
{
    static int done_dev = -1;
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (done_dev == dev) return true;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
    if (!optin_one(k_sytrd_panel, optin) || !optin_one(k_wy_tfactor, optin) || !optin_one(k_dc_deflate, optin) ||
        !optin_one(k_dc_secular, optin) ||
        !optin_one(k_dc_zhat, optin) || !optin_one(k_dc_norms, optin) || !optin_one(k_dc_order, optin))
        return false;
    done_dev = dev;
    return true;
}

}  // namespace

Eig *eig_create(int n, cudaStream_t s)
{
    (void) s;
    if (n < 1 || n > EIG_MAX_N) return nullptr;
    if (!smem_optin()) {
        fprintf(stderr, "[tinyscf] eigensolver: shared-memory opt-in failed: %s\n",
                cudaGetErrorString(cudaGetLastError()));
        return nullptr;
    }
    Eig *E = new Eig();
    E->n = n;
    int dev = 0, nsm = 1, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const size_t dyn = sizeof(double) * (size_t) n;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sytrd_panel, TRD_THREADS, dyn);
    E->G = std::max(1, std::min({nsm * std::max(per, 1), nsm, (n + 7) / 8}));
    if ((long long) E->G * TRD_THREADS / 8 < n) {   // the panel kernel gives every row its own 8 lanes
        fprintf(stderr, "[tinyscf] eigensolver: %d CTAs cannot hold %d rows\n", E->G, n);
        delete E;
        return nullptr;
    }
    E->npanels = (n + TRD_NB - 1) / TRD_NB;
    E->nblk = (n - 1 + BT_NB - 1) / BT_NB;   // blocks of the n - 1 reflectors
    const size_t nn = (size_t) n * n;
    bool ok = ealloc(E, &E->A, nn) && ealloc(E, &E->VT, nn) && ealloc(E, &E->Qb, nn) && ealloc(E, &E->Us, nn) &&
              ealloc(E, &E->PVW, (size_t) 2 * TRD_NB * n) && ealloc(E, &E->PWV, (size_t) 2 * TRD_NB * n) &&
              ealloc(E, &E->Y, (size_t) n * BT_NB) && ealloc(E, &E->Y2, (size_t) n * BT_NB) && ealloc(E, &E->d, n) &&
              ealloc(E, &E->e, n) && ealloc(E, &E->tau, n) && ealloc(E, &E->col, n) &&
              ealloc(E, &E->y, (size_t) ((n + TRD_SEG - 1) / TRD_SEG) * n) &&
              ealloc(E, &E->part, (size_t) E->G * (2 + 2 * TRD_NB)) &&
              ealloc(E, &E->Gb, (size_t) std::max(E->nblk, 1) * GR_KS * BT_NB * BT_NB) &&
              ealloc(E, &E->Tf, (size_t) std::max(E->nblk, 1) * BT_NB * BT_NB) && ealloc(E, &E->bar, 2) &&
              ealloc(E, &E->err, 1) && ealloc(E, &E->acc, 1);
    DcPos &P = E->pos;
    ok = ok && ealloc(E, &P.lam, n) && ealloc(E, &P.ds, n) && ealloc(E, &P.dK, n) && ealloc(E, &P.zK, n) &&
         ealloc(E, &P.lamb, n) && ealloc(E, &P.tau, n) && ealloc(E, &P.zh, n) && ealloc(E, &P.nrm, n) &&
         ealloc(E, &P.lamnew, n) && ealloc(E, &P.perm, n) && ealloc(E, &P.keep, n) && ealloc(E, &P.defl, n) &&
         ealloc(E, &P.rowinfo, n) && ealloc(E, &P.colsrc, n) && ealloc(E, &P.rot, n) && ealloc(E, &P.rotcs, n);
    ok = ok && dc_plan(E);
    if (!ok) {
        fprintf(stderr, "[tinyscf] eigensolver workspace for n = %d: %s\n", n, cudaGetErrorString(cudaGetLastError()));
        eig_destroy(E);
        return nullptr;
    }
    cudaMemset(P.colsrc, 0, sizeof(int) * n);
    cudaMemset(P.perm, 0, sizeof(int) * n);
    cudaMemset(E->bar, 0, sizeof(unsigned long long));
    cudaMemset(E->err, 0, sizeof(int));
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        fprintf(stderr, "[tinyscf] eigensolver set-up for n = %d: %s\n", n, cudaGetErrorString(err));
        eig_destroy(E);
        return nullptr;
    }
    return E;
}

void eig_destroy(Eig *e)
{
    if (!e) return;
    for (void *p : e->allocs) dev_free(p, 0);
    cudaStreamSynchronize(0);
    delete e;
}

int eig_error(Eig *e)
{
    int v = 0;
    if (!e) return ERR_STATE;
    if (cudaMemcpy(&v, e->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return ERR_CUDA;
    return v ? ERR_CUDA : OK;
}

namespace {

int tridiagonalize(Eig *E, const double *d_A, cudaStream_t s)
{
    const int n = E->n;
    const size_t nn = (size_t) n * n;
    TSCF_CUDA_CHECK(cudaMemcpyAsync(E->A, d_A, sizeof(double) * nn, cudaMemcpyDeviceToDevice, s));
    TSCF_CUDA_CHECK(cudaMemsetAsync(E->VT, 0, sizeof(double) * nn, s));
    TSCF_CUDA_CHECK(cudaMemsetAsync(E->tau, 0, sizeof(double) * n, s));
    TSCF_CUDA_CHECK(cudaMemsetAsync(E->e, 0, sizeof(double) * n, s));
    TSCF_CUDA_CHECK(cudaMemsetAsync(E->bar, 0, sizeof(unsigned long long), s));
    const size_t dyn = sizeof(double) * (size_t) n;
    for (int P = 0; P < E->npanels; P++) {
        TrdArgs a;
        a.A = E->A;
        a.VT = E->VT;
        a.PVW = E->PVW;
        a.PWV = E->PWV;
        a.d = E->d;
        a.e = E->e;
        a.tau = E->tau;
        a.col = E->col;
        a.y = E->y;
        a.part = E->part;
        a.bar = E->bar;
        a.err = E->err;
        a.n = n;
        a.p = P * TRD_NB;
        a.cols = std::min(TRD_NB, n - a.p);
        a.G = E->G;
        void *args[] = {&a};
        g_launches++;
        g_eig_launches++;
        TSCF_CUDA_CHECK(cudaLaunchCooperativeKernel((const void *) k_sytrd_panel, dim3(E->G), dim3(TRD_THREADS), args,
                                                    dyn, s));
        const int q = a.p + a.cols, mt = n - q;
        if (mt > 0) {
            // A22 -= V W^T + W V^T = PVW^T PWV over the trailing columns (a full panel: cols = TRD_NB)
            dgemm_untuned(true, false, mt, mt, 2 * TRD_NB, -1.0, E->PVW + q, n, E->PWV + q, n, 1.0,
                          E->A + (size_t) q * n + q, n, s);
            g_eig_launches++;
        }
    }
    return cuda_launch_rc("tridiagonalisation");
}

// Eigenvectors of T into the columns of the returned buffer (E->A or E->Qb).
int divide_conquer(Eig *E, cudaStream_t s, double **out)
{
    const int n = E->n;
    const size_t nn = (size_t) n * n;
    double *buf[2] = {E->A, E->Qb};   // level of depth L writes buf[L % 2], reads its children from the other
    TSCF_CUDA_CHECK(cudaMemsetAsync(buf[0], 0, sizeof(double) * nn, s));
    TSCF_CUDA_CHECK(cudaMemsetAsync(buf[1], 0, sizeof(double) * nn, s));
    TSCF_CUDA_CHECK(cudaMemsetAsync(E->Us, 0, sizeof(double) * nn, s));
    g_launches++;
    g_eig_launches++;
    k_dc_init<<<(n + 255) / 256, 256, 0, s>>>(E->d, E->e, E->pos.lam, buf[0], buf[1], n);
    for (const auto &L : E->levels) {
        const size_t m = (size_t) L.maxm;
        const double *Qin = buf[(L.depth + 1) % 2];
        double *Qout = buf[L.depth % 2];
        k_dc_deflate<<<L.nnodes, 512, 20 * m, s>>>(E->nodes, E->pos, Qin, E->e, n, L.node0);
        k_dc_secular<<<L.nw, 256, 16 * m, s>>>(E->nodes, E->pos, E->tab_w + L.w0);
        k_dc_zhat<<<L.nw, 256, 24 * m, s>>>(E->nodes, E->pos, E->tab_w + L.w0);
        k_dc_norms<<<L.nw, 256, 16 * m, s>>>(E->nodes, E->pos, E->tab_w + L.w0);
        k_dc_order<<<L.nc, DC_CHUNK, 8 * m, s>>>(E->nodes, E->pos, E->tab_c + L.c0);
        k_dc_build<<<L.nw, 256, 0, s>>>(E->nodes, E->pos, E->tab_w + L.w0, E->Us, n);
        k_dc_rotate<<<L.nc, DC_CHUNK, 0, s>>>(E->nodes, E->pos, E->tab_c + L.c0, E->Us, n);
        k_dc_commit_lam<<<L.nc, DC_CHUNK, 0, s>>>(E->nodes, E->pos, E->tab_c + L.c0);
        k_dc_gemm<<<L.nt, 128, 0, s>>>(E->nodes, E->tiles + L.t0, Qin, E->Us, Qout, n);
        g_launches += 9;
        g_eig_launches += 9;
    }
    *out = buf[0];   // the root has depth 0
    return cuda_launch_rc("divide and conquer");
}

// Vout = Z^T Q^T, Z (the tridiagonal's eigenvectors, columns of Zc), Q the
// product of the reflectors, in blocks of BT_NB reflectors from the last:
// Vout <- Vout - (Vout V) T^T V^T.
int back_transform(Eig *E, const double *Zc, double *d_V, cudaStream_t s)
{
    const int n = E->n, nref = n - 1;
    g_launches += 3;
    g_eig_launches += 3;
    k_wy_gram<<<dim3(E->nblk, (BT_NB / 32) * (BT_NB / 32), GR_KS), 256, 0, s>>>(E->VT, E->Gb, n, nref);
    k_wy_tfactor<<<E->nblk, 256, sizeof(double) * (BT_NB * (BT_NB + 1) + BT_NB), s>>>(E->Gb, E->tau, E->Tf, nref);
    k_transpose<<<dim3((n + 31) / 32, (n + 31) / 32), dim3(32, 8), 0, s>>>(Zc, d_V, n);
    for (int B = E->nblk - 1; B >= 0; B--) {
        const int p0 = B * BT_NB, bb = std::min(BT_NB, nref - p0), mv = n - p0 - 1;
        const double *V = E->VT + (size_t) p0 * n + p0 + 1;
        dgemm_untuned(false, true, n, bb, mv, 1.0, d_V + p0 + 1, n, V, n, 0.0, E->Y, BT_NB, s);
        dgemm_untuned(false, true, n, bb, bb, 1.0, E->Y, BT_NB, E->Tf + (size_t) B * BT_NB * BT_NB, BT_NB, 0.0, E->Y2,
                      BT_NB, s);
        dgemm_untuned(false, false, n, mv, bb, -1.0, E->Y2, BT_NB, V, n, 1.0, d_V + p0 + 1, n, s);
        g_eig_launches += 3;
    }
    return cuda_launch_rc("back-transformation");
}

}  // namespace

// Eigenvalues ascending into d_w, eigenvectors as rows of d_V (V[k*n + i] =
// entry i of eigenvector k). d_V may alias d_A.
int eig_run(Eig *E, const double *d_A, double *d_w, double *d_V, cudaStream_t s)
{
    if (!E) return ERR_STATE;
    const int n = E->n;
    if (n == 1) {
        g_launches++;
        g_eig_launches++;
        k_copy_scalar_eig<<<1, 1, 0, s>>>(d_A, d_w, d_V);
        return cuda_launch_rc("eigensolve (n = 1)");
    }
    RC_(tridiagonalize(E, d_A, s));
    double *Z = nullptr;
    RC_(divide_conquer(E, s, &Z));
    RC_(back_transform(E, Z, d_V, s));
    TSCF_CUDA_CHECK(cudaMemcpyAsync(d_w, E->pos.lam, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    return OK;
}

// ------------------------------------------------------------------ dominant subspace
// Rows of U (o x n) become an orthonormal basis of the dominant o-dimensional
// invariant subspace of a symmetric n x n matrix M, by subspace iteration from
// a fixed pseudo-random start: W <- W M, orthonormalised every kOrthoEvery
// products and at the end by Cholesky-QR (G = W W^T = L L^T, W <- L^-1 W,
// with L^-1 from a triangular inverse so the update is one GEMM), the last one
// applied twice for orthogonality to rounding. For a matrix close to a rank-o
// projector (a predicted density in the orthogonal basis) each product
// shrinks the other directions by the ratio of the (o+1)-th to the o-th
// eigenvalue, while the kept directions, with eigenvalues near 1, stay well
// conditioned between orthonormalisations.
namespace {
const int kOrthoEvery = 3;

// W <- L^-1 U for G = U U^T = L L^T (U, W: o x n row-major; G: o x o scratch).
// A failed factorisation sets E->acc on the device.
void chol_qr(Eig *E, const double *U, double *W, double *G, int n, int o, cudaStream_t s)
{
    dgemm(false, true, o, o, n, 1.0, U, n, U, n, 0.0, G, o, s);   // G = U U^T
    k_potrf_lower<<<1, 1024, 0, s>>>(G, o, E->acc);
    k_trtri_lower<<<(o + 127) / 128, 128, 0, s>>>(G, E->Gx, o);
    g_launches += 2;
    // row-major Gx is (L^-1)^T, so W = Gx^T U
    dgemm(true, false, o, n, o, 1.0, E->Gx, o, U, n, 0.0, W, n, s);
}
}  // namespace

int dominant_subspace(Eig *E, const double *d_M, double *d_U, double *d_W, double *d_G, int n, int o, int iters,
                      cudaStream_t s)
{
    if (!E || o <= 0 || o > n || iters < 1) return ERR_INPUT;
    if (E->go < o) {
        if (E->Gx) {
            cudaFree(E->Gx);
            E->allocs.erase(std::find(E->allocs.begin(), E->allocs.end(), (void *) E->Gx));
            E->Gx = nullptr;
        }
        if (!ealloc(E, &E->Gx, (size_t) o * o)) return ERR_ALLOC;
        E->go = o;
    }
    TSCF_CUDA_CHECK(cudaMemsetAsync(E->acc, 0, sizeof(int), s));
    const size_t on = (size_t) o * n;
    double *cur = d_W, *nxt = d_U;   // cur: the basis (or an unorthonormalised product of it)
    k_hash_fill<<<(unsigned) ((on + 255) / 256), 256, 0, s>>>(cur, on);
    g_launches++;
    for (int it = 1; it <= iters; it++) {
        dgemm(false, false, o, n, n, 1.0, cur, n, d_M, n, 0.0, nxt, n, s);   // nxt = cur M (M symmetric)
        if (it % kOrthoEvery == 0 || it == iters) chol_qr(E, nxt, cur, d_G, n, o, s);
        else std::swap(cur, nxt);
    }
    chol_qr(E, cur, nxt, d_G, n, o, s);   // second pass: orthonormal to rounding
    if (nxt != d_U) TSCF_CUDA_CHECK(cudaMemcpyAsync(d_U, nxt, sizeof(double) * on, cudaMemcpyDeviceToDevice, s));
    int acc = 0;
    TSCF_CUDA_CHECK(cudaMemcpyAsync(&acc, E->acc, sizeof(int), cudaMemcpyDeviceToHost, s));
    TSCF_CUDA_CHECK(cudaStreamSynchronize(s));
    return acc == 0 ? OK : ERR_NUMERIC;
}

}  // namespace tscf
