// The learned guess's networks on the GPU: a three-layer MLP per block type
// (SiLU hidden layers), its forward and backward passes as tiled FP32 GEMMs
// with fused bias / activation epilogues, mean-squared-error loss, Adam, the
// trainer that writes the weights file, and prediction: blocks predicted in
// each pair's local frame, rotated into the molecule frame and assembled into
// the density matrix.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "guess.h"
#include "tscf_internal.h"

namespace tscf {

namespace {

// ------------------------------------------------------------------ FP32 GEMM with epilogues
// C[m x n] = op(A) op(B), row-major; 64x64 tile per 256 threads, 4x4 per thread.
// Split-K over blockIdx.z (EPI_STORE only): slice z covers k in [z*kc, (z+1)*kc)
// and writes C + z*m*ldc.
enum { EPI_STORE = 0, EPI_BIAS_SILU = 1, EPI_BIAS = 2, EPI_DSILU = 3 };
constexpr int SB_M = 64, SB_N = 64, SB_K = 16;

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }

template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(256) k_sgemm(int m, int n, int k, int kc, const float *__restrict__ A, int lda,
                                               const float *__restrict__ B, int ldb, float *C, int ldc,
                                               const float *__restrict__ bias, float *Z)
{
    __shared__ float As[SB_K][SB_M + 4];
    __shared__ float Bs[SB_K][SB_N + 4];
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    const int m0 = blockIdx.y * SB_M, n0 = blockIdx.x * SB_N;
    const int kb = blockIdx.z * kc, ke = min(k, kb + kc);
    float acc[4][4] = {};
    for (int k0 = kb; k0 < ke; k0 += SB_K) {
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int l = tid + 256 * r;
            int row, kk;
            if (!TA) { row = l / SB_K; kk = l % SB_K; } else { kk = l / SB_M; row = l % SB_M; }
            int gi = m0 + row, gk = k0 + kk;
            float v = 0.f;
            if (gi < m && gk < ke) v = TA ? A[(size_t) gk * lda + gi] : A[(size_t) gi * lda + gk];
            As[kk][row] = v;
            int col;
            if (!TB) { kk = l / SB_N; col = l % SB_N; } else { col = l / SB_K; kk = l % SB_K; }
            const int gj = n0 + col;
            gk = k0 + kk;
            float w = 0.f;
            if (gj < n && gk < ke) w = TB ? B[(size_t) gj * ldb + gk] : B[(size_t) gk * ldb + gj];
            Bs[kk][col] = w;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < SB_K; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
    float *Cz = C + (size_t) blockIdx.z * m * ldc;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int gi = m0 + ty + 16 * i;
        if (gi >= m) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int gj = n0 + tx + 16 * j;
            if (gj >= n) continue;
            const size_t o = (size_t) gi * ldc + gj;
            float v = acc[i][j];
            if (EPI == EPI_STORE) {
                Cz[o] = v;
            } else if (EPI == EPI_BIAS) {
                C[o] = v + bias[gj];
            } else if (EPI == EPI_BIAS_SILU) {
                v += bias[gj];
                Z[o] = v;
                C[o] = v * sigm(v);
            } else {   // EPI_DSILU: C = v * silu'(Z)
                const float z = Z[o], s = sigm(z);
                C[o] = v * s * (1.0f + z * (1.0f - s));
            }
        }
    }
}

template <int EPI>
void sgemm(bool ta, bool tb, int m, int n, int k, const float *A, int lda, const float *B, int ldb, float *C, int ldc,
           const float *bias, float *Z, int splits, cudaStream_t s)
{
    const int kc = ((k + splits - 1) / splits + SB_K - 1) / SB_K * SB_K;
    dim3 grid((n + SB_N - 1) / SB_N, (m + SB_M - 1) / SB_M, splits);
    g_launches++;
    if (!ta && !tb) k_sgemm<false, false, EPI><<<grid, 256, 0, s>>>(m, n, k, kc, A, lda, B, ldb, C, ldc, bias, Z);
    else if (!ta && tb) k_sgemm<false, true, EPI><<<grid, 256, 0, s>>>(m, n, k, kc, A, lda, B, ldb, C, ldc, bias, Z);
    else if (ta && !tb) k_sgemm<true, false, EPI><<<grid, 256, 0, s>>>(m, n, k, kc, A, lda, B, ldb, C, ldc, bias, Z);
    else k_sgemm<true, true, EPI><<<grid, 256, 0, s>>>(m, n, k, kc, A, lda, B, ldb, C, ldc, bias, Z);
}

// out[i] = sum_z part[z][i] (fixed order)
__global__ void k_sum_parts(const float *part, int nparts, size_t len, float *out)
{
    size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= len) return;
    float s = 0.f;
    for (int z = 0; z < nparts; z++) s += part[(size_t) z * len + i];
    out[i] = s;
}

// column sums of X [rows x cols] (bias gradients), one thread per column
__global__ void k_colsum(const float *X, int rows, int cols, float *out)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols) return;
    float s = 0.f;
    for (int i = 0; i < rows; i++) s += X[(size_t) i * cols + j];
    out[j] = s;
}

// dY = 2 (Y - T) / (rows * cols); per-block partial sums of (Y - T)^2
__global__ void k_mse(const float *Y, const float *T, float *dY, size_t len, float inv, double *loss_part)
{
    __shared__ double sh[256];
    double acc = 0.0;
    for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (size_t) gridDim.x * blockDim.x) {
        const float d = Y[i] - T[i];
        dY[i] = 2.0f * d * inv;
        acc += (double) d * d;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss_part[blockIdx.x] = sh[0];
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, size_t n, float lr, float b1, float b2, float c1,
                       float c2, float eps)
{
    size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_gather_rows(const float *src, const int *idx, int rows, int cols, float *dst)
{
    size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t) rows * cols) return;
    const int r = (int) (i / cols), c = (int) (i % cols);
    dst[i] = src[(size_t) idx[r] * cols + c];
}

constexpr int LOSS_BLOCKS = 148;   // partial sums of the loss (a fixed count: the sum order is fixed)

// Work buffers for one MLP on batches of up to `cap` rows.
struct MlpWork {
    int din, hid, dout, cap;
    float *Z1, *H1, *Z2, *H2, *Y, *dY, *dH, *dH2, *part;
    double *loss_part;
    std::vector<void *> mem;
    int splits;
};

int work_alloc(MlpWork &w, int din, int hid, int dout, int cap)
{
    w.din = din;
    w.hid = hid;
    w.dout = dout;
    w.cap = cap;
    w.splits = std::max(1, std::min(32, cap / 64));
    const size_t ch = (size_t) cap * hid, co = (size_t) cap * dout;
    const size_t pmax = (size_t) w.splits * std::max((size_t) din * hid, std::max((size_t) hid * hid, (size_t) hid * dout));
    float **fb[] = {&w.Z1, &w.H1, &w.Z2, &w.H2, &w.dH, &w.dH2};
    for (float **b : fb) {
        if (cudaMalloc(b, sizeof(float) * ch) != cudaSuccess) return ERR_ALLOC;
        w.mem.push_back(*b);
    }
    float **ob[] = {&w.Y, &w.dY};
    for (float **b : ob) {
        if (cudaMalloc(b, sizeof(float) * co) != cudaSuccess) return ERR_ALLOC;
        w.mem.push_back(*b);
    }
    if (cudaMalloc(&w.part, sizeof(float) * pmax) != cudaSuccess) return ERR_ALLOC;
    w.mem.push_back(w.part);
    if (cudaMalloc(&w.loss_part, sizeof(double) * LOSS_BLOCKS) != cudaSuccess) return ERR_ALLOC;
    w.mem.push_back(w.loss_part);
    return OK;
}

void work_free(MlpWork &w)
{
    for (void *p : w.mem) cudaFree(p);
    w.mem.clear();
}

struct MlpParams {
    const float *W1, *b1, *W2, *b2, *W3, *b3;
};

MlpParams split_params(const float *p, int din, int hid, int dout)
{
    MlpParams q;
    q.W1 = p;
    q.b1 = q.W1 + (size_t) din * hid;
    q.W2 = q.b1 + hid;
    q.b2 = q.W2 + (size_t) hid * hid;
    q.W3 = q.b2 + hid;
    q.b3 = q.W3 + (size_t) hid * dout;
    return q;
}

void mlp_forward(const MlpParams &P, const float *X, int rows, MlpWork &w, cudaStream_t s)
{
    sgemm<EPI_BIAS_SILU>(false, false, rows, w.hid, w.din, X, w.din, P.W1, w.hid, w.H1, w.hid, P.b1, w.Z1, 1, s);
    sgemm<EPI_BIAS_SILU>(false, false, rows, w.hid, w.hid, w.H1, w.hid, P.W2, w.hid, w.H2, w.hid, P.b2, w.Z2, 1, s);
    sgemm<EPI_BIAS>(false, false, rows, w.dout, w.hid, w.H2, w.hid, P.W3, w.dout, w.Y, w.dout, P.b3, nullptr, 1, s);
}

// weight gradient G [k x n] = A^T dZ over `rows`, split over rows, summed in fixed order
void weight_grad(const float *A, int ka, const float *dZ, int n, int rows, MlpWork &w, float *G, cudaStream_t s)
{
    const int sp = std::max(1, std::min(w.splits, rows / 32));
    sgemm<EPI_STORE>(true, false, ka, n, rows, A, ka, dZ, n, w.part, n, nullptr, nullptr, sp, s);
    const size_t len = (size_t) ka * n;
    k_sum_parts<<<(unsigned) ((len + 255) / 256), 256, 0, s>>>(w.part, sp, len, G);
    g_launches++;
}

// loss (mean of squared errors) and full gradient for one batch
void mlp_loss_grad(const MlpParams &P, const float *X, const float *T, int rows, MlpWork &w, float *grad,
                   cudaStream_t s)
{
    mlp_forward(P, X, rows, w, s);
    const size_t len = (size_t) rows * w.dout;
    k_mse<<<LOSS_BLOCKS, 256, 0, s>>>(w.Y, T, w.dY, len, 1.0f / (float) len, w.loss_part);
    g_launches++;
    float *gW1 = grad, *gb1 = gW1 + (size_t) w.din * w.hid, *gW2 = gb1 + w.hid, *gb2 = gW2 + (size_t) w.hid * w.hid,
          *gW3 = gb2 + w.hid, *gb3 = gW3 + (size_t) w.hid * w.dout;
    weight_grad(w.H2, w.hid, w.dY, w.dout, rows, w, gW3, s);
    k_colsum<<<(w.dout + 127) / 128, 128, 0, s>>>(w.dY, rows, w.dout, gb3);
    // dZ2 = (dY W3^T) * silu'(Z2)
    sgemm<EPI_DSILU>(false, true, rows, w.hid, w.dout, w.dY, w.dout, P.W3, w.dout, w.dH2, w.hid, nullptr, w.Z2, 1, s);
    weight_grad(w.H1, w.hid, w.dH2, w.hid, rows, w, gW2, s);
    k_colsum<<<(w.hid + 127) / 128, 128, 0, s>>>(w.dH2, rows, w.hid, gb2);
    // dZ1 = (dZ2 W2^T) * silu'(Z1)
    sgemm<EPI_DSILU>(false, true, rows, w.hid, w.hid, w.dH2, w.hid, P.W2, w.hid, w.dH, w.hid, nullptr, w.Z1, 1, s);
    weight_grad(X, w.din, w.dH, w.hid, rows, w, gW1, s);
    k_colsum<<<(w.hid + 127) / 128, 128, 0, s>>>(w.dH, rows, w.hid, gb1);
    g_launches += 3;
}

double read_loss(const MlpWork &w, cudaStream_t s)
{
    double h[LOSS_BLOCKS];
    cudaMemcpyAsync(h, w.loss_part, sizeof(h), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    double t = 0.0;
    for (double v : h) t += v;
    return t;
}

// ------------------------------------------------------------------ prediction
// One block per pair: D_loc = raw * scale + offset (nf_a x nf_b), then
// D_ab = Pa^T D_loc Pb with P = M(Q^T) = M(Q)^-1, written to (a, b) and,
// transposed, to (b, a); diagonal blocks are symmetrised.
struct PairDev {
    int type, row, off_a, off_b, nf_a, nf_b;
    double Qt[9];   // transposed local frame: M(Qt) takes local functions to the molecule's
};

// Entry (r, c) of M(Q) for an atom with nf Cartesian functions, the same
// products and sums as guess_atom_rotation (host), rounded the same way:
// nf 5 is the shell layout s s p, nf 15 is s s s p p d.
__device__ double rot_entry(const double *Q, int nf, int r, int c)
{
    const int ns = nf == 5 ? 2 : 3;   // leading s functions
    if (r < ns || c < ns) return r == c ? 1.0 : 0.0;
    const int np = nf == 5 ? 1 : 2;   // p shells
    const int pr = (r - ns) / 3, pc = (c - ns) / 3;
    if (pr < np || pc < np) {
        if (pr != pc) return 0.0;
        return Q[((c - ns) % 3) * 3 + (r - ns) % 3];
    }
    const int dr = r - ns - 3 * np, dc = c - ns - 3 * np;   // d shell: components xx xy xz yy yz zz
    const int d0[6] = {0, 0, 0, 1, 1, 2}, d1[6] = {0, 1, 2, 1, 2, 2};
    const int a = d0[dr], b = d1[dr], cc = d0[dc], dd = d1[dc];
    double v = __dmul_rn(Q[cc * 3 + a], Q[dd * 3 + b]);
    if (cc != dd) v = __dadd_rn(v, __dmul_rn(Q[dd * 3 + a], Q[cc * 3 + b]));
    return v;
}

__global__ void k_assemble(const PairDev *pairs, const float *const *Y, const float *const *scale,
                           const float *const *offset, double *D, int nbf)
{
    __shared__ double L[G_MAXF * G_MAXF], T[G_MAXF * G_MAXF], Pa[G_MAXF * G_MAXF], Pb[G_MAXF * G_MAXF];
    const PairDev p = pairs[blockIdx.x];
    const int na = p.nf_a, nb = p.nf_b, nab = na * nb;
    const float *y = Y[p.type] + (size_t) p.row * nab;
    const float *sc = scale[p.type], *of = offset[p.type];
    for (int i = threadIdx.x; i < nab; i += blockDim.x) L[i] = (double) y[i] * sc[i] + of[i];
    for (int i = threadIdx.x; i < na * na; i += blockDim.x) Pa[i] = rot_entry(p.Qt, na, i / na, i % na);
    for (int i = threadIdx.x; i < nb * nb; i += blockDim.x) Pb[i] = rot_entry(p.Qt, nb, i / nb, i % nb);
    __syncthreads();
    for (int i = threadIdx.x; i < nab; i += blockDim.x) {   // T = L Pb
        const int r = i / nb, c = i % nb;
        double s = 0.0;
        for (int k = 0; k < nb; k++) s += L[r * nb + k] * Pb[k * nb + c];
        T[i] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nab; i += blockDim.x) {   // L = Pa^T T
        const int r = i / nb, c = i % nb;
        double s = 0.0;
        for (int k = 0; k < na; k++) s += Pa[k * na + r] * T[k * nb + c];
        L[i] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nab; i += blockDim.x) {
        const int r = i / nb, c = i % nb;
        if (p.off_a == p.off_b) {
            D[(size_t) (p.off_a + r) * nbf + p.off_b + c] = 0.5 * (L[r * nb + c] + L[c * nb + r]);
        } else {
            D[(size_t) (p.off_a + r) * nbf + p.off_b + c] = L[i];
            D[(size_t) (p.off_b + c) * nbf + p.off_a + r] = L[i];
        }
    }
}

const char kMagic[8] = {'T', 'S', 'G', 'U', 'E', 'S', 'S', '1'};

}  // namespace

// ------------------------------------------------------------------ weights file
int guessnet_load(GuessNet **out, const char *path)
{
    FILE *f = fopen(path, "rb");
    if (!f) return ERR_FILEIO;
    char mg[8];
    int hdr[3];
    int rc = OK;
    if (fread(mg, 1, 8, f) != 8 || memcmp(mg, kMagic, 8) != 0 || fread(hdr, sizeof(int), 3, f) != 3 ||
        hdr[2] != G_NTYPES)
        rc = ERR_INPUT;
    GuessNet *net = new GuessNet();
    if (rc == OK) {
        net->din = hdr[0];
        net->hid = hdr[1];
        if (net->din != G_DIN || fread(net->dout, sizeof(int), G_NTYPES, f) != (size_t) G_NTYPES) rc = ERR_INPUT;
    }
    for (int t = 0; rc == OK && t < G_NTYPES; t++) {
        if (net->dout[t] != G_DOUT[t]) { rc = ERR_INPUT; break; }
        const size_t np = mlp_param_count(net->din, net->hid, net->dout[t]);
        std::vector<float> h(np + 2 * (size_t) net->dout[t]);
        if (fread(h.data(), sizeof(float), h.size(), f) != h.size()) { rc = ERR_INPUT; break; }
        if (cudaMalloc(&net->d_params[t], sizeof(float) * h.size()) != cudaSuccess) { rc = ERR_ALLOC; break; }
        cudaMemcpy(net->d_params[t], h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice);
        net->d_scale[t] = net->d_params[t] + np;
        net->d_offset[t] = net->d_scale[t] + net->dout[t];
    }
    fclose(f);
    if (rc != OK) {
        guessnet_free(net);
        return rc;
    }
    *out = net;
    return OK;
}


struct GuessWork {
    int cap_pairs = 0, cap_rows = 0;
    float *dX = nullptr, *dY = nullptr;
    PairDev *dpd = nullptr;
    const float **dptr = nullptr;   // [3][G_NTYPES]: Y, scale, offset of each type
    MlpWork w{};
    std::vector<void *> mem;
};

static void work_release(GuessWork *gw)
{
    if (!gw) return;
    work_free(gw->w);
    for (void *p : gw->mem) cudaFree(p);
    gw->mem.clear();
    gw->cap_pairs = gw->cap_rows = 0;
}

// Buffers for np pairs with at most maxrows of one type (the forward pass
// runs type by type through one MlpWork).
static int work_reserve(GuessNet *net, int np, int maxrows)
{
    if (!net->work) net->work = new GuessWork();
    GuessWork *gw = net->work;
    if (np <= gw->cap_pairs && maxrows <= gw->cap_rows) return OK;
    work_release(gw);
    np = std::max(np, 1);
    maxrows = std::max(maxrows, 1);
    auto dal = [&](void **p, size_t bytes) {
        if (cudaMalloc(p, bytes ? bytes : 16) != cudaSuccess) return false;
        gw->mem.push_back(*p);
        return true;
    };
    if (!dal((void **) &gw->dX, sizeof(float) * (size_t) np * G_DIN) ||
        !dal((void **) &gw->dY, sizeof(float) * (size_t) np * G_MAXF * G_MAXF) ||
        !dal((void **) &gw->dpd, sizeof(PairDev) * np) ||
        !dal((void **) &gw->dptr, sizeof(float *) * 3 * G_NTYPES))
        return ERR_ALLOC;
    int rc = work_alloc(gw->w, net->din, net->hid, G_MAXF * G_MAXF, maxrows);
    if (rc) return rc;
    gw->cap_pairs = np;
    gw->cap_rows = maxrows;
    return OK;
}

int guessnet_predict(GuessNet *net, const std::vector<GuessPair> &pairs, const GuessAtoms &g, double *d_D, int nbf,
                     cudaStream_t s)
{
    const int np = (int) pairs.size();
    // rows of each type contiguous: type t starts at row off[t]
    int cnt[G_NTYPES] = {}, off[G_NTYPES + 1] = {};
    for (const GuessPair &p : pairs) cnt[p.type]++;
    for (int t = 0; t < G_NTYPES; t++) off[t + 1] = off[t] + cnt[t];
    size_t yoff[G_NTYPES + 1] = {};
    for (int t = 0; t < G_NTYPES; t++) yoff[t + 1] = yoff[t] + (size_t) cnt[t] * net->dout[t];
    std::vector<float> X((size_t) np * G_DIN);
    std::vector<PairDev> pd(np);
    int fill[G_NTYPES] = {};
    for (int k = 0; k < np; k++) {
        const GuessPair &p = pairs[k];
        const int row = fill[p.type]++;
        PairDev &q = pd[k];
        q.type = p.type;
        q.row = row;
        q.off_a = p.off_a;
        q.off_b = p.off_b;
        q.nf_a = p.nf_a;
        q.nf_b = p.nf_b;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) q.Qt[i * 3 + j] = p.Qf[j * 3 + i];
        std::memcpy(&X[(size_t) (off[p.type] + row) * G_DIN], p.feat, sizeof(float) * G_DIN);
    }
    int maxrows = 1;
    for (int t = 0; t < G_NTYPES; t++) maxrows = std::max(maxrows, cnt[t]);
    int rc = work_reserve(net, np, maxrows);
    if (rc) return rc;
    GuessWork *gw = net->work;
    cudaMemsetAsync(d_D, 0, sizeof(double) * (size_t) nbf * nbf, s);
    cudaMemcpyAsync(gw->dX, X.data(), sizeof(float) * X.size(), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(gw->dpd, pd.data(), sizeof(PairDev) * np, cudaMemcpyHostToDevice, s);
    const float *hp[3 * G_NTYPES];
    for (int t = 0; t < G_NTYPES; t++) {
        hp[t] = gw->dY + yoff[t];
        hp[G_NTYPES + t] = net->d_scale[t];
        hp[2 * G_NTYPES + t] = net->d_offset[t];
    }
    cudaMemcpyAsync(gw->dptr, hp, sizeof(hp), cudaMemcpyHostToDevice, s);
    for (int t = 0; t < G_NTYPES; t++) {
        if (!cnt[t]) continue;
        gw->w.dout = net->dout[t];
        MlpParams prm = split_params(net->d_params[t], net->din, net->hid, net->dout[t]);
        mlp_forward(prm, gw->dX + (size_t) off[t] * G_DIN, cnt[t], gw->w, s);
        cudaMemcpyAsync(gw->dY + yoff[t], gw->w.Y, sizeof(float) * (size_t) cnt[t] * net->dout[t],
                        cudaMemcpyDeviceToDevice, s);
    }
    if (np > 0) k_assemble<<<np, 128, 0, s>>>(gw->dpd, gw->dptr, gw->dptr + G_NTYPES, gw->dptr + 2 * G_NTYPES, d_D,
                                               nbf);
    g_launches++;
    // the host arrays above are staged by the copies: wait before they go out of scope
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) return ERR_CUDA;
    return OK;
}

void guessnet_free(GuessNet *net)
{
    if (!net) return;
    if (net->work) {
        work_release(net->work);
        delete net->work;
    }
    for (int t = 0; t < G_NTYPES; t++)
        if (net->d_params[t]) cudaFree(net->d_params[t]);
    delete net;
}

// ------------------------------------------------------------------ training
int guessnet_train(const float *feat, const float *target, const int *type, long long n, int epochs, int batch,
                   float lr, unsigned seed, const char *path, float *final_loss)
{
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return ERR_CUDA;
    std::mt19937 rng(seed);
    std::vector<std::vector<float>> blobs(G_NTYPES);
    int rc = OK;
    for (int t = 0; t < G_NTYPES && rc == OK; t++) {
        const int dout = G_DOUT[t];
        std::vector<long long> rows;
        for (long long i = 0; i < n; i++)
            if (type[i] == t) rows.push_back(i);
        const int nt = (int) rows.size();
        const size_t np = mlp_param_count(G_DIN, G_HID, dout);
        std::vector<float> prm(np, 0.f), scale(dout, 1.f), offset(dout, 0.f);
        if (nt > 0) {
            // output normalisation
            std::vector<double> mu(dout, 0.0), var(dout, 0.0);
            for (long long r : rows)
                for (int j = 0; j < dout; j++) mu[j] += target[r * G_MAXF * G_MAXF + j];
            for (int j = 0; j < dout; j++) mu[j] /= nt;
            for (long long r : rows)
                for (int j = 0; j < dout; j++) {
                    double d = target[r * G_MAXF * G_MAXF + j] - mu[j];
                    var[j] += d * d;
                }
            // one scale per type (the RMS deviation over all outputs): the loss
            // then weighs every density element by its absolute error
            double vtot = 0.0;
            for (int j = 0; j < dout; j++) vtot += var[j];
            const double sc = std::max(1e-6, std::sqrt(vtot / ((double) nt * dout)));
            for (int j = 0; j < dout; j++) {
                offset[j] = (float) mu[j];
                scale[j] = (float) sc;
            }
            std::vector<float> hX((size_t) nt * G_DIN), hT((size_t) nt * dout);
            for (int i = 0; i < nt; i++) {
                std::memcpy(&hX[(size_t) i * G_DIN], feat + rows[i] * G_DIN, sizeof(float) * G_DIN);
                for (int j = 0; j < dout; j++)
                    hT[(size_t) i * dout + j] = (target[rows[i] * G_MAXF * G_MAXF + j] - offset[j]) / scale[j];
            }
            // Glorot-uniform weights, zero biases
            auto glorot = [&](float *W, int fi, int fo) {
                std::uniform_real_distribution<float> u(-std::sqrt(6.f / (fi + fo)), std::sqrt(6.f / (fi + fo)));
                for (size_t k = 0; k < (size_t) fi * fo; k++) W[k] = u(rng);
            };
            float *W1 = prm.data(), *W2 = W1 + (size_t) G_DIN * G_HID + G_HID,
                  *W3 = W2 + (size_t) G_HID * G_HID + G_HID;
            glorot(W1, G_DIN, G_HID);
            glorot(W2, G_HID, G_HID);
            glorot(W3, G_HID, dout);
            const int bs = std::min(batch, nt);
            float *dXall = nullptr, *dTall = nullptr, *dXb = nullptr, *dTb = nullptr, *dp = nullptr, *dg = nullptr,
                  *dm = nullptr, *dv = nullptr;
            int *didx = nullptr;
            MlpWork w{};
            std::vector<void *> mem;
            auto dal = [&](void **p, size_t bytes) {
                if (cudaMalloc(p, bytes) != cudaSuccess) return false;
                mem.push_back(*p);
                return true;
            };
            if (!dal((void **) &dXall, sizeof(float) * hX.size()) || !dal((void **) &dTall, sizeof(float) * hT.size()) ||
                !dal((void **) &dXb, sizeof(float) * (size_t) bs * G_DIN) ||
                !dal((void **) &dTb, sizeof(float) * (size_t) bs * dout) || !dal((void **) &dp, sizeof(float) * np) ||
                !dal((void **) &dg, sizeof(float) * np) || !dal((void **) &dm, sizeof(float) * np) ||
                !dal((void **) &dv, sizeof(float) * np) || !dal((void **) &didx, sizeof(int) * (size_t) nt))
                rc = ERR_ALLOC;
            if (rc == OK) rc = work_alloc(w, G_DIN, G_HID, dout, bs);
            if (rc == OK) {
                cudaMemcpyAsync(dXall, hX.data(), sizeof(float) * hX.size(), cudaMemcpyHostToDevice, s);
                cudaMemcpyAsync(dTall, hT.data(), sizeof(float) * hT.size(), cudaMemcpyHostToDevice, s);
                cudaMemcpyAsync(dp, prm.data(), sizeof(float) * np, cudaMemcpyHostToDevice, s);
                cudaMemsetAsync(dm, 0, sizeof(float) * np, s);
                cudaMemsetAsync(dv, 0, sizeof(float) * np, s);
                std::vector<int> perm(nt);
                std::iota(perm.begin(), perm.end(), 0);
                long long step = 0;
                const int nb = nt / bs;   // full batches only
                double last = 0.0;
                MlpParams P = split_params(dp, G_DIN, G_HID, dout);
                for (int ep = 0; ep < epochs; ep++) {
                    std::shuffle(perm.begin(), perm.end(), rng);
                    cudaMemcpyAsync(didx, perm.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, s);
                    // cosine learning-rate decay over the run
                    double tot = 0.0;
                    for (int b = 0; b < nb; b++) {
                        const unsigned gx = (unsigned) (((size_t) bs * G_DIN + 255) / 256),
                                       gt = (unsigned) (((size_t) bs * dout + 255) / 256);
                        k_gather_rows<<<gx, 256, 0, s>>>(dXall, didx + (size_t) b * bs, bs, G_DIN, dXb);
                        k_gather_rows<<<gt, 256, 0, s>>>(dTall, didx + (size_t) b * bs, bs, dout, dTb);
                        mlp_loss_grad(P, dXb, dTb, bs, w, dg, s);
                        step++;
                        const double frac = (double) (ep * nb + b) / std::max(1, epochs * nb);
                        const float lrt = (float) (lr * 0.5 * (1.0 + std::cos(M_PI * frac)));
                        const float c1 = 1.f - std::pow(0.9f, (float) step), c2 = 1.f - std::pow(0.999f, (float) step);
                        k_adam<<<(unsigned) ((np + 255) / 256), 256, 0, s>>>(dp, dg, dm, dv, np, lrt, 0.9f, 0.999f, c1,
                                                                            c2, 1e-8f);
                        g_launches += 3;
                        if (ep == epochs - 1) tot += read_loss(w, s) / ((double) bs * dout);
                    }
                    if (ep == epochs - 1) last = tot / std::max(1, nb);
                }
                cudaMemcpyAsync(prm.data(), dp, sizeof(float) * np, cudaMemcpyDeviceToHost, s);
                if (cudaStreamSynchronize(s) != cudaSuccess) rc = ERR_CUDA;
                if (final_loss) final_loss[t] = (float) last;
            }
            work_free(w);
            for (void *p : mem) cudaFree(p);
        } else if (final_loss) {
            final_loss[t] = 0.f;
        }
        blobs[t] = prm;
        blobs[t].insert(blobs[t].end(), scale.begin(), scale.end());
        blobs[t].insert(blobs[t].end(), offset.begin(), offset.end());
    }
    cudaStreamDestroy(s);
    if (rc != OK) return rc;
    FILE *f = fopen(path, "wb");
    if (!f) return ERR_FILEIO;
    const int hdr[3] = {G_DIN, G_HID, G_NTYPES};
    bool ok = fwrite(kMagic, 1, 8, f) == 8 && fwrite(hdr, sizeof(int), 3, f) == 3 &&
              fwrite(G_DOUT, sizeof(int), G_NTYPES, f) == (size_t) G_NTYPES;
    for (int t = 0; ok && t < G_NTYPES; t++) ok = fwrite(blobs[t].data(), sizeof(float), blobs[t].size(), f) == blobs[t].size();
    fclose(f);
    return ok ? OK : ERR_FILEIO;
}

int guessnet_grad(int din, int hid, int dout, const float *params, const float *X, const float *T, int n, float *grad,
                  float *loss)
{
    const size_t np = mlp_param_count(din, hid, dout);
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return ERR_CUDA;
    float *dp = nullptr, *dX = nullptr, *dT = nullptr, *dg = nullptr;
    MlpWork w{};
    int rc = OK;
    if (cudaMalloc(&dp, sizeof(float) * np) != cudaSuccess || cudaMalloc(&dg, sizeof(float) * np) != cudaSuccess ||
        cudaMalloc(&dX, sizeof(float) * (size_t) n * din) != cudaSuccess ||
        cudaMalloc(&dT, sizeof(float) * (size_t) n * dout) != cudaSuccess)
        rc = ERR_ALLOC;
    if (rc == OK) rc = work_alloc(w, din, hid, dout, n);
    if (rc == OK) {
        cudaMemcpyAsync(dp, params, sizeof(float) * np, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(dX, X, sizeof(float) * (size_t) n * din, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(dT, T, sizeof(float) * (size_t) n * dout, cudaMemcpyHostToDevice, s);
        mlp_loss_grad(split_params(dp, din, hid, dout), dX, dT, n, w, dg, s);
        const double l = read_loss(w, s) / ((double) n * dout);
        cudaMemcpyAsync(grad, dg, sizeof(float) * np, cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) rc = ERR_CUDA;
        *loss = (float) l;
    }
    work_free(w);
    cudaFree(dp);
    cudaFree(dg);
    cudaFree(dX);
    cudaFree(dT);
    cudaStreamDestroy(s);
    return rc;
}

}  // namespace tscf
