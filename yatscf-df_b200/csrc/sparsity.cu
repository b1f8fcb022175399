// Screening structures on the device (TinySCF.c:183-280): the unique shell
// pairs that survive Schwarz screening, and the basis-function pair CSR of
// TinySCF_prepare_sparsity, plus the unique-pair numbering and the upper-pair
// lists the J/K kernels use. Every list keeps the reference's order (row-major
// over the pair index), built by counting per row, an exclusive scan and a
// warp-ballot compaction, so the result is identical to the sequential loops.
#include <cstdio>

#include "tscf_internal.h"

namespace tscf {

namespace {

__global__ void k_max_reduce(const double *x, long long n, double *out)
{
    __shared__ double sh[32];
    double m = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, x[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffff, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffff, m, o));
        if (threadIdx.x == 0) *out = m;
    }
}

// Exclusive scan of n counts into out[0..n] (out[n] = total), one block.
__global__ void __launch_bounds__(1024) k_scan(const int *cnt, int n, int *out)
{
    __shared__ int part[1024];
    const int per = (n + blockDim.x - 1) / blockDim.x, b = threadIdx.x * per, e = min(n, b + per);
    int s = 0;
    for (int i = b; i < e; i++) s += cnt[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < (int) blockDim.x; o <<= 1) {
        const int v = threadIdx.x >= (unsigned) o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int run = part[threadIdx.x] - s;
    for (int i = b; i < e; i++) {
        out[i] = run;
        run += cnt[i];
    }
    if (threadIdx.x == blockDim.x - 1) out[n] = part[threadIdx.x];
}

// Unique shell pairs (TinySCF.c:183-226): pair (M, N >= M) survives when
// sp_scr > eta; it is stored oriented (CMS_Simint.c:308-312: the shell of the
// larger am(.)*5 + am(.) index first) and the list is sorted, i.e. row-major
// over the oriented pair. flags[a * nsh + b] marks oriented pair (a, b).
__global__ void k_uniq_flags(const double *sp_scr, const int *am, int nsh, double eta, int *flags)
{
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long) nsh * nsh) return;
    const int M = (int) (idx / nsh), N = (int) (idx % nsh);
    if (N < M || !(sp_scr[idx] > eta)) return;
    const int mn = am[M] * 5 + am[N], nm = am[N] * 5 + am[M];
    const int a = mn > nm ? M : N, b = mn > nm ? N : M;
    flags[(size_t) a * nsh + b] = 1;
}

// Per row of an n x n predicate: the count of true entries (warp per row).
template <typename Pred>
__device__ void warp_row_count(int row, int n, Pred pred, int *cnt)
{
    const int lane = threadIdx.x & 31;
    int c = 0;
    for (int j = lane; j < n; j += 32) c += pred(j) ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffff, c, o);
    if (lane == 0) cnt[row] = c;
}

__global__ void k_flag_counts(const int *flags, int n, int *cnt)
{
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= n) return;
    warp_row_count(row, n, [&](int j) { return flags[(size_t) row * n + j] != 0; }, cnt);
}

__global__ void k_flag_fill(const int *flags, int n, const int *start, int *first, int *second)
{
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= n) return;
    const int lane = threadIdx.x & 31;
    int base = start[row];
    for (int j0 = 0; j0 < n; j0 += 32) {
        const int j = j0 + lane;
        const bool f = j < n && flags[(size_t) row * n + j] != 0;
        const unsigned bal = __ballot_sync(0xffffffff, f);
        if (f) {
            const int k = base + __popc(bal & ((1u << lane) - 1));
            first[k] = row;
            second[k] = j;
        }
        base += __popc(bal);
    }
}

// Basis-function pairs (TinySCF.c:228-258): row counts of the CSR, of the
// unique pairs (j >= i surviving in either order) and of the CSR's upper entries.
__global__ void k_bf_counts(const double *bf_scr, int n, double eta, int *cnt, int *ucnt, int *upcnt)
{
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= n) return;
    const double *row = bf_scr + (size_t) i * n;
    warp_row_count(i, n, [&](int j) { return row[j] > eta; }, cnt);
    warp_row_count(i, n, [&](int j) { return j >= i && (row[j] > eta || bf_scr[(size_t) j * n + i] > eta); }, ucnt);
    warp_row_count(i, n, [&](int j) { return j >= i && row[j] > eta; }, upcnt);
}

// mask, CSR columns, diagonal entries and the symmetric unique-pair numbering.
__global__ void k_bf_fill(const double *bf_scr, int n, double eta, const int *displs, const int *ustart, int *mask,
                          int *csr_j, int *diag, int *upair)
{
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= n) return;
    const int lane = threadIdx.x & 31;
    const double *row = bf_scr + (size_t) i * n;
    int base = displs[i], ubase = ustart[i];
    for (int j0 = 0; j0 < n; j0 += 32) {
        const int j = j0 + lane;
        const bool f = j < n && row[j] > eta;
        const unsigned bal = __ballot_sync(0xffffffff, f);
        if (j < n) {
            const int k = f ? base + __popc(bal & ((1u << lane) - 1)) : -1;
            mask[(size_t) i * n + j] = k;
            if (f) csr_j[k] = j;
            if (j == i) diag[i] = k;
        }
        base += __popc(bal);
        const bool u = j < n && j >= i && (f || bf_scr[(size_t) j * n + i] > eta);
        const unsigned ubal = __ballot_sync(0xffffffff, u);
        if (u) {
            const int k = ubase + __popc(ubal & ((1u << lane) - 1));
            upair[(size_t) i * n + j] = k;
            upair[(size_t) j * n + i] = k;
        } else if (j < n && j >= i) {
            upair[(size_t) i * n + j] = -1;
            upair[(size_t) j * n + i] = -1;
        }
        ubase += __popc(ubal);
    }
}

// Unique row of each CSR entry and the CSR's upper entries in CSR order.
__global__ void k_bf_fill_upper(const int *csr_j, const int *displs, const int *upstart, const int *upair, int n,
                                int *csr_u, int *up_i, int *up_j, int *up_u)
{
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= n) return;
    const int lane = threadIdx.x & 31;
    const int r0 = displs[i], r1 = displs[i + 1];
    int base = upstart[i];
    for (int q0 = r0; q0 < r1; q0 += 32) {
        const int r = q0 + lane;
        const int j = r < r1 ? csr_j[r] : -1;
        const int u = r < r1 ? upair[(size_t) i * n + j] : -1;
        if (r < r1) csr_u[r] = u;
        const bool f = r < r1 && j >= i;
        const unsigned bal = __ballot_sync(0xffffffff, f);
        if (f) {
            const int k = base + __popc(bal & ((1u << lane) - 1));
            up_i[k] = i;
            up_j[k] = j;
            up_u[k] = u;
        }
        base += __popc(bal);
    }
}

int grid_rows(int n) { return (n + 7) / 8; }   // 8 warps per block of 256 threads

}  // namespace

int device_max(const double *d_x, long long n, double *d_out, cudaStream_t s)
{
    g_launches++;
    k_max_reduce<<<1, 1024, 0, s>>>(d_x, n, d_out);
    return cuda_launch_rc("maximum");
}

int device_unique_shell_pairs(const double *d_sp_scr, const int *d_am, int nsh, double eta, int *d_work,
                              int *d_first, int *d_second, int *count, cudaStream_t s)
{
    const size_t nn = (size_t) nsh * nsh;
    int *flags = d_work, *cnt = d_work + nn, *start = cnt + nsh;
    TSCF_CUDA_CHECK(cudaMemsetAsync(flags, 0, sizeof(int) * nn, s));
    k_uniq_flags<<<(unsigned) ((nn + 255) / 256), 256, 0, s>>>(d_sp_scr, d_am, nsh, eta, flags);
    k_flag_counts<<<grid_rows(nsh), 256, 0, s>>>(flags, nsh, cnt);
    k_scan<<<1, 1024, 0, s>>>(cnt, nsh, start);
    k_flag_fill<<<grid_rows(nsh), 256, 0, s>>>(flags, nsh, start, d_first, d_second);
    g_launches += 4;
    TSCF_CUDA_CHECK(cudaMemcpyAsync(count, start + nsh, sizeof(int), cudaMemcpyDeviceToHost, s));
    return cuda_launch_rc("unique shell pairs");
}

// Pass 1: row counts and their scans (CSR row starts into d_displs); totals =
// {screened ordered pairs, unique pairs, upper CSR entries} (synchronous).
int device_bf_counts(const double *d_bf_scr, int n, double eta, int *d_work, int *d_displs, int totals[3],
                     cudaStream_t s)
{
    int *cnt = d_work, *ucnt = cnt + n, *upcnt = ucnt + n, *ustart = upcnt + n, *upstart = ustart + n + 1;
    k_bf_counts<<<grid_rows(n), 256, 0, s>>>(d_bf_scr, n, eta, cnt, ucnt, upcnt);
    k_scan<<<1, 1024, 0, s>>>(cnt, n, d_displs);
    k_scan<<<1, 1024, 0, s>>>(ucnt, n, ustart);
    k_scan<<<1, 1024, 0, s>>>(upcnt, n, upstart);
    g_launches += 4;
    TSCF_CUDA_CHECK(cudaMemcpyAsync(&totals[0], d_displs + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    TSCF_CUDA_CHECK(cudaMemcpyAsync(&totals[1], ustart + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    TSCF_CUDA_CHECK(cudaMemcpyAsync(&totals[2], upstart + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    TSCF_CUDA_CHECK(cudaStreamSynchronize(s));
    return cuda_launch_rc("basis-function pair counts");
}

// Pass 2 (d_work and d_displs from pass 1): mask, CSR columns, diagonal
// entries, unique-pair numbering, unique row of each CSR entry, upper lists.
int device_bf_fill(const double *d_bf_scr, int n, double eta, const int *d_work, const int *d_displs, int *d_mask,
                   int *d_diag, int *d_upair, int *d_csr_j, int *d_csr_u, int *d_up_i, int *d_up_j, int *d_up_u,
                   cudaStream_t s)
{
    const int *ustart = d_work + 3 * n, *upstart = ustart + n + 1;
    k_bf_fill<<<grid_rows(n), 256, 0, s>>>(d_bf_scr, n, eta, d_displs, ustart, d_mask, d_csr_j, d_diag, d_upair);
    k_bf_fill_upper<<<grid_rows(n), 256, 0, s>>>(d_csr_j, d_displs, upstart, d_upair, n, d_csr_u, d_up_i, d_up_j,
                                                d_up_u);
    g_launches += 2;
    return cuda_launch_rc("basis-function pair sparsity");
}

}  // namespace tscf
