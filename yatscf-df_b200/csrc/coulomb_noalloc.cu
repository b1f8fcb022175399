// A Coulomb (J) build that allocates nothing, for callers that cannot call
// cudaMalloc: a host framework that owns every byte of device memory through
// its own pool (an allocation made behind its back is memory its pool cannot
// see or reclaim, and cudaMalloc can synchronise the device in the middle of
// the framework's own pipeline). The caller passes all inputs and the output
// as device pointers; the
// per-block partial sums, the fitted vector t(P) and the pair weights that the
// J build needs live in the file-scope array below instead of in buffers the
// engine allocates.
//
// Limits: naux <= 4096 auxiliary functions and nup <= 524288 upper pairs; the
// array takes (296 * 4096 + 4096 + 524288) doubles = 13.9 MB on every GPU that
// loads this library, held until the process exits.
//
// The first call on a device looks up the array's device address with that
// device current (cudaGetSymbolAddress) and caches it for the life of the
// process; make that first call before any stream capture. The cached address
// does not survive cudaDeviceReset: do not call this entry point on a device
// after resetting it. Every call shares the one array, which keeps the
// previous call's contents: calls that overlap on the GPU (other streams,
// other host threads) race on it and must be serialised by the caller. No
// part of the array has to start at zero: each call overwrites everything it
// reads.
#include <cstdio>
#include <mutex>

#include "tinyscf_b200.h"
#include "tscf_internal.h"

namespace {

constexpr int kMaxNaux = 4096;
constexpr int kMaxPairs = 524288;
constexpr int kMaxBlocks = 296;   // upper bound of build_J_part_blocks()
constexpr size_t kScratch = (size_t) kMaxBlocks * kMaxNaux + kMaxNaux + kMaxPairs;

__device__ __align__(256) double g_noalloc_scratch[kScratch];

constexpr int kMaxDevices = 64;
double *g_addr[kMaxDevices] = {nullptr};
std::mutex g_mu;

}  // namespace

extern "C" int TinySCF_build_J_noalloc(const double *B, int naux, const int *up_i, const int *up_j, const int *up_u,
                                       int nup, int nbf, const double *D, double *J, void *stream)
{
    if (!B || !up_i || !up_j || !up_u || !D || !J || nbf <= 0 || naux <= 0 || nup <= 0) {
        fprintf(stderr, "[tinyscf] TinySCF_build_J_noalloc: null pointer or empty size\n");
        return TINYSCF_ERR_INPUT;
    }
    if (naux > kMaxNaux || nup > kMaxPairs) {
        fprintf(stderr, "[tinyscf] TinySCF_build_J_noalloc: naux %d (max %d) or nup %d (max %d) is beyond the "
                        "fixed scratch of this entry point\n", naux, kMaxNaux, nup, kMaxPairs);
        return TINYSCF_ERR_UNSUPPORTED;
    }
    // an error already pending on this thread is the caller's: left pending and not reported
    const cudaError_t pending = cudaPeekAtLastError();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TINYSCF_ERR_CUDA;
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_addr[dev]) {
            void *p = nullptr;
            cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (err != cudaSuccess || !p) {
                fprintf(stderr, "[tinyscf] TinySCF_build_J_noalloc: cudaGetSymbolAddress failed: %s\n",
                        cudaGetErrorString(err));
                return TINYSCF_ERR_CUDA;
            }
            g_addr[dev] = (double *) p;
        }
        scratch = g_addr[dev];
    }
    double *part = scratch;
    double *t = part + (size_t) kMaxBlocks * kMaxNaux;
    double *w = t + kMaxNaux;

    tscf::FockPlan p{};
    p.nbf = nbf;
    p.naux = naux;
    p.nup = nup;
    p.up_i = up_i;
    p.up_j = up_j;
    p.up_u = up_u;
    p.B = B;
    const int nblk = tscf::build_J_part_blocks(p);
    cudaStream_t s = (cudaStream_t) stream;
    // J entries of screened pairs are never written by the J kernels: clear the output.
    if (cudaMemsetAsync(J, 0, sizeof(double) * (size_t) nbf * nbf, s) != cudaSuccess) return TINYSCF_ERR_CUDA;
    tscf::build_J(p, D, J, t, part, nblk, w, s);
    const cudaError_t launched = cudaPeekAtLastError();
    return (launched == cudaSuccess || launched == pending) ? TINYSCF_OK : TINYSCF_ERR_CUDA;
}
