// Internal declarations shared by the host driver (tinyscf.cpp) and the CUDA
// modules. Nothing here is part of the public C ABI (include/*.h).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include <atomic>
#include <functional>

namespace tscf {

// Number of engine kernels launched by this process (host-side count, read by
// the benchmark); atomic, since the allocation-free J entry point may run on
// other host threads than an engine instance.
extern std::atomic<long long> g_launches;
// The part of g_launches that the eigensolver (eigh.cu) launched.
extern std::atomic<long long> g_eig_launches;

// ---------------------------------------------------------------- limits
constexpr int MAX_L_ORB = 2;           // orbital shells up to d
constexpr int MAX_L_AUX = 3;           // auxiliary shells up to f
constexpr int MAXDIIS  = 10;          // TinySCF.h:8
constexpr int BOYS_MMAX = 8;           // highest F_m needed: (dd|dd) Schwarz quartets
constexpr int BOYS_TAYLOR = 7;         // Taylor terms of the tabulated Boys function
constexpr double BOYS_DT = 0.05;       // grid spacing in T
constexpr double BOYS_TMAX = 60.0;     // beyond: asymptotic form
constexpr int BOYS_NGRID = 1201;       // BOYS_TMAX / BOYS_DT + 1

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int ncum(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) * (l + 3) / 6; }

// Status codes returned by the *_status entry points (0 = success).
enum Status : int {
    OK = 0,
    ERR_CUDA = 1,
    ERR_FILEIO = 2,
    ERR_INPUT = 3,
    ERR_UNSUPPORTED = 4,
    ERR_ALLOC = 5,
    ERR_NUMERIC = 6,
    ERR_STATE = 7,
};

// Device view of a shell table (structure of arrays, all device pointers).
struct DevShells {
    int nsh;
    const int *am;        // [nsh]
    const int *nprim;     // [nsh]
    const int *poff;      // [nsh] offset into alpha/coef
    const int *bfoff;     // [nsh+1] first basis function of each shell
    const double *cen;    // [3*nsh] Bohr
    const double *alpha;  // [total prims]
    const double *coef;   // [total prims], normalised (x^l component unit norm)
};

// ---------------------------------------------------------------- integrals (ints.cu)
void boys_table_init(cudaStream_t s);   // uploads the Boys table once per process/device

// Shell ids grouped by angular momentum: d_ids (device) lists the shells of
// AM 0, then 1, ...; h_start (host) holds the group boundaries [maxL+2].

// S and Hcore = T + V for all shell pairs; S, H row-major nbf x nbf.
void launch_one_electron_grouped(const DevShells &sh, const int *d_ids, const int *h_start, int natoms,
                                 const double *d_Z, const double *d_xyz, double *d_S, double *d_H, int nbf,
                                 cudaStream_t s);

// Schwarz screening values for every ordered shell pair (M,N):
// bf_scr[(bfM+iM)*nbf + bfN+iN] = |(mn|mn)| read with the reference's index
// (TinySCF.c:153), sp_scr[M*nsh+N] = max over the block.
void launch_schwarz_grouped(const DevShells &sh, const int *d_ids, const int *h_start, double *d_sp_scr,
                            double *d_bf_scr, int nbf, cudaStream_t s);

// max_p (p|p) for each aux shell.
void launch_df_scrval(const DevShells &aux, double *d_out, cudaStream_t s);

// 3-centre integrals (mn|P) for the listed shell pairs into the unique-pair
// tensor pqA_u[u][P] (u from upair_index[iM*nbf+iN], -1 = absent).
struct ThreeCenterPlan {
    const int2 *pairs;        // [npairs] shell pair (M,N), grouped by AM class
    int npairs;
    const int *class_start;   // host: [nclass+1] pair ranges of each (la,lb) class
    const int *class_la, *class_lb;
    int nclass;
    const int *aux_by_am;     // device: aux shell ids grouped by AM
    const int *aux_am_start;  // host: [MAX_L_AUX+2]
    const double *sp_scr;     // device: [nsh*nsh]
    const double *df_scr;     // device: [naux_sh]
    double scrtol2;
    const int *upair_index;   // device: [nbf*nbf]
    int nbf, naux;
};
void launch_three_center(const DevShells &sh, const DevShells &aux, const ThreeCenterPlan &plan,
                         double *d_pqA_u, cudaStream_t s);

// (P|Q) for aux shell pairs with df_scr[P]*df_scr[Q] >= scrtol2, mirrored; Jpq row-major naux x naux.
void launch_two_center_grouped(const DevShells &aux, const int *d_ids, const int *h_start, const double *d_df_scr,
                               double scrtol2, double *d_Jpq, int naux, cudaStream_t s);

// ---------------------------------------------------------------- screening structures (sparsity.cu)
// *d_out = max of n doubles.
int device_max(const double *d_x, long long n, double *d_out, cudaStream_t s);
// Unique shell pairs of TinySCF.c:183-226 (sp_scr > eta, oriented by the
// am(.)*5 + am(.) index, sorted) into d_first / d_second; *count (host) is
// written once the stream reaches it. d_work: nsh^2 + 2 nsh + 1 ints.
int device_unique_shell_pairs(const double *d_sp_scr, const int *d_am, int nsh, double eta, int *d_work,
                              int *d_first, int *d_second, int *count, cudaStream_t s);
// The bf-pair CSR of TinySCF.c:228-258 (bf_scr > eta) in two passes; d_work:
// 5 n + 2 ints, d_displs: n + 1. Pass 1 returns the totals {ordered pairs,
// unique pairs, upper CSR entries}; pass 2 fills the lists sized from them.
int device_bf_counts(const double *d_bf_scr, int n, double eta, int *d_work, int *d_displs, int totals[3],
                     cudaStream_t s);
int device_bf_fill(const double *d_bf_scr, int n, double eta, const int *d_work, const int *d_displs, int *d_mask,
                   int *d_diag, int *d_upair, int *d_csr_j, int *d_csr_u, int *d_up_i, int *d_up_j, int *d_up_u,
                   cudaStream_t s);

// ---------------------------------------------------------------- dense FP64 (linalg.cu)
// C = alpha * op(A) * op(B) + beta * C, row-major, op = transpose if ta/tb.
void dgemm(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, int lda,
           const double *B, int ldb, double beta, double *C, int ldc, cudaStream_t s);

// The same product with the tile picked from the call shape (no tuning run).
void dgemm_untuned(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, int lda,
                   const double *B, int ldb, double beta, double *C, int ldc, cudaStream_t s);
// ERR_CUDA (with a message) when a launch since the last check failed; the error is not cleared.
int cuda_launch_rc(const char *what);
// Streaming multiprocessors of the current device (queried once per device).
int num_sms();

// Device buffers of the engine (linalg.cu): from the device's stream-ordered
// pool, kept reserved across engines, unless TINYSCF_MEMPOOL=0. dev_malloc
// returns once the buffer is usable on any stream; dev_free is stream-ordered
// on s (the caller synchronises before reusing the memory elsewhere).
int  dev_malloc(void **p, size_t bytes, cudaStream_t s);
void dev_free(void *p, cudaStream_t s);
int  dev_trim(int device);   // return the pool's unused memory to the device

// Symmetric eigen-decomposition (eigh.cu; ascending eigenvalues). A is
// row-major n x n symmetric; on return V holds eigenvectors as ROWS (V[k*n + i]
// = i-th entry of eigenvector k); V may alias A. Workspace (four n x n
// matrices) is owned by the Eig object; n <= EIG_MAX_N. Asynchronous on s;
// eig_error() (synchronous) reports a grid barrier of the tridiagonalisation
// that gave up waiting.
constexpr int EIG_MAX_N = 8192;
struct Eig;
Eig *eig_create(int n, cudaStream_t s);
void eig_destroy(Eig *e);
int  eig_run(Eig *e, const double *d_A, double *d_w, double *d_V, cudaStream_t s);
int  eig_error(Eig *e);

// Orthonormal rows U (o x n) spanning the dominant o-dimensional invariant
// subspace of a symmetric M (n x n): iters products with M from a fixed
// pseudo-random start, orthonormalised by Cholesky-QR every few products and
// twice at the end; W (o x n) and G (o x o) are scratch; the Cholesky factor
// and its inverse are this library's kernels. ERR_NUMERIC when a Cholesky
// factor fails (the caller then solves the eigenproblem instead).
int dominant_subspace(Eig *e, const double *d_M, double *d_U, double *d_W, double *d_G, int n, int o, int iters,
                      cudaStream_t s);
// X = U diag(f(w)) U^T with f(w) = w^-1/2, U from eigenvectors in rows.
void inv_sqrt_from_eig(const double *d_w, const double *d_V, double *d_X, double *d_tmp, int n, cudaStream_t s);

// LAPACK dpstf2 semantics (unblocked pivoted Cholesky, lower, first-max pivot),
// applied to a row-major symmetric matrix in place; rank to *d_rank. d_blk
// (optional, n ints; d_blk_work: n ints of scratch): a block id per row when A
// is block diagonal in those blocks; the result is the same, bit for bit.
void pivoted_cholesky(double *d_A, int n, double tol, int *d_piv, int *d_rank, double *d_work, cudaStream_t s,
                      const int *d_blk = nullptr, int *d_blk_work = nullptr);
// TinySCF_D2Cocc's copy of the factor into Cocc (TinySCF.c:297-319).
void d2cocc_copy(const double *d_chol, const int *d_rank, double *d_Cocc, int nbf, int nocc, cudaStream_t s);

// Elementwise helpers.
void fill(double *d, double v, size_t n, cudaStream_t s);
void scale_copy(const double *src, double *dst, double a, size_t n, cudaStream_t s);

// ---------------------------------------------------------------- Fock build (fock.cu)
struct FockPlan {
    int nbf, naux, nocc;
    int nnz;                  // ordered screened pairs (reference CSR)
    int nup;                  // ordered pairs (i, j>=i) used by J
    const int *csr_j;         // [nnz] column j of each CSR entry
    const int *csr_displs;    // [nbf+1]
    const int *csr_u;         // [nnz] unique-pair row of each CSR entry
    const int *up_i, *up_j;   // [nup] upper CSR entries (i <= j)
    const int *up_u;          // [nup] their unique-pair rows
    const double *B;          // DF tensor, [nu][naux] unique pairs
};
// J = symmetrised Coulomb matrix from D (build_Fock.c:37-130).
// d_t (naux) and d_part (scratch, nblk*naux) are caller buffers.
void build_J(const FockPlan &p, const double *d_D, double *d_J, double *d_t, double *d_part, int part_blocks,
             double *d_w, cudaStream_t s);
int  build_J_part_blocks(const FockPlan &p);
// J from an FP32 copy of the DF tensor (FP64 products and sums): half the HBM
// traffic, ~1e-7 relative error; the mixed-precision form's iterations use it
void build_J_f32(const FockPlan &p, const float *B32, const double *d_D, double *d_J, double *d_t, double *d_part,
                 int part_blocks, double *d_w, cudaStream_t s);
void convert_f32(const double *in, float *out, size_t n, cudaStream_t s);
// K from Cocc (build_Fock.c:244-347): T(i,s,P) = sum_j C(j,s) B(ij,P) ...
// wide = 1: 64 x 256 FFMA tiles (k_halftransform_wide), 2: 64 x 256 DMMA tiles
// (k_halftransform_dmma), 3: the same DMMA tiles in persistent CTAs with a
// cp.async pipeline over the CSR chunks (k_halftransform_pipe), 4: 168 x 128
// DMMA tiles over 12 warps in the same pipeline (k_halftransform_pipe2), 0:
// 64 x 64 FFMA tiles
// d_rowmax (wide = 3 or 4, else ignored): max_q |T(i, q)| of every row as
// double bits, for the integer-tensor-core K.
void build_K_halftransform(const FockPlan &p, const double *d_Cocc, double *d_T, cudaStream_t s, int wide = 0,
                           unsigned long long *d_rowmax = nullptr);
// ... then K = T T^T over upper 64x64 tiles (d_tiles: (bi,bj), bi <= bj), split-K, mirrored.
// tile = 64 (k_syrk_part, FFMA), 128 (k_syrk_part128, FFMA) or KSYRK_DMMA
// (k_syrk_dmma: 128 x 128 tiles on the FP64 tensor cores); d_tiles lists the
// upper tile pairs for that tile size (128 for KSYRK_DMMA)
constexpr int KSYRK_DMMA = 129;
void build_K_syrk(const FockPlan &p, const double *d_T, double *d_K, double *d_Kpart, int ksplit,
                  const int2 *d_tiles, cudaStream_t s, int tile = 64);
size_t build_K_part_elems(const FockPlan &p, int ksplit);
// F = H + 2J - K and e_part[b] = partial sums of D .* (F + H) (TinySCF.c:367-376).
void build_F_energy(const double *d_H, const double *d_J, const double *d_K, const double *d_D,
                    double *d_F, double *d_epart, int n, cudaStream_t s);
constexpr int ENERGY_BLOCKS = 296;
// ---------------------------------------------------------------- mixed-precision K (kmixed.cu)
struct KMix;
// Needs p.B, p.csr_j, p.csr_u, p.nbf, p.naux, p.nocc and the host CSR row starts.
int  kmix_create(KMix **out, const FockPlan &p, const int *h_displs, cudaStream_t s);
void kmix_destroy(KMix *k);
void kmix_reset(KMix *k, cudaStream_t s);
// K (FP64, accumulated across calls) from the occupied factor Cocc; S is the overlap.
// mark (optional) is called with 0 before the half-transform kernel, 1 between
// it and the G GEMM, 2 after the G GEMM (device timers around the two).
int  kmix_build(KMix *k, const double *Cocc, const double *S, double *K, cudaStream_t s,
                const std::function<void(int)> &mark = nullptr);
int  kmix_error_flag();
// Many molecules' incremental K builds with one half-transform launch and one
// G GEMM launch over all of them (the alignments and reductions stay per
// molecule). ks: the molecules' KMix objects (owned by the caller).
struct KMixBatch;
int  kmix_batch_create(KMixBatch **out, KMix *const *ks, int n, cudaStream_t s);
void kmix_batch_destroy(KMixBatch *b);
// active[m] (host): molecules to build; Cocc[m], S[m] their inputs, K[m] their K (FP64, accumulated).
int  kmix_batch_build(KMixBatch *b, const int *active, const double *const *Cocc, const double *const *S,
                      double *const *K, cudaStream_t s);
// Runs the G GEMM kernel's bounded waits out on purpose (no copies issued,
// waits of wait_cycles clock cycles); *code receives the recorded wait code.
int  kmix_wait_probe(KMix *k, long long wait_cycles, int *code, cudaStream_t s);

// ---------------------------------------------------------------- K = T T^T on the integer tensor cores (ozaki.cu)
struct OzSyrk;
// T is nbf x Q (row pitch Q); workspace: the residue planes (nmod x nbf x Q bytes, padded).
int  oz_create(OzSyrk **out, int nbf, long long Q, cudaStream_t s);
void oz_destroy(OzSyrk *o);
// K (nbf x nbf, both triangles) = T T^T to FP64 accuracy. d_rowmax: the rows'
// max |T| as double bits when the half-transform produced them (oz_rowmax),
// else nullptr (the rows are scanned).
int  oz_syrk(OzSyrk *o, const double *d_T, double *d_K, cudaStream_t s, const unsigned long long *d_rowmax = nullptr);
unsigned long long *oz_rowmax(OzSyrk *o);
int  oz_error_flag();
// {moduli, beta, tiles, K ranges, chunks per range, padded rows}
void oz_info(const OzSyrk *o, int info[6]);

// ---------------------------------------------------------------- DIIS / density (scf.cu)
constexpr int DIIS_DOT_BLOCKS = 512;      // most blocks of the DIIS residual dots
struct DiisState {            // device-resident DIIS bookkeeping (DIIS.c:12-123)
    int len;
    int bmax_id;
    int idx;
    int pad;
    double bmax;
    double B[(MAXDIIS + 1) * (MAXDIIS + 1)];
    double coef[MAXDIIS + 1];
    double dots[MAXDIIS];
    double part[DIIS_DOT_BLOCKS * MAXDIIS];   // per-block partial sums of the dots
};
void diis_init(DiisState *d_st, cudaStream_t s);
void diis_step(DiisState *d_st, int max_diis, const double *d_F, const double *d_D, const double *d_S,
               const double *d_X, double *d_Fout, double *d_F0, double *d_R, double *d_tmp, double *d_tmp2,
               int n, cudaStream_t s);
// diis_step when D = Cocc Cocc^T: the commutator from n x n_occ products (needs 2 n_occ <= n).
void diis_step_cocc(DiisState *d_st, int max_diis, const double *d_F, const double *d_Cocc, int o, const double *d_S,
                    const double *d_X, double *d_Fout, double *d_F0, double *d_R, double *d_tmp, double *d_tmp2, int n,
                    cudaStream_t s);
void xtfx(const double *d_X, const double *d_F, double *d_out, double *d_tmp, int n, cudaStream_t s);
void energy_reduce(const double *d_epart, double *d_E, cudaStream_t s);
// Occupied-subspace refinement between full eigensolves (scf.cu).
struct SubspaceWork {
    double *A, *UA, *R, *Cv, *M, *Y, *Z, *T, *W, *res;
};
int subspace_refine(const double *d_Fp, const double *d_Vstale, const double *d_wstale, double *d_U, int n, int o,
                    SubspaceWork &w, double tol, int max_steps, int *steps_out, double *res_out, cudaStream_t s);
// Refinement inside a stream capture: the steps run in a WHILE conditional
// node whose condition a device kernel sets from the residual. d_ctl->tol and
// ->max_steps are inputs; ->step, ->res and ->converged are written.
struct RefineCtl {
    double res, prev, tol;
    int step, max_steps, converged;
};
int subspace_refine_capture(const double *d_Fp, const double *d_Vstale, const double *d_wstale, double *d_U, int n,
                            int o, SubspaceWork &w, RefineCtl *d_ctl, cudaStream_t s, cudaStream_t s_body,
                            long long *body_launches);
void density_from_rows(const double *d_X, const double *d_U, double *d_Cocc, double *d_D, int n, int nocc,
                       cudaStream_t s);
// Cocc = X * V[0:nocc]^T (eigenvectors in rows), D = Cocc Cocc^T.
void density_from_eig(const double *d_X, const double *d_V, double *d_Cocc, double *d_D, int n, int nocc,
                      cudaStream_t s);

}  // namespace tscf

#define RC_(x)                      \
    do {                            \
        const int rc__ = (x);       \
        if (rc__) return rc__;      \
    } while (0)

#define TSCF_CUDA_CHECK(x)                                                            \
    do {                                                                              \
        cudaError_t e__ = (x);                                                        \
        if (e__ != cudaSuccess) {                                                     \
            fprintf(stderr, "[tinyscf] CUDA error %s at %s:%d: %s\n", #x, __FILE__,   \
                    __LINE__, cudaGetErrorString(e__));                               \
            return tscf::ERR_CUDA;                                                    \
        }                                                                             \
    } while (0)
