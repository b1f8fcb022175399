/*
 * Extensions of the B200 engine beyond the reference's TinySCF API. None of
 * these exist in the reference; they give FFI callers status codes instead of
 * abort(), let tests feed a density in, and expose device timings.
 */
#ifndef TINYSCF_B200_EXT_H
#define TINYSCF_B200_EXT_H

#include <stddef.h>
#include "TinySCF.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (0 = success). */
#define TINYSCF_OK              0
#define TINYSCF_ERR_CUDA        1
#define TINYSCF_ERR_FILEIO      2
#define TINYSCF_ERR_INPUT       3
#define TINYSCF_ERR_UNSUPPORTED 4
#define TINYSCF_ERR_ALLOC       5
#define TINYSCF_ERR_NUMERIC     6
#define TINYSCF_ERR_STATE       7

/* Device-event timers (milliseconds of the last call of each phase). */
enum {
    TINYSCF_T_HCORE = 0,     /* S, Hcore, X                          */
    TINYSCF_T_SCHWARZ,       /* Schwarz quartets + DF screening      */
    TINYSCF_T_GUESS,         /* SAD upload + pivoted Cholesky        */
    TINYSCF_T_3C,            /* 3-centre integrals                   */
    TINYSCF_T_2C,            /* (P|Q)                                */
    TINYSCF_T_INVSQRT,       /* (P|Q)^-1/2                           */
    TINYSCF_T_DFGEMM,        /* B = (mn|P) (P|Q)^-1/2                */
    TINYSCF_T_J,             /* J build                              */
    TINYSCF_T_K_HT,          /* K occupied half-transform            */
    TINYSCF_T_K_SYRK,        /* K = T T^T                            */
    TINYSCF_T_FOCK,          /* F = H + 2J - K and energy            */
    TINYSCF_T_DIIS,          /* DIIS                                 */
    TINYSCF_T_DENSITY,       /* eigensolve + density                 */
    TINYSCF_T_ITER,          /* one SCF iteration                    */
    TINYSCF_T_SCF,           /* the whole TinySCF_do_SCF             */
    TINYSCF_T_K_MIXED,       /* mixed-precision incremental K        */
    TINYSCF_T_FINAL,         /* final FP64 Fock build (mixed mode)   */
    TINYSCF_T_K_HALF,        /* mixed K: tensor-core half-transform  */
    TINYSCF_T_K_GEMM,        /* mixed K: tensor-core G = dT S^T      */
    TINYSCF_T_COUNT
};

/* malloc a zeroed struct for callers that cannot use sizeof (FFI);
 * free_TinySCF releases it, as it does a caller-malloc'd struct. */
TINYSCF_API TinySCF_t TinySCF_alloc(void);
/* sizeof(struct TinySCF_struct) as compiled into the library, for FFI mirrors. */
TINYSCF_API size_t TinySCF_struct_size(void);
TINYSCF_API const char *TinySCF_status_string(int status);

/* Status-returning twins of the TinySCF API (same semantics, no abort). */
TINYSCF_API int TinySCF_init_status(TinySCF_t t, const char *bas_fname, const char *df_bas_fname,
                        const char *xyz_fname, int niters);
TINYSCF_API int TinySCF_compute_Hcore_Ovlp_mat_status(TinySCF_t t);
TINYSCF_API int TinySCF_compute_sq_Schwarz_scrvals_status(TinySCF_t t);
TINYSCF_API int TinySCF_prepare_sparsity_status(TinySCF_t t);
TINYSCF_API int TinySCF_get_initial_guess_status(TinySCF_t t);
TINYSCF_API int TinySCF_build_DF_tensor_status(TinySCF_t t);
TINYSCF_API int TinySCF_build_FockMat_status(TinySCF_t t);
TINYSCF_API int TinySCF_DIIS_status(TinySCF_t t);
TINYSCF_API int TinySCF_build_DenMat_status(TinySCF_t t);
TINYSCF_API int TinySCF_do_SCF_status(TinySCF_t t);
TINYSCF_API int TinySCF_free_status(TinySCF_t t);

/* Upload a density (nbf x nbf) and its factor (nbf x n_occ; NULL keeps the
 * current one) from host memory; used before TinySCF_build_FockMat. */
TINYSCF_API int TinySCF_set_density(TinySCF_t t, const double *D, const double *Cocc);
/* Upload a Fock matrix (nbf x nbf): the input of TinySCF_DIIS, or, with
 * orthogonal != 0, the X^T F X input of TinySCF_build_DenMat. */
TINYSCF_API int TinySCF_set_fock(TinySCF_t t, const double *F, int orthogonal);
/* Copy S, Hcore, X, F, D, J, K, Cocc, eigval and DIIS state to the host mirrors. */
TINYSCF_API int TinySCF_sync_host(TinySCF_t t);
/* Copy the DF tensor in the reference's layout: rows in bf_pair CSR order
 * (nnz rows), df_nbf columns. out must hold num_bf_pair_scr * df_nbf doubles. */
TINYSCF_API int TinySCF_get_df_tensor(TinySCF_t t, double *out);
/* Timers: writes min(n, TINYSCF_T_COUNT) values in milliseconds (last call). */
TINYSCF_API int TinySCF_get_timings(TinySCF_t t, double *ms, int n);
/* Accumulated timers since the last reset: total milliseconds and number of
 * timed calls per phase (per SCF iteration for the per-iteration phases). */
TINYSCF_API int TinySCF_get_timing_stats(TinySCF_t t, double *sum_ms, long long *count, int n);
TINYSCF_API int TinySCF_reset_timing_stats(TinySCF_t t);
/* Counters: [0] engine kernels launched by this process, [1] bytes copied
 * host->device, [2] bytes copied device->host by this engine instance,
 * [3] full eigensolves and [4] occupied-subspace refinement steps taken by
 * the density builds of this instance, [5] (shell pair, aux shell) tuples the
 * last 3-centre integral build launched (before screening), [6] restarts of
 * TinySCF_do_SCF from the SAD guess by its divergence guard (an energy that is
 * not finite, or one rising by more than 1e-6 Eh four iterations in a row;
 * a second divergence in the same solve returns TINYSCF_ERR_NUMERIC), [7] FP64
 * exchange products K = T T^T this instance ran on the integer tensor cores
 * (Ozaki scheme II: int8 residues of T modulo 15 coprime moduli, exact int32
 * products, Chinese-remainder reconstruction; chosen by the autotuner when
 * faster, forced on or off by the environment variable TINYSCF_OZAKI=1 / 0). */
TINYSCF_API int TinySCF_get_counters(TinySCF_t t, long long *out, int n);
/* Coulomb matrix J from a density D without allocating anything: for callers
 * that cannot call cudaMalloc (a host framework that owns all device memory
 * through its own pool, which an allocation made behind its back would
 * escape). No counterpart in the reference. All pointers are device pointers: B holds one
 * DF-tensor row of naux doubles per pair, up_i/up_j/up_u list the nup upper
 * pairs (i <= j) and the B row of each, D and J are nbf x nbf row-major;
 * stream is a cudaStream_t (NULL = default stream). The call is asynchronous.
 * Scratch is a fixed 13.9 MB __device__ array inside the library (held on
 * every GPU that loads it until exit), so naux <= 4096 and nup <= 524288;
 * larger sizes return TINYSCF_ERR_UNSUPPORTED. The first call on a device
 * looks the array up and caches its address for the process (make it before
 * any stream capture; not valid after cudaDeviceReset of that device); calls
 * that overlap on the GPU share the array and race. The return code covers
 * the arguments, that look-up and the launches (an error already pending on
 * the calling thread is left pending and not reported); faults while the
 * kernels run surface at the caller's next synchronisation. */
TINYSCF_API int TinySCF_build_J_noalloc(const double *B, int naux, const int *up_i, const int *up_j,
                                        const int *up_u, int nup, int nbf, const double *D, double *J,
                                        void *stream);
/* Precision of the exchange build. TINYSCF_K_FP64 (default): FP64 on the CUDA
 * cores, the reference's arithmetic. TINYSCF_K_MIXED: incremental builds from
 * the change of the occupied orbitals on the tcgen05 tensor cores (split-BF16
 * operands, FP32 accumulation, FP64 K), J of the iterations from an FP32 copy
 * of the DF tensor (FP64 arithmetic), then one FP64 Fock build at convergence
 * whose energy is the result. In mixed mode each Fock build
 * updates K from the previous build's orbitals; TinySCF_reset_scf restarts. */
#define TINYSCF_K_FP64  0
#define TINYSCF_K_MIXED 1
TINYSCF_API int TinySCF_set_k_precision(TinySCF_t t, int mode);
/* Density solver of the SCF loop. TINYSCF_DENSITY_EIG (default): a full
 * eigendecomposition of X^T F X every iteration, as build_density.c:37-69.
 * TINYSCF_DENSITY_REFINE: once a full eigensolve has been taken, later
 * iterations refine the previous occupied subspace against the new Fock
 * matrix (residual preconditioned with the last full eigenbasis, Loewdin
 * re-orthonormalisation) until max|(I-P)F'U^T| < 1e-9 Eh, and fall back to a
 * full eigensolve when that does not converge within a few steps. D is the
 * same aufbau density as long as no orbital level crosses the HOMO-LUMO gap
 * between full eigensolves; eigval and the columns of Cocc then hold the last
 * full eigensolve's eigenvalues and an orthonormal (not canonical) occupied
 * basis. */
#define TINYSCF_DENSITY_EIG    0
#define TINYSCF_DENSITY_REFINE 1
TINYSCF_API int TinySCF_set_density_solver(TinySCF_t t, int mode);
/* CUDA-graph SCF iterations. With on = 1, TinySCF_do_SCF captures one
 * iteration from iteration 3 on (DIIS active and run once eagerly, so the
 * autotuner has seen every shape) into a CUDA graph: J, K,
 * Fock and energy, DIIS and, with TINYSCF_DENSITY_REFINE, the density with its
 * refinement loop as a device-controlled conditional (WHILE) node; each later
 * iteration is one graph launch. The full eigensolve of TINYSCF_DENSITY_EIG
 * (and the refinement's fallback) runs outside the graph. The graph is
 * recaptured when the K precision or density solver changes. */
TINYSCF_API int TinySCF_set_graph(TinySCF_t t, int on);
/* Initial guess. TINYSCF_GUESS_SAD (default): the reference's superposition
 * of atomic densities with its pivoted-Cholesky Cocc (TinySCF.c:282-364).
 * TINYSCF_GUESS_LEARNED: atom-pair density blocks predicted by the MLPs in the
 * weights file (block types: diagonal H / C,N,O; off-diagonal pairs closer
 * than 4 A), assembled and projected onto the idempotent density of the n_occ
 * leading natural orbitals; molecules with other elements or shell layouts
 * fall back to SAD. weights may be NULL to keep a loaded network. Takes effect
 * at the next TinySCF_get_initial_guess / TinySCF_reset_scf. */
#define TINYSCF_GUESS_SAD     0
#define TINYSCF_GUESS_LEARNED 1
/* The SAD density put through the same projection as the learned one (the
 * ablation that isolates what the network adds). */
#define TINYSCF_GUESS_SAD_PROJECTED 2
TINYSCF_API int TinySCF_set_guess(TinySCF_t t, int mode, const char *weights);
/* Which guess the last TinySCF_get_initial_guess used (or -status). */
TINYSCF_API int TinySCF_guess_used(TinySCF_t t);
/* Training data from a density D (host, nbf x nbf, e.g. a converged one):
 * for every atom pair of the molecule its 128 features, its target block in
 * the pair's local frame (225 floats, row-major nf_a x nf_b) and its block
 * type. With feat == NULL returns the number of pairs; else fills up to cap
 * pairs and returns the count (negative status on error). */
TINYSCF_API long long TinySCF_guess_dataset(TinySCF_t t, const double *D, float *feat, float *target, int *type,
                                            long long cap);
/* The learned guess's atom-pair blocks for a molecule (no GPU needed):
 * natoms atoms with 0-based element indices elem (H = 0, C = 5, N = 6, O = 7),
 * Bohr coordinates xyz (natoms x 3) and, per atom, nshell[a] shell angular
 * momenta in basis order in shell_am (all atoms' lists concatenated). For
 * block k < cap writes ab[2k], ab[2k+1] (its atoms, the one with more
 * functions first; equal atoms for a diagonal block), type[k] (0-4),
 * frame[9k..9k+8] (3 x 3 row-major, rows the local axes e_x, e_y, e_z) and
 * feat[128k..128k+127] (the invariant features the networks read); any of
 * the four may be NULL, all four NULL returns the count alone. Returns the
 * number of blocks, -TINYSCF_ERR_UNSUPPORTED when an element or shell layout
 * is not covered, -TINYSCF_ERR_INPUT when cap is too small. */
TINYSCF_API long long TinySCF_guess_pairs(int natoms, const int *elem, const double *xyz, const int *nshell,
                                          const int *shell_am, int *ab, int *type, double *frame, float *feat,
                                          long long cap);
/* The basis rotation the learned guess uses for one atom (no GPU needed):
 * with molecule coordinates x_m = Q^T x_l (Q: 3 x 3 row-major, rows the local
 * axes), writes M (nf x nf row-major, nf = sum of Cartesian components of the
 * shells, s/p/d only) such that the atom's functions obey phi_m = M phi_l. */
TINYSCF_API int TinySCF_guess_rotation(const int *shell_am, int nshells, const double *Q, double *M);
/* Train the five block-type MLPs (128-192-192-out, SiLU) with Adam on the GPU
 * from host arrays as TinySCF_guess_dataset writes them and save the weights
 * file at path; final_loss (5 floats) receives each type's last-epoch MSE in
 * normalised units. */
TINYSCF_API int TinySCF_guess_train(const float *feat, const float *target, const int *type, long long n, int epochs,
                                    int batch, float lr, unsigned seed, const char *path, float *final_loss);
/* Mean-squared-error loss and its gradient for one MLP (parameters laid out
 * W1[din][hid], b1, W2[hid][hid], b2, W3[hid][dout], b3) on n rows, computed
 * by the training kernels: host in, host out. */
TINYSCF_API int TinySCF_guess_mlp_grad(int din, int hid, int dout, const float *params, const float *X, const float *T,
                                       int n, float *grad, float *loss);
/* Autotuner (on unless TINYSCF_AUTOTUNE=0): the first time a shape is met
 * outside a stream capture, the candidates for these knobs are timed on the
 * device and the fastest kept for the process (and saved to / loaded from the
 * file named by TINYSCF_TUNE_FILE): the block size and thread order of each
 * 3-centre integral AM class, the tile shape of each FP64 GEMM shape
 * (FFMA 64x64, 32x32, 128x64, or 128x128 / 64x64 / 32x32 with K split over
 * the warps on the FP64 tensor cores), the tile and split count of the FP64
 * exchange rank-k product, the exchange half-transform (FFMA 64x64 or 64x256,
 * DMMA 64x256, or DMMA 64x256 in persistent CTAs with a cp.async pipeline)
 * and the row blocks of the J first pass.
 * All candidates compute the same values (the FP64 tensor-core tiles up to
 * rounding in the last bits). */
TINYSCF_API int TinySCF_set_autotune(int on);
/* Free and total device memory in bytes (cudaMemGetInfo) of a CUDA device,
 * for callers that size batches of molecules to what fits. Free includes the
 * memory that freed engines left in the engines' pool (below). */
TINYSCF_API int TinySCF_device_memory(int device, long long *free_bytes, long long *total_bytes);
/* The engines' large device buffers come from the device's stream-ordered
 * memory pool, which keeps memory reserved after an engine is freed so that
 * the next engine reuses it without new mappings (TINYSCF_MEMPOOL=0 in the
 * environment uses cudaMalloc / cudaFree instead). This returns the pool's
 * unused memory to the device. */
TINYSCF_API int TinySCF_trim_memory(int device);
/* The tuner's table as text ("key -> choice (ms) [candidate: ms]..."); writes
 * at most len bytes into buf and returns the full length. */
TINYSCF_API int TinySCF_autotune_report(char *buf, int len);
/* Batched SCF over many molecules of uneven size. Each molecule is a handle
 * set up through the single-molecule calls (up to TinySCF_build_DF_tensor,
 * any initial guess; FP64 exchange, or TINYSCF_K_MIXED: then its exchange is
 * the tensor-core incremental build, one molecule at a time, and one batched
 * FP64 Fock build on the converged densities gives its energy, as
 * TinySCF_do_SCF does). TinySCF_batch_do_SCF then iterates all of
 * them together: every SCF phase (J, K, Fock + energy, DIIS, density) is one
 * launch over all molecules still iterating; the density eigensolves run
 * molecule by molecule on the engine's eigensolver. Each molecule follows its own
 * reference loop (ene_tol, niters, iteration count, DIIS history) and ends
 * with its host mirrors filled as after TinySCF_do_SCF. The handles must stay
 * alive until TinySCF_batch_free (which frees only the batch). */
typedef struct TinySCF_batch_struct *TinySCF_batch_t;
TINYSCF_API int TinySCF_batch_create(TinySCF_batch_t *out, TinySCF_t *mols, int nmol);
TINYSCF_API int TinySCF_batch_do_SCF(TinySCF_batch_t b);
/* Device time of the last TinySCF_batch_do_SCF (ms), its number of batched
 * iterations (the slowest molecule's count) and the kernels it launched
 * outside the per-molecule eigensolves. */
TINYSCF_API int TinySCF_batch_stats(TinySCF_batch_t b, double *scf_ms, int *iterations, long long *launches);
/* Device time (ms) of the last TinySCF_batch_do_SCF by phase: [0] J,
 * [1] K, [2] Fock + energy, [3] DIIS, [4] density, [5] final FP64 Fock build
 * of the molecules set to TINYSCF_K_MIXED; min(n, 6) values. */
TINYSCF_API int TinySCF_batch_phase_ms(TinySCF_batch_t b, double *ms, int n);
TINYSCF_API int TinySCF_batch_free(TinySCF_batch_t b);
/* Aux-partitioned Fock builds: one molecule over several GPUs, one process
 * and handle per GPU (no counterpart in the reference, which runs on one
 * node's cores). Called before TinySCF_build_DF_tensor, TinySCF_set_aux_slice
 * makes the handle build and hold only the DF tensor's aux columns [p0, p1)
 * (B = pqA (P|Q)^-1/2 restricted to those columns); TinySCF_build_FockMat then
 * gives the slice's partial J and K, whose sums over a partition of
 * [0, naux) are the full J and K (both are sums over the aux index).
 * TinySCF_set_JK takes the summed J and K (host, nbf x nbf) and recomputes F
 * and the energy as TinySCF_build_FockMat does; TinySCF_DIIS and
 * TinySCF_build_DenMat follow unchanged. TinySCF_do_SCF refuses a sliced
 * handle: the caller runs the loop with one reduction of [J | K] per
 * iteration (yatscf-df_b200/auxsplit.py does, over torch.distributed). */
TINYSCF_API int TinySCF_set_aux_slice(TinySCF_t t, int p0, int p1);
TINYSCF_API int TinySCF_set_JK(TinySCF_t t, const double *J, const double *K);
/* Checks the tensor-core exchange kernels' bounded waits (no counterpart in
 * the reference, which has no device code): runs one CTA of the G GEMM kernel
 * of a handle set to TINYSCF_K_MIXED with no copies issued, so that its MMA
 * and epilogue waits, limited to wait_cycles clock cycles, run out with
 * nothing in flight; the kernel records the wait's code, frees its tensor
 * memory and returns. *code receives that code (0 if no wait gave up); the
 * flag is cleared afterwards and the handle stays usable. */
TINYSCF_API int TinySCF_kmix_wait_probe(TinySCF_t t, long long wait_cycles, int *code);
/* The engine's FP64 symmetric eigensolver on host buffers: A (n x n,
 * row-major, symmetric) -> w (n eigenvalues, ascending) and V (n x n, row k =
 * eigenvector k). It is what replaces the reference's LAPACKE_dsyev calls
 * (TinySCF.c:65 for X = S^-1/2, build_DF_tensor.c:217 for (P|Q)^-1/2,
 * build_density.c:54 for the Fock eigensolve): Householder
 * tridiagonalisation, divide and conquer, back-transformation, all as this
 * library's kernels. n <= 8192. Allocates and frees its own workspace on the
 * device; synchronous. TINYSCF_ERR_CUDA if a grid barrier of the
 * tridiagonalisation gave up waiting. */
TINYSCF_API int TinySCF_eigh(int device, int n, const double *A, double *w, double *V);
/* K = T T^T (T: n x q, row-major; K: n x n, both triangles) on host buffers,
 * by the integer-tensor-core product the engine's FP64 exchange uses when
 * TINYSCF_OZAKI selects it (the rank-k step of build_Fock.c:317-341): each row
 * of T scaled by a power of two and rounded to a 49-bit integer, its residues
 * modulo 15 coprime moduli <= 256 multiplied as int8 with exact int32 sums,
 * the sums rebuilt by the Chinese remainder theorem and rounded once to FP64.
 * Allocates and frees its own workspace (about 15 n q bytes); synchronous. */
TINYSCF_API int TinySCF_syrk_int8(int device, int n, long long q, const double *T, double *K);
/* Back to the state right after TinySCF_get_initial_guess (SAD density, its
 * factor, empty DIIS history), keeping integrals and the DF tensor. */
TINYSCF_API int TinySCF_reset_scf(TinySCF_t t);

#ifdef __cplusplus
}
#endif

#endif
