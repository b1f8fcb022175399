/*
 * TinySCF C API of the B200 DF-RHF engine — drop-in for the reference's
 * TinySCF.h (huanghua1994/YATSCF-DF, TinySCF.h:1-140).
 *
 * Same entry points, same argument meaning, same call order as the
 * reference's main.c:28-46. The struct keeps the reference's public field
 * names (sizes, screening arrays, host matrices, SCF state); MKL and Simint
 * types are gone (TinySCF.h:4-6,55,92-96) and device state lives behind the
 * opaque `dev` pointer. All matrices are row-major doubles, as in the
 * reference. Host matrices are mirrors of device buffers: they are filled by
 * every public call that produces them, and at the end of TinySCF_do_SCF.
 *
 * Error convention: like the reference, the void entry points report fatal
 * errors on stderr and abort(); every entry point also has a *_status twin
 * (tinyscf_b200.h) that returns a status code instead and leaves the process
 * running.
 */
#ifndef TINYSCF_B200_TINYSCF_H
#define TINYSCF_B200_TINYSCF_H

#ifdef __cplusplus
extern "C" {
#endif

/* Symbols exported by libtinyscf_b200.so (it is built with hidden visibility). */
#ifndef TINYSCF_API
#define TINYSCF_API __attribute__((visibility("default")))
#endif

#define MAX_DIIS 10     /* TinySCF.h:8 */
#define MIN_DIIS 2      /* TinySCF.h:9 (unused, as in the reference) */

struct TinySCF_struct
{
    /* Chemical system info (TinySCF.h:19-25) */
    void *basis, *df_basis;     /* opaque parsed basis sets                          */
    int natoms, nshells;
    int nbasfuncs, n_occ;
    int charge, electron;
    int df_nbf, df_nshells;

    /* Auxiliary variables (TinySCF.h:28-31) */
    int nshellpairs;            /* nshells * nshells                                 */
    int num_uniq_sp;            /* unique shell pairs surviving screening            */
    int mat_size;               /* nbasfuncs * nbasfuncs                             */
    int max_dim;

    /* SCF iteration info (TinySCF.h:34-37) */
    int niters, iter;
    double nuc_energy;
    double HF_energy;           /* electronic energy; total = HF_energy + nuc_energy */
    double ene_tol;             /* 1e-11, TinySCF_init_free.c:75                     */

    /* Screening (TinySCF.h:40-53) */
    double shell_scrtol2;       /* 1e-22, TinySCF_init_free.c:78                     */
    double max_scrval;
    double max_df_scrval;
    double *sp_scrval;          /* [nshells*nshells]                                 */
    double *bf_pair_scrval;     /* [nbf*nbf]                                         */
    int    *uniq_sp_lid;
    int    *uniq_sp_rid;
    double *df_sp_scrval;       /* [df_nshells]                                      */
    int    *bf_pair_mask;       /* [nbf*nbf], CSR position or -1                     */
    int    *bf_pair_j;          /* [nnz]                                             */
    int    *bf_pair_diag;       /* [nbf]                                             */
    int    *bf_mask_displs;     /* [nbf+1]                                           */
    int    num_bf_pair_scr;     /* nnz                                               */

    /* Shell -> basis function maps (TinySCF.h:57-60) */
    int *shell_bf_sind, *shell_bf_num;
    int *df_shell_bf_sind, *df_shell_bf_num;

    /* Host mirrors of the SCF matrices (TinySCF.h:63-73) */
    double *Hcore_mat, *S_mat, *F_mat, *D_mat, *J_mat, *K_mat, *X_mat;
    double *Cocc_mat;           /* [nbf*n_occ]                                       */
    double *eigval;             /* [nbf]                                             */
    int    *ev_idx;             /* [nbf]                                             */
    double *tmp_mat;

    /* DIIS bookkeeping (TinySCF.h:86-88), mirrored from the device */
    int    DIIS_len, DIIS_bmax_id;
    double DIIS_bmax;
    int    max_diis;            /* DIIS depth, 1..MAX_DIIS (default MAX_DIIS)        */

    /* Statistics (TinySCF.h:99) */
    double mem_size, init_time, S_Hcore_time, shell_scr_time;

    /* B200 engine state */
    int   status;               /* last status code, 0 = success                     */
    int   device;               /* CUDA device ordinal                               */
    int   verbose;              /* 0 = silent, 1 = the reference's stdout lines      */
    void *dev;                  /* opaque device state                               */
};

typedef struct TinySCF_struct* TinySCF_t;

/* TinySCF.h:107-110 / TinySCF_init_free.c:14-208 */
TINYSCF_API void init_TinySCF(TinySCF_t TinySCF, char *bas_fname, char *df_bas_fname, char *xyz_fname, const int niters);

/* TinySCF.h:112-113 / TinySCF_init_free.c:211-268: frees all buffers AND the struct */
TINYSCF_API void free_TinySCF(TinySCF_t TinySCF);

/* TinySCF.h:115-120 / TinySCF_init_free.c:270-342: no MKL batch arrays on the
 * device path; kept so main.c's call sequence compiles and runs unchanged. */
TINYSCF_API void TinySCF_init_batch_dgemm_arrays(TinySCF_t TinySCF);
TINYSCF_API void TinySCF_free_batch_dgemm_arrays(TinySCF_t TinySCF);

/* TinySCF.h:122-125 / TinySCF.c:20-83 */
TINYSCF_API void TinySCF_compute_Hcore_Ovlp_mat(TinySCF_t TinySCF);

/* TinySCF.h:127-129 / TinySCF.c:112-226 */
TINYSCF_API void TinySCF_compute_sq_Schwarz_scrvals(TinySCF_t TinySCF);

/* TinySCF.h:131-132 / TinySCF.c:228-280 */
TINYSCF_API void TinySCF_prepare_sparsity(TinySCF_t TinySCF);

/* TinySCF.h:134-135 / TinySCF.c:324-364 (and TinySCF_D2Cocc, :282-322) */
TINYSCF_API void TinySCF_get_initial_guess(TinySCF_t TinySCF);

/* TinySCF.h:137-138 / TinySCF.c:378-435 */
TINYSCF_API void TinySCF_do_SCF(TinySCF_t TinySCF);

#ifdef __cplusplus
}
#endif

#endif
