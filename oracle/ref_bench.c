/*
 * ORACLE — test infrastructure only (the CPU baseline of bench.py).
 *
 * Times the reference's own CPU implementation through its API, in the order
 * of main.c:28-46: setup once, then <nsolves> SCF solves from the SAD guess,
 * each converged to |dE| < ene_tol (TinySCF.c:386). Between solves the guess
 * and the DIIS history are restored as init_TinySCF leaves them
 * (TinySCF_init_free.c:174-184, TinySCF.c:324-364).
 *
 *   ref_bench <basis.gbs> <df_basis.gbs> <mol.xyz> <niters> <ene_tol> <nsolves>
 *
 * The reference's own stdout is kept; the summary goes to stderr:
 *   SETUP <s>   SOLVE <k> <iters> <energy> <s>
 */
#include <float.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "CMS.h"
#include "TinySCF.h"
#include "build_DF_tensor.h"
#include "utils.h"

int main(int argc, char **argv)
{
    if (argc < 7)
    {
        fprintf(stderr, "usage: %s <basis> <df_basis> <xyz> <niters> <ene_tol> <nsolves>\n", argv[0]);
        return 255;
    }
    double ene_tol = atof(argv[5]);
    int nsolves = atoi(argv[6]);
    double t0 = get_wtime_sec();
    TinySCF_t t = (TinySCF_t) malloc(sizeof(struct TinySCF_struct));
    init_TinySCF(t, argv[1], argv[2], argv[3], atoi(argv[4]));
    TinySCF_init_batch_dgemm_arrays(t);
    TinySCF_compute_Hcore_Ovlp_mat(t);
    TinySCF_compute_sq_Schwarz_scrvals(t);
    TinySCF_prepare_sparsity(t);
    TinySCF_get_initial_guess(t);
    TinySCF_build_DF_tensor(t);
    double t1 = get_wtime_sec();
    fprintf(stderr, "SETUP %.6f\n", t1 - t0);
    size_t msz = sizeof(double) * (size_t) t->mat_size;
    for (int k = 0; k < nsolves; k++)
    {
        if (k > 0)
        {
            TinySCF_get_initial_guess(t);
            memset(t->F0_mat, 0, msz * MAX_DIIS);
            memset(t->R_mat, 0, msz * MAX_DIIS);
            t->DIIS_len = 0;
            for (int i = 0; i < (MAX_DIIS + 1) * (MAX_DIIS + 1); i++) t->B_mat[i] = -1.0;
            for (int i = 0; i < (MAX_DIIS + 1); i++) t->B_mat[i * (MAX_DIIS + 1) + i] = 0.0;
            t->DIIS_bmax_id = 0;
            t->DIIS_bmax = -DBL_MAX;
        }
        t->ene_tol = ene_tol;
        double s0 = get_wtime_sec();
        TinySCF_do_SCF(t);
        double s1 = get_wtime_sec();
        fflush(stdout);
        fprintf(stderr, "SOLVE %d %d %.12f %.6f\n", k, t->iter, t->HF_energy + t->nuc_energy, s1 - s0);
    }
    TinySCF_free_batch_dgemm_arrays(t);
    free_TinySCF(t);
    return 0;
}
