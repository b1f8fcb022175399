/*
 * ORACLE — test infrastructure only.
 *
 * A driver for the reference's own SCF code (compiled unchanged from the
 * reference sources by oracle/Makefile). It calls the TinySCF API in the
 * order of main.c:28-46 and runs the loop of TinySCF_do_SCF
 * (TinySCF.c:378-435) itself so that it can dump every intermediate matrix:
 *
 *   ref_dump <basis.gbs> <df_basis.gbs> <mol.xyz> <niters> <outdir> [dump_df_tensor]
 *
 * Files written to <outdir> (little-endian binary, row-major):
 *   meta.txt                 sizes, nuclear energy, iteration count
 *   S.bin H.bin X.bin        nbf x nbf
 *   D0.bin Cocc0.bin         SAD guess and its (quirky) pivoted-Cholesky factor
 *   mask.i32 pairj.i32 displs.i32   bf-pair CSR (TinySCF.c:228-258)
 *   Jpq.bin                  (P|Q)^-1/2, naux x naux
 *   B.bin                    DF tensor nnz x naux (only with dump_df_tensor)
 *   it<k>_{J,K,F,Fo,D,Cocc}.bin and energies.txt per iteration
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#include "CMS.h"
#include "TinySCF.h"
#include "build_DF_tensor.h"
#include "build_Fock.h"
#include "build_density.h"
#include "DIIS.h"

static char outdir[4096];

static void dump(const char *name, const void *p, size_t bytes)
{
    char fn[4352];
    snprintf(fn, sizeof(fn), "%s/%s", outdir, name);
    FILE *f = fopen(fn, "wb");
    if (!f) { perror(fn); exit(2); }
    fwrite(p, 1, bytes, f);
    fclose(f);
}

int main(int argc, char **argv)
{
    if (argc < 6)
    {
        fprintf(stderr, "usage: %s <basis> <df_basis> <xyz> <niters> <outdir> [dump_df_tensor]\n", argv[0]);
        return 255;
    }
    snprintf(outdir, sizeof(outdir), "%s", argv[5]);
    int dumpB = (argc > 6) ? atoi(argv[6]) : 0;

    TinySCF_t t = (TinySCF_t) malloc(sizeof(struct TinySCF_struct));
    init_TinySCF(t, argv[1], argv[2], argv[3], atoi(argv[4]));
    TinySCF_init_batch_dgemm_arrays(t);
    TinySCF_compute_Hcore_Ovlp_mat(t);
    TinySCF_compute_sq_Schwarz_scrvals(t);
    TinySCF_prepare_sparsity(t);
    TinySCF_get_initial_guess(t);

    int nbf = t->nbasfuncs, naux = t->df_nbf, nocc = t->n_occ;
    size_t msz = sizeof(double) * nbf * nbf;
    int nnz = t->bf_mask_displs[nbf];
    dump("S.bin", t->S_mat, msz);
    dump("H.bin", t->Hcore_mat, msz);
    dump("X.bin", t->X_mat, msz);
    dump("D0.bin", t->D_mat, msz);
    dump("Cocc0.bin", t->Cocc_mat, sizeof(double) * nbf * nocc);
    dump("mask.i32", t->bf_pair_mask, sizeof(int) * nbf * nbf);
    dump("pairj.i32", t->bf_pair_j, sizeof(int) * nnz);
    dump("displs.i32", t->bf_mask_displs, sizeof(int) * (nbf + 1));

    TinySCF_build_DF_tensor(t);
    dump("Jpq.bin", t->Jpq, sizeof(double) * naux * naux);
    if (dumpB) dump("B.bin", t->df_tensor, sizeof(double) * (size_t) nnz * naux);

    /* The loop of TinySCF_do_SCF (TinySCF.c:378-435), with dumps. */
    char fn[256];
    char efn[4352];
    snprintf(efn, sizeof(efn), "%s/energies.txt", outdir);
    FILE *ef = fopen(efn, "w");
    t->iter = 0;
    double prev_energy = 0, energy_delta = 223;
    while ((t->iter < t->niters) && (energy_delta >= t->ene_tol))
    {
        TinySCF_build_FockMat(t);
        snprintf(fn, sizeof(fn), "it%d_J.bin", t->iter); dump(fn, t->J_mat, msz);
        snprintf(fn, sizeof(fn), "it%d_K.bin", t->iter); dump(fn, t->K_mat, msz);
        snprintf(fn, sizeof(fn), "it%d_F.bin", t->iter); dump(fn, t->F_mat, msz);
        double energy = 0.0;
        for (int i = 0; i < nbf * nbf; i++) energy += t->D_mat[i] * (t->F_mat[i] + t->Hcore_mat[i]);
        t->HF_energy = energy;
        energy_delta = fabs(t->HF_energy - prev_energy);
        prev_energy = t->HF_energy;
        TinySCF_DIIS(t);
        snprintf(fn, sizeof(fn), "it%d_Fo.bin", t->iter); dump(fn, t->F_mat, msz);
        TinySCF_build_DenMat(t);
        snprintf(fn, sizeof(fn), "it%d_D.bin", t->iter); dump(fn, t->D_mat, msz);
        snprintf(fn, sizeof(fn), "it%d_Cocc.bin", t->iter); dump(fn, t->Cocc_mat, sizeof(double) * nbf * nocc);
        fprintf(ef, "%d %.17g %.17g\n", t->iter, t->HF_energy + t->nuc_energy, t->HF_energy);
        if (t->iter == 0) energy_delta = 223;
        t->iter++;
    }
    fclose(ef);

    char mfn[4352];
    snprintf(mfn, sizeof(mfn), "%s/meta.txt", outdir);
    FILE *mf = fopen(mfn, "w");
    fprintf(mf, "nbf %d\nnaux %d\nnocc %d\nnnz %d\nnshells %d\nnum_uniq_sp %d\nniters %d\nnuc_energy %.17g\n",
            nbf, naux, nocc, nnz, t->nshells, t->num_uniq_sp, t->iter, t->nuc_energy);
    fclose(mf);

    TinySCF_free_batch_dgemm_arrays(t);
    free_TinySCF(t);
    return 0;
}
