/*
 * ORACLE — test infrastructure only.
 *
 * Implements the libCMS Simint middleware API (libCMS/CMS_Simint.h:61-112)
 * on top of the oracle's McMurchie–Davidson engine (ints.c), so the
 * reference's own SCF sources compile and run unchanged without the
 * un-vendored Simint library. Only the entry points the reference's hot path
 * calls are provided:
 *
 *   CMS_createSimint / CMS_destroySimint          CMS_Simint.c:36-239, 241-306
 *   CMS_computeShellQuartet_Simint                CMS_Simint.c:338-399
 *   CMS_computePairOvl_Simint                     CMS_Simint.c:403-421
 *   CMS_computePairCoreH_Simint                   CMS_Simint.c:425-461
 *   CMS_Simint_getShellpairAMIndex                CMS_Simint.c:308-312
 *   CMS_Simint_{create,free}ThreadMultishellpair  CMS_Simint.c:314-334
 *   CMS_Simint_resetStatisInfo                    CMS_Simint.c:463-472
 *   CMS_Simint_computeDFShellQuartetBatch         CMS_Simint.c:499-566
 *   CMS_Simint_computeDFShellPair                 CMS_Simint.c:570-630
 *   CMS_Simint_getDFShellpairScreenVal            CMS_Simint.c:632-637
 *
 * Differences from Simint, by design:
 *   - no primitive screening: every quartet is computed (Simint drops
 *     primitive quartets below 1e-14, CMS_Simint.c:147-148), so nints is never 0;
 *   - the DF screening value of aux shell P is max_p (p|p) over its Cartesian
 *     components, with the unit shell on both sides — the quantity the
 *     reference multiplies with max (mn|mn) and compares against 1e-22
 *     (build_DF_tensor.c:100, TinySCF.c:183).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#include "CMS.h"
#include "ints.h"

/* Simint's shell type is opaque to the reference (pointer members only). */
struct simint_shell
{
    oi_shell sh;
    double *alpha, *coef;
};

static void make_shell(struct simint_shell *s, int am, int nprim, double x, double y, double z,
                       const double *alpha, const double *cc, int normalize)
{
    s->alpha = (double *) malloc(sizeof(double) * nprim);
    s->coef  = (double *) malloc(sizeof(double) * nprim);
    memcpy(s->alpha, alpha, sizeof(double) * nprim);
    if (normalize) oi_normalize(am, nprim, alpha, cc, s->coef);
    else memcpy(s->coef, cc, sizeof(double) * nprim);
    s->sh.am = am; s->sh.nprim = nprim;
    s->sh.x = x; s->sh.y = y; s->sh.z = z;
    s->sh.alpha = s->alpha; s->sh.coef = s->coef;
}

CMSStatus_t CMS_createSimint(BasisSet_t basis, BasisSet_t df_basis, Simint_t *simint, int nthreads)
{
    CMS_ASSERT(nthreads > 0);
    Simint_t s = (Simint_t) calloc(1, sizeof(struct Simint));
    CMS_ASSERT(s != NULL);

    s->nthreads  = nthreads;
    s->max_am    = basis->max_momentum;
    s->df_max_am = df_basis->max_momentum;
    if (s->df_max_am > s->max_am) s->max_am = s->df_max_am;

    int max_ncart = (s->max_am + 1) * (s->max_am + 2) / 2;
    int maxsize = max_ncart * max_ncart * max_ncart * max_ncart;
    maxsize = (maxsize + 7) / 8 * 8;
    s->outmem_per_thread = maxsize * _Simint_NSHELL_SIMD + 8;
    s->outbuf = (double *) malloc(sizeof(double) * (size_t) s->outmem_per_thread * nthreads);
    CMS_ASSERT(s->outbuf != NULL);

    s->nshells = basis->nshells;
    s->shells = (struct simint_shell *) calloc(basis->nshells, sizeof(struct simint_shell));
    for (int i = 0; i < (int) basis->nshells; i++)
        make_shell(&s->shells[i], basis->momentum[i], basis->nexp[i],
                   basis->xyz0[i * 4 + 0], basis->xyz0[i * 4 + 1], basis->xyz0[i * 4 + 2],
                   basis->exp[i], basis->cc[i], 1);

    /* The last DF shell is the unit shell (CMS_Simint.c:131-141). */
    s->df_nshells = df_basis->nshells;
    s->df_shells = (struct simint_shell *) calloc(df_basis->nshells + 1, sizeof(struct simint_shell));
    for (int i = 0; i < (int) df_basis->nshells; i++)
        make_shell(&s->df_shells[i], df_basis->momentum[i], df_basis->nexp[i],
                   df_basis->xyz0[i * 4 + 0], df_basis->xyz0[i * 4 + 1], df_basis->xyz0[i * 4 + 2],
                   df_basis->exp[i], df_basis->cc[i], 1);
    {
        double a0 = 0.0, c1 = 1.0;
        make_shell(&s->df_shells[df_basis->nshells], 0, 1, 0.0, 0.0, 0.0, &a0, &c1, 0);
    }
    printf("Simint screen method    = none (oracle McMurchie-Davidson engine)\n");

    /* Group DF shells by angular momentum (CMS_Simint.c:184-204). */
    s->df_am_shell_id   = (int *) malloc(sizeof(int) * s->df_nshells);
    s->df_am_shell_spos = (int *) calloc(s->df_max_am + 2, sizeof(int));
    s->df_am_shell_num  = (int *) calloc(s->df_max_am + 1, sizeof(int));
    for (int i = 0; i < s->df_nshells; i++) s->df_am_shell_num[s->df_shells[i].sh.am]++;
    for (int i = 1; i <= s->df_max_am + 1; i++)
        s->df_am_shell_spos[i] = s->df_am_shell_spos[i - 1] + s->df_am_shell_num[i - 1];
    memset(s->df_am_shell_num, 0, sizeof(int) * (s->df_max_am + 1));
    for (int i = 0; i < s->df_nshells; i++)
    {
        int am = s->df_shells[i].sh.am;
        s->df_am_shell_id[s->df_am_shell_spos[am] + s->df_am_shell_num[am]] = i;
        s->df_am_shell_num[am]++;
    }

    /* The screening value of each aux shell, stored in the otherwise unused
     * workbuf pointer slot. */
    double *df_scr = (double *) malloc(sizeof(double) * (s->df_nshells > 0 ? s->df_nshells : 1));
    const oi_shell *unit = &s->df_shells[s->df_nshells].sh;
    for (int i = 0; i < s->df_nshells; i++)
    {
        const oi_shell *P = &s->df_shells[i].sh;
        int n = oi_ncart(P->am);
        double *buf = (double *) malloc(sizeof(double) * n * n);
        oi_eri(P, unit, P, unit, buf);
        double mx = 0.0;
        for (int k = 0; k < n; k++) if (fabs(buf[k * n + k]) > mx) mx = fabs(buf[k * n + k]);
        df_scr[i] = mx;
        free(buf);
    }
    s->workbuf = df_scr;

    int stat_info_size = sizeof(double) * nthreads;
    s->num_multi_shellpairs = (double *) calloc(1, stat_info_size);
    s->sum_nprim            = (double *) calloc(1, stat_info_size);
    s->num_screened_prim    = (double *) calloc(1, stat_info_size);
    s->num_unscreened_prim  = (double *) calloc(1, stat_info_size);
    s->num_screened_vec     = (double *) calloc(1, stat_info_size);
    s->num_unscreened_vec   = (double *) calloc(1, stat_info_size);

    *simint = s;
    return CMS_STATUS_SUCCESS;
}

CMSStatus_t CMS_destroySimint(Simint_t s, int show_stat)
{
    (void) show_stat;
    for (int i = 0; i < s->nshells; i++) { free(s->shells[i].alpha); free(s->shells[i].coef); }
    for (int i = 0; i <= s->df_nshells; i++) { free(s->df_shells[i].alpha); free(s->df_shells[i].coef); }
    free(s->shells); free(s->df_shells);
    free(s->df_am_shell_id); free(s->df_am_shell_spos); free(s->df_am_shell_num);
    free(s->workbuf); free(s->outbuf);
    free(s->num_multi_shellpairs); free(s->sum_nprim);
    free(s->num_screened_prim); free(s->num_unscreened_prim);
    free(s->num_screened_vec); free(s->num_unscreened_vec);
    free(s);
    return CMS_STATUS_SUCCESS;
}

int CMS_Simint_getShellpairAMIndex(Simint_t simint, int P, int Q)
{
    return simint->shells[P].sh.am * ((_Simint_OSTEI_MAXAM) + 1) + simint->shells[Q].sh.am;
}

void CMS_Simint_createThreadMultishellpair(void **thread_multi_shellpair)
{
    *thread_multi_shellpair = malloc(8);
}

void CMS_Simint_freeThreadMultishellpair(void **thread_multi_shellpair)
{
    free(*thread_multi_shellpair);
}

void CMS_Simint_resetStatisInfo(Simint_t simint)
{
    (void) simint;
}

static double *thread_out(Simint_t s, int tid)
{
    return s->outbuf + (size_t) tid * s->outmem_per_thread;
}

CMSStatus_t CMS_computeShellQuartet_Simint(Simint_t simint, int tid, int A, int B, int C, int D,
                                           double **integrals, int *nints)
{
    double *out = thread_out(simint, tid);
    const struct simint_shell *sh = simint->shells;
    oi_eri(&sh[A].sh, &sh[B].sh, &sh[C].sh, &sh[D].sh, out);
    *integrals = out;
    *nints = oi_ncart(sh[A].sh.am) * oi_ncart(sh[B].sh.am) * oi_ncart(sh[C].sh.am) * oi_ncart(sh[D].sh.am);
    return CMS_STATUS_SUCCESS;
}

CMSStatus_t CMS_computePairOvl_Simint(BasisSet_t basis, Simint_t simint, int tid,
                                      int A, int B, double **integrals, int *nints)
{
    (void) basis;
    double *out = thread_out(simint, tid);
    oi_overlap(&simint->shells[A].sh, &simint->shells[B].sh, out);
    *integrals = out;
    *nints = oi_ncart(simint->shells[A].sh.am) * oi_ncart(simint->shells[B].sh.am);
    return CMS_STATUS_SUCCESS;
}

CMSStatus_t CMS_computePairCoreH_Simint(BasisSet_t basis, Simint_t simint, int tid,
                                        int A, int B, double **integrals, int *nints)
{
    double *out = thread_out(simint, tid);
    int n = oi_ncart(simint->shells[A].sh.am) * oi_ncart(simint->shells[B].sh.am);
    double *tmp = (double *) malloc(sizeof(double) * n);
    double *xyz = (double *) malloc(sizeof(double) * 3 * basis->natoms);
    for (int i = 0; i < basis->natoms; i++)
    {
        xyz[3 * i] = basis->xn[i]; xyz[3 * i + 1] = basis->yn[i]; xyz[3 * i + 2] = basis->zn[i];
    }
    oi_kinetic(&simint->shells[A].sh, &simint->shells[B].sh, tmp);
    oi_potential(&simint->shells[A].sh, &simint->shells[B].sh, basis->natoms, basis->charge, xyz, out);
    for (int i = 0; i < n; i++) out[i] += tmp[i];
    free(tmp); free(xyz);
    *integrals = out;
    *nints = n;
    return CMS_STATUS_SUCCESS;
}

CMSStatus_t CMS_Simint_computeDFShellQuartetBatch(Simint_t simint, int tid, int M, int N, int *P_list, int npairs,
                                                  double **thread_batch_integrals, int *thread_batch_nints,
                                                  void **thread_multi_shellpair)
{
    (void) thread_multi_shellpair;
    double *out = thread_out(simint, tid);
    const struct simint_shell *sh = simint->shells;
    const oi_shell *unit = &simint->df_shells[simint->df_nshells].sh;
    int size = oi_ncart(sh[M].sh.am) * oi_ncart(sh[N].sh.am) * oi_ncart(simint->df_shells[P_list[0]].sh.am);
    for (int i = 0; i < npairs; i++)
        oi_eri(&sh[M].sh, &sh[N].sh, &simint->df_shells[P_list[i]].sh, unit, out + (size_t) i * size);
    *thread_batch_integrals = out;
    *thread_batch_nints = size;
    return CMS_STATUS_SUCCESS;
}

CMSStatus_t CMS_Simint_computeDFShellPair(Simint_t simint, int tid, int M, int N,
                                          double **integrals, int *nints)
{
    double *out = thread_out(simint, tid);
    const oi_shell *unit = &simint->df_shells[simint->df_nshells].sh;
    oi_eri(&simint->df_shells[M].sh, unit, &simint->df_shells[N].sh, unit, out);
    *integrals = out;
    *nints = oi_ncart(simint->df_shells[M].sh.am) * oi_ncart(simint->df_shells[N].sh.am);
    return CMS_STATUS_SUCCESS;
}

double CMS_Simint_getDFShellpairScreenVal(Simint_t simint, int i)
{
    return simint->workbuf[i];
}
