/*
 * ORACLE — test infrastructure only.
 *
 * Bulk integral loops of the reference, restated in C over the oracle engine
 * (ints.c) so the numpy restatement (oracle.py) does not loop over millions of
 * shell triplets in Python. Each function follows the reference loop it names.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "ints.h"

typedef struct
{
    int nsh;
    const int *am, *nprim, *off;   /* per shell; off indexes alpha/coef      */
    const double *cen;             /* 3 * nsh, Bohr                          */
    const double *alpha, *coef;    /* coef already normalised                */
} ob_basis;

static oi_shell get_shell(const ob_basis *b, int i)
{
    oi_shell s;
    s.am = b->am[i]; s.nprim = b->nprim[i];
    s.x = b->cen[3 * i]; s.y = b->cen[3 * i + 1]; s.z = b->cen[3 * i + 2];
    s.alpha = b->alpha + b->off[i]; s.coef = b->coef + b->off[i];
    return s;
}

static void bf_offsets(const ob_basis *b, int *sind)
{
    sind[0] = 0;
    for (int i = 0; i < b->nsh; i++) sind[i + 1] = sind[i] + oi_ncart(b->am[i]);
}

static const double unit_alpha = 0.0, unit_coef = 1.0;
static oi_shell unit_shell(void)
{
    oi_shell s;
    s.am = 0; s.nprim = 1; s.x = s.y = s.z = 0.0;
    s.alpha = &unit_alpha; s.coef = &unit_coef;
    return s;
}

/* S and Hcore = T + V over all shell pairs (TinySCF.c:20-56). */
void ob_one_electron(const ob_basis *b, int natoms, const double *Z, const double *xyz,
                     double *S, double *H)
{
    int *sind = (int *) malloc(sizeof(int) * (b->nsh + 1));
    bf_offsets(b, sind);
    int nbf = sind[b->nsh];
    #pragma omp parallel for schedule(dynamic)
    for (int M = 0; M < b->nsh; M++)
    {
        double buf[28 * 28], tbuf[28 * 28];
        oi_shell A = get_shell(b, M);
        for (int N = 0; N < b->nsh; N++)
        {
            oi_shell B = get_shell(b, N);
            int nA = oi_ncart(A.am), nB = oi_ncart(B.am);
            oi_overlap(&A, &B, buf);
            for (int i = 0; i < nA; i++)
                for (int j = 0; j < nB; j++) S[(size_t) (sind[M] + i) * nbf + sind[N] + j] = buf[i * nB + j];
            oi_kinetic(&A, &B, tbuf);
            oi_potential(&A, &B, natoms, Z, xyz, buf);
            for (int i = 0; i < nA; i++)
                for (int j = 0; j < nB; j++)
                    H[(size_t) (sind[M] + i) * nbf + sind[N] + j] = buf[i * nB + j] + tbuf[i * nB + j];
        }
    }
    free(sind);
}

/* Schwarz values (TinySCF.c:128-165). The reference reads the quartet block
 * at iN*(dM*dN*dM+dM) + iM*(dN*dM+1) (TinySCF.c:153), which is the (mn|mn)
 * diagonal only when dM == dN or one of them is 1; quirk != 0 reproduces that
 * index, quirk == 0 reads the true diagonal. */
void ob_schwarz(const ob_basis *b, int quirk, double *sp_scrval, double *bf_scrval)
{
    int *sind = (int *) malloc(sizeof(int) * (b->nsh + 1));
    bf_offsets(b, sind);
    int nbf = sind[b->nsh];
    #pragma omp parallel for schedule(dynamic)
    for (int M = 0; M < b->nsh; M++)
    {
        double *buf = (double *) malloc(sizeof(double) * 28 * 28 * 28 * 28);
        oi_shell A = get_shell(b, M);
        int dM = oi_ncart(A.am);
        for (int N = 0; N < b->nsh; N++)
        {
            oi_shell B = get_shell(b, N);
            int dN = oi_ncart(B.am);
            oi_eri(&A, &B, &A, &B, buf);
            double mx = 0.0;
            for (int iM = 0; iM < dM; iM++)
                for (int iN = 0; iN < dN; iN++)
                {
                    int idx = quirk ? iN * (dM * dN * dM + dM) + iM * (dN * dM + 1)
                                    : iM * (dN * dM * dN + dN) + iN * (dM * dN + 1);
                    double v = fabs(buf[idx]);
                    bf_scrval[(size_t) (sind[M] + iM) * nbf + sind[N] + iN] = v;
                    if (v > mx) mx = v;
                }
            sp_scrval[M * b->nsh + N] = mx;
        }
        free(buf);
    }
    free(sind);
}

/* max_p (p|p) per aux shell: the DF screening value of the oracle's
 * CMS_Simint_getDFShellpairScreenVal. */
void ob_df_scrval(const ob_basis *aux, double *out)
{
    oi_shell U = unit_shell();
    for (int i = 0; i < aux->nsh; i++)
    {
        oi_shell P = get_shell(aux, i);
        int n = oi_ncart(P.am);
        double buf[28 * 28];
        oi_eri(&P, &U, &P, &U, buf);
        double mx = 0.0;
        for (int k = 0; k < n; k++) if (fabs(buf[k * n + k]) > mx) mx = fabs(buf[k * n + k]);
        out[i] = mx;
    }
}

/* 3-centre integrals scattered into pqA rows (ij) and (ji)
 * (build_DF_tensor.c:14-47, 49-150). Triplets with
 * sp_scrval(M,N) * df_scrval(P) < scrtol2 are skipped (:100) and stay zero;
 * rows of screened bf pairs (mask -1) are dropped — the reference writes them
 * out of bounds. */
void ob_3center(const ob_basis *b, const ob_basis *aux, const int *uniq_l, const int *uniq_r, int nuniq,
                const double *sp_scrval, const double *df_scrval, double scrtol2,
                const int *mask, double *pqA)
{
    int *sind = (int *) malloc(sizeof(int) * (b->nsh + 1));
    int *asind = (int *) malloc(sizeof(int) * (aux->nsh + 1));
    bf_offsets(b, sind); bf_offsets(aux, asind);
    int nbf = sind[b->nsh], naux = asind[aux->nsh];
    oi_shell U = unit_shell();
    #pragma omp parallel for schedule(dynamic)
    for (int iMN = 0; iMN < nuniq; iMN++)
    {
        double buf[6 * 6 * 28];
        int M = uniq_l[iMN], N = uniq_r[iMN];
        oi_shell A = get_shell(b, M), B = get_shell(b, N);
        int dM = oi_ncart(A.am), dN = oi_ncart(B.am);
        double scr0 = sp_scrval[M * b->nsh + N];
        for (int P = 0; P < aux->nsh; P++)
        {
            if (scr0 * df_scrval[P] < scrtol2) continue;
            oi_shell C = get_shell(aux, P);
            int dP = oi_ncart(C.am);
            oi_eri(&A, &B, &C, &U, buf);
            for (int im = 0; im < dM; im++)
                for (int in = 0; in < dN; in++)
                {
                    int iM = sind[M] + im, iN = sind[N] + in;
                    int r0 = mask[iM * nbf + iN], r1 = mask[iN * nbf + iM];
                    const double *src = buf + (im * dN + in) * dP;
                    if (r0 >= 0) memcpy(pqA + (size_t) r0 * naux + asind[P], src, sizeof(double) * dP);
                    if (r1 >= 0) memcpy(pqA + (size_t) r1 * naux + asind[P], src, sizeof(double) * dP);
                }
        }
    }
    free(sind); free(asind);
}

/* (P|Q) for screened upper shell pairs, mirrored (build_DF_tensor.c:152-203). */
void ob_2center(const ob_basis *aux, const double *df_scrval, double scrtol2, double *Jpq)
{
    int *asind = (int *) malloc(sizeof(int) * (aux->nsh + 1));
    bf_offsets(aux, asind);
    int naux = asind[aux->nsh];
    oi_shell U = unit_shell();
    #pragma omp parallel for schedule(dynamic)
    for (int M = 0; M < aux->nsh; M++)
    {
        double buf[28 * 28];
        oi_shell A = get_shell(aux, M);
        int dM = oi_ncart(A.am);
        for (int N = M; N < aux->nsh; N++)
        {
            if (df_scrval[M] * df_scrval[N] < scrtol2) continue;
            oi_shell B = get_shell(aux, N);
            int dN = oi_ncart(B.am);
            oi_eri(&A, &U, &B, &U, buf);
            for (int i = 0; i < dM; i++)
                for (int j = 0; j < dN; j++)
                {
                    double v = buf[i * dN + j];
                    Jpq[(size_t) (asind[M] + i) * naux + asind[N] + j] = v;
                    Jpq[(size_t) (asind[N] + j) * naux + asind[M] + i] = v;
                }
        }
    }
    free(asind);
}
