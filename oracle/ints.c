/*
 * ORACLE — test infrastructure only (see ints.h). McMurchie–Davidson
 * Cartesian Gaussian integrals in plain C, written from the published method
 * (Helgaker, Jørgensen, Olsen, "Molecular Electronic-Structure Theory", ch. 9):
 * Hermite expansion coefficients E^{ij}_t, Hermite Coulomb integrals R^n_{tuv}
 * and the Boys function F_m(T).
 *
 * It stands in for the integrals the reference gets from Simint
 * (libCMS/CMS_Simint.c:363 4-centre, :411 overlap, :441 kinetic, :444 nuclear
 * attraction, :527 batched 3-centre, :595 2-centre).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "ints.h"

#define EMAX 7     /* i, j <= 6 (kinetic needs lb+2)     */
#define TMAX 13    /* t <= i + j                          */

int oi_ncart(int l) { return (l + 1) * (l + 2) / 2; }

static void cart_list(int l, int c[][3])
{
    int n = 0;
    for (int lx = l; lx >= 0; lx--)
        for (int ly = l - lx; ly >= 0; ly--)
        {
            c[n][0] = lx; c[n][1] = ly; c[n][2] = l - lx - ly;
            n++;
        }
}

/* Boys function: series for F_mmax (all terms positive, no cancellation),
 * downward recursion F_m = (2T F_{m+1} + e^-T) / (2m+1); asymptotic form
 * when e^-T is below double precision relative to F_m. */
void oi_boys(int mmax, double T, double *F)
{
    if (T < 100.0)
    {
        double term = 1.0 / (2 * mmax + 1), sum = term;
        for (int k = 1; k < 4000; k++)
        {
            term *= 2.0 * T / (2 * mmax + 2 * k + 1);
            sum  += term;
            if (term < 1e-18 * sum) break;
        }
        double eT = exp(-T);
        F[mmax] = eT * sum;
        for (int m = mmax - 1; m >= 0; m--)
            F[m] = (2.0 * T * F[m + 1] + eT) / (2 * m + 1);
    } else {
        double f = 0.5 * sqrt(M_PI / T);
        F[0] = f;
        for (int m = 1; m <= mmax; m++)
        {
            f *= (2 * m - 1) / (2.0 * T);
            F[m] = f;
        }
    }
}

static double dfact(int n)  /* n!! for n >= -1 */
{
    double r = 1.0;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}

void oi_normalize(int am, int nprim, const double *alpha, const double *coef_in, double *coef_out)
{
    double df = dfact(2 * am - 1);
    for (int k = 0; k < nprim; k++)
    {
        double a = alpha[k];
        coef_out[k] = coef_in[k] * pow(2.0 * a / M_PI, 0.75) * pow(4.0 * a, 0.5 * am) / sqrt(df);
    }
    double s = 0.0;
    for (int k = 0; k < nprim; k++)
        for (int l = 0; l < nprim; l++)
        {
            double p = alpha[k] + alpha[l];
            s += coef_out[k] * coef_out[l] * pow(M_PI / p, 1.5) * df / pow(2.0 * p, am);
        }
    double f = 1.0 / sqrt(s);
    for (int k = 0; k < nprim; k++) coef_out[k] *= f;
}

/* 1D Hermite expansion coefficients E[i][j][t], i <= la, j <= lb. */
static void make_E(int la, int lb, double p, double XPA, double XPB, double K,
                   double E[EMAX][EMAX][TMAX])
{
    double ip2 = 0.5 / p;
    for (int i = 0; i <= la; i++)
        for (int j = 0; j <= lb; j++)
            for (int t = 0; t <= i + j + 1 && t < TMAX; t++) E[i][j][t] = 0.0;
    E[0][0][0] = K;
    for (int i = 0; i < la; i++)
        for (int t = 0; t <= i + 1; t++)
        {
            double v = 0.0;
            if (t > 0)     v += ip2 * E[i][0][t - 1];
            if (t <= i)    v += XPA * E[i][0][t];
            if (t + 1 <= i) v += (t + 1) * E[i][0][t + 1];
            E[i + 1][0][t] = v;
        }
    for (int j = 0; j < lb; j++)
        for (int i = 0; i <= la; i++)
            for (int t = 0; t <= i + j + 1; t++)
            {
                double v = 0.0;
                if (t > 0)          v += ip2 * E[i][j][t - 1];
                if (t <= i + j)     v += XPB * E[i][j][t];
                if (t + 1 <= i + j) v += (t + 1) * E[i][j][t + 1];
                E[i][j + 1][t] = v;
            }
}

/* Per-thread scratch so the hot loops do not call malloc. */
static __thread double *tl_buf = NULL;
static __thread size_t  tl_cap = 0;
static double *scratch(size_t n)
{
    if (n > tl_cap)
    {
        free(tl_buf);
        tl_buf = (double *) malloc(n * sizeof(double));
        tl_cap = n;
    }
    return tl_buf;
}

/* Hermite Coulomb integrals R^n_{tuv}, n,t,u,v <= L, flat cube of side L+1. */
static void make_R(int L, double alpha, double X, double Y, double Z, double *R)
{
    const int D = L + 1;
#define RI(n, t, u, v) R[((((size_t) (n)) * D + (t)) * D + (u)) * D + (v)]
    double F[32];
    oi_boys(L, alpha * (X * X + Y * Y + Z * Z), F);
    double m2a = -2.0 * alpha, pw = 1.0;
    for (int n = 0; n <= L; n++)
    {
        RI(n, 0, 0, 0) = pw * F[n];
        pw *= m2a;
    }
    for (int n = L - 1; n >= 0; n--)
    {
        int M = L - n;
        for (int t = 0; t <= M; t++)
            for (int u = 0; u <= M - t; u++)
                for (int v = 0; v <= M - t - u; v++)
                {
                    if (t + u + v == 0) continue;
                    double val;
                    if (t > 0)
                    {
                        val = X * RI(n + 1, t - 1, u, v);
                        if (t > 1) val += (t - 1) * RI(n + 1, t - 2, u, v);
                    } else if (u > 0) {
                        val = Y * RI(n + 1, t, u - 1, v);
                        if (u > 1) val += (u - 1) * RI(n + 1, t, u - 2, v);
                    } else {
                        val = Z * RI(n + 1, t, u, v - 1);
                        if (v > 1) val += (v - 1) * RI(n + 1, t, u, v - 2);
                    }
                    RI(n, t, u, v) = val;
                }
    }
}

typedef struct
{
    double p, P[3];
    double E[3][EMAX][EMAX][TMAX];
} prim_pair;

static void make_pair(const oi_shell *A, int ka, const oi_shell *B, int kb, int extra_b, prim_pair *pp)
{
    double a = A->alpha[ka], b = B->alpha[kb];
    double p = a + b, mu = (p > 0.0) ? a * b / p : 0.0;
    double Ac[3] = {A->x, A->y, A->z}, Bc[3] = {B->x, B->y, B->z};
    pp->p = p;
    for (int d = 0; d < 3; d++)
    {
        double Pd = (a * Ac[d] + b * Bc[d]) / p;
        pp->P[d] = Pd;
        double XAB = Ac[d] - Bc[d];
        make_E(A->am, B->am + extra_b, p, Pd - Ac[d], Pd - Bc[d], exp(-mu * XAB * XAB), pp->E[d]);
    }
}

void oi_overlap(const oi_shell *A, const oi_shell *B, double *out)
{
    int ca[28][3], cb[28][3];
    int nA = oi_ncart(A->am), nB = oi_ncart(B->am);
    cart_list(A->am, ca); cart_list(B->am, cb);
    memset(out, 0, sizeof(double) * nA * nB);
    prim_pair pp;
    for (int ka = 0; ka < A->nprim; ka++)
        for (int kb = 0; kb < B->nprim; kb++)
        {
            make_pair(A, ka, B, kb, 0, &pp);
            double pref = A->coef[ka] * B->coef[kb] * pow(M_PI / pp.p, 1.5);
            for (int i = 0; i < nA; i++)
                for (int j = 0; j < nB; j++)
                    out[i * nB + j] += pref * pp.E[0][ca[i][0]][cb[j][0]][0]
                                            * pp.E[1][ca[i][1]][cb[j][1]][0]
                                            * pp.E[2][ca[i][2]][cb[j][2]][0];
        }
}

void oi_kinetic(const oi_shell *A, const oi_shell *B, double *out)
{
    int ca[28][3], cb[28][3];
    int nA = oi_ncart(A->am), nB = oi_ncart(B->am);
    cart_list(A->am, ca); cart_list(B->am, cb);
    memset(out, 0, sizeof(double) * nA * nB);
    prim_pair pp;
    for (int ka = 0; ka < A->nprim; ka++)
        for (int kb = 0; kb < B->nprim; kb++)
        {
            make_pair(A, ka, B, kb, 2, &pp);
            double b = B->alpha[kb];
            double pref = A->coef[ka] * B->coef[kb] * pow(M_PI / pp.p, 1.5);
            for (int i = 0; i < nA; i++)
                for (int j = 0; j < nB; j++)
                {
                    double s[3], t[3];
                    for (int d = 0; d < 3; d++)
                    {
                        int ii = ca[i][d], jj = cb[j][d];
                        double (*E)[EMAX][TMAX] = pp.E[d];
                        s[d] = E[ii][jj][0];
                        double v = -2.0 * b * b * E[ii][jj + 2][0] + b * (2 * jj + 1) * E[ii][jj][0];
                        if (jj >= 2) v -= 0.5 * jj * (jj - 1) * E[ii][jj - 2][0];
                        t[d] = v;
                    }
                    out[i * nB + j] += pref * (t[0] * s[1] * s[2] + s[0] * t[1] * s[2] + s[0] * s[1] * t[2]);
                }
        }
}

void oi_potential(const oi_shell *A, const oi_shell *B, int natoms,
                  const double *Z, const double *xyz, double *out)
{
    int ca[28][3], cb[28][3];
    int nA = oi_ncart(A->am), nB = oi_ncart(B->am);
    cart_list(A->am, ca); cart_list(B->am, cb);
    memset(out, 0, sizeof(double) * nA * nB);
    int L = A->am + B->am, D = L + 1;
    double *R = scratch((size_t) D * D * D * D);
    prim_pair pp;
    for (int ka = 0; ka < A->nprim; ka++)
        for (int kb = 0; kb < B->nprim; kb++)
        {
            make_pair(A, ka, B, kb, 0, &pp);
            double pref = A->coef[ka] * B->coef[kb] * 2.0 * M_PI / pp.p;
            for (int c = 0; c < natoms; c++)
            {
                make_R(L, pp.p, pp.P[0] - xyz[3 * c], pp.P[1] - xyz[3 * c + 1], pp.P[2] - xyz[3 * c + 2], R);
                double f = -Z[c] * pref;
                for (int i = 0; i < nA; i++)
                    for (int j = 0; j < nB; j++)
                    {
                        int ix = ca[i][0] + cb[j][0], iy = ca[i][1] + cb[j][1], iz = ca[i][2] + cb[j][2];
                        double sum = 0.0;
                        for (int t = 0; t <= ix; t++)
                        {
                            double ex = pp.E[0][ca[i][0]][cb[j][0]][t];
                            for (int u = 0; u <= iy; u++)
                            {
                                double exy = ex * pp.E[1][ca[i][1]][cb[j][1]][u];
                                for (int v = 0; v <= iz; v++)
                                    sum += exy * pp.E[2][ca[i][2]][cb[j][2]][v] * RI(0, t, u, v);
                            }
                        }
                        out[i * nB + j] += f * sum;
                    }
            }
        }
}

void oi_eri(const oi_shell *A, const oi_shell *B, const oi_shell *C, const oi_shell *D_, double *out)
{
    int ca[28][3], cb[28][3], cc[28][3], cd[28][3];
    int nA = oi_ncart(A->am), nB = oi_ncart(B->am), nC = oi_ncart(C->am), nD = oi_ncart(D_->am);
    cart_list(A->am, ca); cart_list(B->am, cb); cart_list(C->am, cc); cart_list(D_->am, cd);
    int nAB = nA * nB, nCD = nC * nD;
    memset(out, 0, sizeof(double) * nAB * nCD);
    int LAB = A->am + B->am, LCD = C->am + D_->am, L = LAB + LCD, D = L + 1;
    int H = LAB + 1;                               /* Hermite box side for the bra */
    size_t rsz = (size_t) D * D * D * D;
    size_t gsz = (size_t) nCD * H * H * H;
    double *buf = scratch(rsz + gsz);
    double *R = buf, *G = buf + rsz;
    prim_pair pab, pcd;
    for (int ka = 0; ka < A->nprim; ka++)
    for (int kb = 0; kb < B->nprim; kb++)
    {
        make_pair(A, ka, B, kb, 0, &pab);
        for (int kc = 0; kc < C->nprim; kc++)
        for (int kd = 0; kd < D_->nprim; kd++)
        {
            make_pair(C, kc, D_, kd, 0, &pcd);
            double p = pab.p, q = pcd.p, alpha = p * q / (p + q);
            double pref = 2.0 * pow(M_PI, 2.5) / (p * q * sqrt(p + q))
                        * A->coef[ka] * B->coef[kb] * C->coef[kc] * D_->coef[kd];
            make_R(L, alpha, pab.P[0] - pcd.P[0], pab.P[1] - pcd.P[1], pab.P[2] - pcd.P[2], R);
            /* contract the ket Hermite expansion first: G[cd][t][u][v] */
            for (int k = 0; k < nC; k++)
            for (int l = 0; l < nD; l++)
            {
                int icd = k * nD + l;
                int jx = cc[k][0] + cd[l][0], jy = cc[k][1] + cd[l][1], jz = cc[k][2] + cd[l][2];
                double *g = G + (size_t) icd * H * H * H;
                for (int t = 0; t <= LAB; t++)
                for (int u = 0; u <= LAB - t; u++)
                for (int v = 0; v <= LAB - t - u; v++)
                {
                    double s = 0.0;
                    for (int tau = 0; tau <= jx; tau++)
                    {
                        double ex = pcd.E[0][cc[k][0]][cd[l][0]][tau];
                        if (ex == 0.0) continue;
                        for (int nu = 0; nu <= jy; nu++)
                        {
                            double exy = ex * pcd.E[1][cc[k][1]][cd[l][1]][nu];
                            for (int phi = 0; phi <= jz; phi++)
                            {
                                double e = exy * pcd.E[2][cc[k][2]][cd[l][2]][phi];
                                if ((tau + nu + phi) & 1) e = -e;
                                s += e * RI(0, t + tau, u + nu, v + phi);
                            }
                        }
                    }
                    g[(t * H + u) * H + v] = s;
                }
            }
            for (int i = 0; i < nA; i++)
            for (int j = 0; j < nB; j++)
            {
                int ix = ca[i][0] + cb[j][0], iy = ca[i][1] + cb[j][1], iz = ca[i][2] + cb[j][2];
                double *o = out + (size_t) (i * nB + j) * nCD;
                for (int icd = 0; icd < nCD; icd++)
                {
                    const double *g = G + (size_t) icd * H * H * H;
                    double s = 0.0;
                    for (int t = 0; t <= ix; t++)
                    {
                        double ex = pab.E[0][ca[i][0]][cb[j][0]][t];
                        for (int u = 0; u <= iy; u++)
                        {
                            double exy = ex * pab.E[1][ca[i][1]][cb[j][1]][u];
                            for (int v = 0; v <= iz; v++)
                                s += exy * pab.E[2][ca[i][2]][cb[j][2]][v] * g[(t * H + u) * H + v];
                        }
                    }
                    o[icd] += pref * s;
                }
            }
        }
    }
}
#undef RI
