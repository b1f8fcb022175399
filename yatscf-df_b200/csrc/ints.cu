// FP64 Gaussian integrals on sm_100a: Obara–Saika vertical recursion (VRR),
// Head-Gordon–Pople electron transfer (ETR) and horizontal recursion (HRR)
// over a tabulated Boys function. Replaces the Simint calls of the reference
// (libCMS/CMS_Simint.c:363 4-centre, :411 overlap, :441/:444 kinetic+nuclear,
// :527 batched 3-centre, :595 2-centre).
//
// Work is bucketed by angular-momentum class so every warp runs one class:
// one launch per (la,lb[,lc]) class, one thread per shell pair (1e, Schwarz),
// per (shell pair, aux shell) triplet (3-centre) or per aux pair (2-centre).
//
// Conventions: Cartesian components in lexicographic order (xx,xy,xz,yy,yz,zz);
// contracted shells normalised so the x^l component has unit norm; the
// "unit shell" (exponent 0, coefficient 1) turns 4-centre into 3-/2-centre
// integrals, as in libCMS/CMS_Simint.c:131-141.
#include <cmath>
#include <cstdio>
#include <vector>

#include "tscf_internal.h"
#include "tune.h"

namespace tscf {

// ------------------------------------------------------------------ tables
// Cartesian components of every level l <= 8 in cumulative order:
// index ncum(l-1) + n(n+1)/2 + lz with n = l - lx.
__constant__ unsigned char c_comp[165][3];
__device__ double g_boys[BOYS_NGRID * 16];

static bool g_tables_ready[64] = {false};

static void host_boys_column(double T, double *F, int mmax)
{
    // Series for F_mmax (positive terms only) in long double, then downward recursion.
    long double term = 1.0L / (2 * mmax + 1), sum = term;
    for (int k = 1; k < 5000; k++) {
        term *= 2.0L * T / (2 * mmax + 2 * k + 1);
        sum += term;
        if (term < 1e-22L * sum) break;
    }
    long double eT = expl(-(long double) T);
    long double f = eT * sum;
    F[mmax] = (double) f;
    for (int m = mmax - 1; m >= 0; m--) {
        f = (2.0L * T * f + eT) / (2 * m + 1);
        F[m] = (double) f;
    }
}

void boys_table_init(cudaStream_t s)
{
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && g_tables_ready[dev]) return;
    std::vector<double> tab(BOYS_NGRID * 16);
    for (int k = 0; k < BOYS_NGRID; k++) host_boys_column(k * BOYS_DT, &tab[k * 16], 15);
    unsigned char comp[165][3];
    int idx = 0;
    for (int l = 0; l <= 8; l++)
        for (int lx = l; lx >= 0; lx--)
            for (int ly = l - lx; ly >= 0; ly--) {
                comp[idx][0] = (unsigned char) lx;
                comp[idx][1] = (unsigned char) ly;
                comp[idx][2] = (unsigned char) (l - lx - ly);
                idx++;
            }
    cudaMemcpyToSymbolAsync(g_boys, tab.data(), sizeof(double) * tab.size(), 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(c_comp, comp, sizeof(comp), 0, cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    if (dev < 64) g_tables_ready[dev] = true;
}

// F_m(T), m = 0..mmax: 7-term Taylor expansion of F_mmax about the nearest grid
// point (dF_m/dT = -F_{m+1}), downward recursion F_m = (2T F_{m+1} + e^-T)/(2m+1);
// asymptotic form (2m-1)!!/2^(m+1) sqrt(pi/T^(2m+1)) beyond T = 60.
__device__ __forceinline__ void boys(int mmax, double T, double *F)
{
    if (T >= BOYS_TMAX) {
        double f = 0.5 * sqrt(M_PI / T);
        F[0] = f;
        double i2t = 0.5 / T;
        for (int m = 1; m <= mmax; m++) {
            f *= (2 * m - 1) * i2t;
            F[m] = f;
        }
        return;
    }
    int k = __double2int_rn(T * (1.0 / BOYS_DT));
    double d = k * BOYS_DT - T;                       // -(T - T_k)
    const double *row = g_boys + k * 16 + mmax;
    double f = row[6];
    f = row[5] + f * d * (1.0 / 6.0);
    f = row[4] + f * d * (1.0 / 5.0);
    f = row[3] + f * d * (1.0 / 4.0);
    f = row[2] + f * d * (1.0 / 3.0);
    f = row[1] + f * d * (1.0 / 2.0);
    f = row[0] + f * d;
    F[mmax] = f;
    if (mmax > 0) {
        double eT = exp(-T);
        double t2 = 2.0 * T;
        for (int m = mmax - 1; m >= 0; m--) {
            f = (t2 * f + eT) / (2 * m + 1);
            F[m] = f;
        }
    }
}

__device__ __forceinline__ int cidx(int lx, int lz, int l)
{
    int n = l - lx;
    return n * (n + 1) / 2 + lz;
}
__device__ __forceinline__ int cum_of(int lx, int ly, int lz)
{
    int l = lx + ly + lz;
    return ncum(l - 1) + cidx(lx, lz, l);
}

// ------------------------------------------------------------------ VRR
// [e|0]^(0) for all e with |e| <= L into e0[ncum(L)]:
// [e+1_i]^(m) = PA_i [e]^(m) + WP_i [e]^(m+1) + e_i/(2z) ([e-1_i]^(m) - rz [e-1_i]^(m+1)).
// (For nuclear attraction pass WP = -PC and rz = 1.)
template <int LT>
struct VrrSize {
    __host__ __device__ static constexpr int w()
    {
        int best = 1;
        for (int l = 0; l <= LT; l++) {
            int v = ncart(l) * (LT - l + 1);
            if (v > best) best = v;
        }
        return best;
    }
};

template <int LT>
__device__ __forceinline__ void vrr_e0(int L, const double *F, double pref, const double PA[3], const double WP[3],
                                       double inv2z, double rz, double *e0)
{
    constexpr int W = VrrSize<LT>::w();
    double lev[3][W];
    for (int m = 0; m <= L; m++) lev[0][m] = pref * F[m];
    e0[0] = lev[0][0];
    for (int l = 1; l <= L; l++) {
        double *cur = lev[l % 3];
        const double *p1 = lev[(l + 2) % 3];
        const double *p2 = lev[(l + 1) % 3];
        const int M = L - l;
        const int base = ncum(l - 1);
        for (int c = 0; c < ncart(l); c++) {
            int lx = c_comp[base + c][0], ly = c_comp[base + c][1], lz = c_comp[base + c][2];
            int i = lx > 0 ? 0 : (ly > 0 ? 1 : 2);
            int ai = (i == 0 ? lx : (i == 1 ? ly : lz)) - 1;   // i-th index of the lower function
            int ux = lx - (i == 0), uz = lz - (i == 2);
            int c1 = cidx(ux, uz, l - 1);
            const double *q1 = p1 + c1 * (M + 2);
            double *o = cur + c * (M + 1);
            if (ai > 0) {
                int vx = ux - (i == 0), vz = uz - (i == 2);
                int c2 = cidx(vx, vz, l - 2);
                const double *q2 = p2 + c2 * (M + 3);
                double f = ai * inv2z;
                for (int m = 0; m <= M; m++)
                    o[m] = PA[i] * q1[m] + WP[i] * q1[m + 1] + f * (q2[m] - rz * q2[m + 1]);
            } else {
                for (int m = 0; m <= M; m++) o[m] = PA[i] * q1[m] + WP[i] * q1[m + 1];
            }
            e0[base + c] = o[0];
        }
    }
}

// ------------------------------------------------------------------ ETR + accumulate
// From [e|0] (|e| <= L) build [e|f] for |f| up to lc+ld with the electron
// transfer relation (m = 0 only)
//   [e|f+1_i] = cAB_i [e|f] + e_i/(2eta)[e-1_i|f] + f_i/(2eta)[e|f-1_i] - (zeta/eta)[e+1_i|f],
//   cAB_i = -(beta AB_i + delta CD_i)/eta,
// and add [e|f] for e in [la, la+lb], f in [lc, lc+ld] into acc[e][f].
template <int LT, int LF>
struct EtrSize {
    __host__ __device__ static constexpr int w()
    {
        int best = 1;
        for (int f = 0; f <= LF; f++) {
            int v = ncum(LT - f) * ncart(f);
            if (v > best) best = v;
        }
        return best;
    }
};

template <int LT, int LF>
__device__ __forceinline__ void etr_accumulate(int L, int la, int Le, int lc, int Lf, const double *e0,
                                               const double cAB[3], double inv2eta, double zeta_eta,
                                               double *acc, int NFa)
{
    const int eoff = ncum(la - 1), eend = ncum(Le), foff = ncum(lc - 1);
    if (lc == 0)
        for (int e = eoff; e < eend; e++) acc[(e - eoff) * NFa] += e0[e];
    if (Lf == 0) return;
    constexpr int W = EtrSize<LT, LF>::w();
    double buf[3][W];
    // level 0 lives in e0 (stride 1)
    for (int f = 0; f < Lf; f++) {
        const double *cur = (f == 0) ? e0 : buf[f % 3];
        const double *prev = (f == 1) ? e0 : buf[(f + 2) % 3];
        double *nxt = buf[(f + 1) % 3];
        const int nf = ncart(f), nf1 = ncart(f + 1), nfm = (f >= 1) ? ncart(f - 1) : 1;
        const int nE = ncum(L - f - 1);
        const int gbase = ncum(f);
        for (int g = 0; g < nf1; g++) {
            int gx = c_comp[gbase + g][0], gy = c_comp[gbase + g][1], gz = c_comp[gbase + g][2];
            int i = gx > 0 ? 0 : (gy > 0 ? 1 : 2);
            int hx = gx - (i == 0), hy = gy - (i == 1), hz = gz - (i == 2);
            int hi = (i == 0 ? hx : (i == 1 ? hy : hz));
            int ch = cidx(hx, hz, f);
            int ch2 = (hi > 0) ? cidx(hx - (i == 0), hz - (i == 2), f - 1) : 0;
            double fh = hi * inv2eta;
            bool acc_level = (f + 1 >= lc);
            int gacc = ncum(f) - foff + g;
            for (int e = 0; e < nE; e++) {
                int ex = c_comp[e][0], ey = c_comp[e][1], ez = c_comp[e][2];
                int ei = (i == 0 ? ex : (i == 1 ? ey : ez));
                int eup = cum_of(ex + (i == 0), ey + (i == 1), ez + (i == 2));
                double v = cAB[i] * cur[e * nf + ch] - zeta_eta * cur[eup * nf + ch];
                if (ei > 0) {
                    int edn = cum_of(ex - (i == 0), ey - (i == 1), ez - (i == 2));
                    v += ei * inv2eta * cur[edn * nf + ch];
                }
                if (hi > 0) v += fh * prev[e * nfm + ch2];
                nxt[e * nf1 + g] = v;
                if (acc_level && e >= eoff && e < eend) acc[(e - eoff) * NFa + gacc] += v;
            }
        }
    }
}

// HRR leaves of (a,b| for lb <= 2: (a,b| = sum_k w_k (e_k,0| with AB = A - B.
__device__ __forceinline__ int hrr_leaves(int ax, int ay, int az, int bx, int by, int bz, const double AB[3],
                                          int *e, double *w)
{
    int lb = bx + by + bz;
    if (lb == 0) {
        e[0] = cum_of(ax, ay, az);
        w[0] = 1.0;
        return 1;
    }
    int i = bx > 0 ? 0 : (by > 0 ? 1 : 2);
    int di[3] = {i == 0, i == 1, i == 2};
    if (lb == 1) {
        e[0] = cum_of(ax + di[0], ay + di[1], az + di[2]);
        w[0] = 1.0;
        e[1] = cum_of(ax, ay, az);
        w[1] = AB[i];
        return 2;
    }
    int rx = bx - di[0], ry = by - di[1];
    int j = rx > 0 ? 0 : (ry > 0 ? 1 : 2);
    int dj[3] = {j == 0, j == 1, j == 2};
    e[0] = cum_of(ax + di[0] + dj[0], ay + di[1] + dj[1], az + di[2] + dj[2]);
    w[0] = 1.0;
    e[1] = cum_of(ax + di[0], ay + di[1], az + di[2]);
    w[1] = AB[j];
    e[2] = cum_of(ax + dj[0], ay + dj[1], az + dj[2]);
    w[2] = AB[i];
    e[3] = cum_of(ax, ay, az);
    w[3] = AB[i] * AB[j];
    return 4;
}

struct Sh {
    int am, np;
    double x, y, z;
    const double *al, *co;
};
__device__ __forceinline__ Sh load_shell(const DevShells &s, int i)
{
    Sh r;
    r.am = s.am[i];
    r.np = s.nprim[i];
    r.x = s.cen[3 * i];
    r.y = s.cen[3 * i + 1];
    r.z = s.cen[3 * i + 2];
    r.al = s.alpha + s.poff[i];
    r.co = s.coef + s.poff[i];
    return r;
}
__device__ __forceinline__ Sh unit_shell()
{
    Sh r;
    r.am = 0;
    r.np = 1;
    r.x = r.y = r.z = 0.0;
    r.al = nullptr;
    r.co = nullptr;
    return r;
}

// Contracted [e|f] accumulator for (ab|cd): acc[e in la..la+lb][f in lc..lc+ld].
// d may be the unit shell (ud = true), b may be the unit shell (ub = true).
template <int LT, int LF>
__device__ void quartet_acc(const Sh &A, const Sh &B, bool ub, const Sh &C, const Sh &D, bool ud, double *acc,
                            int NEa, int NFa)
{
    const int la = A.am, lb = B.am, lc = C.am, ld = D.am;
    const int L = la + lb + lc + ld, Le = la + lb, Lf = lc + ld;
    for (int k = 0; k < NEa * NFa; k++) acc[k] = 0.0;
    const double AB[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
    const double CD[3] = {C.x - D.x, C.y - D.y, C.z - D.z};
    const double AB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    const double CD2 = CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2];
    double F[LT + 1];
    double e0[ncum(LT)];
    const int npb = ub ? 1 : B.np, npd = ud ? 1 : D.np;
    for (int ka = 0; ka < A.np; ka++) {
        const double a = A.al[ka], ca = A.co[ka];
        for (int kb = 0; kb < npb; kb++) {
            const double b = ub ? 0.0 : B.al[kb], cb = ub ? 1.0 : B.co[kb];
            const double z = a + b, iz = 1.0 / z;
            const double P[3] = {(a * A.x + b * B.x) * iz, (a * A.y + b * B.y) * iz, (a * A.z + b * B.z) * iz};
            const double Kab = ca * cb * exp(-a * b * iz * AB2);
            const double PA[3] = {P[0] - A.x, P[1] - A.y, P[2] - A.z};
            for (int kc = 0; kc < C.np; kc++) {
                const double c = C.al[kc], cc = C.co[kc];
                for (int kd = 0; kd < npd; kd++) {
                    const double d = ud ? 0.0 : D.al[kd], cd = ud ? 1.0 : D.co[kd];
                    const double eta = c + d, ie = 1.0 / eta;
                    const double Q[3] = {(c * C.x + d * D.x) * ie, (c * C.y + d * D.y) * ie, (c * C.z + d * D.z) * ie};
                    const double Kcd = cc * cd * exp(-c * d * ie * CD2);
                    const double izt = 1.0 / (z + eta);
                    const double rho = z * eta * izt;
                    const double W[3] = {(z * P[0] + eta * Q[0]) * izt, (z * P[1] + eta * Q[1]) * izt,
                                         (z * P[2] + eta * Q[2]) * izt};
                    const double PQ2 = (P[0] - Q[0]) * (P[0] - Q[0]) + (P[1] - Q[1]) * (P[1] - Q[1]) +
                                       (P[2] - Q[2]) * (P[2] - Q[2]);
                    const double pref = 2.0 * 17.493418327624862 /* pi^2.5 */ * iz * ie * sqrt(izt) * Kab * Kcd;
                    boys(L, rho * PQ2, F);
                    const double WP[3] = {W[0] - P[0], W[1] - P[1], W[2] - P[2]};
                    vrr_e0<LT>(L, F, pref, PA, WP, 0.5 * iz, rho * iz, e0);
                    const double cAB[3] = {-(b * AB[0] + d * CD[0]) * ie, -(b * AB[1] + d * CD[1]) * ie,
                                           -(b * AB[2] + d * CD[2]) * ie};
                    etr_accumulate<LT, LF>(L, la, Le, lc, Lf, e0, cAB, 0.5 * ie, z * ie, acc, NFa);
                }
            }
        }
    }
}

// ------------------------------------------------------------------ 3-centre kernel
// One thread per (shell pair in class, aux shell of AM lc). Writes pqA_u rows.
// aux_major = 0: consecutive threads take consecutive aux shells of one pair;
// 1: consecutive pairs for one aux shell. The block size and this order are
// picked per AM class by the autotuner (launch_3c_class).
template <int LA, int LB, int LC>
__global__ void __launch_bounds__(256) k_three_center(DevShells sh, DevShells aux, const int2 *pairs, int pair0,
                                                      int npairs, const int *aux_ids, int naux_am,
                                                      const double *sp_scr, const double *df_scr, double scrtol2,
                                                      const int *upair_index, int nbf, int naux, double *pqA,
                                                      int aux_major)
{
    const long long tid = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long long) npairs * naux_am) return;
    const int ip = aux_major ? (int) (tid % npairs) : (int) (tid / naux_am);
    const int iq = aux_major ? (int) (tid / npairs) : (int) (tid % naux_am);
    const int2 mn = pairs[pair0 + ip];
    const int P = aux_ids[iq];
    const double s0 = sp_scr[mn.x * sh.nsh + mn.y];
    if (s0 * df_scr[P] < scrtol2) return;                         // build_DF_tensor.c:100
    constexpr int LT = LA + LB + LC;
    constexpr int NEa = ncum(LA + LB) - ncum(LA - 1);
    constexpr int NFa = ncart(LC);
    double acc[NEa * NFa];
    const Sh A = load_shell(sh, mn.x), B = load_shell(sh, mn.y), C = load_shell(aux, P);
    const Sh U = unit_shell();
    quartet_acc<(LT > 0 ? LT : 1), LC>(A, B, false, C, U, true, acc, NEa, NFa);
    const double AB[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
    const int bfM = sh.bfoff[mn.x], bfN = sh.bfoff[mn.y], bfP = aux.bfoff[P];
    const int eoff = ncum(LA - 1);
    const bool same = (mn.x == mn.y);
    const int baseA = ncum(LA - 1), baseB = ncum(LB - 1);
    for (int ia = 0; ia < ncart(LA); ia++) {
        const int ax = c_comp[baseA + ia][0], ay = c_comp[baseA + ia][1], az = c_comp[baseA + ia][2];
        for (int ib = 0; ib < ncart(LB); ib++) {
            if (same && ia < ib) continue;        // the reference keeps the iM > iN value (build_DF_tensor.c:28-44)
            const int u = upair_index[(bfM + ia) * nbf + bfN + ib];
            if (u < 0) continue;
            int le[4];
            double lw[4];
            const int nl = hrr_leaves(ax, ay, az, c_comp[baseB + ib][0], c_comp[baseB + ib][1], c_comp[baseB + ib][2],
                                      AB, le, lw);
            double *dst = pqA + (size_t) u * naux + bfP;
            for (int p = 0; p < NFa; p++) {
                double v = 0.0;
                for (int k = 0; k < nl; k++) v += lw[k] * acc[(le[k] - eoff) * NFa + p];
                dst[p] = v;
            }
        }
    }
}

template <int LA, int LB, int LC>
static void launch_3c_class(const DevShells &sh, const DevShells &aux, const ThreeCenterPlan &pl, int pair0,
                            int npairs, int lc_start, int naux_am, double *pqA, cudaStream_t s)
{
    long long n = (long long) npairs * naux_am;
    if (n == 0) return;
    auto run = [&](int c) {
        const int bs = 64 << (c % 3), order = c / 3;
        const int blocks = (int) ((n + bs - 1) / bs);
        k_three_center<LA, LB, LC><<<blocks, bs, 0, s>>>(sh, aux, pl.pairs, pair0, npairs, pl.aux_by_am + lc_start,
                                                         naux_am, pl.sp_scr, pl.df_scr, pl.scrtol2, pl.upair_index,
                                                         pl.nbf, pl.naux, pqA, order);
        g_launches++;
    };
    // every candidate writes the same values, so re-running while tuning is harmless
    char key[64];
    snprintf(key, sizeof(key), "3c:%d%d%d:%s", LA, LB, LC, n < 65536 ? "small" : "large");
    int c = tune_lookup(key);
    if (c < 0 && tune_enabled()) {
        tune_run(key, {0, 1, 2, 3, 4, 5}, run, s, 1);
        return;
    }
    run(c < 0 ? 1 : c);
}

template <int LA, int LB>
static void launch_3c_lc(const DevShells &sh, const DevShells &aux, const ThreeCenterPlan &pl, int pair0, int np,
                         double *pqA, cudaStream_t s)
{
    for (int lc = 0; lc <= MAX_L_AUX; lc++) {
        int st = pl.aux_am_start[lc], cnt = pl.aux_am_start[lc + 1] - st;
        switch (lc) {
        case 0: launch_3c_class<LA, LB, 0>(sh, aux, pl, pair0, np, st, cnt, pqA, s); break;
        case 1: launch_3c_class<LA, LB, 1>(sh, aux, pl, pair0, np, st, cnt, pqA, s); break;
        case 2: launch_3c_class<LA, LB, 2>(sh, aux, pl, pair0, np, st, cnt, pqA, s); break;
        case 3: launch_3c_class<LA, LB, 3>(sh, aux, pl, pair0, np, st, cnt, pqA, s); break;
        }
    }
}

void launch_three_center(const DevShells &sh, const DevShells &aux, const ThreeCenterPlan &pl, double *pqA,
                         cudaStream_t s)
{
    for (int c = 0; c < pl.nclass; c++) {
        int p0 = pl.class_start[c], np = pl.class_start[c + 1] - p0;
        if (np == 0) continue;
        int la = pl.class_la[c], lb = pl.class_lb[c];
        int key = la * 3 + lb;
        switch (key) {
        case 0: launch_3c_lc<0, 0>(sh, aux, pl, p0, np, pqA, s); break;
        case 3: launch_3c_lc<1, 0>(sh, aux, pl, p0, np, pqA, s); break;
        case 4: launch_3c_lc<1, 1>(sh, aux, pl, p0, np, pqA, s); break;
        case 6: launch_3c_lc<2, 0>(sh, aux, pl, p0, np, pqA, s); break;
        case 7: launch_3c_lc<2, 1>(sh, aux, pl, p0, np, pqA, s); break;
        case 8: launch_3c_lc<2, 2>(sh, aux, pl, p0, np, pqA, s); break;
        default: break;   // la < lb never occurs: pairs are oriented with am(M) >= am(N)
        }
    }
}

// ------------------------------------------------------------------ 2-centre kernel
template <int LP, int LQ>
__global__ void __launch_bounds__(128) k_two_center(DevShells aux, const int *idsP, int nP, const int *idsQ, int nQ,
                                                    const double *df_scr, double scrtol2, double *Jpq, int naux)
{
    const long long tid = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long long) nP * nQ) return;
    const int P = idsP[tid / nQ], Q = idsQ[tid % nQ];
    if (P > Q) return;
    if (df_scr[P] * df_scr[Q] < scrtol2) return;                   // build_DF_tensor.c:176
    constexpr int NEa = ncart(LP), NFa = ncart(LQ);
    double acc[NEa * NFa];
    const Sh A = load_shell(aux, P), C = load_shell(aux, Q), U = unit_shell();
    quartet_acc<(LP + LQ > 0 ? LP + LQ : 1), LQ>(A, U, true, C, U, true, acc, NEa, NFa);
    const int bp = aux.bfoff[P], bq = aux.bfoff[Q];
    for (int i = 0; i < NEa; i++)
        for (int j = 0; j < NFa; j++) {
            double v = acc[i * NFa + j];
            Jpq[(size_t) (bp + i) * naux + bq + j] = v;
            Jpq[(size_t) (bq + j) * naux + bp + i] = v;
        }
}


struct AuxGroups {
    const int *ids;          // device ids grouped by AM
    const int *start;        // host [MAX_L_AUX+2]
};

template <int LP>
static void launch_2c_row(const DevShells &aux, const AuxGroups &g, const double *df_scr, double scrtol2, double *Jpq,
                          int naux, cudaStream_t s)
{
    for (int lq = 0; lq <= MAX_L_AUX; lq++) {
        int p0 = g.start[LP], nP = g.start[LP + 1] - p0;
        int q0 = g.start[lq], nQ = g.start[lq + 1] - q0;
        long long n = (long long) nP * nQ;
        if (n == 0) continue;
        int blocks = (int) ((n + 127) / 128);
        switch (lq) {
        case 0: k_two_center<LP, 0><<<blocks, 128, 0, s>>>(aux, g.ids + p0, nP, g.ids + q0, nQ, df_scr, scrtol2, Jpq, naux); break;
        case 1: k_two_center<LP, 1><<<blocks, 128, 0, s>>>(aux, g.ids + p0, nP, g.ids + q0, nQ, df_scr, scrtol2, Jpq, naux); break;
        case 2: k_two_center<LP, 2><<<blocks, 128, 0, s>>>(aux, g.ids + p0, nP, g.ids + q0, nQ, df_scr, scrtol2, Jpq, naux); break;
        case 3: k_two_center<LP, 3><<<blocks, 128, 0, s>>>(aux, g.ids + p0, nP, g.ids + q0, nQ, df_scr, scrtol2, Jpq, naux); break;
        }
    }
}

void launch_two_center_grouped(const DevShells &aux, const int *d_ids, const int *h_start, const double *d_df_scr,
                               double scrtol2, double *d_Jpq, int naux, cudaStream_t s)
{
    AuxGroups g{d_ids, h_start};
    launch_2c_row<0>(aux, g, d_df_scr, scrtol2, d_Jpq, naux, s);
    launch_2c_row<1>(aux, g, d_df_scr, scrtol2, d_Jpq, naux, s);
    launch_2c_row<2>(aux, g, d_df_scr, scrtol2, d_Jpq, naux, s);
    launch_2c_row<3>(aux, g, d_df_scr, scrtol2, d_Jpq, naux, s);
}

// max_p (p|p) per aux shell (the DF screening value).
__global__ void k_df_scrval(DevShells aux, double *out)
{
    int P = blockIdx.x * blockDim.x + threadIdx.x;
    if (P >= aux.nsh) return;
    const Sh A = load_shell(aux, P), U = unit_shell();
    double acc[ncart(MAX_L_AUX) * ncart(MAX_L_AUX)];
    const int n = ncart(A.am);
    quartet_acc<2 * MAX_L_AUX, MAX_L_AUX>(A, U, true, A, U, true, acc, n, n);
    double mx = 0.0;
    for (int k = 0; k < n; k++) mx = fmax(mx, fabs(acc[k * n + k]));
    out[P] = mx;
}

void launch_df_scrval(const DevShells &aux, double *d_out, cudaStream_t s)
{
    k_df_scrval<<<(aux.nsh + 63) / 64, 64, 0, s>>>(aux, d_out);
}

// ------------------------------------------------------------------ Schwarz kernel
// (MN|MN): only the diagonal (mn|mn) elements are formed, each from its HRR
// leaves on both sides. bf_scr[iM][iN] takes the element the reference reads
// at iN*(dM*dN*dM+dM) + iM*(dN*dM+1) (TinySCF.c:153): the diagonal of the
// component pair k = iN*dM + iM in the [dM][dN] ordering.
template <int LM, int LN>
__global__ void __launch_bounds__(64) k_schwarz(DevShells sh, const int *idsM, int nM, const int *idsN, int nN,
                                                double *sp_scr, double *bf_scr, int nbf)
{
    const long long tid = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long long) nM * nN) return;
    const int M = idsM[tid / nN], N = idsN[tid % nN];
    constexpr int dM = ncart(LM), dN = ncart(LN);
    constexpr int NEa = ncum(LM + LN) - ncum(LM - 1);
    double acc[NEa * NEa];
    const Sh A = load_shell(sh, M), B = load_shell(sh, N);
    quartet_acc<(2 * (LM + LN) > 0 ? 2 * (LM + LN) : 1), LM + LN>(A, B, false, A, B, false, acc, NEa, NEa);
    const double AB[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
    const int eoff = ncum(LM - 1);
    const int baseA = ncum(LM - 1), baseB = ncum(LN - 1);
    double diag[dM * dN];
    double mx = 0.0;
    for (int a = 0; a < dM; a++)
        for (int b = 0; b < dN; b++) {
            int le[4];
            double lw[4];
            int nl = hrr_leaves(c_comp[baseA + a][0], c_comp[baseA + a][1], c_comp[baseA + a][2],
                                c_comp[baseB + b][0], c_comp[baseB + b][1], c_comp[baseB + b][2], AB, le, lw);
            double v = 0.0;
            for (int x = 0; x < nl; x++)
                for (int y = 0; y < nl; y++) v += lw[x] * lw[y] * acc[(le[x] - eoff) * NEa + (le[y] - eoff)];
            v = fabs(v);
            diag[a * dN + b] = v;
            mx = fmax(mx, v);
        }
    const int bfM = sh.bfoff[M], bfN = sh.bfoff[N];
    for (int iM = 0; iM < dM; iM++)
        for (int iN = 0; iN < dN; iN++) bf_scr[(size_t) (bfM + iM) * nbf + bfN + iN] = diag[iN * dM + iM];
    sp_scr[M * sh.nsh + N] = mx;
}

template <int LM>
static void launch_schwarz_row(const DevShells &sh, const int *ids, const int *start, double *sp, double *bf, int nbf,
                               cudaStream_t s)
{
    for (int ln = 0; ln <= MAX_L_ORB; ln++) {
        int m0 = start[LM], nM = start[LM + 1] - m0, n0 = start[ln], nN = start[ln + 1] - n0;
        long long n = (long long) nM * nN;
        if (n == 0) continue;
        int blocks = (int) ((n + 63) / 64);
        switch (ln) {
        case 0: k_schwarz<LM, 0><<<blocks, 64, 0, s>>>(sh, ids + m0, nM, ids + n0, nN, sp, bf, nbf); break;
        case 1: k_schwarz<LM, 1><<<blocks, 64, 0, s>>>(sh, ids + m0, nM, ids + n0, nN, sp, bf, nbf); break;
        case 2: k_schwarz<LM, 2><<<blocks, 64, 0, s>>>(sh, ids + m0, nM, ids + n0, nN, sp, bf, nbf); break;
        }
    }
}

void launch_schwarz_grouped(const DevShells &sh, const int *d_ids, const int *h_start, double *d_sp, double *d_bf,
                            int nbf, cudaStream_t s)
{
    launch_schwarz_row<0>(sh, d_ids, h_start, d_sp, d_bf, nbf, s);
    launch_schwarz_row<1>(sh, d_ids, h_start, d_sp, d_bf, nbf, s);
    launch_schwarz_row<2>(sh, d_ids, h_start, d_sp, d_bf, nbf, s);
}


// ------------------------------------------------------------------ one-electron kernel
// S (1D Obara–Saika overlaps), T (from overlaps with b+-2 in one direction),
// V (Obara–Saika nuclear-attraction VRR over [e|A^(m)|0] + HRR leaves).
template <int LM, int LN>
__global__ void __launch_bounds__(64) k_one_electron(DevShells sh, const int *idsM, int nM, const int *idsN, int nN,
                                                     int natoms, const double *Z, const double *xyz, double *S,
                                                     double *H, int nbf)
{
    const long long tid = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long long) nM * nN) return;
    const int M = idsM[tid / nN], N = idsN[tid % nN];
    // S and H are symmetric: each unordered pair once (the shell of lower AM,
    // or the lower index within one AM class, first), its block mirrored
    if (LM == LN && M > N) return;
    constexpr int dM = ncart(LM), dN = ncart(LN), LE = LM + LN;
    constexpr int NEa = ncum(LE) - ncum(LM - 1);
    const Sh A = load_shell(sh, M), B = load_shell(sh, N);
    const double AB[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
    const double AB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    double Sv[dM * dN], Tv[dM * dN], Vacc[NEa];
    for (int k = 0; k < dM * dN; k++) Sv[k] = Tv[k] = 0.0;
    for (int k = 0; k < NEa; k++) Vacc[k] = 0.0;
    const int baseA = ncum(LM - 1), baseB = ncum(LN - 1);
    double F[LE + 1];
    double e0[ncum(LE > 0 ? LE : 1)];
    for (int ka = 0; ka < A.np; ka++) {
        const double a = A.al[ka];
        for (int kb = 0; kb < B.np; kb++) {
            const double b = B.al[kb];
            const double z = a + b, iz = 1.0 / z;
            const double P[3] = {(a * A.x + b * B.x) * iz, (a * A.y + b * B.y) * iz, (a * A.z + b * B.z) * iz};
            const double K = A.co[ka] * B.co[kb] * exp(-a * b * iz * AB2);
            // 1D overlaps s[d][i][j], i <= LM, j <= LN + 2
            double s1[3][LM + 1][LN + 3];
            const double sq = sqrt(M_PI * iz);
            for (int d = 0; d < 3; d++) {
                const double PAd = P[d] - (d == 0 ? A.x : (d == 1 ? A.y : A.z));
                const double PBd = P[d] - (d == 0 ? B.x : (d == 1 ? B.y : B.z));
                s1[d][0][0] = sq;
                for (int i = 0; i <= LM; i++)
                    for (int j = 0; j <= LN + 2; j++) {
                        if (i == 0 && j == 0) continue;
                        double v;
                        if (i > 0) {
                            v = PAd * s1[d][i - 1][j];
                            double t = 0.0;
                            if (i > 1) t += (i - 1) * s1[d][i - 2][j];
                            if (j > 0) t += j * s1[d][i - 1][j - 1];
                            v += 0.5 * iz * t;
                        } else {
                            v = PBd * s1[d][0][j - 1];
                            if (j > 1) v += 0.5 * iz * (j - 1) * s1[d][0][j - 2];
                        }
                        s1[d][i][j] = v;
                    }
            }
            for (int ia = 0; ia < dM; ia++) {
                int aa[3] = {c_comp[baseA + ia][0], c_comp[baseA + ia][1], c_comp[baseA + ia][2]};
                for (int ib = 0; ib < dN; ib++) {
                    int bb[3] = {c_comp[baseB + ib][0], c_comp[baseB + ib][1], c_comp[baseB + ib][2]};
                    double sx = s1[0][aa[0]][bb[0]], sy = s1[1][aa[1]][bb[1]], sz = s1[2][aa[2]][bb[2]];
                    Sv[ia * dN + ib] += K * sx * sy * sz;
                    double t[3];
                    for (int d = 0; d < 3; d++) {
                        int j = bb[d];
                        double v = -2.0 * b * b * s1[d][aa[d]][j + 2] + b * (2 * j + 1) * s1[d][aa[d]][j];
                        if (j >= 2) v -= 0.5 * j * (j - 1) * s1[d][aa[d]][j - 2];
                        t[d] = v;
                    }
                    Tv[ia * dN + ib] += K * (t[0] * sy * sz + sx * t[1] * sz + sx * sy * t[2]);
                }
            }
            // nuclear attraction
            const double PA[3] = {P[0] - A.x, P[1] - A.y, P[2] - A.z};
            for (int c = 0; c < natoms; c++) {
                const double PC[3] = {P[0] - xyz[3 * c], P[1] - xyz[3 * c + 1], P[2] - xyz[3 * c + 2]};
                const double mPC[3] = {-PC[0], -PC[1], -PC[2]};
                boys(LE, z * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]), F);
                vrr_e0<(LE > 0 ? LE : 1)>(LE, F, -Z[c] * 2.0 * M_PI * iz * K, PA, mPC, 0.5 * iz, 1.0, e0);
                for (int e = ncum(LM - 1); e < ncum(LE); e++) Vacc[e - ncum(LM - 1)] += e0[e];
            }
        }
    }
    const int bfM = sh.bfoff[M], bfN = sh.bfoff[N];
    const int eoff = ncum(LM - 1);
    for (int ia = 0; ia < dM; ia++)
        for (int ib = 0; ib < dN; ib++) {
            int le[4];
            double lw[4];
            int nl = hrr_leaves(c_comp[baseA + ia][0], c_comp[baseA + ia][1], c_comp[baseA + ia][2],
                                c_comp[baseB + ib][0], c_comp[baseB + ib][1], c_comp[baseB + ib][2], AB, le, lw);
            double v = 0.0;
            for (int k = 0; k < nl; k++) v += lw[k] * Vacc[le[k] - eoff];
            size_t o = (size_t) (bfM + ia) * nbf + bfN + ib, ot = (size_t) (bfN + ib) * nbf + bfM + ia;
            const double sv = Sv[ia * dN + ib], hv = Tv[ia * dN + ib] + v;
            S[o] = sv;
            H[o] = hv;
            S[ot] = sv;
            H[ot] = hv;
        }
}

template <int LM>
static void launch_1e_row(const DevShells &sh, const int *ids, const int *start, int natoms, const double *Z,
                          const double *xyz, double *S, double *H, int nbf, cudaStream_t s)
{
    for (int ln = LM; ln <= MAX_L_ORB; ln++) {   // classes (LM, LN >= LM); the kernel mirrors each block
        int m0 = start[LM], nM = start[LM + 1] - m0, n0 = start[ln], nN = start[ln + 1] - n0;
        long long n = (long long) nM * nN;
        if (n == 0) continue;
        int blocks = (int) ((n + 63) / 64);
        switch (ln) {
        case 0: k_one_electron<LM, 0><<<blocks, 64, 0, s>>>(sh, ids + m0, nM, ids + n0, nN, natoms, Z, xyz, S, H, nbf); break;
        case 1: k_one_electron<LM, 1><<<blocks, 64, 0, s>>>(sh, ids + m0, nM, ids + n0, nN, natoms, Z, xyz, S, H, nbf); break;
        case 2: k_one_electron<LM, 2><<<blocks, 64, 0, s>>>(sh, ids + m0, nM, ids + n0, nN, natoms, Z, xyz, S, H, nbf); break;
        }
    }
}

void launch_one_electron_grouped(const DevShells &sh, const int *d_ids, const int *h_start, int natoms,
                                 const double *d_Z, const double *d_xyz, double *d_S, double *d_H, int nbf,
                                 cudaStream_t s)
{
    launch_1e_row<0>(sh, d_ids, h_start, natoms, d_Z, d_xyz, d_S, d_H, nbf, s);
    launch_1e_row<1>(sh, d_ids, h_start, natoms, d_Z, d_xyz, d_S, d_H, nbf, s);
    launch_1e_row<2>(sh, d_ids, h_start, natoms, d_Z, d_xyz, d_S, d_H, nbf, s);
}


}  // namespace tscf
