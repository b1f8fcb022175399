/*
 * ORACLE — test infrastructure only. Nothing in the product links this file;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * and there only to check results.
 *
 * Cartesian Gaussian integral engine (McMurchie–Davidson) restating the
 * integrals the reference obtains from the un-vendored Simint library
 * (libCMS/CMS_Simint.c:363,411,441,444,527,595). Simint itself is absent, so
 * integral-level parity with Simint is unpinned; this engine is pinned by
 * closed forms, mpmath Boys values and symmetry checks (tests/test_oracle_ints.py).
 *
 * Conventions (shared with the device engine, stated once here):
 *   - Cartesian components in lexicographic order: for l=2: xx, xy, xz, yy, yz, zz.
 *   - Contracted shells are scaled so the x^l component has unit norm.
 *   - The "unit shell" (am 0, one primitive, exponent 0, coefficient 1, not
 *     normalised; libCMS/CMS_Simint.c:131-141) turns 4-centre code into
 *     3-centre (ab|P) and 2-centre (P|Q) integrals.
 *   - Output blocks are row-major [a][b] (1e), [a][b][c][d] (ERI), the layout
 *     the reference reads (build_DF_tensor.c:26,34,195; TinySCF.c:49,53).
 */
#ifndef ORACLE_INTS_H
#define ORACLE_INTS_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct
{
    int am;             /* angular momentum                                   */
    int nprim;          /* number of primitives                               */
    double x, y, z;     /* centre in Bohr                                     */
    const double *alpha;/* exponents [nprim]                                  */
    const double *coef; /* normalised contraction coefficients [nprim]        */
} oi_shell;

int  oi_ncart(int l);

/* F_m(T) for m = 0..mmax, written to F[0..mmax]. */
void oi_boys(int mmax, double T, double *F);

/* Scale raw contraction coefficients so the x^l component is unit-normalised. */
void oi_normalize(int am, int nprim, const double *alpha, const double *coef_in, double *coef_out);

void oi_overlap  (const oi_shell *A, const oi_shell *B, double *out);
void oi_kinetic  (const oi_shell *A, const oi_shell *B, double *out);
void oi_potential(const oi_shell *A, const oi_shell *B, int natoms,
                  const double *Z, const double *xyz, double *out);
void oi_eri      (const oi_shell *A, const oi_shell *B,
                  const oi_shell *C, const oi_shell *D, double *out);

#ifdef __cplusplus
}
#endif

#endif
