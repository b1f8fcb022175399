/* Drop-in for the reference's build_density.h:6-8 (build_density.c:12-69). */
#ifndef TINYSCF_B200_BUILD_DENSITY_H
#define TINYSCF_B200_BUILD_DENSITY_H
#include "TinySCF.h"
#ifdef __cplusplus
extern "C" {
#endif
/* Host helper, same behaviour as the reference's (build_density.c:12-35),
 * including its index-swap slip on exactly equal eigenvalues. */
TINYSCF_API void quickSort_eigval(double *eigval, int *ev_idx, int l, int r);
/* eig(F'), C = X C0, n_occ lowest, D = Cocc Cocc^T — on the device. */
TINYSCF_API void TinySCF_build_DenMat(TinySCF_t TinySCF);
#ifdef __cplusplus
}
#endif
#endif
