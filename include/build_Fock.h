/* Drop-in for the reference's build_Fock.h:6 (build_Fock.c:349-396):
 * J, K and F = Hcore + 2J - K from the current D_mat / Cocc_mat. */
#ifndef TINYSCF_B200_BUILD_FOCK_H
#define TINYSCF_B200_BUILD_FOCK_H
#include "TinySCF.h"
#ifdef __cplusplus
extern "C" {
#endif
TINYSCF_API void TinySCF_build_FockMat(TinySCF_t TinySCF);
#ifdef __cplusplus
}
#endif
#endif
