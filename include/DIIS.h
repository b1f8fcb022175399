/* Drop-in for the reference's DIIS.h:6 (DIIS.c:12-123): commutator DIIS in
 * the orthogonal basis, replacement of the historically largest residual. */
#ifndef TINYSCF_B200_DIIS_H
#define TINYSCF_B200_DIIS_H
#include "TinySCF.h"
#ifdef __cplusplus
extern "C" {
#endif
TINYSCF_API void TinySCF_DIIS(TinySCF_t TinySCF);
#ifdef __cplusplus
}
#endif
#endif
