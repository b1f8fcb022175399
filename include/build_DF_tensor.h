/* Drop-in for the reference's build_DF_tensor.h:6 (build_DF_tensor.c:256-287):
 * 3-centre integrals, (P|Q), (P|Q)^-1/2 and the DF tensor, all on the device. */
#ifndef TINYSCF_B200_BUILD_DF_TENSOR_H
#define TINYSCF_B200_BUILD_DF_TENSOR_H
#include "TinySCF.h"
#ifdef __cplusplus
extern "C" {
#endif
TINYSCF_API void TinySCF_build_DF_tensor(TinySCF_t TinySCF);
#ifdef __cplusplus
}
#endif
#endif
