// Batched (many-molecule) SCF: per-molecule device descriptors, per-phase work
// lists and the phase launchers of batch.cu.
#pragma once
#include "tscf_internal.h"

namespace tscf {

struct MolDev {
    int nbf, naux, nocc, nup, jblk, ksplit, max_diis, ktile;   // ktile: 64, 128 or KSYRK_DMMA
    const int *up_i, *up_j, *up_u, *csr_j, *csr_u, *displs;
    const int2 *tiles;   // upper tile pairs for ktile
    const double *B, *H, *S, *X;
    const float *B32;   // FP32 copy of B for the mixed-precision molecules' J (null otherwise)
    double *D, *J, *K, *F, *Fp, *Cocc, *T, *Kpart, *Jt, *Jpart, *Jw, *epart, *E, *tmp, *tmp2, *F0, *R, *eigA;
    DiisState *diis;
};

// items numbered molecule by molecule: molecule m owns [start[m], start[m+1])
struct WorkList {
    const int *start;   // device, nmol + 1 entries
    int nmol;
    int total;
};

struct GemmDesc {
    int m, n, k, lda, ldb, ldc;
    const double *A, *B;
    double *C;
    double alpha, beta;
};

struct BatchGemm {
    const GemmDesc *descs = nullptr;   // device, one per molecule
    WorkList wl{};
    bool ta = false, tb = false;
};

struct BatchPlan {
    const MolDev *mols = nullptr;   // device
    const int *active = nullptr;    // device, 1 while the molecule iterates
    int nmol = 0, naux_max = 0;
    // half / half_wide and syrk / syrk128 hold the items of the molecules that
    // use that tile (the other molecules contribute none)
    WorkList nup256, jblk, naux256, nup64, half, half_wide, half_dmma, syrk, syrk128, syrk_dmma, nn256, efb;
    BatchGemm g_xtf, g_tx_fp, g_fd, g_fds, g_xtt, g_t2x, g_tx_t2, g_cocc, g_dens;
};

// use32: the molecules that have an FP32 copy of B read it (the iterations of
// the mixed-precision form); 0 for the FP64 J of their final build
void batch_j(const BatchPlan &b, cudaStream_t s, int use32 = 1);
// kact: per-molecule flags of the molecules whose exchange is built here (FP64)
void batch_k(const BatchPlan &b, const int *kact, cudaStream_t s);
void batch_fock(const BatchPlan &b, double *d_Eall, cudaStream_t s);
void batch_diis(const BatchPlan &b, bool full, cudaStream_t s);
void batch_gemm(const BatchGemm &g, const int *d_active, cudaStream_t s);
// F' of the molecules flagged in mask into their eigensolver slots
void batch_copy_fp(const BatchPlan &b, const int *mask, cudaStream_t s);
void diis_solve_batched(const MolDev *d_mols, const int *d_active, int nmol, cudaStream_t s);

}  // namespace tscf
