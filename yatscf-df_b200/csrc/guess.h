// Learned initial guess: atom-pair density blocks predicted by small MLPs in
// a local frame of each pair, rotated into the molecule's frame and projected
// onto an idempotent density (no counterpart in the reference, whose guess is
// the superposition of atomic densities, TinySCF.c:324-364).
//
// Block types (first atom = the one with more basis functions, ties by index):
//   0 diagonal, heavy atom (C/N/O: s s s p p d = 15 Cartesian functions)
//   1 diagonal, H (s s p = 5)
//   2 heavy-heavy, 3 heavy-H, 4 H-H  (off-diagonal, distance < kPairCut)
// Other elements or shell layouts are not covered: the caller falls back to SAD.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace tscf {

constexpr int G_DIN = 128;        // feature width (113 used, zero padded)
constexpr int G_HID = 192;        // hidden width of both hidden layers
constexpr int G_NTYPES = 5;
constexpr int G_MAXF = 15;        // functions per atom covered
constexpr int G_NENV = 12;        // environment atoms per pair
constexpr double kPairCut = 4.0;  // Angstrom: off-diagonal blocks beyond this are zero
constexpr double kEnvCut = 5.0;   // Angstrom: environment radius
extern const int G_DOUT[G_NTYPES];
extern const int G_NFA[G_NTYPES];
extern const int G_NFB[G_NTYPES];

// parameters of one type's MLP, floats in this order:
// W1 [din][hid], b1 [hid], W2 [hid][hid], b2 [hid], W3 [hid][dout], b3 [dout]
inline size_t mlp_param_count(int din, int hid, int dout)
{
    return (size_t) din * hid + hid + (size_t) hid * hid + hid + (size_t) hid * dout + dout;
}

struct GuessAtoms {
    int natoms = 0;
    const int *eid = nullptr;       // 0-based element index (H = 0)
    const double *xyz = nullptr;    // Bohr
    const int *bf0 = nullptr;       // first basis function of each atom
    std::vector<std::vector<int>> shell_am;   // shell angular momenta of each atom, in basis order
};

struct GuessPair {
    int a = 0, b = 0, type = 0;
    int off_a = 0, off_b = 0, nf_a = 0, nf_b = 0;
    float feat[G_DIN];
    double Qf[9];   // local frame: rows are e_x, e_y, e_z in molecule coordinates
};

// Pairs, frames and features. Returns 0, or nonzero when an atom's element or
// shell layout is not covered by the block types.
int guess_pairs(const GuessAtoms &g, std::vector<GuessPair> &out);

// M(Q) for the Cartesian functions of one atom: phi_molecule = M phi_local.
void guess_atom_rotation(const std::vector<int> &shell_am, const double *Q, double *M, int nf);

// Target block in the local frame: D_loc = M_a^T D_ab M_b (D row-major nbf x nbf).
void guess_local_block(const GuessAtoms &g, const GuessPair &p, const double *D, int nbf, float *out);

struct GuessWork;   // device workspace of guessnet_predict, grown on demand and kept

struct GuessNet {
    int din = G_DIN, hid = G_HID;
    int dout[G_NTYPES];
    float *d_params[G_NTYPES] = {};
    float *d_scale[G_NTYPES] = {}, *d_offset[G_NTYPES] = {};   // y = raw * scale + offset
    GuessWork *work = nullptr;
};

int guessnet_load(GuessNet **net, const char *path);
void guessnet_free(GuessNet *net);

// Predict the blocks of the given pairs and write the (symmetric) density
// into d_D (zeroed first). Runs on stream s; returns 0 or an error status.
int guessnet_predict(GuessNet *net, const std::vector<GuessPair> &pairs, const GuessAtoms &g, double *d_D,
                     int nbf, cudaStream_t s);

// Train all five types on host data and write the weights file.
int guessnet_train(const float *feat, const float *target, const int *type, long long n, int epochs, int batch,
                   float lr, unsigned seed, const char *path, float *final_loss);

// Loss and gradient of one MLP on a batch (host in/out): gradient check.
int guessnet_grad(int din, int hid, int dout, const float *params, const float *X, const float *T, int n,
                  float *grad, float *loss);

}  // namespace tscf
