// Host side of the learned initial guess: atom pairs, local frames, invariant
// features, and the Cartesian rotation of basis-function blocks. The frames
// and features are functions of the geometry alone, so training data (built
// from converged densities) and prediction see the same inputs.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

#include "guess.h"

namespace tscf {

const int G_DOUT[G_NTYPES] = {225, 25, 225, 75, 25};
const int G_NFA[G_NTYPES] = {15, 5, 15, 15, 5};
const int G_NFB[G_NTYPES] = {15, 5, 15, 5, 5};

namespace {

const double BOHR2A = 0.52917720859;
const int kGuessThreads = 8;   // host threads that build the pair features of a large molecule

// one-hot slot of the covered elements (0-based element index: H 0, C 5, N 6, O 7)
int elem_slot(int eid)
{
    switch (eid) {
    case 0: return 0;
    case 5: return 1;
    case 6: return 2;
    case 7: return 3;
    default: return -1;
    }
}

// 0 = H layout (s s p), 1 = heavy layout (s s s p p d), -1 = not covered
int layout_kind(const std::vector<int> &am)
{
    static const int h[] = {0, 0, 1}, x[] = {0, 0, 0, 1, 1, 2};
    if (am.size() == 3 && std::equal(am.begin(), am.end(), h)) return 0;
    if (am.size() == 6 && std::equal(am.begin(), am.end(), x)) return 1;
    return -1;
}

void sub(const double *a, const double *b, double *o) { for (int k = 0; k < 3; k++) o[k] = a[k] - b[k]; }
double dot(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
void cross(const double *a, const double *b, double *o)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
bool unit(double *a)
{
    double n = std::sqrt(dot(a, a));
    if (n < 1e-12) return false;
    for (int k = 0; k < 3; k++) a[k] /= n;
    return true;
}

// Frame with e_z = z (unit) and e_x towards the first candidate point whose
// distance from the z axis through `origin` exceeds 0.25 A (Bohr inputs).
// Frame with e_z = z (unit) and e_x towards the point x_atom projected off
// the z axis through `origin`; with no such point (x_atom null) any
// perpendicular (the block is then symmetric about z).
void make_frame(const double *origin, const double *z, const double *x_atom, double *Q)
{
    double ex[3] = {0, 0, 0};
    if (x_atom) {
        sub(x_atom, origin, ex);
        double t = dot(ex, z);
        for (int k = 0; k < 3; k++) ex[k] -= t * z[k];
        unit(ex);
    } else {
        int m = 0;
        for (int k = 1; k < 3; k++)
            if (std::fabs(z[k]) < std::fabs(z[m])) m = k;
        double e[3] = {0, 0, 0};
        e[m] = 1.0;
        double t = dot(e, z);
        for (int k = 0; k < 3; k++) ex[k] = e[k] - t * z[k];
        unit(ex);
    }
    double ey[3];
    cross(z, ex, ey);
    for (int k = 0; k < 3; k++) {
        Q[k] = ex[k];
        Q[3 + k] = ey[k];
        Q[6 + k] = z[k];
    }
}

// Distances in sort keys are quantised to 1e-4 A so that atoms at equal
// distance (a rigid monomer's two H, say) are ordered by index, the same way
// for every orientation of the molecule.
std::pair<long long, int> dkey(double r_angstrom, int idx) { return {std::llround(r_angstrom * 1e4), idx}; }

// The atom that fixes e_x: among all atoms but skip0 and skip1, the one with the
// smallest key (distance from `origin`, then index) whose distance from the
// z axis through `origin` exceeds 0.25 A; -1 when there is none. One pass
// over the atoms instead of sorting them.
int x_atom(const GuessAtoms &g, const double *origin, const double *z, int skip0, int skip1)
{
    int best = -1;
    std::pair<long long, int> bkey;
    for (int c = 0; c < g.natoms; c++) {
        if (c == skip0 || c == skip1) continue;
        double v[3];
        sub(g.xyz + 3 * c, origin, v);
        const std::pair<long long, int> key = dkey(std::sqrt(dot(v, v)) * BOHR2A, c);
        if (best >= 0 && !(key < bkey)) continue;
        const double t = dot(v, z);
        for (int k = 0; k < 3; k++) v[k] -= t * z[k];
        if (std::sqrt(dot(v, v)) * BOHR2A > 0.25) {
            best = c;
            bkey = key;
        }
    }
    return best;
}

double cutoff_fn(double r, double rc) { return r >= rc ? 0.0 : 0.5 * (std::cos(M_PI * r / rc) + 1.0); }

void features(const GuessAtoms &g, int a, int b, const double *origin, const double *Q, float *f,
              std::vector<std::pair<long long, int>> &env)
{
    std::memset(f, 0, sizeof(float) * G_DIN);
    f[elem_slot(g.eid[a])] = 1.0f;
    f[4 + elem_slot(g.eid[b])] = 1.0f;
    f[8] = (a == b) ? 1.0f : 0.0f;
    if (a != b) {
        double v[3];
        sub(g.xyz + 3 * b, g.xyz + 3 * a, v);
        double r = std::sqrt(dot(v, v)) * BOHR2A;
        for (int k = 0; k < 8; k++) {
            double c = 0.5 + 0.5 * k, d = (r - c) / 0.5;
            f[9 + k] = (float) std::exp(-d * d);
        }
    }
    // environment: nearest other atoms to the origin within kEnvCut, in the local frame
    env.clear();
    for (int c = 0; c < g.natoms; c++) {
        if (c == a || c == b) continue;
        double v[3];
        sub(g.xyz + 3 * c, origin, v);
        double r = std::sqrt(dot(v, v)) * BOHR2A;
        if (r < kEnvCut) env.push_back(dkey(r, c));
    }
    const int ne = std::min((int) env.size(), G_NENV);
    std::partial_sort(env.begin(), env.begin() + ne, env.end());
    for (int k = 0; k < ne; k++) {
        const int c = env[k].second;
        double v[3];
        sub(g.xyz + 3 * c, origin, v);
        const double r = std::sqrt(dot(v, v)) * BOHR2A, fc = cutoff_fn(r, kEnvCut);
        float *o = f + 17 + 8 * k;
        for (int d = 0; d < 3; d++) o[d] = (float) (fc * dot(Q + 3 * d, v) * BOHR2A / kEnvCut);
        int sl = elem_slot(g.eid[c]);
        if (sl >= 0) o[3 + sl] = (float) fc;
        o[7] = (float) fc;
    }
}

// Frame and features of block (a, b): a == b is a diagonal block (origin at
// the atom, z to the nearest neighbour, x to the next off-axis one); a != b
// is off-diagonal (origin at the midpoint, z from a to b).
void fill_pair(const GuessAtoms &g, const std::vector<int> &nf, int a, int b, GuessPair &p,
               std::vector<std::pair<long long, int>> &env)
{
    p.a = a;
    p.b = b;
    p.off_a = g.bf0[a];
    p.off_b = g.bf0[b];
    p.nf_a = nf[a];
    p.nf_b = nf[b];
    if (a == b) {
        p.type = nf[a] == 15 ? 0 : 1;
        int near = -1;
        std::pair<long long, int> nkey;
        for (int c = 0; c < g.natoms; c++)
            if (c != a) {
                double v[3];
                sub(g.xyz + 3 * c, g.xyz + 3 * a, v);
                const std::pair<long long, int> key = dkey(std::sqrt(dot(v, v)) * BOHR2A, c);
                if (near < 0 || key < nkey) {
                    near = c;
                    nkey = key;
                }
            }
        if (near < 0) {
            const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
            std::memcpy(p.Qf, I, sizeof(I));
        } else {
            double z[3];
            sub(g.xyz + 3 * near, g.xyz + 3 * a, z);
            unit(z);
            const int x = x_atom(g, g.xyz + 3 * a, z, a, near);
            make_frame(g.xyz + 3 * a, z, x >= 0 ? g.xyz + 3 * x : nullptr, p.Qf);
        }
        features(g, a, a, g.xyz + 3 * a, p.Qf, p.feat, env);
        return;
    }
    p.type = (nf[a] == 15 && nf[b] == 15) ? 2 : (nf[a] == 15 ? 3 : 4);
    double mid[3], z[3];
    for (int k = 0; k < 3; k++) mid[k] = 0.5 * (g.xyz[3 * a + k] + g.xyz[3 * b + k]);
    sub(g.xyz + 3 * b, g.xyz + 3 * a, z);
    unit(z);
    const int x = x_atom(g, mid, z, a, b);
    make_frame(mid, z, x >= 0 ? g.xyz + 3 * x : nullptr, p.Qf);
    features(g, a, b, mid, p.Qf, p.feat, env);
}

}  // namespace

int guess_pairs(const GuessAtoms &g, std::vector<GuessPair> &out)
{
    out.clear();
    const int na = g.natoms;
    std::vector<int> nf(na);
    for (int a = 0; a < na; a++) {
        const int kind = layout_kind(g.shell_am[a]);
        if (kind < 0 || elem_slot(g.eid[a]) < 0) return 1;
        nf[a] = kind ? 15 : 5;
    }
    // blocks in output order: the diagonal ones, then pairs i < j closer than
    // kPairCut with the atom of more functions first
    std::vector<std::pair<int, int>> ab;
    for (int a = 0; a < na; a++) ab.emplace_back(a, a);
    const double cut = kPairCut / BOHR2A;
    for (int i = 0; i < na; i++)
        for (int j = i + 1; j < na; j++) {
            double v[3];
            sub(g.xyz + 3 * j, g.xyz + 3 * i, v);
            if (std::sqrt(dot(v, v)) >= cut) continue;
            if (nf[j] > nf[i]) ab.emplace_back(j, i);
            else ab.emplace_back(i, j);
        }
    out.resize(ab.size());
    // each block is independent: a few host threads share them (a block
    // costs O(natoms), so small molecules stay on the calling thread)
    const long long work = (long long) ab.size() * na;
    const int hw = (int) std::max(1u, std::thread::hardware_concurrency());
    const int nth = (int) std::min<long long>(std::min(hw, kGuessThreads), std::max(1LL, work / 16384));
    auto run = [&](int t) {
        std::vector<std::pair<long long, int>> env;
        for (size_t k = t; k < ab.size(); k += nth) fill_pair(g, nf, ab[k].first, ab[k].second, out[k], env);
    };
    if (nth == 1) {
        run(0);
        return 0;
    }
    std::vector<std::thread> th;
    std::vector<int> here{0};   // shares run on this thread (all of them if no thread can be started)
    for (int t = 1; t < nth; t++) {
        try {
            th.emplace_back(run, t);
        } catch (...) {
            here.push_back(t);
        }
    }
    for (int t : here) run(t);
    for (std::thread &x : th) x.join();
    return 0;
}

// Molecule coordinates x_m = Q^T x_l. A p function's polynomial x_m,a is then
// sum_c Q[c][a] x_l,c; a Cartesian d function x_m,a x_m,b (one normalisation
// constant for all six components) is sum_cd Q[c][a] Q[d][b] x_l,c x_l,d.
void guess_atom_rotation(const std::vector<int> &shell_am, const double *Q, double *M, int nf)
{
    std::memset(M, 0, sizeof(double) * nf * nf);
    static const int dpair[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
    int o = 0;
    for (int l : shell_am) {
        if (l == 0) {
            M[o * nf + o] = 1.0;
            o += 1;
        } else if (l == 1) {
            for (int a = 0; a < 3; a++)
                for (int c = 0; c < 3; c++) M[(o + a) * nf + o + c] = Q[c * 3 + a];
            o += 3;
        } else {
            for (int r = 0; r < 6; r++) {
                const int a = dpair[r][0], b = dpair[r][1];
                for (int s = 0; s < 6; s++) {
                    const int c = dpair[s][0], d = dpair[s][1];
                    double v = Q[c * 3 + a] * Q[d * 3 + b];
                    if (c != d) v += Q[d * 3 + a] * Q[c * 3 + b];
                    M[(o + r) * nf + o + s] = v;
                }
            }
            o += 6;
        }
    }
}

void guess_local_block(const GuessAtoms &g, const GuessPair &p, const double *D, int nbf, float *out)
{
    double Ma[G_MAXF * G_MAXF], Mb[G_MAXF * G_MAXF], T[G_MAXF * G_MAXF];
    guess_atom_rotation(g.shell_am[p.a], p.Qf, Ma, p.nf_a);
    guess_atom_rotation(g.shell_am[p.b], p.Qf, Mb, p.nf_b);
    // T = D_ab M_b, out = M_a^T T
    for (int i = 0; i < p.nf_a; i++)
        for (int j = 0; j < p.nf_b; j++) {
            double s = 0.0;
            for (int k = 0; k < p.nf_b; k++) s += D[(size_t) (p.off_a + i) * nbf + p.off_b + k] * Mb[k * p.nf_b + j];
            T[i * p.nf_b + j] = s;
        }
    for (int i = 0; i < p.nf_a; i++)
        for (int j = 0; j < p.nf_b; j++) {
            double s = 0.0;
            for (int k = 0; k < p.nf_a; k++) s += Ma[k * p.nf_a + i] * T[k * p.nf_b + j];
            out[i * p.nf_b + j] = (float) s;
        }
}

}  // namespace tscf
