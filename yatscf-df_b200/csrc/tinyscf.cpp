// Host side of the B200 DF-RHF engine: the TinySCF C API (include/TinySCF.h
// and friends) over the sm_100a kernels of ints.cu, linalg.cu, fock.cu and
// scf.cu. Input parsing follows libCMS (CMS_BasisSet.c) so the same .gbs/.xyz
// and SAD files give the same shells, charges and guesses; the screening and
// sparsity bookkeeping follows TinySCF.c:112-280 on the host (small, O(nbf^2)),
// everything O(nbf^2 * naux) and up runs on the device.
#include <algorithm>
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <sys/mman.h>

#include "TinySCF.h"
#include "DIIS.h"
#include "build_DF_tensor.h"
#include "build_Fock.h"
#include "build_density.h"
#include "tinyscf_b200.h"
#include "tscf_internal.h"
#include "guess.h"
#include "batch.h"
#include "tune.h"


using namespace tscf;

namespace {

const double A2BOHR = 1.0 / 0.52917720859;   // CMS_BasisSet.c:39
const int ELEN = 50;
// occupied-subspace refinement: residual bound (Eh) and step limit before a full eigensolve
const double kRefineTol = 1e-9;
const int kRefineSteps = 6;
// subspace iterations that project the learned guess onto an idempotent density
const int kGuessSubspaceIters = 6;
const char *ETABLE[ELEN] = {"H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al",
                            "Si", "P",  "S",  "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe",
                            "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",
                            "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn"};
const char MTABLE[] = "SPDFG";

struct ShellDef {
    int am;
    std::vector<double> ex, cc;
};

struct BasisDef {
    std::map<int, std::vector<ShellDef>> elem;   // 0-based element index -> shells
    std::string dir;
};

struct Molecule {
    int natoms = 0, Q = 0, nelec = 0;
    std::vector<int> eid;        // 0-based element index
    std::vector<double> xyz;     // Bohr
    double enuc = 0.0;
};

struct HostShells {
    int nsh = 0, nbf = 0, maxam = 0;
    std::vector<int> am, nprim, poff, bfoff, atom_of;
    std::vector<double> cen, alpha, coef;
    std::vector<int> atom_bf0, atom_bf1;
};

int elem_index(const char *s)
{
    for (int i = 0; i < ELEN; i++)
        if (strcmp(s, ETABLE[i]) == 0) return i;
    return -1;
}

// CMS_import_molecule (CMS_BasisSet.c:310-426)
int parse_xyz(const char *fn, Molecule &m)
{
    FILE *f = fopen(fn, "r");
    if (!f) return ERR_FILEIO;
    char line[1024], str[1024];
    int rc = OK;
    if (!fgets(line, sizeof(line), f) || sscanf(line, "%d", &m.natoms) != 1 || m.natoms <= 0) rc = ERR_INPUT;
    if (rc == OK && !fgets(line, sizeof(line), f)) rc = ERR_INPUT;
    if (rc == OK) m.Q = (int) atof(line);
    while (rc == OK && fgets(line, sizeof(line), f)) {
        double x, y, z;
        int nsc = sscanf(line, "%1023s %lf %lf %lf", str, &x, &y, &z);
        if (nsc < 1 || !isalpha((unsigned char) str[0])) continue;
        int e = (strlen(str) <= 2) ? elem_index(str) : -1;
        if (e < 0 || nsc < 4) { rc = ERR_INPUT; break; }
        if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z)) { rc = ERR_INPUT; break; }
        m.eid.push_back(e);
        m.xyz.push_back(x * A2BOHR);
        m.xyz.push_back(y * A2BOHR);
        m.xyz.push_back(z * A2BOHR);
        m.nelec += e + 1;
    }
    fclose(f);
    if (rc != OK) return rc;
    if ((int) m.eid.size() != m.natoms) return ERR_INPUT;
    m.enuc = 0.0;
    for (int a = 0; a < m.natoms; a++)
        for (int b = a + 1; b < m.natoms; b++) {
            double dx = m.xyz[3 * a] - m.xyz[3 * b], dy = m.xyz[3 * a + 1] - m.xyz[3 * b + 1],
                   dz = m.xyz[3 * a + 2] - m.xyz[3 * b + 2];
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            if (!(r > 1e-6)) return ERR_INPUT;   // coincident nuclei: infinite repulsion
            m.enuc += (m.eid[a] + 1.0) * (m.eid[b] + 1.0) / r;
        }
    return OK;
}

// CMS_import_basis (CMS_BasisSet.c:439-642): SP-type shells split into S, P, ...
int parse_gbs(const char *fn, BasisDef &b)
{
    FILE *f = fopen(fn, "r");
    if (!f) return ERR_FILEIO;
    std::vector<std::string> lines;
    char buf[1024];
    while (fgets(buf, sizeof(buf), f)) lines.push_back(buf);
    fclose(f);
    if (lines.empty()) return ERR_INPUT;
    char str[1024] = {0};
    if (sscanf(lines[0].c_str(), "%1023s", str) == 1 && strcmp(str, "spherical") == 0)
        return ERR_UNSUPPORTED;   // the engine is Cartesian-only, like Simint's path in the reference
    size_t i = 1;
    while (i < lines.size()) {
        const std::string &L = lines[i++];
        if (L.empty() || !isalpha((unsigned char) L[0])) continue;
        sscanf(L.c_str(), "%1023s", str);
        int e = elem_index(str);
        if (e < 0) return ERR_INPUT;
        std::vector<ShellDef> shells;
        while (i < lines.size()) {
            const std::string &S = lines[i++];
            if (!S.empty() && isalpha((unsigned char) S[0])) {
                int nexp = 0;
                double beta = 0;
                char kind[64] = {0};
                if (sscanf(S.c_str(), "%63s %d %lf", kind, &nexp, &beta) < 2) return ERR_INPUT;
                int ns = (int) strlen(kind);
                if (nexp <= 0 || ns <= 0 || ns > 3) return ERR_INPUT;
                if (i + nexp > lines.size()) return ERR_INPUT;
                std::vector<double> ex(nexp), cc[3];
                for (int k = 0; k < 3; k++) cc[k].assign(nexp, 0.0);
                for (int p = 0; p < nexp; p++) {
                    const std::string &R = lines[i + p];
                    if (R.empty() || R[0] == '*' || isalpha((unsigned char) R[0])) return ERR_INPUT;
                    // an exponent and ns finite coefficients; Fortran 'D' exponents
                    // (1.0D+01) read as 'E'
                    std::string Rn = R;
                    for (char &c : Rn)
                        if (c == 'D' || c == 'd') c = 'E';
                    double v[4] = {0, 0, 0, 0};
                    const int got = sscanf(Rn.c_str(), "%lf %lf %lf %lf", &v[0], &v[1], &v[2], &v[3]);
                    if (got < 1 + ns || !std::isfinite(v[0]) || !(v[0] > 0.0)) return ERR_INPUT;
                    for (int k = 0; k < ns; k++)
                        if (!std::isfinite(v[1 + k])) return ERR_INPUT;
                    ex[p] = v[0];
                    for (int k = 0; k < 3; k++) cc[k][p] = v[1 + k];
                }
                i += nexp;
                for (int k = 0; k < ns; k++) {
                    const char *pos = strchr(MTABLE, kind[k]);
                    if (!pos || kind[k] == 0) return ERR_INPUT;
                    ShellDef d;
                    d.am = (int) (pos - MTABLE);
                    d.ex = ex;
                    d.cc = cc[k];
                    shells.push_back(d);
                }
            }
            if (!S.empty() && S[0] == '*') break;
        }
        b.elem[e] = shells;
    }
    std::string p(fn);
    size_t sl = p.find_last_of('/');
    b.dir = (sl == std::string::npos) ? std::string(".") : p.substr(0, sl);
    return OK;
}

// CMS_import_guess (CMS_BasisSet.c:657-746): one value per line; a missing,
// short or (one-sidedly) asymmetric file gives a zero block.
std::vector<double> load_sad(const BasisDef &b, int e, int nf)
{
    std::vector<double> g((size_t) nf * nf, 0.0);
    std::string fn = b.dir + "/" + ETABLE[e] + ".dat";
    FILE *f = fopen(fn.c_str(), "r");
    if (!f) return g;
    char line[1024];
    bool bad = false;
    for (int k = 0; k < nf * nf; k++) {
        if (!fgets(line, sizeof(line), f)) { bad = true; break; }
        sscanf(line, "%le", &g[k]);
    }
    fclose(f);
    if (!bad)
        for (int j = 0; j < nf && !bad; j++)
            for (int k = 0; k < nf; k++)
                if (g[(size_t) j * nf + k] - g[(size_t) k * nf + j] > 1e-12) { bad = true; break; }
    if (bad) std::fill(g.begin(), g.end(), 0.0);
    return g;
}

double dfact(int n)
{
    double r = 1.0;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}

// Contracted-shell normalisation with unit-norm x^l component.
void normalize(int am, const std::vector<double> &al, const std::vector<double> &cc, std::vector<double> &out)
{
    const int n = (int) al.size();
    const double df = dfact(2 * am - 1);
    out.resize(n);
    for (int k = 0; k < n; k++)
        out[k] = cc[k] * pow(2.0 * al[k] / M_PI, 0.75) * pow(4.0 * al[k], 0.5 * am) / sqrt(df);
    double s = 0.0;
    for (int k = 0; k < n; k++)
        for (int l = 0; l < n; l++) {
            double p = al[k] + al[l];
            s += out[k] * out[l] * pow(M_PI / p, 1.5) * df / pow(2.0 * p, am);
        }
    double fct = 1.0 / sqrt(s);
    for (auto &v : out) v *= fct;
}

int build_shells(const Molecule &m, const BasisDef &b, HostShells &h)
{
    h = HostShells();
    for (int a = 0; a < m.natoms; a++) {
        auto it = b.elem.find(m.eid[a]);
        if (it == b.elem.end()) return ERR_INPUT;
        h.atom_bf0.push_back(h.nbf);
        for (const ShellDef &d : it->second) {
            std::vector<double> cn;
            normalize(d.am, d.ex, d.cc, cn);
            h.am.push_back(d.am);
            h.nprim.push_back((int) d.ex.size());
            h.poff.push_back((int) h.alpha.size());
            h.bfoff.push_back(h.nbf);
            h.atom_of.push_back(a);
            for (int k = 0; k < 3; k++) h.cen.push_back(m.xyz[3 * a + k]);
            h.alpha.insert(h.alpha.end(), d.ex.begin(), d.ex.end());
            h.coef.insert(h.coef.end(), cn.begin(), cn.end());
            h.nbf += ncart(d.am);
            h.maxam = std::max(h.maxam, d.am);
            h.nsh++;
        }
        h.atom_bf1.push_back(h.nbf);
    }
    h.bfoff.push_back(h.nbf);
    return OK;
}

// ------------------------------------------------------------------ device state
struct DevArrays {
    int *am = nullptr, *np = nullptr, *poff = nullptr, *bfoff = nullptr, *ids = nullptr;
    double *cen = nullptr, *al = nullptr, *co = nullptr;
    std::vector<int> am_start;
    DevShells view() const
    {
        return DevShells{0, am, np, poff, bfoff, cen, al, co};
    }
};

struct Engine {
    Molecule mol;
    BasisDef bas, dfbas;
    HostShells sh, ash;
    cudaStream_t s = nullptr;
    cudaEvent_t ev0[TINYSCF_T_COUNT], ev1[TINYSCF_T_COUNT];
    bool ev_used[TINYSCF_T_COUNT];
    double timers[TINYSCF_T_COUNT];
    double tsum[TINYSCF_T_COUNT];
    long long tcnt[TINYSCF_T_COUNT];
    long long h2d = 0, d2h = 0;       // bytes moved by explicit host<->device copies
    DevArrays dsh, dash;
    double *Z = nullptr, *xyz = nullptr;
    size_t nn = 0;
    double *S = nullptr, *H = nullptr, *X = nullptr, *F = nullptr, *Fp = nullptr, *D = nullptr, *J = nullptr,
           *K = nullptr, *Cocc = nullptr, *tmp = nullptr, *tmp2 = nullptr, *w = nullptr, *V = nullptr;
    double *F0 = nullptr, *R = nullptr;
    DiisState *diis = nullptr;
    double *sp_scr = nullptr, *bf_scr = nullptr, *df_scr = nullptr;
    int *piv = nullptr, *rank = nullptr;
    int *bf_atom = nullptr, *bf_atom_work = nullptr;   // atom of each basis function (SAD blocks)
    double *pwork = nullptr;
    // sparsity
    int nnz = 0, nu = 0, nup = 0;
    int *csr_j = nullptr, *csr_displs = nullptr, *csr_u = nullptr, *up_i = nullptr, *up_j = nullptr,
        *up_u = nullptr, *upair = nullptr;
    int2 *pairs3c = nullptr;
    std::vector<int> cls_start, cls_la, cls_lb;
    double *B = nullptr;
    int aux_p0 = 0, aux_ns = 0;   // aux columns [aux_p0, aux_p0 + aux_ns) of the DF tensor held (0: all)
    double *T = nullptr, *Kpart = nullptr;
    int2 *tiles = nullptr;
    int ksplit = 1, ksplit_max = 1, ksplit64 = 1, ktile = 64, khwide = 0;
    int2 *tiles128 = nullptr;
    bool d_from_cocc = false;   // D = Cocc Cocc^T (set by the engine's density builds, cleared by SAD / set_density)
    OzSyrk *oz = nullptr;   // K = T T^T on the integer tensor cores (used when kozaki)
    bool kozaki = false;
    long long n_ozaki = 0;  // K = T T^T builds that ran on the integer tensor cores
    double *Jt = nullptr, *Jpart = nullptr, *Jw = nullptr;
    int jblk = 1, jblk_max = 1;
    double *epart = nullptr, *E = nullptr;
    Eig *eig = nullptr;
    int kprec = TINYSCF_K_FP64;
    int dmode = TINYSCF_DENSITY_EIG;
    double *U = nullptr;          // occupied rows (nocc x nbf) in the orthogonal basis
    bool have_eig = false;        // V, w hold a full eigensolve of an earlier F'
    long long guard_restarts = 0; // SCF restarts from the SAD guess by the divergence guard
    SubspaceWork sw{};
    long long n_eig = 0, n_refine = 0;
    long long n3c_quartets = 0;   // (shell pair, aux shell) tuples of the last DF build
    // CUDA-graph iteration (Fock, DIIS and, with the refinement solver, the density)
    bool use_graph = false;
    bool capturing = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int graph_key = -1;
    bool gev_used[TINYSCF_T_COUNT];
    long long g_top = 0, g_body = 0;  // kernels per launch outside / per step inside the refinement loop
    cudaStream_t s_body = nullptr;
    RefineCtl *rctl = nullptr;        // device
    RefineCtl *h_rctl = nullptr;      // pinned host copy written by the graph
    double *h_E = nullptr;            // pinned host copy of the energy written by the graph
    // learned initial guess
    int guess_mode = TINYSCF_GUESS_SAD;
    int guess_used = TINYSCF_GUESS_SAD;
    GuessNet *gnet = nullptr;
    KMix *kmix = nullptr;
    double *Kmix = nullptr;
    float *B32 = nullptr;         // FP32 copy of the DF tensor for the mixed form's J
    int stage = 0;            // 1 hcore, 2 schwarz, 3 sparsity, 4 guess, 5 df
    bool F_is_orth = false;   // which buffer currently plays the reference's F_mat
    std::vector<void *> allocs;

    FockPlan plan() const
    {
        FockPlan p;
        p.nbf = sh.nbf;
        p.naux = aux_ns > 0 ? aux_ns : ash.nbf;
        p.nocc = 0;
        p.nnz = nnz;
        p.nup = nup;
        p.csr_j = csr_j;
        p.csr_displs = csr_displs;
        p.csr_u = csr_u;
        p.up_i = up_i;
        p.up_j = up_j;
        p.up_u = up_u;
        p.B = B;
        return p;
    }
};

Engine *E_(TinySCF_t t) { return (Engine *) t->dev; }

template <typename T>
int dalloc(Engine *e, T **p, size_t count)
{
    void *q = nullptr;
    if (dev_malloc(&q, sizeof(T) * (count ? count : 1), e->s) != OK) {
        fprintf(stderr, "[tinyscf] device allocation of %zu bytes failed\n", sizeof(T) * count);
        return ERR_ALLOC;
    }
    e->allocs.push_back(q);
    *p = (T *) q;
    return OK;
}

void dfree(Engine *e, void *p)
{
    if (!p) return;
    cudaStreamSynchronize(e->s);
    dev_free(p, e->s);
    auto it = std::find(e->allocs.begin(), e->allocs.end(), p);
    if (it != e->allocs.end()) e->allocs.erase(it);
}

void d2h(Engine *e, void *dst, const void *src, size_t bytes)
{
    cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
    e->d2h += (long long) bytes;
}

template <typename T>
int upload(Engine *e, T **p, const std::vector<T> &v)
{
    int rc = dalloc(e, p, v.size());
    if (rc) return rc;
    e->h2d += (long long) (sizeof(T) * v.size());
    if (!v.empty() && cudaMemcpyAsync(*p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, e->s) != cudaSuccess)
        return ERR_CUDA;
    return OK;
}

// Inside a stream capture the timer events become event-record nodes of the
// graph, so each graph launch times its phases like an eager iteration.
void tstart(Engine *e, int k)
{
    if (e->capturing) cudaEventRecordWithFlags(e->ev0[k], e->s, cudaEventRecordExternal);
    else cudaEventRecord(e->ev0[k], e->s);
}
void tstop(Engine *e, int k)
{
    if (e->capturing) {
        cudaEventRecordWithFlags(e->ev1[k], e->s, cudaEventRecordExternal);
        e->gev_used[k] = true;
    } else {
        cudaEventRecord(e->ev1[k], e->s);
        e->ev_used[k] = true;
    }
}
void tcollect(Engine *e)
{
    for (int k = 0; k < TINYSCF_T_COUNT; k++)
        if (e->ev_used[k]) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, e->ev0[k], e->ev1[k]) == cudaSuccess) {
                e->timers[k] = ms;
                e->tsum[k] += ms;
                e->tcnt[k]++;
            }
            e->ev_used[k] = false;
        }
}

int cuda_rc(const char *what)
{
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        fprintf(stderr, "[tinyscf] CUDA error after %s: %s\n", what, cudaGetErrorString(err));
        return ERR_CUDA;
    }
    return OK;
}

int sync_rc(Engine *e, const char *what)
{
    cudaError_t err = cudaStreamSynchronize(e->s);
    if (err == cudaSuccess) err = cudaGetLastError();
    if (err != cudaSuccess) {
        fprintf(stderr, "[tinyscf] CUDA error in %s: %s\n", what, cudaGetErrorString(err));
        return ERR_CUDA;
    }
    return OK;
}

int upload_shells(Engine *e, const HostShells &h, int maxl, DevArrays &d)
{
    int rc;
    if ((rc = upload(e, &d.am, h.am)) || (rc = upload(e, &d.np, h.nprim)) || (rc = upload(e, &d.poff, h.poff)) ||
        (rc = upload(e, &d.bfoff, h.bfoff)) || (rc = upload(e, &d.cen, h.cen)) || (rc = upload(e, &d.al, h.alpha)) ||
        (rc = upload(e, &d.co, h.coef)))
        return rc;
    std::vector<int> ids;
    d.am_start.assign(maxl + 2, 0);
    for (int l = 0; l <= maxl; l++) {
        d.am_start[l] = (int) ids.size();
        for (int i = 0; i < h.nsh; i++)
            if (h.am[i] == l) ids.push_back(i);
    }
    d.am_start[maxl + 1] = (int) ids.size();
    return upload(e, &d.ids, ids);
}

DevShells shells_view(const DevArrays &d, int nsh)
{
    DevShells v = d.view();
    v.nsh = nsh;
    return v;
}

// Host mirrors: 64-byte aligned and zero-filled. Blocks of 128 KB and more
// are fresh anonymous mappings, which are zero without being touched
// (transparent huge pages asked for, so the first write of a large one faults
// 2 MB at a time): an nbf x nbf mirror costs page faults only when a call
// first fills it. Smaller blocks come from the heap. afree tells the two apart
// by a registry of the mappings (any other pointer goes to free()).
constexpr size_t ABIG = (size_t) 128 << 10;

// The registry is never destroyed, so engines freed while the process exits still find it.
std::map<void *, size_t> &amaps()
{
    static auto *m = new std::map<void *, size_t>();
    return *m;
}

std::mutex &amaps_mu()
{
    static auto *mu = new std::mutex();
    return *mu;
}

void *amalloc(size_t bytes)
{
    if (bytes == 0) bytes = 64;
    if (bytes >= ABIG) {
        void *b = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
        if (b == MAP_FAILED) return nullptr;
        madvise(b, bytes, MADV_HUGEPAGE);   // advice only: ignored where huge pages are off
        std::lock_guard<std::mutex> lk(amaps_mu());
        amaps()[b] = bytes;
        return b;
    }
    void *b = nullptr;
    if (posix_memalign(&b, 64, bytes)) return nullptr;
    memset(b, 0, bytes);
    return b;
}

void afree(void *p)
{
    if (!p) return;
    size_t len = 0;
    {
        std::lock_guard<std::mutex> lk(amaps_mu());
        auto it = amaps().find(p);
        if (it != amaps().end()) {
            len = it->second;
            amaps().erase(it);
        }
    }
    if (len) munmap(p, len);
    else free(p);
}

#define RC(x)                    \
    do {                         \
        int rc__ = (x);          \
        if (rc__) return rc__;   \
    } while (0)

// ------------------------------------------------------------------ init
int init_impl(TinySCF_t t, const char *bas_fname, const char *df_bas_fname, const char *xyz_fname, int niters)
{
    double st = 0;
    {
        struct timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        st = ts.tv_sec + 1e-9 * ts.tv_nsec;
    }
    memset(t, 0, sizeof(*t));
    const char *vb = getenv("TINYSCF_VERBOSE");
    t->verbose = vb ? atoi(vb) : 1;
    const char *dv = getenv("TINYSCF_DEVICE");
    t->device = dv ? atoi(dv) : 0;
    Engine *e = new Engine();
    t->dev = e;
    RC(parse_xyz(xyz_fname, e->mol));
    RC(parse_gbs(bas_fname, e->bas));
    RC(parse_gbs(df_bas_fname, e->dfbas));
    RC(build_shells(e->mol, e->bas, e->sh));
    RC(build_shells(e->mol, e->dfbas, e->ash));
    if (e->sh.maxam > MAX_L_ORB || e->ash.maxam > MAX_L_AUX) {
        fprintf(stderr, "[tinyscf] shells beyond d (orbital) / f (auxiliary) are not supported\n");
        return ERR_UNSUPPORTED;
    }
    if (e->ash.nbf > 8192) {   // the J kernels keep one column group of 16 x 512 aux functions per thread block
        fprintf(stderr, "[tinyscf] %d auxiliary functions: at most 8192 are supported\n", e->ash.nbf);
        return ERR_UNSUPPORTED;
    }
    const int nbf = e->sh.nbf, naux = e->ash.nbf;
    t->natoms = e->mol.natoms;
    t->nshells = e->sh.nsh;
    t->nbasfuncs = nbf;
    t->n_occ = (e->mol.nelec - e->mol.Q) / 2;   // CMS_BasisSet.c:788-791
    t->charge = e->mol.Q;
    t->electron = e->mol.nelec;
    t->df_nbf = naux;
    t->df_nshells = e->ash.nsh;
    t->nshellpairs = t->nshells * t->nshells;
    t->mat_size = nbf * nbf;
    t->num_uniq_sp = (t->nshells + 1) * t->nshells / 2;
    t->max_dim = ncart(e->sh.maxam);
    t->niters = niters;
    t->iter = 0;
    t->ene_tol = 1e-11;
    t->shell_scrtol2 = 1e-11 * 1e-11;
    t->max_diis = MAX_DIIS;
    t->nuc_energy = e->mol.enuc;
    if (t->n_occ <= 0 || t->n_occ > nbf) return ERR_INPUT;
    if (t->verbose) {
        printf("Job information:\n");
        printf("    basis set            = %s\n", bas_fname);
        printf("    DF basis set         = %s\n", df_bas_fname);
        printf("    molecule             = %s\n", xyz_fname);
        printf("    # atoms              = %d\n", t->natoms);
        printf("    # shells             = %d\n", t->nshells);
        printf("    # basis functions    = %d\n", t->nbasfuncs);
        printf("    # DF shells          = %d\n", t->df_nshells);
        printf("    # DF basis functions = %d\n", t->df_nbf);
        printf("    # occupied orbits    = %d\n", t->n_occ);
        printf("    # charge             = %d\n", t->charge);
        printf("    # electrons          = %d\n", t->electron);
    }

    // host mirrors
    size_t nn = (size_t) nbf * nbf;
    t->sp_scrval = (double *) amalloc(sizeof(double) * t->nshellpairs);
    t->bf_pair_scrval = (double *) amalloc(sizeof(double) * nn);
    t->df_sp_scrval = (double *) amalloc(sizeof(double) * t->df_nshells);
    t->uniq_sp_lid = (int *) amalloc(sizeof(int) * t->num_uniq_sp);
    t->uniq_sp_rid = (int *) amalloc(sizeof(int) * t->num_uniq_sp);
    t->bf_pair_mask = (int *) amalloc(sizeof(int) * nn);
    t->bf_pair_j = (int *) amalloc(sizeof(int) * nn);
    t->bf_pair_diag = (int *) amalloc(sizeof(int) * nbf);
    t->bf_mask_displs = (int *) amalloc(sizeof(int) * (nbf + 1));
    t->shell_bf_sind = (int *) amalloc(sizeof(int) * (t->nshells + 1));
    t->shell_bf_num = (int *) amalloc(sizeof(int) * t->nshells);
    t->df_shell_bf_sind = (int *) amalloc(sizeof(int) * (t->df_nshells + 1));
    t->df_shell_bf_num = (int *) amalloc(sizeof(int) * t->df_nshells);
    for (int i = 0; i <= t->nshells; i++) t->shell_bf_sind[i] = e->sh.bfoff[i];
    for (int i = 0; i < t->nshells; i++) t->shell_bf_num[i] = ncart(e->sh.am[i]);
    for (int i = 0; i <= t->df_nshells; i++) t->df_shell_bf_sind[i] = e->ash.bfoff[i];
    for (int i = 0; i < t->df_nshells; i++) t->df_shell_bf_num[i] = ncart(e->ash.am[i]);
    double **mats[] = {&t->Hcore_mat, &t->S_mat, &t->F_mat, &t->D_mat, &t->J_mat, &t->K_mat, &t->X_mat, &t->tmp_mat};
    for (double **m : mats) *m = (double *) amalloc(sizeof(double) * nn);
    t->Cocc_mat = (double *) amalloc(sizeof(double) * nbf * t->n_occ);
    t->eigval = (double *) amalloc(sizeof(double) * nbf);
    t->ev_idx = (int *) amalloc(sizeof(int) * nbf);
    for (int i = 0; i < nbf; i++) t->ev_idx[i] = i;
    t->DIIS_bmax = -DBL_MAX;

    // device
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        fprintf(stderr, "[tinyscf] no CUDA device available: the engine has no CPU path\n");
        return ERR_CUDA;
    }
    if (t->device < 0 || t->device >= ndev) t->device = 0;
    TSCF_CUDA_CHECK(cudaSetDevice(t->device));
    TSCF_CUDA_CHECK(cudaStreamCreateWithFlags(&e->s, cudaStreamNonBlocking));
    for (int k = 0; k < TINYSCF_T_COUNT; k++) {
        TSCF_CUDA_CHECK(cudaEventCreate(&e->ev0[k]));
        TSCF_CUDA_CHECK(cudaEventCreate(&e->ev1[k]));
        e->ev_used[k] = false;
        e->timers[k] = 0.0;
        e->tsum[k] = 0.0;
        e->tcnt[k] = 0;
    }
    boys_table_init(e->s);
    RC(upload_shells(e, e->sh, MAX_L_ORB, e->dsh));
    RC(upload_shells(e, e->ash, MAX_L_AUX, e->dash));
    std::vector<double> Z(e->mol.natoms);
    for (int a = 0; a < e->mol.natoms; a++) Z[a] = e->mol.eid[a] + 1.0;
    RC(upload(e, &e->Z, Z));
    RC(upload(e, &e->xyz, e->mol.xyz));
    e->nn = nn;
    double **dm[] = {&e->S, &e->H, &e->X, &e->F, &e->Fp, &e->D, &e->J, &e->K, &e->tmp, &e->tmp2, &e->V};
    for (double **m : dm) {
        RC(dalloc(e, m, nn));
        cudaMemsetAsync(*m, 0, sizeof(double) * nn, e->s);
    }
    RC(dalloc(e, &e->Cocc, (size_t) nbf * t->n_occ));
    RC(dalloc(e, &e->w, nbf));
    RC(dalloc(e, &e->F0, nn * MAX_DIIS));
    RC(dalloc(e, &e->R, nn * MAX_DIIS));
    cudaMemsetAsync(e->F0, 0, sizeof(double) * nn * MAX_DIIS, e->s);
    cudaMemsetAsync(e->R, 0, sizeof(double) * nn * MAX_DIIS, e->s);
    RC(dalloc(e, &e->diis, 1));
    diis_init(e->diis, e->s);
    RC(dalloc(e, &e->sp_scr, (size_t) t->nshellpairs));
    RC(dalloc(e, &e->bf_scr, nn));
    RC(dalloc(e, &e->df_scr, (size_t) t->df_nshells));
    RC(dalloc(e, &e->piv, nbf));
    RC(dalloc(e, &e->rank, 1));
    RC(dalloc(e, &e->pwork, 2 * (size_t) nbf));
    RC(dalloc(e, &e->epart, ENERGY_BLOCKS));
    RC(dalloc(e, &e->E, 1));
    e->eig = eig_create(nbf, e->s);
    if (!e->eig) return ERR_CUDA;
    RC(sync_rc(e, "init"));
    t->mem_size = (double) nn * 8 * (13 + 2 * MAX_DIIS);
    {
        struct timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        t->init_time = ts.tv_sec + 1e-9 * ts.tv_nsec - st;
    }
    return OK;
}

// ------------------------------------------------------------------ Hcore, S, X (TinySCF.c:20-83)
int hcore_impl(TinySCF_t t)
{
    Engine *e = E_(t);
    if (!e) return ERR_STATE;
    const int nbf = t->nbasfuncs;
    tstart(e, TINYSCF_T_HCORE);
    DevShells v = shells_view(e->dsh, e->sh.nsh);
    launch_one_electron_grouped(v, e->dsh.ids, e->dsh.am_start.data(), e->mol.natoms, e->Z, e->xyz, e->S, e->H, nbf,
                                e->s);
    RC(cuda_rc("one-electron integrals"));
    RC(eig_run(e->eig, e->S, e->w, e->V, e->s));
    inv_sqrt_from_eig(e->w, e->V, e->X, e->tmp, nbf, e->s);
    tstop(e, TINYSCF_T_HCORE);
    RC(sync_rc(e, "Hcore/S/X"));
    tcollect(e);
    t->S_Hcore_time = e->timers[TINYSCF_T_HCORE] * 1e-3;
    d2h(e, t->S_mat, e->S, sizeof(double) * e->nn);
    d2h(e, t->Hcore_mat, e->H, sizeof(double) * e->nn);
    d2h(e, t->X_mat, e->X, sizeof(double) * e->nn);
    if (t->verbose)
        printf("TinySCF precompute Hcore, S, and X matrices over,  elapsed time = %.3lf (s)\n", t->S_Hcore_time);
    e->stage = std::max(e->stage, 1);
    return OK;
}

// ------------------------------------------------------------------ Schwarz (TinySCF.c:112-226)
int schwarz_impl(TinySCF_t t)
{
    Engine *e = E_(t);
    if (!e) return ERR_STATE;
    const int nbf = t->nbasfuncs, nsh = t->nshells;
    tstart(e, TINYSCF_T_SCHWARZ);
    DevShells v = shells_view(e->dsh, nsh), av = shells_view(e->dash, t->df_nshells);
    launch_schwarz_grouped(v, e->dsh.ids, e->dsh.am_start.data(), e->sp_scr, e->bf_scr, nbf, e->s);
    launch_df_scrval(av, e->df_scr, e->s);
    tstop(e, TINYSCF_T_SCHWARZ);
    RC(cuda_rc("Schwarz quartets"));
    RC(sync_rc(e, "Schwarz"));
    tcollect(e);
    // maxima and the unique shell pairs on the device (TinySCF.c:112-226); host mirrors of the results
    double *mx_d = nullptr;
    int *wk = nullptr, *first = nullptr, *second = nullptr;
    RC(dalloc(e, &mx_d, 2));
    RC(dalloc(e, &wk, (size_t) nsh * nsh + 2 * nsh + 1));
    RC(dalloc(e, &first, (size_t) nsh * (nsh + 1) / 2));
    RC(dalloc(e, &second, (size_t) nsh * (nsh + 1) / 2));
    RC(device_max(e->sp_scr, (long long) nsh * nsh, mx_d, e->s));
    RC(device_max(e->df_scr, t->df_nshells, mx_d + 1, e->s));
    double mx[2] = {0.0, 0.0};
    TSCF_CUDA_CHECK(cudaMemcpyAsync(mx, mx_d, sizeof(mx), cudaMemcpyDeviceToHost, e->s));
    RC(sync_rc(e, "screening maxima"));
    t->max_scrval = mx[0];
    t->max_df_scrval = mx[1];
    const double eta = t->shell_scrtol2 / t->max_df_scrval;
    int npairs = 0;
    RC(device_unique_shell_pairs(e->sp_scr, e->dsh.am, nsh, eta, wk, first, second, &npairs, e->s));
    RC(sync_rc(e, "unique shell pairs"));
    t->num_uniq_sp = npairs;
    d2h(e, t->uniq_sp_lid, first, sizeof(int) * npairs);
    d2h(e, t->uniq_sp_rid, second, sizeof(int) * npairs);
    d2h(e, t->sp_scrval, e->sp_scr, sizeof(double) * nsh * nsh);
    d2h(e, t->bf_pair_scrval, e->bf_scr, sizeof(double) * e->nn);
    d2h(e, t->df_sp_scrval, e->df_scr, sizeof(double) * t->df_nshells);
    dfree(e, mx_d);
    dfree(e, wk);
    dfree(e, first);
    dfree(e, second);
    t->shell_scr_time = e->timers[TINYSCF_T_SCHWARZ] * 1e-3;
    if (t->verbose)
        printf("TinySCF precompute shell screening info over,      elapsed time = %.3lf (s)\n", t->shell_scr_time);
    e->stage = std::max(e->stage, 2);
    return OK;
}

// ------------------------------------------------------------------ sparsity (TinySCF.c:228-280)
int sparsity_impl(TinySCF_t t)
{
    Engine *e = E_(t);
    if (!e || e->stage < 2) return ERR_STATE;
    const int nbf = t->nbasfuncs, naux = t->df_nbf, nocc = t->n_occ;
    const double eta = t->shell_scrtol2 / t->max_df_scrval;
    // the bf-pair CSR (TinySCF.c:228-258), the unique pairs and the upper lists on the device
    int *wk = nullptr, *mask = nullptr, *diag = nullptr;
    RC(dalloc(e, &wk, (size_t) 5 * nbf + 2));
    RC(dalloc(e, &mask, e->nn));
    RC(dalloc(e, &diag, nbf));
    RC(dalloc(e, &e->csr_displs, nbf + 1));
    RC(dalloc(e, &e->upair, e->nn));
    int totals[3] = {0, 0, 0};
    RC(device_bf_counts(e->bf_scr, nbf, eta, wk, e->csr_displs, totals, e->s));
    const int nnz = totals[0], nu = totals[1], nup = totals[2];
    RC(dalloc(e, &e->csr_j, nnz));
    RC(dalloc(e, &e->csr_u, nnz));
    RC(dalloc(e, &e->up_i, nup));
    RC(dalloc(e, &e->up_j, nup));
    RC(dalloc(e, &e->up_u, nup));
    RC(device_bf_fill(e->bf_scr, nbf, eta, wk, e->csr_displs, mask, diag, e->upair, e->csr_j, e->csr_u, e->up_i,
                      e->up_j, e->up_u, e->s));
    RC(sync_rc(e, "sparsity"));
    d2h(e, t->bf_pair_mask, mask, sizeof(int) * e->nn);
    d2h(e, t->bf_pair_j, e->csr_j, sizeof(int) * nnz);
    d2h(e, t->bf_mask_displs, e->csr_displs, sizeof(int) * (nbf + 1));
    d2h(e, t->bf_pair_diag, diag, sizeof(int) * nbf);
    dfree(e, wk);
    dfree(e, mask);
    dfree(e, diag);
    t->num_bf_pair_scr = nnz;
    e->nnz = nnz;
    e->nu = nu;
    e->nup = nup;
    // 3-centre work list: unique shell pairs grouped by (am(M), am(N)) class
    std::vector<int2> pl;
    e->cls_start.clear();
    e->cls_la.clear();
    e->cls_lb.clear();
    for (int la = 0; la <= MAX_L_ORB; la++)
        for (int lb = 0; lb <= la; lb++) {
            e->cls_start.push_back((int) pl.size());
            e->cls_la.push_back(la);
            e->cls_lb.push_back(lb);
            for (int k = 0; k < t->num_uniq_sp; k++) {
                int M = t->uniq_sp_lid[k], N = t->uniq_sp_rid[k];
                if (e->sh.am[M] == la && e->sh.am[N] == lb) pl.push_back(make_int2(M, N));
            }
        }
    e->cls_start.push_back((int) pl.size());
    RC(upload(e, &e->pairs3c, pl));
    // DF tensor, K and J buffers
    RC(dalloc(e, &e->B, (size_t) nu * naux));
    RC(dalloc(e, &e->T, (size_t) nbf * nocc * naux));
    const int nt = (nbf + 63) / 64, ntiles = nt * (nt + 1) / 2;
    const int nt2 = (nbf + 127) / 128, ntiles2 = nt2 * (nt2 + 1) / 2;
    const int nsm = num_sms();
    e->ksplit = std::max(1, std::min(64, (4 * nsm + ntiles - 1) / ntiles));
    e->ksplit64 = e->ksplit;
    const int h128 = std::max(1, std::min(64, (2 * nsm + ntiles2 - 1) / ntiles2));
    e->ksplit_max = std::min(64, 2 * std::max(e->ksplit, h128));   // room for the autotuner's candidates
    // untuned defaults by size: the larger register tiles pay off once there are enough of them
    if (nbf >= 384) {
        e->ktile = KSYRK_DMMA;
        e->ksplit = h128;
    }
    e->khwide = nbf >= 384 ? 2 : 0;
    RC(dalloc(e, &e->Kpart, (size_t) e->ksplit_max * nbf * nbf));
    {
        std::vector<int2> tl, tl2;
        for (int a = 0; a < nt; a++)
            for (int b = a; b < nt; b++) tl.push_back(make_int2(a, b));
        for (int a = 0; a < nt2; a++)
            for (int b = a; b < nt2; b++) tl2.push_back(make_int2(a, b));
        RC(upload(e, &e->tiles, tl));
        RC(upload(e, &e->tiles128, tl2));
    }
    FockPlan p = e->plan();
    e->jblk = build_J_part_blocks(p);
    e->jblk_max = std::max(e->jblk, std::min(4 * num_sms(), std::max(1, e->nup)));
    RC(dalloc(e, &e->Jt, naux));
    RC(dalloc(e, &e->Jpart, (size_t) e->jblk_max * naux));
    RC(dalloc(e, &e->Jw, std::max(1, e->nup)));
    RC(sync_rc(e, "sparsity"));
    t->mem_size = (double) nu * naux * 8 + (double) nbf * nocc * naux * 8 + 24.0 * e->nn * 8;
    if (t->verbose) {
        printf("TinySCF handling shell pair sparsity over,         elapsed time = %.3lf (s)\n", 0.0);
        printf("TinySCF memory allocation and initialization over, elapsed time = %.3lf (s)\n", 0.0);
        printf("TinySCF regular + density fitting memory usage = %.2lf MB \n", t->mem_size / 1048576.0);
        printf("#### Sparsity of basis function pairs = %lf, %lf\n", (double) t->num_uniq_sp / t->nshellpairs,
               (double) nnz / t->mat_size);
    }
    e->stage = std::max(e->stage, 3);
    return OK;
}

// ------------------------------------------------------------------ guess (TinySCF.c:282-364)
// SAD density (TinySCF.c:324-364): atomic blocks from the .dat files, scaled
// by 0.5 (and by the charge factor for ions).
void sad_blocks(Engine *e, TinySCF_t t, std::vector<double> &D)
{
    const int nbf = t->nbasfuncs;
    for (int a = 0; a < t->natoms; a++) {
        int el = e->mol.eid[a];
        int b0 = e->sh.atom_bf0[a], b1 = e->sh.atom_bf1[a], nf = b1 - b0;
        std::vector<double> g = load_sad(e->bas, el, nf);
        for (int i = 0; i < nf; i++)
            for (int j = 0; j < nf; j++) D[(size_t) (b0 + i) * nbf + b0 + j] = g[(size_t) i * nf + j];
    }
    double R = 1.0;
    if (t->charge != 0 && t->electron != 0) R = (double) (t->electron - t->charge) / (double) t->electron;
    R *= 0.5;
    for (auto &v : D) v *= R;
}

GuessAtoms guess_atoms(Engine *e)
{
    GuessAtoms g;
    g.natoms = e->mol.natoms;
    g.eid = e->mol.eid.data();
    g.xyz = e->mol.xyz.data();
    g.bf0 = e->sh.atom_bf0.data();
    g.shell_am.assign(g.natoms, {});
    for (int k = 0; k < e->sh.nsh; k++) g.shell_am[e->sh.atom_of[k]].push_back(e->sh.am[k]);
    return g;
}

// Predicted density blocks, then the idempotent density closest in the
// orthogonal basis: the n_occ-dimensional dominant subspace U of S^1/2 D S^1/2
// (S^1/2 = S X; subspace iteration for the learned guess, a full eigensolve
// for projected SAD), Cocc = X U^T, D = Cocc Cocc^T. Returns ERR_UNSUPPORTED when
// an atom is not covered by the network (the caller then uses SAD).
int learned_guess(TinySCF_t t)
{
    Engine *e = E_(t);
    const int n = t->nbasfuncs, o = t->n_occ;
    if (o <= 0 || o > n) return ERR_UNSUPPORTED;
    tstart(e, TINYSCF_T_GUESS);   // the timer spans the host-side features too
    std::vector<GuessPair> pairs;
    if (e->guess_mode == TINYSCF_GUESS_LEARNED) {
        GuessAtoms g = guess_atoms(e);
        if (guess_pairs(g, pairs)) return ERR_UNSUPPORTED;
        RC(guessnet_predict(e->gnet, pairs, g, e->D, n, e->s));
    } else {
        std::vector<double> D((size_t) n * n, 0.0);
        sad_blocks(e, t, D);
        TSCF_CUDA_CHECK(cudaMemcpyAsync(e->D, D.data(), sizeof(double) * D.size(), cudaMemcpyHostToDevice, e->s));
        e->h2d += (long long) (sizeof(double) * D.size());
    }
    dgemm(false, false, n, n, n, 1.0, e->S, n, e->X, n, 0.0, e->tmp, n, e->s);      // S^1/2
    dgemm(false, false, n, n, n, 1.0, e->tmp, n, e->D, n, 0.0, e->tmp2, n, e->s);
    dgemm(false, false, n, n, n, 1.0, e->tmp2, n, e->tmp, n, 0.0, e->F, n, e->s);   // S^1/2 D S^1/2
    int prc = ERR_NUMERIC;
    if (e->guess_mode == TINYSCF_GUESS_LEARNED) {
        // the prediction is close to a rank-n_occ projector: a few subspace
        // iterations find its occupied space at a fraction of an eigensolve
        prc = dominant_subspace(e->eig, e->F, e->V, e->tmp, e->tmp2, n, o, kGuessSubspaceIters, e->s);
        if (prc != OK && prc != ERR_NUMERIC) return prc;
        if (prc == OK) { density_from_rows(e->X, e->V, e->Cocc, e->D, n, o, e->s); e->d_from_cocc = true; }
    }
    if (prc != OK) {   // projected SAD, or a Gram matrix that lost definiteness
        RC(eig_run(e->eig, e->F, e->w, e->V, e->s));
        { density_from_eig(e->X, e->V + (size_t) (n - o) * n, e->Cocc, e->D, n, o, e->s); e->d_from_cocc = true; }
    }
    tstop(e, TINYSCF_T_GUESS);
    RC(cuda_rc("learned initial guess"));
    RC(sync_rc(e, "learned initial guess"));
    tcollect(e);
    d2h(e, t->D_mat, e->D, sizeof(double) * e->nn);
    d2h(e, t->Cocc_mat, e->Cocc, sizeof(double) * n * o);
    if (t->verbose)
        printf("TinySCF %s initial guess: %zu atom-pair blocks, %.3lf (s)\n",
               e->guess_mode == TINYSCF_GUESS_LEARNED ? "learned" : "projected SAD", pairs.size(),
               e->timers[TINYSCF_T_GUESS] * 1e-3);
    return OK;
}

int guess_impl(TinySCF_t t)
{
    Engine *e = E_(t);
    if (!e) return ERR_STATE;
    const int nbf = t->nbasfuncs, nocc = t->n_occ;
    e->have_eig = false;
    if ((e->guess_mode == TINYSCF_GUESS_LEARNED && e->gnet && e->stage >= 1) ||
        (e->guess_mode == TINYSCF_GUESS_SAD_PROJECTED && e->stage >= 1)) {
        int rc = learned_guess(t);
        if (rc == OK) {
            e->guess_used = e->guess_mode;
            e->stage = std::max(e->stage, 4);
            return OK;
        }
        if (rc != ERR_UNSUPPORTED) return rc;
        if (t->verbose) printf("TinySCF learned initial guess: an atom is not covered, using SAD\n");
    }
    e->guess_used = TINYSCF_GUESS_SAD;
    e->d_from_cocc = false;   // the SAD density is not Cocc Cocc^T
    tstart(e, TINYSCF_T_GUESS);   // the timer spans reading the SAD blocks too
    std::vector<double> D((size_t) nbf * nbf, 0.0);
    sad_blocks(e, t, D);
    TSCF_CUDA_CHECK(cudaMemcpyAsync(e->D, D.data(), sizeof(double) * D.size(), cudaMemcpyHostToDevice, e->s));
    e->h2d += (long long) (sizeof(double) * D.size());
    TSCF_CUDA_CHECK(cudaMemcpyAsync(e->tmp, e->D, sizeof(double) * D.size(), cudaMemcpyDeviceToDevice, e->s));
    // the SAD density is block diagonal by atom: the factorisation skips the
    // other atoms' exact zeros (TINYSCF_PSTF_BLOCKS=0: the dense kernel)
    const char *pb = getenv("TINYSCF_PSTF_BLOCKS");
    if (!(pb && pb[0] == '0')) {
        if (!e->bf_atom) {
            std::vector<int> ba(nbf, 0);
            for (int a = 0; a < t->natoms; a++)
                for (int b = e->sh.atom_bf0[a]; b < e->sh.atom_bf1[a]; b++) ba[b] = a;
            RC(upload(e, &e->bf_atom, ba));
            RC(dalloc(e, &e->bf_atom_work, nbf));
        }
        pivoted_cholesky(e->tmp, nbf, 1e-12, e->piv, e->rank, e->pwork, e->s, e->bf_atom, e->bf_atom_work);
    } else {
        pivoted_cholesky(e->tmp, nbf, 1e-12, e->piv, e->rank, e->pwork, e->s);
    }
    d2cocc_copy(e->tmp, e->rank, e->Cocc, nbf, nocc, e->s);
    tstop(e, TINYSCF_T_GUESS);
    RC(cuda_rc("initial guess"));
    RC(sync_rc(e, "initial guess"));
    tcollect(e);
    memcpy(t->D_mat, D.data(), sizeof(double) * D.size());
    d2h(e, t->Cocc_mat, e->Cocc, sizeof(double) * nbf * nocc);
    if (t->verbose)
        printf("TinySCF SAD initial guess: D mat / Cocc mat used %lf, %lf (s)\n", 0.0,
               e->timers[TINYSCF_T_GUESS] * 1e-3);
    e->stage = std::max(e->stage, 4);
    return OK;
}

// ------------------------------------------------------------------ autotuning of the Fock build
// The split count of the FP64 exchange (K = T T^T) and the number of row
// blocks of the J first pass are timed on this molecule's buffers (their
// contents do not matter for the timing; the first Fock build rewrites J and
// K) and the fastest kept; later molecules of the same sizes reuse the choice.
// K = T T^T on the integer tensor cores (ozaki.cu): TINYSCF_OZAKI=1 always,
// 0 never, otherwise when the autotuner times it faster than the FP64 kernels.
static int ozaki_mode()
{
    const char *v = getenv("TINYSCF_OZAKI");
    if (v && v[0] == '0') return 0;
    if (v && v[0] == '1') return 1;
    return -1;
}

static int ensure_oz(Engine *e, TinySCF_t t)
{
    if (e->oz) return OK;
    return oz_create(&e->oz, t->nbasfuncs, (long long) t->n_occ * e->plan().naux, e->s);
}

static bool use_oz(const Engine *e)
{
    const int om = ozaki_mode();
    return e->oz && (om == 1 || (om < 0 && e->kozaki));
}

int autotune_fock(TinySCF_t t)
{
    Engine *e = E_(t);
    if (ozaki_mode() == 1) RC(ensure_oz(e, t));
    if (!tune_enabled()) return OK;
    FockPlan p = e->plan();
    p.nocc = t->n_occ;
    char key[96];
    // candidates: tile * 1000 + split count
    snprintf(key, sizeof(key), "ksyrk:%d:%d:%d", t->nbasfuncs, t->n_occ, t->df_nbf);
    int c = tune_lookup(key);
    if (c < 0) {
        const int nt2 = (t->nbasfuncs + 127) / 128, ntiles2 = nt2 * (nt2 + 1) / 2;
        const int h128 = std::max(1, std::min(64, (2 * num_sms() + ntiles2 - 1) / ntiles2));
        std::vector<int> cand;
        for (int v : {std::max(1, e->ksplit64 / 2), e->ksplit64, std::min(e->ksplit_max, 2 * e->ksplit64)})
            if (std::find(cand.begin(), cand.end(), 64000 + v) == cand.end()) cand.push_back(64000 + v);
        for (int v : {std::max(1, h128 / 2), h128, std::min(e->ksplit_max, 2 * h128)}) {
            if (std::find(cand.begin(), cand.end(), 128000 + v) == cand.end()) cand.push_back(128000 + v);
            if (std::find(cand.begin(), cand.end(), KSYRK_DMMA * 1000 + v) == cand.end())
                cand.push_back(KSYRK_DMMA * 1000 + v);
        }
        c = tune_run(key, cand, [&](int k) {
            const int tile = k / 1000;
            build_K_syrk(p, e->T, e->K, e->Kpart, k % 1000, tile == 64 ? e->tiles : e->tiles128, e->s, tile);
        }, e->s);
    }
    if ((c / 1000 == 64 || c / 1000 == 128 || c / 1000 == KSYRK_DMMA) && c % 1000 >= 1 && c % 1000 <= e->ksplit_max) {
        e->ktile = c / 1000;
        e->ksplit = c % 1000;
        if (e->ktile == 64) e->ksplit64 = e->ksplit;
    }
    if (ozaki_mode() < 0 && t->nbasfuncs >= 128) {
        snprintf(key, sizeof(key), "ksyrk_oz:%d:%d:%d", t->nbasfuncs, t->n_occ, p.naux);
        c = tune_lookup(key);
        if (c != 0) {
            if (ensure_oz(e, t) != OK) {
                cudaGetLastError();
                c = 0;
            } else if (c < 0) {
                c = tune_run(key, {0, 1}, [&](int v) {
                    if (v) oz_syrk(e->oz, e->T, e->K, e->s);
                    else build_K_syrk(p, e->T, e->K, e->Kpart, e->ksplit, e->ktile == 64 ? e->tiles : e->tiles128,
                                      e->s, e->ktile);
                }, e->s);
            }
        }
        e->kozaki = c == 1;
        if (!e->kozaki && e->oz) {
            RC(sync_rc(e, "autotuning"));
            oz_destroy(e->oz);
            e->oz = nullptr;
        }
    }
    snprintf(key, sizeof(key), "khalf:%d:%d:%d:%d", t->nbasfuncs, t->n_occ, t->df_nbf, e->nnz);
    c = tune_lookup(key);
    if (const char *v = getenv("TINYSCF_KHALF"))   // a fixed half-transform variant (0-4) instead of timing them
        if (v[0] >= '0' && v[0] <= '4' && v[1] == 0) c = v[0] - '0';
    if (c < 0)
        c = tune_run(key, {0, 1, 2, 3, 4}, [&](int w) { build_K_halftransform(p, e->Cocc, e->T, e->s, w); }, e->s);
    if (c >= 0 && c <= 4) e->khwide = c;
    snprintf(key, sizeof(key), "jrows:%d:%d", e->nup, t->df_nbf);
    c = tune_lookup(key);
    if (c < 0) {
        std::vector<int> cand;
        const int nsm = num_sms();
        for (int v : {nsm, 2 * nsm, 4 * nsm})
            if (v <= e->jblk_max && std::find(cand.begin(), cand.end(), v) == cand.end()) cand.push_back(v);
        if (cand.empty()) cand.push_back(e->jblk);
        c = tune_run(key, cand, [&](int nb) { build_J(p, e->D, e->J, e->Jt, e->Jpart, nb, e->Jw, e->s); }, e->s);
    }
    if (c >= 1 && c <= e->jblk_max) e->jblk = c;
    return sync_rc(e, "autotuning");
}

// ------------------------------------------------------------------ DF tensor (build_DF_tensor.c:256-287)
int df_impl(TinySCF_t t)
{
    Engine *e = E_(t);
    if (!e || e->stage < 3) return ERR_STATE;
    const int nbf = t->nbasfuncs, naux = t->df_nbf;
    if (t->verbose) printf("---------- DF tensor construction ----------\n");
    double *pqA = nullptr, *Jpq = nullptr, *Jw = nullptr, *JV = nullptr, *Jinv = nullptr;
    RC(dalloc(e, &pqA, (size_t) e->nu * naux));
    TSCF_CUDA_CHECK(cudaMemsetAsync(pqA, 0, sizeof(double) * (size_t) e->nu * naux, e->s));
    ThreeCenterPlan pl;
    pl.pairs = e->pairs3c;
    pl.npairs = e->cls_start.back();
    pl.class_start = e->cls_start.data();
    pl.class_la = e->cls_la.data();
    pl.class_lb = e->cls_lb.data();
    pl.nclass = (int) e->cls_la.size();
    pl.aux_by_am = e->dash.ids;
    pl.aux_am_start = e->dash.am_start.data();
    pl.sp_scr = e->sp_scr;
    pl.df_scr = e->df_scr;
    pl.scrtol2 = t->shell_scrtol2;
    pl.upair_index = e->upair;
    pl.nbf = nbf;
    pl.naux = naux;
    DevShells v = shells_view(e->dsh, t->nshells), av = shells_view(e->dash, t->df_nshells);
    tstart(e, TINYSCF_T_3C);
    launch_three_center(v, av, pl, pqA, e->s);
    e->n3c_quartets = (long long) pl.npairs * t->df_nshells;
    tstop(e, TINYSCF_T_3C);
    RC(cuda_rc("3-centre integrals"));
    RC(dalloc(e, &Jpq, (size_t) naux * naux));
    RC(dalloc(e, &JV, (size_t) naux * naux));
    RC(dalloc(e, &Jinv, (size_t) naux * naux));
    RC(dalloc(e, &Jw, naux));
    TSCF_CUDA_CHECK(cudaMemsetAsync(Jpq, 0, sizeof(double) * (size_t) naux * naux, e->s));
    tstart(e, TINYSCF_T_2C);
    launch_two_center_grouped(av, e->dash.ids, e->dash.am_start.data(), e->df_scr, t->shell_scrtol2, Jpq, naux, e->s);
    tstop(e, TINYSCF_T_2C);
    RC(cuda_rc("2-centre integrals"));
    tstart(e, TINYSCF_T_INVSQRT);
    Eig *eg = eig_create(naux, e->s);
    if (!eg) return ERR_CUDA;
    int erc = eig_run(eg, Jpq, Jw, JV, e->s);
    inv_sqrt_from_eig(Jw, JV, Jinv, Jpq, naux, e->s);
    tstop(e, TINYSCF_T_INVSQRT);
    if (erc) { eig_destroy(eg); return erc; }
    tstart(e, TINYSCF_T_DFGEMM);
    // B = pqA (P|Q)^-1/2, or its aux columns [aux_p0, aux_p0 + aux_ns) for an aux-partitioned handle
    const int ncol = e->aux_ns > 0 ? e->aux_ns : naux;
    dgemm(false, false, e->nu, ncol, naux, 1.0, pqA, naux, Jinv + e->aux_p0, naux, 0.0, e->B, ncol, e->s);
    tstop(e, TINYSCF_T_DFGEMM);
    RC(cuda_rc("DF tensor GEMM"));
    int rc = sync_rc(e, "DF tensor");
    eig_destroy(eg);
    dfree(e, pqA);
    dfree(e, Jpq);
    dfree(e, JV);
    dfree(e, Jinv);
    dfree(e, Jw);
    if (rc) return rc;
    tcollect(e);
    if (t->verbose) {
        printf("* 3-center integral : %.3lf (s)\n", e->timers[TINYSCF_T_3C] * 1e-3);
        printf("* 2-center integral : %.3lf (s)\n", e->timers[TINYSCF_T_2C] * 1e-3);
        printf("* matrix inv-sqrt   : %.3lf (s)\n", e->timers[TINYSCF_T_INVSQRT] * 1e-3);
        printf("* build DF tensor   : %.3lf (s)\n", e->timers[TINYSCF_T_DFGEMM] * 1e-3);
        printf("---------- DF tensor construction finished ----------\n");
    }
    e->stage = std::max(e->stage, 5);
    return autotune_fock(t);
}

// ------------------------------------------------------------------ Fock (build_Fock.c:349-396)
int fock_device(TinySCF_t t, bool force_fp64 = false)
{
    Engine *e = E_(t);
    FockPlan p = e->plan();
    p.nocc = t->n_occ;
    tstart(e, TINYSCF_T_J);
    if (e->kprec == TINYSCF_K_MIXED && !force_fp64 && e->B32)
        build_J_f32(p, e->B32, e->D, e->J, e->Jt, e->Jpart, e->jblk, e->Jw, e->s);
    else
        build_J(p, e->D, e->J, e->Jt, e->Jpart, e->jblk, e->Jw, e->s);
    tstop(e, TINYSCF_T_J);
    const double *Kuse = e->K;
    if (e->kprec == TINYSCF_K_MIXED && !force_fp64) {
        tstart(e, TINYSCF_T_K_MIXED);
        RC(kmix_build(e->kmix, e->Cocc, e->S, e->Kmix, e->s, [&](int w) {
            if (w == 0) tstart(e, TINYSCF_T_K_HALF);
            else if (w == 1) {
                tstop(e, TINYSCF_T_K_HALF);
                tstart(e, TINYSCF_T_K_GEMM);
            } else {
                tstop(e, TINYSCF_T_K_GEMM);
            }
        }));
        tstop(e, TINYSCF_T_K_MIXED);
        Kuse = e->Kmix;
    } else {
        // with the pipelined half-transform and the integer-tensor-core K, the
        // row maxima that K's scaling needs come out of the half-transform
        unsigned long long *rm = (use_oz(e) && e->khwide >= 3) ? oz_rowmax(e->oz) : nullptr;
        tstart(e, TINYSCF_T_K_HT);
        build_K_halftransform(p, e->Cocc, e->T, e->s, e->khwide, rm);
        tstop(e, TINYSCF_T_K_HT);
        tstart(e, TINYSCF_T_K_SYRK);
        if (use_oz(e)) {
            RC(oz_syrk(e->oz, e->T, e->K, e->s, rm));
            e->n_ozaki++;
        } else
            build_K_syrk(p, e->T, e->K, e->Kpart, e->ksplit, e->ktile == 64 ? e->tiles : e->tiles128, e->s,
                         e->ktile);
        tstop(e, TINYSCF_T_K_SYRK);
    }
    if (Kuse != e->K)
        cudaMemcpyAsync(e->K, Kuse, sizeof(double) * e->nn, cudaMemcpyDeviceToDevice, e->s);
    tstart(e, TINYSCF_T_FOCK);
    build_F_energy(e->H, e->J, e->K, e->D, e->F, e->epart, t->nbasfuncs, e->s);
    energy_reduce(e->epart, e->E, e->s);
    tstop(e, TINYSCF_T_FOCK);
    e->F_is_orth = false;
    return cuda_rc("Fock build");
}

int fock_impl(TinySCF_t t, bool to_host)
{
    Engine *e = E_(t);
    if (!e || e->stage < 5) return ERR_STATE;
    RC(fock_device(t));
    RC(sync_rc(e, "Fock build"));
    tcollect(e);
    if (to_host) {
        d2h(e, t->J_mat, e->J, sizeof(double) * e->nn);
        d2h(e, t->K_mat, e->K, sizeof(double) * e->nn);
        d2h(e, t->F_mat, e->F, sizeof(double) * e->nn);
        d2h(e, &t->HF_energy, e->E, sizeof(double));
    }
    return OK;
}

// ------------------------------------------------------------------ DIIS (DIIS.c:12-123)
int diis_device(TinySCF_t t)
{
    Engine *e = E_(t);
    const int n = t->nbasfuncs;
    tstart(e, TINYSCF_T_DIIS);
    if (t->iter <= 1) {
        xtfx(e->X, e->F, e->Fp, e->tmp, n, e->s);
    } else {
        int md = t->max_diis;
        if (md < 1 || md > MAX_DIIS) md = MAX_DIIS;
        const int o = t->n_occ;
        if (e->d_from_cocc && o > 0 && 2 * o <= n)
            diis_step_cocc(e->diis, md, e->F, e->Cocc, o, e->S, e->X, e->Fp, e->F0, e->R, e->tmp, e->tmp2, n, e->s);
        else
            diis_step(e->diis, md, e->F, e->D, e->S, e->X, e->Fp, e->F0, e->R, e->tmp, e->tmp2, n, e->s);
    }
    tstop(e, TINYSCF_T_DIIS);
    e->F_is_orth = true;
    return cuda_rc("DIIS");
}

int diis_impl(TinySCF_t t, bool to_host)
{
    Engine *e = E_(t);
    if (!e || e->stage < 1) return ERR_STATE;
    RC(diis_device(t));
    RC(sync_rc(e, "DIIS"));
    tcollect(e);
    if (to_host) d2h(e, t->F_mat, e->Fp, sizeof(double) * e->nn);
    return OK;
}

// ------------------------------------------------------------------ density (build_density.c:37-69)
int density_device(TinySCF_t t)
{
    Engine *e = E_(t);
    const int n = t->nbasfuncs, o = t->n_occ;
    tstart(e, TINYSCF_T_DENSITY);
    const double *Fo = e->F_is_orth ? e->Fp : e->F;
    if (e->dmode == TINYSCF_DENSITY_REFINE && e->have_eig && o > 0 && o < n) {
        int steps = 0;
        double res = 0.0;
        RC(subspace_refine(Fo, e->V, e->w, e->U, n, o, e->sw, kRefineTol, kRefineSteps, &steps, &res, e->s));
        e->n_refine += steps;
        if (res < kRefineTol) {
            { density_from_rows(e->X, e->U, e->Cocc, e->D, n, o, e->s); e->d_from_cocc = true; }
            tstop(e, TINYSCF_T_DENSITY);
            return cuda_rc("density (subspace refinement)");
        }
    }
    RC(eig_run(e->eig, Fo, e->w, e->V, e->s));
    { density_from_eig(e->X, e->V, e->Cocc, e->D, n, o, e->s); e->d_from_cocc = true; }
    e->n_eig++;
    if (e->dmode == TINYSCF_DENSITY_REFINE && o > 0) {
        TSCF_CUDA_CHECK(cudaMemcpyAsync(e->U, e->V, sizeof(double) * (size_t) o * n, cudaMemcpyDeviceToDevice, e->s));
        e->have_eig = true;
    }
    tstop(e, TINYSCF_T_DENSITY);
    return cuda_rc("density");
}

int density_impl(TinySCF_t t, bool to_host)
{
    Engine *e = E_(t);
    if (!e || e->stage < 1) return ERR_STATE;
    RC(density_device(t));
    RC(sync_rc(e, "density"));
    tcollect(e);
    if (to_host) {
        d2h(e, t->D_mat, e->D, sizeof(double) * e->nn);
        d2h(e, t->Cocc_mat, e->Cocc, sizeof(double) * t->nbasfuncs * t->n_occ);
        d2h(e, t->eigval, e->w, sizeof(double) * t->nbasfuncs);
    }
    return OK;
}

int sync_host_impl(TinySCF_t t)
{
    Engine *e = E_(t);
    if (!e) return ERR_STATE;
    RC(sync_rc(e, "sync"));
    const int nbf = t->nbasfuncs;
    d2h(e, t->S_mat, e->S, sizeof(double) * e->nn);
    d2h(e, t->Hcore_mat, e->H, sizeof(double) * e->nn);
    d2h(e, t->X_mat, e->X, sizeof(double) * e->nn);
    d2h(e, t->F_mat, e->F_is_orth ? e->Fp : e->F, sizeof(double) * e->nn);
    d2h(e, t->D_mat, e->D, sizeof(double) * e->nn);
    d2h(e, t->J_mat, e->J, sizeof(double) * e->nn);
    d2h(e, t->K_mat, e->K, sizeof(double) * e->nn);
    d2h(e, t->Cocc_mat, e->Cocc, sizeof(double) * nbf * t->n_occ);
    d2h(e, t->eigval, e->w, sizeof(double) * nbf);
    DiisState st;
    d2h(e, &st, e->diis, sizeof(st));
    t->DIIS_len = st.len;
    t->DIIS_bmax_id = st.bmax_id;
    t->DIIS_bmax = st.bmax;
    return cuda_rc("sync to host");
}

// ------------------------------------------------------------------ CUDA-graph iteration
void graph_release(Engine *e)
{
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->gexec = nullptr;
    e->graph = nullptr;
    e->graph_key = -1;
}

// Capture one SCF iteration once DIIS has run eagerly once (t->iter >= 3): J, K (FP64 or
// mixed), Fock + energy, DIIS, and with the refinement solver the density with
// its step loop as a device-controlled WHILE node. The full-eigensolve density
// stays outside the graph (the eigensolver library is not captured).
int graph_capture(TinySCF_t t)
{
    Engine *e = E_(t);
    const int n = t->nbasfuncs, o = t->n_occ;
    graph_release(e);
    if (!e->s_body) TSCF_CUDA_CHECK(cudaStreamCreateWithFlags(&e->s_body, cudaStreamNonBlocking));
    if (!e->h_rctl) {
        TSCF_CUDA_CHECK(cudaMallocHost(&e->h_rctl, sizeof(RefineCtl)));
        TSCF_CUDA_CHECK(cudaMallocHost(&e->h_E, sizeof(double)));
        RC(dalloc(e, &e->rctl, 1));
    }
    const bool refine = e->dmode == TINYSCF_DENSITY_REFINE && o > 0 && o < n;
    if (refine) {
        RefineCtl c{};
        c.tol = kRefineTol;
        c.max_steps = kRefineSteps;
        TSCF_CUDA_CHECK(cudaMemcpyAsync(e->rctl, &c, sizeof(c), cudaMemcpyHostToDevice, e->s));
        TSCF_CUDA_CHECK(cudaStreamSynchronize(e->s));
    }
    for (int k = 0; k < TINYSCF_T_COUNT; k++) e->gev_used[k] = false;
    TSCF_CUDA_CHECK(cudaStreamBeginCapture(e->s, cudaStreamCaptureModeRelaxed));
    e->capturing = true;
    const long long l0 = g_launches;
    int rc = fock_device(t);
    if (!rc) rc = diis_device(t);
    if (!rc && refine) {
        tstart(e, TINYSCF_T_DENSITY);
        rc = subspace_refine_capture(e->Fp, e->V, e->w, e->U, n, o, e->sw, e->rctl, e->s, e->s_body, &e->g_body);
        if (!rc) {
            { density_from_rows(e->X, e->U, e->Cocc, e->D, n, o, e->s); e->d_from_cocc = true; }
            cudaMemcpyAsync(e->h_rctl, e->rctl, sizeof(RefineCtl), cudaMemcpyDeviceToHost, e->s);
        }
        tstop(e, TINYSCF_T_DENSITY);
    }
    if (!rc) cudaMemcpyAsync(e->h_E, e->E, sizeof(double), cudaMemcpyDeviceToHost, e->s);
    e->g_top = g_launches - l0;
    g_launches = l0;
    e->capturing = false;
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(e->s, &g);
    if (rc || ce != cudaSuccess) {
        cudaGetLastError();
        if (g) cudaGraphDestroy(g);
        fprintf(stderr, "[tinyscf] capture of the SCF iteration failed: %s\n",
                ce != cudaSuccess ? cudaGetErrorString(ce) : TinySCF_status_string(rc));
        return rc ? rc : ERR_CUDA;
    }
    e->graph = g;
    TSCF_CUDA_CHECK(cudaGraphInstantiate(&e->gexec, g, 0));
    e->graph_key = e->kprec * 2 + e->dmode;
    return OK;
}

// One SCF iteration (t->iter >= 3) through the captured graph; E receives the
// energy. Falls back to a full eigensolve when the refinement loop stopped
// without converging.
int graph_iteration(TinySCF_t t, double *E)
{
    Engine *e = E_(t);
    const int n = t->nbasfuncs, o = t->n_occ;
    if (!e->gexec || e->graph_key != e->kprec * 2 + e->dmode) RC(graph_capture(t));
    const bool refine = e->dmode == TINYSCF_DENSITY_REFINE && o > 0 && o < n;
    cudaEventRecord(e->ev0[TINYSCF_T_ITER], e->s);
    TSCF_CUDA_CHECK(cudaGraphLaunch(e->gexec, e->s));
    for (int k = 0; k < TINYSCF_T_COUNT; k++)
        if (e->gev_used[k]) e->ev_used[k] = true;
    e->F_is_orth = true;
    if (!refine) {
        RC(density_device(t));
    } else {
        TSCF_CUDA_CHECK(cudaStreamSynchronize(e->s));
        const RefineCtl c = *e->h_rctl;
        e->n_refine += c.step;
        g_launches += e->g_body * c.step;
        if (!c.converged) {
            // same as the eager solver's fallback: full eigensolve of this F'
            // (the DENSITY timer keeps the start the graph recorded)
            RC(eig_run(e->eig, e->Fp, e->w, e->V, e->s));
            { density_from_eig(e->X, e->V, e->Cocc, e->D, n, o, e->s); e->d_from_cocc = true; }
            TSCF_CUDA_CHECK(cudaMemcpyAsync(e->U, e->V, sizeof(double) * (size_t) o * n, cudaMemcpyDeviceToDevice, e->s));
            e->n_eig++;
            tstop(e, TINYSCF_T_DENSITY);
        }
    }
    g_launches += e->g_top;
    cudaEventRecord(e->ev1[TINYSCF_T_ITER], e->s);
    e->ev_used[TINYSCF_T_ITER] = true;
    RC(sync_rc(e, "SCF iteration (graph)"));
    *E = *e->h_E;
    e->d2h += (long long) sizeof(double);
    return OK;
}

// ------------------------------------------------------------------ SCF loop (TinySCF.c:378-435)
// Divergence guard of the SCF loop: an energy that is not finite, or that
// rises by more than kGuardRise Eh kGuardRises iterations in a row (from
// iteration 2, where DIIS starts), restarts the solve once from the SAD guess
// with an empty DIIS history; a second divergence in the same solve ends it
// with ERR_NUMERIC. A converging SCF never triggers it (rises there are
// rounding, far below kGuardRise), so it leaves the reference's iteration
// sequence untouched.
constexpr int kGuardRises = 4;
constexpr double kGuardRise = 1e-6;

int restart_from_sad(TinySCF_t t)
{
    Engine *e = E_(t);
    const int mode = e->guess_mode;
    e->guess_mode = TINYSCF_GUESS_SAD;
    const int rc = TinySCF_reset_scf(t);
    e->guess_mode = mode;
    e->guard_restarts++;
    return rc;
}

int scf_impl(TinySCF_t t)
{
    Engine *e = E_(t);
    if (!e || e->stage < 5) return ERR_STATE;
    if (e->aux_ns > 0) {
        fprintf(stderr, "[tinyscf] TinySCF_do_SCF: this handle holds a slice of the aux index; run the loop with a "
                        "reduction of J and K over the slices (TinySCF_set_JK)\n");
        return ERR_STATE;
    }
    if (t->verbose) {
        printf("TinySCF SCF iteration started...\n");
        printf("Nuclear energy = %.10lf\n", t->nuc_energy);
    }
    cudaEvent_t scf0, scf1;
    cudaEventCreate(&scf0);
    cudaEventCreate(&scf1);
    cudaEventRecord(scf0, e->s);
    t->iter = 0;
    double prev_energy = 0, energy_delta = 223;
    int rises = 0, restarts = 0;
    while ((t->iter < t->niters) && (energy_delta >= t->ene_tol)) {
        if (t->verbose) printf("--------------- Iteration %d ---------------\n", t->iter);
        double E = 0.0;
        if (e->use_graph && t->iter >= 3) {   // iteration 2 runs eagerly: its shapes get tuned before the capture
            RC(graph_iteration(t, &E));
        } else {
            tstart(e, TINYSCF_T_ITER);
            RC(fock_device(t));
            RC(diis_device(t));
            RC(density_device(t));
            tstop(e, TINYSCF_T_ITER);
            TSCF_CUDA_CHECK(cudaMemcpyAsync(&E, e->E, sizeof(double), cudaMemcpyDeviceToHost, e->s));
            e->d2h += (long long) sizeof(double);
            RC(sync_rc(e, "SCF iteration"));
        }
        tcollect(e);
        t->HF_energy = E;
        rises = (t->iter >= 2 && E > prev_energy + kGuardRise) ? rises + 1 : 0;
        if (!std::isfinite(E) || rises >= kGuardRises) {
            if (restarts > 0) {
                fprintf(stderr, "[tinyscf] SCF diverged again at iteration %d (energy %.10g): giving up\n", t->iter,
                        E + t->nuc_energy);
                return ERR_NUMERIC;
            }
            fprintf(stderr, "[tinyscf] SCF diverging at iteration %d (energy %.10g): restarting from the SAD guess\n",
                    t->iter, E + t->nuc_energy);
            RC(restart_from_sad(t));
            restarts++;
            rises = 0;
            prev_energy = 0;
            energy_delta = 223;
            t->iter = 0;
            continue;
        }
        energy_delta = fabs(t->HF_energy - prev_energy);
        prev_energy = t->HF_energy;
        if (t->verbose) {
            const double *tm = e->timers;
            printf("* Build Fock matrix     : %.3lf (s)\n", (tm[TINYSCF_T_J] + tm[TINYSCF_T_K_HT] + tm[TINYSCF_T_K_SYRK] + tm[TINYSCF_T_FOCK]) * 1e-3);
            printf("|---- J matrix          |---- %.3lf (s)\n", tm[TINYSCF_T_J] * 1e-3);
            printf("|---- aux. K tensor     |---- %.3lf (s)\n", tm[TINYSCF_T_K_HT] * 1e-3);
            printf("|---- K matrix          |---- %.3lf (s)\n", tm[TINYSCF_T_K_SYRK] * 1e-3);
            printf("* DIIS procedure        : %.3lf (s)\n", tm[TINYSCF_T_DIIS] * 1e-3);
            printf("* Build density matrix  : %.3lf (s)\n", tm[TINYSCF_T_DENSITY] * 1e-3);
            printf("* Iteration runtime     = %.3lf (s)\n", tm[TINYSCF_T_ITER] * 1e-3);
            printf("* Energy = %.10lf (%.10lf)", t->HF_energy + t->nuc_energy, t->HF_energy);
            if (t->iter > 0) printf(", delta = %e\n", energy_delta);
            else printf("\n");
        }
        if (t->iter == 0) energy_delta = 223;
        t->iter++;
    }
    if (e->kprec == TINYSCF_K_MIXED) {
        // one FP64 Fock build on the converged density; its energy is the result
        tstart(e, TINYSCF_T_FINAL);
        RC(fock_device(t, true));
        tstop(e, TINYSCF_T_FINAL);
        double E = 0.0;
        TSCF_CUDA_CHECK(cudaMemcpyAsync(&E, e->E, sizeof(double), cudaMemcpyDeviceToHost, e->s));
        e->d2h += (long long) sizeof(double);
        RC(sync_rc(e, "final FP64 Fock build"));
        tcollect(e);
        if (t->verbose)
            printf("* Final FP64 Fock build: Energy = %.10lf (%.10lf), mixed-precision energy was %.10lf\n",
                   E + t->nuc_energy, E, t->HF_energy + t->nuc_energy);
        t->HF_energy = E;
        int fl = kmix_error_flag();
        if (fl) {
            fprintf(stderr, "[tinyscf] tensor-core K: a bounded wait timed out (code %d)\n", fl);
            return ERR_CUDA;
        }
    }
    if (e->oz) {
        const int fl = oz_error_flag();
        if (fl) {
            fprintf(stderr, "[tinyscf] integer tensor-core K: a bounded wait timed out (code %d)\n", fl);
            return ERR_CUDA;
        }
    }
    cudaEventRecord(scf1, e->s);
    cudaEventSynchronize(scf1);
    float ms = 0;
    cudaEventElapsedTime(&ms, scf0, scf1);
    e->timers[TINYSCF_T_SCF] = ms;
    cudaEventDestroy(scf0);
    cudaEventDestroy(scf1);
    if (t->verbose) printf("--------------- SCF iterations finished ---------------\n");
    return sync_host_impl(t);
}

// Host wall-clock seconds (for the release breakdown of TINYSCF_VERBOSE >= 2).
static double wall_s()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

void free_impl(TinySCF_t t)
{
    // with verbose >= 2, the wall time of each release step (ms)
    const bool report = t->verbose >= 2;
    double tl = wall_s(), ms[8] = {};
    auto lap = [&](int k) {
        const double now = wall_s();
        ms[k] += 1e3 * (now - tl);
        tl = now;
    };
    Engine *e = E_(t);
    if (e) {
        if (e->s) cudaStreamSynchronize(e->s);
        lap(0);
        graph_release(e);
        if (e->s_body) cudaStreamDestroy(e->s_body);
        lap(1);
        if (e->h_rctl) cudaFreeHost(e->h_rctl);
        if (e->h_E) cudaFreeHost(e->h_E);
        lap(2);
        guessnet_free(e->gnet);
        lap(3);
        eig_destroy(e->eig);
        kmix_destroy(e->kmix);
        oz_destroy(e->oz);
        lap(4);
        for (void *p : e->allocs) dev_free(p, e->s);
        e->allocs.clear();
        if (e->s) cudaStreamSynchronize(e->s);
        lap(5);
        if (e->s) {
            for (int k = 0; k < TINYSCF_T_COUNT; k++) {
                cudaEventDestroy(e->ev0[k]);
                cudaEventDestroy(e->ev1[k]);
            }
            cudaStreamDestroy(e->s);
        }
        delete e;
        t->dev = nullptr;
        lap(6);
    }
    void *hp[] = {t->sp_scrval, t->bf_pair_scrval, t->df_sp_scrval, t->uniq_sp_lid, t->uniq_sp_rid, t->bf_pair_mask,
                  t->bf_pair_j, t->bf_pair_diag, t->bf_mask_displs, t->shell_bf_sind, t->shell_bf_num,
                  t->df_shell_bf_sind, t->df_shell_bf_num, t->Hcore_mat, t->S_mat, t->F_mat, t->D_mat, t->J_mat,
                  t->K_mat, t->X_mat, t->tmp_mat, t->Cocc_mat, t->eigval, t->ev_idx};
    for (void *p : hp) afree(p);
    lap(7);
    if (report)
        printf("* release (ms): sync %.2f, graphs %.2f, pinned %.2f, guess net %.2f, eig/K-mix/rank-k %.2f, "
               "buffers %.2f, events/stream %.2f, host mirrors %.2f\n",
               ms[0], ms[1], ms[2], ms[3], ms[4], ms[5], ms[6], ms[7]);
}

void die(const char *fn, int rc)
{
    fprintf(stderr, "[tinyscf] %s failed: %s\n", fn, TinySCF_status_string(rc));
    abort();
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

TinySCF_t TinySCF_alloc(void)
{
    return (TinySCF_t) calloc(1, sizeof(struct TinySCF_struct));
}

size_t TinySCF_struct_size(void) { return sizeof(struct TinySCF_struct); }

const char *TinySCF_status_string(int status)
{
    switch (status) {
    case TINYSCF_OK: return "success";
    case TINYSCF_ERR_CUDA: return "CUDA error";
    case TINYSCF_ERR_FILEIO: return "cannot open input file";
    case TINYSCF_ERR_INPUT: return "invalid input";
    case TINYSCF_ERR_UNSUPPORTED: return "unsupported input";
    case TINYSCF_ERR_ALLOC: return "device allocation failed";
    case TINYSCF_ERR_NUMERIC: return "numerical failure";
    case TINYSCF_ERR_STATE: return "call out of order";
    default: return "unknown status";
    }
}

#define STATUS_WRAP(name, call)            \
    int name(TinySCF_t t)                  \
    {                                      \
        if (!t) return TINYSCF_ERR_STATE;  \
        int rc = (call);                   \
        t->status = rc;                    \
        return rc;                         \
    }

int TinySCF_init_status(TinySCF_t t, const char *bas, const char *dfbas, const char *xyz, int niters)
{
    if (!t) return TINYSCF_ERR_STATE;
    int rc = init_impl(t, bas, dfbas, xyz, niters);
    t->status = rc;
    return rc;
}
STATUS_WRAP(TinySCF_compute_Hcore_Ovlp_mat_status, hcore_impl(t))
STATUS_WRAP(TinySCF_compute_sq_Schwarz_scrvals_status, schwarz_impl(t))
STATUS_WRAP(TinySCF_prepare_sparsity_status, sparsity_impl(t))
STATUS_WRAP(TinySCF_get_initial_guess_status, guess_impl(t))
STATUS_WRAP(TinySCF_build_DF_tensor_status, df_impl(t))
STATUS_WRAP(TinySCF_build_FockMat_status, fock_impl(t, true))
STATUS_WRAP(TinySCF_DIIS_status, diis_impl(t, true))
STATUS_WRAP(TinySCF_build_DenMat_status, density_impl(t, true))
STATUS_WRAP(TinySCF_do_SCF_status, scf_impl(t))

int TinySCF_free_status(TinySCF_t t)
{
    if (!t) return TINYSCF_ERR_STATE;
    free_impl(t);
    free(t);
    return TINYSCF_OK;
}

int TinySCF_set_density(TinySCF_t t, const double *D, const double *Cocc)
{
    if (!t || !t->dev) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    if (D && cudaMemcpy(e->D, D, sizeof(double) * e->nn, cudaMemcpyHostToDevice) != cudaSuccess) return TINYSCF_ERR_CUDA;
    if (D || Cocc) e->d_from_cocc = false;   // a caller's pair need not satisfy D = Cocc Cocc^T
    if (Cocc && cudaMemcpy(e->Cocc, Cocc, sizeof(double) * t->nbasfuncs * t->n_occ, cudaMemcpyHostToDevice) != cudaSuccess)
        return TINYSCF_ERR_CUDA;
    if (D) memcpy(t->D_mat, D, sizeof(double) * e->nn);
    if (Cocc) memcpy(t->Cocc_mat, Cocc, sizeof(double) * t->nbasfuncs * t->n_occ);
    return TINYSCF_OK;
}

int TinySCF_set_fock(TinySCF_t t, const double *F, int orthogonal)
{
    if (!t || !t->dev || !F) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    if (cudaMemcpy(orthogonal ? e->Fp : e->F, F, sizeof(double) * e->nn, cudaMemcpyHostToDevice) != cudaSuccess)
        return TINYSCF_ERR_CUDA;
    e->F_is_orth = orthogonal != 0;
    memcpy(t->F_mat, F, sizeof(double) * e->nn);
    return TINYSCF_OK;
}

int TinySCF_sync_host(TinySCF_t t)
{
    if (!t || !t->dev) return TINYSCF_ERR_STATE;
    return sync_host_impl(t);
}

int TinySCF_get_df_tensor(TinySCF_t t, double *out)
{
    if (!t || !t->dev || !out) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    if (e->stage < 5) return TINYSCF_ERR_STATE;
    const int naux = e->aux_ns > 0 ? e->aux_ns : t->df_nbf;
    // one row per ordered CSR entry, gathered from the unique-pair tensor
    std::vector<int> cu(e->nnz);
    d2h(e, cu.data(), e->csr_u, sizeof(int) * e->nnz);
    for (int k = 0; k < e->nnz; k++)
        if (cudaMemcpy(out + (size_t) k * naux, e->B + (size_t) cu[k] * naux, sizeof(double) * naux,
                       cudaMemcpyDeviceToHost) != cudaSuccess)
            return TINYSCF_ERR_CUDA;
    return TINYSCF_OK;
}

int TinySCF_set_k_precision(TinySCF_t t, int mode)
{
    if (!t || !t->dev) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    if (mode != TINYSCF_K_FP64 && mode != TINYSCF_K_MIXED) return TINYSCF_ERR_INPUT;
    if (mode == TINYSCF_K_MIXED) {
        if (e->stage < 5) return TINYSCF_ERR_STATE;   // needs the DF tensor
        if (!e->kmix) {
            FockPlan p = e->plan();
            p.nocc = t->n_occ;
            int rc = kmix_create(&e->kmix, p, t->bf_mask_displs, e->s);
            if (rc) return rc;
            rc = dalloc(e, &e->Kmix, e->nn);
            if (rc) return rc;
            rc = dalloc(e, &e->B32, (size_t) e->nu * p.naux);
            if (rc) return rc;
            convert_f32(e->B, e->B32, (size_t) e->nu * p.naux, e->s);
        }
        kmix_reset(e->kmix, e->s);
        if (sync_rc(e, "mixed K set-up")) return TINYSCF_ERR_CUDA;
    }
    e->kprec = mode;
    return TINYSCF_OK;
}

int TinySCF_set_density_solver(TinySCF_t t, int mode)
{
    if (!t || !t->dev) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    if (mode != TINYSCF_DENSITY_EIG && mode != TINYSCF_DENSITY_REFINE) return TINYSCF_ERR_INPUT;
    if (e->stage < 1) return TINYSCF_ERR_STATE;
    const int n = t->nbasfuncs, o = t->n_occ;
    if (mode == TINYSCF_DENSITY_REFINE && !e->U && o > 0) {
        const size_t no = (size_t) n * o, oo = (size_t) o * o;
        double **bufs[] = {&e->U, &e->sw.A, &e->sw.R, &e->sw.Cv};
        for (double **b : bufs)
            if (dalloc(e, b, no)) return TINYSCF_ERR_ALLOC;
        double **small[] = {&e->sw.UA, &e->sw.M, &e->sw.Y, &e->sw.Z, &e->sw.T, &e->sw.W};
        for (double **b : small)
            if (dalloc(e, b, oo)) return TINYSCF_ERR_ALLOC;
        if (dalloc(e, &e->sw.res, 1)) return TINYSCF_ERR_ALLOC;
    }
    e->dmode = mode;
    e->have_eig = false;
    return TINYSCF_OK;
}

int TinySCF_set_graph(TinySCF_t t, int on)
{
    if (!t || !t->dev) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    if (on != 0 && on != 1) return TINYSCF_ERR_INPUT;
    if (!on) {
        cudaStreamSynchronize(e->s);
        graph_release(e);
    }
    e->use_graph = on != 0;
    return TINYSCF_OK;
}

int TinySCF_set_guess(TinySCF_t t, int mode, const char *weights)
{
    if (!t || !t->dev) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    if (mode != TINYSCF_GUESS_SAD && mode != TINYSCF_GUESS_LEARNED && mode != TINYSCF_GUESS_SAD_PROJECTED)
        return TINYSCF_ERR_INPUT;
    if (weights) {
        GuessNet *net = nullptr;
        int rc = guessnet_load(&net, weights);
        if (rc) {
            fprintf(stderr, "[tinyscf] cannot load guess network weights from %s: %s\n", weights,
                    TinySCF_status_string(rc));
            return rc;
        }
        guessnet_free(e->gnet);
        e->gnet = net;
    }
    if (mode == TINYSCF_GUESS_LEARNED && !e->gnet) return TINYSCF_ERR_STATE;
    e->guess_mode = mode;
    return TINYSCF_OK;
}

int TinySCF_guess_used(TinySCF_t t)
{
    if (!t || !t->dev) return -TINYSCF_ERR_STATE;
    return E_(t)->guess_used;
}

long long TinySCF_guess_dataset(TinySCF_t t, const double *D, float *feat, float *target, int *type, long long cap)
{
    if (!t || !t->dev || !D) return -TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    GuessAtoms g = guess_atoms(e);
    std::vector<GuessPair> pairs;
    if (guess_pairs(g, pairs)) return -TINYSCF_ERR_UNSUPPORTED;
    if (!feat) return (long long) pairs.size();
    if ((long long) pairs.size() > cap) return -TINYSCF_ERR_INPUT;
    for (size_t k = 0; k < pairs.size(); k++) {
        std::memcpy(feat + k * G_DIN, pairs[k].feat, sizeof(float) * G_DIN);
        float *o = target + k * G_MAXF * G_MAXF;
        std::memset(o, 0, sizeof(float) * G_MAXF * G_MAXF);
        guess_local_block(g, pairs[k], D, t->nbasfuncs, o);
        type[k] = pairs[k].type;
    }
    return (long long) pairs.size();
}

long long TinySCF_guess_pairs(int natoms, const int *elem, const double *xyz, const int *nshell, const int *shell_am,
                              int *ab, int *type, double *frame, float *feat, long long cap)
{
    if (natoms <= 0 || !elem || !xyz || !nshell || !shell_am || cap < 0) return -TINYSCF_ERR_INPUT;
    GuessAtoms g;
    g.natoms = natoms;
    g.eid = elem;
    g.xyz = xyz;
    std::vector<int> bf0(natoms);
    g.shell_am.assign(natoms, {});
    int sh = 0, nf = 0;
    for (int a = 0; a < natoms; a++) {
        if (nshell[a] < 0) return -TINYSCF_ERR_INPUT;
        bf0[a] = nf;
        for (int k = 0; k < nshell[a]; k++, sh++) {
            const int l = shell_am[sh];
            if (l < 0 || l > 2) return -TINYSCF_ERR_UNSUPPORTED;
            g.shell_am[a].push_back(l);
            nf += (l + 1) * (l + 2) / 2;
        }
    }
    g.bf0 = bf0.data();
    std::vector<GuessPair> pairs;
    if (guess_pairs(g, pairs)) return -TINYSCF_ERR_UNSUPPORTED;
    const long long n = (long long) pairs.size();
    if (!ab && !type && !frame && !feat) return n;
    if (n > cap) return -TINYSCF_ERR_INPUT;
    for (long long k = 0; k < n; k++) {
        const GuessPair &p = pairs[k];
        if (ab) {
            ab[2 * k] = p.a;
            ab[2 * k + 1] = p.b;
        }
        if (type) type[k] = p.type;
        if (frame) std::memcpy(frame + 9 * k, p.Qf, sizeof(p.Qf));
        if (feat) std::memcpy(feat + (size_t) k * G_DIN, p.feat, sizeof(p.feat));
    }
    return n;
}

int TinySCF_guess_rotation(const int *shell_am, int nshells, const double *Q, double *M)
{
    if (!shell_am || !Q || !M || nshells <= 0) return TINYSCF_ERR_INPUT;
    std::vector<int> am(shell_am, shell_am + nshells);
    int nf = 0;
    for (int l : am) {
        if (l < 0 || l > 2) return TINYSCF_ERR_UNSUPPORTED;
        nf += (l + 1) * (l + 2) / 2;
    }
    guess_atom_rotation(am, Q, M, nf);
    return TINYSCF_OK;
}

int TinySCF_guess_train(const float *feat, const float *target, const int *type, long long n, int epochs, int batch,
                        float lr, unsigned seed, const char *path, float *final_loss)
{
    if (!feat || !target || !type || n <= 0 || epochs <= 0 || batch <= 0 || !path) return TINYSCF_ERR_INPUT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return TINYSCF_ERR_CUDA;
    }
    return guessnet_train(feat, target, type, n, epochs, batch, lr, seed, path, final_loss);
}

int TinySCF_guess_mlp_grad(int din, int hid, int dout, const float *params, const float *X, const float *T, int n,
                           float *grad, float *loss)
{
    if (!params || !X || !T || !grad || !loss || din <= 0 || hid <= 0 || dout <= 0 || n <= 0) return TINYSCF_ERR_INPUT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return TINYSCF_ERR_CUDA;
    }
    return guessnet_grad(din, hid, dout, params, X, T, n, grad, loss);
}

int TinySCF_reset_scf(TinySCF_t t)
{
    if (!t || !t->dev) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    if (e->stage < 4) return TINYSCF_ERR_STATE;
    int verbose = t->verbose;
    t->verbose = 0;
    int rc = guess_impl(t);
    t->verbose = verbose;
    if (rc) return rc;
    diis_init(e->diis, e->s);
    cudaMemsetAsync(e->F0, 0, sizeof(double) * e->nn * MAX_DIIS, e->s);
    cudaMemsetAsync(e->R, 0, sizeof(double) * e->nn * MAX_DIIS, e->s);
    if (e->kmix) kmix_reset(e->kmix, e->s);
    e->have_eig = false;
    t->iter = 0;
    t->DIIS_len = 0;
    t->DIIS_bmax_id = 0;
    t->DIIS_bmax = -DBL_MAX;
    return sync_rc(e, "reset");
}

int TinySCF_get_timing_stats(TinySCF_t t, double *sum_ms, long long *count, int n)
{
    if (!t || !t->dev) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    for (int k = 0; k < n && k < TINYSCF_T_COUNT; k++) {
        if (sum_ms) sum_ms[k] = e->tsum[k];
        if (count) count[k] = e->tcnt[k];
    }
    return TINYSCF_OK;
}

int TinySCF_reset_timing_stats(TinySCF_t t)
{
    if (!t || !t->dev) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    for (int k = 0; k < TINYSCF_T_COUNT; k++) {
        e->tsum[k] = 0.0;
        e->tcnt[k] = 0;
    }
    return TINYSCF_OK;
}

int TinySCF_get_counters(TinySCF_t t, long long *out, int n)
{
    if (!t || !t->dev || !out) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    long long v[8] = {g_launches, e->h2d,         e->d2h,           e->n_eig,
                      e->n_refine, e->n3c_quartets, e->guard_restarts, e->n_ozaki};
    for (int k = 0; k < n && k < 8; k++) out[k] = v[k];
    return TINYSCF_OK;
}

int TinySCF_get_timings(TinySCF_t t, double *ms, int n)
{
    if (!t || !t->dev || !ms) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    for (int k = 0; k < n && k < TINYSCF_T_COUNT; k++) ms[k] = e->timers[k];
    return TINYSCF_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ batched SCF
// Many molecules, each set up through the single-molecule API, iterate
// together: every SCF phase is one launch over all molecules still iterating
// (batch.cu), the density eigensolves run per molecule on the engine's own
// eigensolver. Each molecule follows the reference loop
// (TinySCF.c:378-435) with its own ene_tol, niters and convergence.
struct TinySCF_batch_struct {
    std::vector<TinySCF_t> mols;
    cudaStream_t s = nullptr;
    BatchPlan plan;
    std::vector<void *> mem;
    struct Group {
        int n = 0;
        std::vector<int> members;
        double *A = nullptr, *W = nullptr;
        Eig *eig = nullptr;
    };
    std::vector<Group> groups;
    double *d_Eall = nullptr;
    int *d_active = nullptr;
    int *d_kact = nullptr;             // molecules whose K the batched FP64 kernels build this iteration
    int *d_need = nullptr;             // molecules whose density takes an eigensolve this iteration
    std::vector<char> mixed;           // molecules with the tensor-core incremental K
    KMixBatch *kmb = nullptr;          // their K builds, one launch per tensor-core kernel (null: one by one)
    std::vector<int> kmb_mol, kmb_act; // batch index and active flag of each of them
    std::vector<const double *> kmb_C, kmb_S;
    std::vector<double *> kmb_K;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double scf_ms = 0.0;
    int iterations = 0;
    long long launches = 0;
    // per-phase device time of the last batched SCF: J, K, Fock + energy, DIIS, density,
    // final FP64 Fock build of the mixed-precision molecules
    cudaEvent_t pev[6] = {};
    double phase_ms[6] = {};
};

namespace {

template <typename T>
int balloc(TinySCF_batch_t b, T **p, size_t count)
{
    void *q = nullptr;
    if (cudaMalloc(&q, sizeof(T) * (count ? count : 1)) != cudaSuccess) {
        cudaGetLastError();
        return ERR_ALLOC;
    }
    b->mem.push_back(q);
    *p = (T *) q;
    return OK;
}

int make_list(TinySCF_batch_t b, const std::vector<int> &counts, WorkList &wl)
{
    std::vector<int> st(counts.size() + 1, 0);
    for (size_t k = 0; k < counts.size(); k++) st[k + 1] = st[k] + counts[k];
    int *d = nullptr;
    RC(balloc(b, &d, st.size()));
    if (cudaMemcpy(d, st.data(), sizeof(int) * st.size(), cudaMemcpyHostToDevice) != cudaSuccess) return ERR_CUDA;
    wl.start = d;
    wl.nmol = (int) counts.size();
    wl.total = st.back();
    return OK;
}

int make_gemm(TinySCF_batch_t b, const std::vector<GemmDesc> &descs, bool ta, bool tb, BatchGemm &g)
{
    std::vector<int> counts;
    for (const GemmDesc &d : descs) counts.push_back(((d.m + 63) / 64) * ((d.n + 63) / 64));
    RC(make_list(b, counts, g.wl));
    GemmDesc *dd = nullptr;
    RC(balloc(b, &dd, descs.size()));
    if (cudaMemcpy(dd, descs.data(), sizeof(GemmDesc) * descs.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return ERR_CUDA;
    g.descs = dd;
    g.ta = ta;
    g.tb = tb;
    return OK;
}

int batch_create_impl(TinySCF_batch_t b, TinySCF_t *ts, int nmol)
{
    const int dev = ts[0]->device;
    for (int k = 0; k < nmol; k++) {
        if (!ts[k] || !ts[k]->dev || E_(ts[k])->stage < 5 || ts[k]->device != dev) return ERR_STATE;
        b->mols.push_back(ts[k]);
    }
    TSCF_CUDA_CHECK(cudaSetDevice(dev));
    TSCF_CUDA_CHECK(cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking));
    TSCF_CUDA_CHECK(cudaEventCreate(&b->ev0));
    TSCF_CUDA_CHECK(cudaEventCreate(&b->ev1));
    for (auto &ev : b->pev) TSCF_CUDA_CHECK(cudaEventCreate(&ev));
    // eigensolver groups of equal basis size
    std::map<int, int> gid;
    std::vector<int> slot(nmol);
    for (int k = 0; k < nmol; k++) {
        const int n = ts[k]->nbasfuncs;
        if (!gid.count(n)) {
            gid[n] = (int) b->groups.size();
            b->groups.push_back({});
            b->groups.back().n = n;
        }
        auto &g = b->groups[gid[n]];
        slot[k] = (int) g.members.size();
        g.members.push_back(k);
    }
    for (auto &g : b->groups) {
        const int64_t cnt = (int64_t) g.members.size(), n = g.n;
        RC(balloc(b, &g.A, (size_t) cnt * n * n));
        RC(balloc(b, &g.W, (size_t) cnt * n));
        g.eig = eig_create(g.n, b->s);
        if (!g.eig) return ERR_ALLOC;
    }
    // per-molecule descriptors and work lists
    std::vector<MolDev> md(nmol);
    std::vector<int> c_nup256, c_jblk, c_naux256, c_nup64, c_half, c_halfw, c_halfd, c_syrk, c_syrk128, c_syrkd, c_nn256,
        c_efb;
    std::vector<GemmDesc> xtf, txfp, fd, fds, xtt, t2x, txt2, cocc, dens;
    int naux_max = 1;
    for (int k = 0; k < nmol; k++) {
        TinySCF_t t = ts[k];
        Engine *e = E_(t);
        const int n = t->nbasfuncs, o = t->n_occ, na = t->df_nbf;
        auto &g = b->groups[gid[n]];
        MolDev &m = md[k];
        memset(&m, 0, sizeof(m));
        m.nbf = n;
        m.naux = na;
        m.nocc = o;
        m.nup = e->nup;
        m.jblk = e->jblk;
        m.ksplit = e->ksplit;
        m.ktile = e->ktile;
        m.max_diis = (t->max_diis < 1 || t->max_diis > MAX_DIIS) ? MAX_DIIS : t->max_diis;
        m.up_i = e->up_i;
        m.up_j = e->up_j;
        m.up_u = e->up_u;
        m.csr_j = e->csr_j;
        m.csr_u = e->csr_u;
        m.displs = e->csr_displs;
        m.tiles = e->ktile == 64 ? e->tiles : e->tiles128;
        m.B = e->B;
        m.B32 = (e->kprec == TINYSCF_K_MIXED) ? e->B32 : nullptr;
        m.H = e->H;
        m.S = e->S;
        m.X = e->X;
        m.D = e->D;
        m.J = e->J;
        m.K = e->K;
        m.F = e->F;
        m.Fp = e->Fp;
        m.Cocc = e->Cocc;
        m.T = e->T;
        m.Kpart = e->Kpart;
        m.Jt = e->Jt;
        m.Jpart = e->Jpart;
        m.Jw = e->Jw;
        m.epart = e->epart;
        m.E = e->E;
        m.tmp = e->tmp;
        m.tmp2 = e->tmp2;
        m.F0 = e->F0;
        m.R = e->R;
        m.diis = e->diis;
        m.eigA = g.A + (size_t) slot[k] * n * n;
        naux_max = std::max(naux_max, na);
        const int nt = (n + 63) / 64;
        const size_t nn = (size_t) n * n;
        c_nup256.push_back((e->nup + 255) / 256);
        c_jblk.push_back(e->jblk);
        c_naux256.push_back((na + 255) / 256);
        c_nup64.push_back((e->nup + 63) / 64);
        c_half.push_back(e->khwide ? 0 : n * ((o + 63) / 64) * ((na + 63) / 64));
        c_halfw.push_back(e->khwide == 1 ? n * ((o + 63) / 64) * ((na + 255) / 256) : 0);
        c_halfd.push_back(e->khwide >= 2 ? n * ((o + 63) / 64) * ((na + 255) / 256) : 0);   // DMMA tiles
        const int nt2 = (n + 127) / 128;
        c_syrk.push_back(e->ktile == 64 ? nt * (nt + 1) / 2 * e->ksplit : 0);
        c_syrk128.push_back(e->ktile == 128 ? nt2 * (nt2 + 1) / 2 * e->ksplit : 0);
        c_syrkd.push_back(e->ktile == KSYRK_DMMA ? nt2 * (nt2 + 1) / 2 * e->ksplit : 0);
        c_nn256.push_back((int) ((nn + 255) / 256));
        c_efb.push_back(ENERGY_BLOCKS);
        xtf.push_back({n, n, n, n, n, n, e->X, e->F, e->tmp, 1.0, 0.0});
        txfp.push_back({n, n, n, n, n, n, e->tmp, e->X, e->Fp, 1.0, 0.0});
        fd.push_back({n, n, n, n, n, n, e->F, e->D, e->tmp, 1.0, 0.0});
        fds.push_back({n, n, n, n, n, n, e->tmp, e->S, e->tmp2, 1.0, 0.0});
        xtt.push_back({n, n, n, n, n, n, e->X, e->tmp, e->tmp2, 1.0, 0.0});
        t2x.push_back({n, n, n, n, n, n, e->tmp2, e->X, e->tmp, 1.0, 0.0});
        txt2.push_back({n, n, n, n, n, n, e->tmp, e->X, e->tmp2, 1.0, 0.0});
        cocc.push_back({n, o, n, n, n, o, e->X, m.eigA, e->Cocc, 1.0, 0.0});
        dens.push_back({n, n, o, o, o, n, e->Cocc, e->Cocc, e->D, 1.0, 0.0});
    }
    BatchPlan &p = b->plan;
    p.nmol = nmol;
    p.naux_max = naux_max;
    MolDev *dm = nullptr;
    RC(balloc(b, &dm, nmol));
    TSCF_CUDA_CHECK(cudaMemcpy(dm, md.data(), sizeof(MolDev) * nmol, cudaMemcpyHostToDevice));
    p.mols = dm;
    int *da = nullptr;
    RC(balloc(b, &da, nmol));
    p.active = da;
    b->d_active = da;
    RC(balloc(b, &b->d_Eall, nmol));
    RC(balloc(b, &b->d_kact, nmol));
    RC(balloc(b, &b->d_need, nmol));
    b->mixed.assign(nmol, 0);
    for (int k = 0; k < nmol; k++) b->mixed[k] = E_(ts[k])->kprec == TINYSCF_K_MIXED && E_(ts[k])->kmix != nullptr;
    {   // TINYSCF_BATCH_KMIX=1: the mixed molecules' K in one launch per kernel (default: one molecule
        // at a time, which measured faster on the 256 water clusters: 4.2 s against 5.0 s of K)
        const char *v = getenv("TINYSCF_BATCH_KMIX");
        std::vector<KMix *> ks;
        for (int k = 0; k < nmol; k++)
            if (b->mixed[k]) {
                Engine *e = E_(ts[k]);
                ks.push_back(e->kmix);
                b->kmb_mol.push_back(k);
                b->kmb_C.push_back(e->Cocc);
                b->kmb_S.push_back(e->S);
                b->kmb_K.push_back(e->Kmix);
            }
        b->kmb_act.assign(ks.size(), 0);
        if (!ks.empty() && v && v[0] == '1') RC(kmix_batch_create(&b->kmb, ks.data(), (int) ks.size(), b->s));
    }
    RC(make_list(b, c_nup256, p.nup256));
    RC(make_list(b, c_jblk, p.jblk));
    RC(make_list(b, c_naux256, p.naux256));
    RC(make_list(b, c_nup64, p.nup64));
    RC(make_list(b, c_half, p.half));
    RC(make_list(b, c_halfw, p.half_wide));
    RC(make_list(b, c_halfd, p.half_dmma));
    RC(make_list(b, c_syrk, p.syrk));
    RC(make_list(b, c_syrk128, p.syrk128));
    RC(make_list(b, c_syrkd, p.syrk_dmma));
    RC(make_list(b, c_nn256, p.nn256));
    RC(make_list(b, c_efb, p.efb));
    RC(make_gemm(b, xtf, true, false, p.g_xtf));
    RC(make_gemm(b, txfp, false, false, p.g_tx_fp));
    RC(make_gemm(b, fd, false, false, p.g_fd));
    RC(make_gemm(b, fds, false, false, p.g_fds));
    RC(make_gemm(b, xtt, true, false, p.g_xtt));
    RC(make_gemm(b, t2x, false, false, p.g_t2x));
    RC(make_gemm(b, txt2, false, false, p.g_tx_t2));
    RC(make_gemm(b, cocc, false, true, p.g_cocc));
    RC(make_gemm(b, dens, false, true, p.g_dens));
    return OK;
}

// Eigensolves of the flagged molecules, one per molecule with the engine's
// solver of its group's size.
int batch_eigs(TinySCF_batch_t b, const std::vector<int> &need)
{
    for (auto &g : b->groups) {
        const int64_t cnt = (int64_t) g.members.size(), n = g.n;
        for (int64_t k = 0; k < cnt; k++)
            if (need[g.members[k]]) RC(eig_run(g.eig, g.A + k * n * n, g.W + k * n, g.A + k * n * n, b->s));
    }
    return OK;
}

int batch_scf_impl(TinySCF_batch_t b)
{
    const int nmol = (int) b->mols.size();
    std::vector<int> act(nmol, 0);
    std::vector<double> prev(nmol, 0.0), delta(nmol, 223.0), Eh(nmol, 0.0);
    for (int k = 0; k < nmol; k++) {
        TinySCF_t t = b->mols[k];
        t->iter = 0;
        act[k] = (t->niters > 0) ? 1 : 0;
        // the loop consumes the guess (or the state a reset left) exactly like do_SCF
        TSCF_CUDA_CHECK(cudaStreamSynchronize(E_(t)->s));
    }
    std::vector<int> kact(nmol, 0), need(nmol, 0);
    for (int k = 0; k < nmol; k++) E_(b->mols[k])->have_eig = false;   // each batched solve starts from eigensolves
    auto upload_flags = [&]() {
        for (int k = 0; k < nmol; k++) kact[k] = act[k] && !b->mixed[k];
        cudaMemcpyAsync(b->d_active, act.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice, b->s);
        return cudaMemcpyAsync(b->d_kact, kact.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice, b->s);
    };
    TSCF_CUDA_CHECK(upload_flags());
    const long long l0 = g_launches, le0 = g_eig_launches;
    for (double &v : b->phase_ms) v = 0.0;
    for (int k = 0; k < nmol; k++)   // a molecule's incremental K restarts with each batched solve
        if (b->mixed[k]) kmix_reset(E_(b->mols[k])->kmix, b->s);
    cudaEventRecord(b->ev0, b->s);
    int it = 0;
    for (;; it++) {
        bool any = false;
        for (int v : act) any |= v != 0;
        if (!any) break;
        cudaEventRecord(b->pev[0], b->s);
        batch_j(b->plan, b->s);
        cudaEventRecord(b->pev[1], b->s);
        batch_k(b->plan, b->d_kact, b->s);
        if (b->kmb) {   // tensor-core incremental exchange of every mixed molecule: one launch per kernel
            for (size_t j = 0; j < b->kmb_mol.size(); j++) b->kmb_act[j] = act[b->kmb_mol[j]];
            RC(kmix_batch_build(b->kmb, b->kmb_act.data(), b->kmb_C.data(), b->kmb_S.data(), b->kmb_K.data(), b->s));
        }
        for (int k = 0; k < nmol; k++) {
            if (!act[k] || !b->mixed[k]) continue;
            Engine *e = E_(b->mols[k]);
            if (!b->kmb) RC(kmix_build(e->kmix, e->Cocc, e->S, e->Kmix, b->s));   // one molecule at a time
            TSCF_CUDA_CHECK(cudaMemcpyAsync(e->K, e->Kmix, sizeof(double) * e->nn, cudaMemcpyDeviceToDevice, b->s));
        }
        cudaEventRecord(b->pev[2], b->s);
        batch_fock(b->plan, b->d_Eall, b->s);
        cudaEventRecord(b->pev[3], b->s);
        batch_diis(b->plan, it >= 2, b->s);
        cudaEventRecord(b->pev[4], b->s);
        // density: molecules set to TINYSCF_DENSITY_REFINE first refine their
        // occupied subspace (host-checked steps, one molecule at a time); the
        // rest, and those whose refinement did not converge, take eigensolves
        for (int k = 0; k < nmol; k++) {
            need[k] = act[k];
            if (!act[k]) continue;
            Engine *e = E_(b->mols[k]);
            const int n = b->mols[k]->nbasfuncs, o = b->mols[k]->n_occ;
            if (e->dmode != TINYSCF_DENSITY_REFINE || !e->have_eig || o <= 0 || o >= n) continue;
            int steps = 0;
            double res = 0.0;
            RC(subspace_refine(e->Fp, e->V, e->w, e->U, n, o, e->sw, kRefineTol, kRefineSteps, &steps, &res, b->s));
            e->n_refine += steps;
            if (res < kRefineTol) {
                { density_from_rows(e->X, e->U, e->Cocc, e->D, n, o, b->s); e->d_from_cocc = true; }
                need[k] = 0;
            }
        }
        TSCF_CUDA_CHECK(cudaMemcpyAsync(b->d_need, need.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice, b->s));
        batch_copy_fp(b->plan, b->d_need, b->s);
        RC(batch_eigs(b, need));
        batch_gemm(b->plan.g_cocc, b->d_need, b->s);
        batch_gemm(b->plan.g_dens, b->d_need, b->s);
        for (auto &g : b->groups)   // new eigenbases of the refinement molecules
            for (size_t q = 0; q < g.members.size(); q++) {
                const int k = g.members[q];
                Engine *e = E_(b->mols[k]);
                if (!need[k]) continue;
                e->n_eig++;
                if (e->dmode != TINYSCF_DENSITY_REFINE || !e->U) continue;
                const int n = g.n, o = b->mols[k]->n_occ;
                TSCF_CUDA_CHECK(cudaMemcpyAsync(e->V, g.A + q * (size_t) n * n, sizeof(double) * (size_t) n * n,
                                                cudaMemcpyDeviceToDevice, b->s));
                TSCF_CUDA_CHECK(cudaMemcpyAsync(e->w, g.W + q * (size_t) n, sizeof(double) * n,
                                                cudaMemcpyDeviceToDevice, b->s));
                TSCF_CUDA_CHECK(cudaMemcpyAsync(e->U, e->V, sizeof(double) * (size_t) o * n, cudaMemcpyDeviceToDevice,
                                                b->s));
                e->have_eig = true;
            }
        cudaEventRecord(b->pev[5], b->s);
        TSCF_CUDA_CHECK(cudaMemcpyAsync(Eh.data(), b->d_Eall, sizeof(double) * nmol, cudaMemcpyDeviceToHost, b->s));
        TSCF_CUDA_CHECK(cudaStreamSynchronize(b->s));
        for (int q = 0; q < 5; q++) {
            float pm = 0.f;
            cudaEventElapsedTime(&pm, b->pev[q], b->pev[q + 1]);
            b->phase_ms[q] += pm;
        }
        TSCF_CUDA_CHECK(cudaGetLastError());
        for (int k = 0; k < nmol; k++) {
            if (!act[k]) continue;
            TinySCF_t t = b->mols[k];
            t->HF_energy = Eh[k];
            if (!std::isfinite(Eh[k])) return ERR_NUMERIC;
            delta[k] = fabs(Eh[k] - prev[k]);
            prev[k] = Eh[k];
            if (t->iter == 0) delta[k] = 223;
            t->iter++;
            if (!(t->iter < t->niters && delta[k] >= t->ene_tol)) act[k] = 0;
        }
        TSCF_CUDA_CHECK(upload_flags());
    }
    // one FP64 Fock build on the converged density of every mixed-precision molecule;
    // its energy is the result (as TinySCF_do_SCF does for one molecule)
    bool any_mixed = false;
    for (int k = 0; k < nmol; k++) {
        act[k] = b->mixed[k];
        any_mixed |= b->mixed[k] != 0;
    }
    if (any_mixed) {
        TSCF_CUDA_CHECK(cudaMemcpyAsync(b->d_active, act.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice, b->s));
        TSCF_CUDA_CHECK(cudaMemcpyAsync(b->d_kact, act.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice, b->s));
        cudaEventRecord(b->pev[0], b->s);
        batch_j(b->plan, b->s, 0);
        batch_k(b->plan, b->d_kact, b->s);
        batch_fock(b->plan, b->d_Eall, b->s);
        cudaEventRecord(b->pev[1], b->s);
        TSCF_CUDA_CHECK(cudaMemcpyAsync(Eh.data(), b->d_Eall, sizeof(double) * nmol, cudaMemcpyDeviceToHost, b->s));
        TSCF_CUDA_CHECK(cudaStreamSynchronize(b->s));
        float pm = 0.f;
        cudaEventElapsedTime(&pm, b->pev[0], b->pev[1]);
        b->phase_ms[5] += pm;
        for (int k = 0; k < nmol; k++)
            if (b->mixed[k]) b->mols[k]->HF_energy = Eh[k];
        const int fl = kmix_error_flag();
        if (fl) {
            fprintf(stderr, "[tinyscf] tensor-core K: a bounded wait timed out (code %d)\n", fl);
            return ERR_CUDA;
        }
    }
    cudaEventRecord(b->ev1, b->s);
    TSCF_CUDA_CHECK(cudaEventSynchronize(b->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->scf_ms = ms;
    b->iterations = it;
    b->launches = (g_launches - l0) - (g_eig_launches - le0);
    // eigenvalues (of the last full eigensolve) and host mirrors of every molecule
    for (auto &g : b->groups)
        for (size_t k = 0; k < g.members.size(); k++) {
            Engine *e = E_(b->mols[g.members[k]]);
            if (e->dmode == TINYSCF_DENSITY_REFINE && e->U) continue;   // w already holds it
            TSCF_CUDA_CHECK(cudaMemcpyAsync(e->w, g.W + k * g.n, sizeof(double) * g.n, cudaMemcpyDeviceToDevice, b->s));
        }
    TSCF_CUDA_CHECK(cudaStreamSynchronize(b->s));
    for (int k = 0; k < nmol; k++) {
        Engine *e = E_(b->mols[k]);
        e->F_is_orth = !b->mixed[k];   // after the final build F holds H + 2J - K
        e->have_eig = false;
        RC(sync_host_impl(b->mols[k]));
    }
    return OK;
}

void batch_free_impl(TinySCF_batch_t b)
{
    if (b->s) cudaStreamSynchronize(b->s);
    kmix_batch_destroy(b->kmb);
    for (auto &g : b->groups) eig_destroy(g.eig);
    for (void *p : b->mem) cudaFree(p);
    for (auto &ev : b->pev)
        if (ev) cudaEventDestroy(ev);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->s) cudaStreamDestroy(b->s);
}

}  // namespace

extern "C" {

int TinySCF_device_memory(int device, long long *free_bytes, long long *total_bytes)
{
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) {
        cudaGetLastError();
        return TINYSCF_ERR_CUDA;
    }
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return TINYSCF_ERR_CUDA;
    size_t f = 0, tot = 0;
    cudaError_t err = cudaMemGetInfo(&f, &tot);
    cudaMemPool_t pool;   // memory the engines' pool holds but does not use is free for them too
    if (err == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, device >= 0 ? device : cur) == cudaSuccess) {
        uint64_t reserved = 0, used = 0;
        if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
            f += (size_t) (reserved - used);
    }
    cudaGetLastError();
    cudaSetDevice(cur);
    if (err != cudaSuccess) return TINYSCF_ERR_CUDA;
    if (free_bytes) *free_bytes = (long long) f;
    if (total_bytes) *total_bytes = (long long) tot;
    return TINYSCF_OK;
}

int TinySCF_set_autotune(int on)
{
    tune_set_enabled(on != 0);
    return TINYSCF_OK;
}

int TinySCF_autotune_report(char *buf, int len)
{
    std::string r = tune_report();
    if (buf && len > 0) {
        snprintf(buf, (size_t) len, "%s", r.c_str());
    }
    return (int) r.size();
}

int TinySCF_batch_create(TinySCF_batch_t *out, TinySCF_t *mols, int nmol)
{
    if (!out || !mols || nmol <= 0) return TINYSCF_ERR_INPUT;
    TinySCF_batch_t b = new TinySCF_batch_struct();
    int rc = batch_create_impl(b, mols, nmol);
    if (rc) {
        batch_free_impl(b);
        delete b;
        return rc;
    }
    *out = b;
    return TINYSCF_OK;
}

int TinySCF_batch_do_SCF(TinySCF_batch_t b)
{
    if (!b) return TINYSCF_ERR_STATE;
    return batch_scf_impl(b);
}

int TinySCF_batch_stats(TinySCF_batch_t b, double *scf_ms, int *iterations, long long *launches)
{
    if (!b) return TINYSCF_ERR_STATE;
    if (scf_ms) *scf_ms = b->scf_ms;
    if (iterations) *iterations = b->iterations;
    if (launches) *launches = b->launches;
    return TINYSCF_OK;
}

int TinySCF_batch_phase_ms(TinySCF_batch_t b, double *ms, int n)
{
    if (!b || !ms) return TINYSCF_ERR_STATE;
    for (int q = 0; q < n && q < 6; q++) ms[q] = b->phase_ms[q];
    return TINYSCF_OK;
}

int TinySCF_batch_free(TinySCF_batch_t b)
{
    if (!b) return TINYSCF_ERR_STATE;
    batch_free_impl(b);
    delete b;
    return TINYSCF_OK;
}

int TinySCF_set_aux_slice(TinySCF_t t, int p0, int p1)
{
    if (!t || !t->dev) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    if (e->stage >= 5) return TINYSCF_ERR_STATE;   // before the DF tensor is built
    if (p0 < 0 || p1 <= p0 || p1 > t->df_nbf) return TINYSCF_ERR_INPUT;
    e->aux_p0 = p0;
    e->aux_ns = (p0 == 0 && p1 == t->df_nbf) ? 0 : p1 - p0;
    return TINYSCF_OK;
}

int TinySCF_set_JK(TinySCF_t t, const double *J, const double *K)
{
    if (!t || !t->dev || !J || !K) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    if (e->stage < 5) return TINYSCF_ERR_STATE;
    const size_t bytes = sizeof(double) * e->nn;
    if (cudaMemcpyAsync(e->J, J, bytes, cudaMemcpyHostToDevice, e->s) != cudaSuccess ||
        cudaMemcpyAsync(e->K, K, bytes, cudaMemcpyHostToDevice, e->s) != cudaSuccess)
        return TINYSCF_ERR_CUDA;
    e->h2d += (long long) (2 * bytes);
    tstart(e, TINYSCF_T_FOCK);
    build_F_energy(e->H, e->J, e->K, e->D, e->F, e->epart, t->nbasfuncs, e->s);
    energy_reduce(e->epart, e->E, e->s);
    tstop(e, TINYSCF_T_FOCK);
    e->F_is_orth = false;
    if (cuda_rc("Fock assembly") || sync_rc(e, "Fock assembly")) return TINYSCF_ERR_CUDA;
    tcollect(e);
    memcpy(t->J_mat, J, bytes);
    memcpy(t->K_mat, K, bytes);
    d2h(e, t->F_mat, e->F, bytes);
    d2h(e, &t->HF_energy, e->E, sizeof(double));
    return TINYSCF_OK;
}

int TinySCF_kmix_wait_probe(TinySCF_t t, long long wait_cycles, int *code)
{
    if (!t || !t->dev || !code) return TINYSCF_ERR_STATE;
    Engine *e = E_(t);
    if (!e->kmix) return TINYSCF_ERR_STATE;
    return kmix_wait_probe(e->kmix, wait_cycles, code, e->s);
}

int TinySCF_eigh(int device, int n, const double *A, double *w, double *V)
{
    if (n < 1 || n > EIG_MAX_N || !A || !w || !V) return TINYSCF_ERR_INPUT;
    if (cudaSetDevice(device) != cudaSuccess) return TINYSCF_ERR_CUDA;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return TINYSCF_ERR_CUDA;
    const size_t nn = (size_t) n * n;
    double *dA = nullptr, *dw = nullptr, *dV = nullptr;
    Eig *eg = nullptr;
    int rc = TINYSCF_OK;
    if (cudaMalloc(&dA, sizeof(double) * nn) != cudaSuccess || cudaMalloc(&dw, sizeof(double) * n) != cudaSuccess ||
        cudaMalloc(&dV, sizeof(double) * nn) != cudaSuccess || !(eg = eig_create(n, s))) {
        rc = TINYSCF_ERR_ALLOC;
    } else if (cudaMemcpyAsync(dA, A, sizeof(double) * nn, cudaMemcpyHostToDevice, s) != cudaSuccess) {
        rc = TINYSCF_ERR_CUDA;
    } else {
        rc = eig_run(eg, dA, dw, dV, s);
        if (rc == OK && (cudaMemcpyAsync(w, dw, sizeof(double) * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                         cudaMemcpyAsync(V, dV, sizeof(double) * nn, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                         cudaStreamSynchronize(s) != cudaSuccess))
            rc = TINYSCF_ERR_CUDA;
        if (rc == OK) rc = eig_error(eg);
    }
    eig_destroy(eg);
    cudaFree(dA);
    cudaFree(dw);
    cudaFree(dV);
    cudaStreamDestroy(s);
    return rc;
}

int TinySCF_trim_memory(int device)
{
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) {
        cudaGetLastError();
        return TINYSCF_ERR_CUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess) return TINYSCF_ERR_CUDA;
    const int rc = dev_trim(device);
    cudaSetDevice(cur);
    return rc == OK ? TINYSCF_OK : TINYSCF_ERR_CUDA;
}

int TinySCF_syrk_int8(int device, int n, long long q, const double *T, double *K)
{
    if (n < 1 || q < 1 || !T || !K) return TINYSCF_ERR_INPUT;
    if (cudaSetDevice(device) != cudaSuccess) return TINYSCF_ERR_CUDA;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return TINYSCF_ERR_CUDA;
    double *dT = nullptr, *dK = nullptr;
    OzSyrk *oz = nullptr;
    int rc = TINYSCF_OK;
    if (cudaMalloc(&dT, sizeof(double) * (size_t) n * q) != cudaSuccess ||
        cudaMalloc(&dK, sizeof(double) * (size_t) n * n) != cudaSuccess) {
        cudaGetLastError();
        rc = TINYSCF_ERR_ALLOC;
    } else if ((rc = oz_create(&oz, n, q, s)) == OK) {
        if (cudaMemcpyAsync(dT, T, sizeof(double) * (size_t) n * q, cudaMemcpyHostToDevice, s) != cudaSuccess)
            rc = TINYSCF_ERR_CUDA;
        else if ((rc = oz_syrk(oz, dT, dK, s)) == OK &&
                 (cudaMemcpyAsync(K, dK, sizeof(double) * (size_t) n * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                  cudaStreamSynchronize(s) != cudaSuccess))
            rc = TINYSCF_ERR_CUDA;
        if (rc == OK && oz_error_flag()) rc = TINYSCF_ERR_CUDA;
    }
    oz_destroy(oz);
    cudaFree(dT);
    cudaFree(dK);
    cudaStreamDestroy(s);
    return rc;
}

// ---- the reference's void API (abort on failure, like its asserts)
void init_TinySCF(TinySCF_t t, char *bas, char *dfbas, char *xyz, const int niters)
{
    int rc = TinySCF_init_status(t, bas, dfbas, xyz, niters);
    if (rc) die("init_TinySCF", rc);
}
void free_TinySCF(TinySCF_t t) { TinySCF_free_status(t); }
void TinySCF_init_batch_dgemm_arrays(TinySCF_t t) { (void) t; }
void TinySCF_free_batch_dgemm_arrays(TinySCF_t t) { (void) t; }
void TinySCF_compute_Hcore_Ovlp_mat(TinySCF_t t)
{
    int rc = TinySCF_compute_Hcore_Ovlp_mat_status(t);
    if (rc) die("TinySCF_compute_Hcore_Ovlp_mat", rc);
}
void TinySCF_compute_sq_Schwarz_scrvals(TinySCF_t t)
{
    int rc = TinySCF_compute_sq_Schwarz_scrvals_status(t);
    if (rc) die("TinySCF_compute_sq_Schwarz_scrvals", rc);
}
void TinySCF_prepare_sparsity(TinySCF_t t)
{
    int rc = TinySCF_prepare_sparsity_status(t);
    if (rc) die("TinySCF_prepare_sparsity", rc);
}
void TinySCF_get_initial_guess(TinySCF_t t)
{
    int rc = TinySCF_get_initial_guess_status(t);
    if (rc) die("TinySCF_get_initial_guess", rc);
}
void TinySCF_build_DF_tensor(TinySCF_t t)
{
    int rc = TinySCF_build_DF_tensor_status(t);
    if (rc) die("TinySCF_build_DF_tensor", rc);
}
void TinySCF_build_FockMat(TinySCF_t t)
{
    int rc = TinySCF_build_FockMat_status(t);
    if (rc) die("TinySCF_build_FockMat", rc);
}
void TinySCF_DIIS(TinySCF_t t)
{
    int rc = TinySCF_DIIS_status(t);
    if (rc) die("TinySCF_DIIS", rc);
}
void TinySCF_build_DenMat(TinySCF_t t)
{
    int rc = TinySCF_build_DenMat_status(t);
    if (rc) die("TinySCF_build_DenMat", rc);
}
void TinySCF_do_SCF(TinySCF_t t)
{
    int rc = TinySCF_do_SCF_status(t);
    if (rc) die("TinySCF_do_SCF", rc);
}

// build_density.c:12-35, the reference's host helper, behaviour kept as is.
void quickSort_eigval(double *eigval, int *ev_idx, int l, int r)
{
    int i = l, j = r;
    double mid = eigval[(i + j) / 2], dswap;
    while (i <= j) {
        while (eigval[i] < mid) i++;
        while (eigval[j] > mid) j--;
        if (i <= j) {
            ev_idx[i] = ev_idx[j];
            ev_idx[j] = ev_idx[i];
            dswap = eigval[i];
            eigval[i] = eigval[j];
            eigval[j] = dswap;
            i++;
            j--;
        }
    }
    if (i < r) quickSort_eigval(eigval, ev_idx, i, r);
    if (j > l) quickSort_eigval(eigval, ev_idx, l, j);
}

}  // extern "C"
