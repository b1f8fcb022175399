"""ORACLE — test infrastructure only.

A numpy restatement of the reference's DF-RHF path (huanghua1994/YATSCF-DF),
used only by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline
leg, and there only to check results, never as the computation measured or
shipped. Every function names the reference file:line it
follows. Integrals come from the oracle's own McMurchie–Davidson engine
(ints.c, oracle_bulk.c via ctypes) because the reference's Simint is not
available; linear algebra is numpy/scipy LAPACK, standing in for MKL.

The restatement is pinned against the reference's own C sources compiled by
``oracle/Makefile`` (``oracle/_ref/ref_dump``) on the same inputs: see
tests/test_oracle_golden.py and the fixtures in tests/golden/ (written by
tests/golden/make_fixtures.py).
"""
import ctypes
import math
import os
import re

import numpy as np
from scipy.linalg import lapack

HERE = os.path.dirname(os.path.abspath(__file__))

A2BOHR = 1.0 / 0.52917720859          # CMS_BasisSet.c:39
ETABLE = ["H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne",
          "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar", "K", "Ca",
          "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn",
          "Ga", "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y", "Zr",
          "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn"]   # CMS_BasisSet.c:43-55
MTABLE = "SPDFG"                       # CMS_BasisSet.c:57
MAX_DIIS = 10                          # TinySCF.h:8
ENE_TOL = 1e-11                        # TinySCF_init_free.c:75
SHELL_SCRTOL2 = 1e-11 * 1e-11          # TinySCF_init_free.c:78


def ncart(l):
    return (l + 1) * (l + 2) // 2


_FLOAT_PREFIX = re.compile(r"^[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?")


def _atof(s):
    """C atof()/sscanf("%lf"): the longest leading float prefix, 0.0 if none
    (so a Fortran "0.45D-03" reads as 0.45, as it does in the reference)."""
    m = _FLOAT_PREFIX.match(s.strip())
    return float(m.group(0)) if m else 0.0


# ---------------------------------------------------------------- input files
def parse_xyz(path):
    """CMS_import_molecule (CMS_BasisSet.c:310-426): Angstrom -> Bohr, charge
    from the comment line, nuclear repulsion energy."""
    with open(path) as f:
        lines = f.read().splitlines()
    natoms = int(lines[0].split()[0])
    Q = int(_atof(lines[1]))
    sym, xyz = [], []
    for line in lines[2:]:
        tok = line.split()
        if not tok or not tok[0][0].isalpha():
            continue
        if tok[0] not in ETABLE:
            raise ValueError("atom %s is not supported" % tok[0])
        sym.append(tok[0])
        xyz.append([float(tok[1]) * A2BOHR, float(tok[2]) * A2BOHR, float(tok[3]) * A2BOHR])
    if len(sym) != natoms:
        raise ValueError("natoms does not match the header")
    Z = np.array([ETABLE.index(s) + 1 for s in sym], dtype=np.float64)
    xyz = np.array(xyz, dtype=np.float64)
    enuc = 0.0
    for a in range(natoms):
        for b in range(a + 1, natoms):
            enuc += Z[a] * Z[b] / math.sqrt(float(np.sum((xyz[a] - xyz[b]) ** 2)))
    return dict(sym=sym, Z=Z, xyz=xyz, Q=Q, enuc=enuc, nelec=int(Z.sum()))


def parse_gbs(path):
    """CMS_import_basis (CMS_BasisSet.c:439-642): element -> list of
    (am, exponents, raw coefficients); SP shells split into S then P."""
    with open(path) as f:
        lines = f.read().splitlines()
    basis, i = {}, 1
    while i < len(lines):
        line = lines[i]
        i += 1
        if not line or not line[0].isalpha():
            continue
        el = line.split()[0]
        shells = []
        while i < len(lines):
            line = lines[i]
            i += 1
            if line and line[0].isalpha():
                tok = line.split()
                kind, nexp = tok[0], int(_atof(tok[1]))
                rows = [[_atof(v) for v in lines[i + k].split()[:4]] for k in range(nexp)]
                i += nexp
                for sub, letter in enumerate(kind):
                    am = MTABLE.index(letter)
                    shells.append((am, np.array([r[0] for r in rows]), np.array([r[1 + sub] for r in rows])))
            if line.startswith("*"):
                break
        basis[el] = shells
    return basis


def load_sad(gbs_path, el, nfunc):
    """CMS_import_guess (CMS_BasisSet.c:657-746): <dir>/<El>.dat, one value per
    line; zero block if missing, short, or failing the one-sided symmetry test."""
    fn = os.path.join(os.path.dirname(gbs_path), el + ".dat")
    if not os.path.exists(fn):
        return np.zeros((nfunc, nfunc))
    with open(fn) as f:
        vals = f.read().split()
    if len(vals) < nfunc * nfunc:
        return np.zeros((nfunc, nfunc))
    g = np.array([float(v) for v in vals[:nfunc * nfunc]]).reshape(nfunc, nfunc)
    if np.any(g - g.T > 1e-12):
        return np.zeros((nfunc, nfunc))
    return g


# ------------------------------------------------------------ integral engine
class _OBBasis(ctypes.Structure):
    _fields_ = [("nsh", ctypes.c_int),
                ("am", ctypes.c_void_p), ("nprim", ctypes.c_void_p), ("off", ctypes.c_void_p),
                ("cen", ctypes.c_void_p), ("alpha", ctypes.c_void_p), ("coef", ctypes.c_void_p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(os.path.join(HERE, "liboracle.so"))
        _lib.oi_boys.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_void_p]
        _lib.oi_normalize.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        vp, bp = ctypes.c_void_p, ctypes.POINTER(_OBBasis)
        _lib.ob_one_electron.argtypes = [bp, ctypes.c_int, vp, vp, vp, vp]
        _lib.ob_schwarz.argtypes = [bp, ctypes.c_int, vp, vp]
        _lib.ob_df_scrval.argtypes = [bp, vp]
        _lib.ob_3center.argtypes = [bp, bp, vp, vp, ctypes.c_int, vp, vp, ctypes.c_double, vp, vp]
        _lib.ob_2center.argtypes = [bp, vp, ctypes.c_double, vp]
        for f in ("ob_one_electron", "ob_schwarz", "ob_df_scrval", "ob_3center", "ob_2center", "oi_boys", "oi_normalize"):
            getattr(_lib, f).restype = None
    return _lib


def _p(a):
    return a.ctypes.data


class Shells:
    """Shell table of a molecule (CMS_parse_molecule, CMS_BasisSet.c:192-299)
    with normalised coefficients (the Simint step of CMS_Simint.c:143-145)."""

    def __init__(self, mol, basis):
        am, nprim, off, cen, alpha, coef = [], [], [], [], [], []
        self.atom_bf = []
        nbf = 0
        for a, el in enumerate(mol["sym"]):
            if el not in basis:
                raise ValueError("element %s missing from basis" % el)
            start = nbf
            for (l, ex, cc) in basis[el]:
                cn = np.zeros(len(ex))
                lib().oi_normalize(l, len(ex), _p(np.ascontiguousarray(ex)), _p(np.ascontiguousarray(cc)), _p(cn))
                off.append(len(alpha))
                am.append(l)
                nprim.append(len(ex))
                cen.extend(mol["xyz"][a])
                alpha.extend(ex)
                coef.extend(cn)
                nbf += ncart(l)
            self.atom_bf.append((start, nbf))
        self.am = np.array(am, dtype=np.int32)
        self.nprim = np.array(nprim, dtype=np.int32)
        self.off = np.array(off, dtype=np.int32)
        self.cen = np.array(cen, dtype=np.float64)
        self.alpha = np.array(alpha, dtype=np.float64)
        self.coef = np.array(coef, dtype=np.float64)
        self.nsh = len(am)
        self.nbf = nbf
        self.sind = np.concatenate([[0], np.cumsum([ncart(l) for l in am])]).astype(np.int32)
        self.c = _OBBasis(self.nsh, _p(self.am), _p(self.nprim), _p(self.off),
                          _p(self.cen), _p(self.alpha), _p(self.coef))


def boys(mmax, T):
    F = np.zeros(mmax + 1)
    lib().oi_boys(mmax, float(T), _p(F))
    return F


# ------------------------------------------------------------ the SCF engine
class OracleSCF:
    """State and steps of struct TinySCF_struct (TinySCF.h:12-100)."""

    def __init__(self, bas_fname, df_bas_fname, xyz_fname, niters, max_diis=MAX_DIIS,
                 schwarz_quirk=True):
        # init_TinySCF (TinySCF_init_free.c:14-208)
        self.mol = parse_xyz(xyz_fname)
        self.basis = parse_gbs(bas_fname)
        self.df_basis = parse_gbs(df_bas_fname)
        self.bas_fname = bas_fname
        self.sh = Shells(self.mol, self.basis)
        self.dsh = Shells(self.mol, self.df_basis)
        self.nbf, self.naux = self.sh.nbf, self.dsh.nbf
        self.n_occ = int((self.mol["nelec"] - self.mol["Q"]) / 2)   # CMS_BasisSet.c:788-791
        self.charge, self.electron = self.mol["Q"], self.mol["nelec"]
        self.niters = niters
        self.max_diis = max_diis
        self.schwarz_quirk = schwarz_quirk
        self.nuc_energy = self.mol["enuc"]
        self._diis_reset()

    def _diis_reset(self):
        n, m = self.nbf, self.max_diis
        self.F0 = np.zeros((m, n, n))
        self.R = np.zeros((m, n, n))
        self.B = -np.ones((m + 1, m + 1))             # TinySCF_init_free.c:178-182
        np.fill_diagonal(self.B, 0.0)
        self.diis_len, self.bmax_id, self.bmax = 0, 0, -np.finfo(np.float64).max

    # TinySCF_compute_Hcore_Ovlp_mat (TinySCF.c:20-83)
    def compute_Hcore_Ovlp_mat(self):
        n = self.nbf
        self.S = np.zeros((n, n))
        self.H = np.zeros((n, n))
        lib().ob_one_electron(ctypes.byref(self.sh.c), len(self.mol["sym"]), _p(self.mol["Z"]),
                              _p(np.ascontiguousarray(self.mol["xyz"])), _p(self.S), _p(self.H))
        w, U = np.linalg.eigh(self.S)
        self.X = (U * (1.0 / np.sqrt(w))) @ U.T

    # TinySCF_compute_sq_Schwarz_scrvals (TinySCF.c:112-226)
    def compute_sq_Schwarz_scrvals(self):
        nsh, n = self.sh.nsh, self.nbf
        self.sp_scrval = np.zeros(nsh * nsh)
        self.bf_pair_scrval = np.zeros(n * n)
        lib().ob_schwarz(ctypes.byref(self.sh.c), int(self.schwarz_quirk), _p(self.sp_scrval), _p(self.bf_pair_scrval))
        self.max_scrval = self.sp_scrval.max()
        self.df_sp_scrval = np.zeros(self.dsh.nsh)
        lib().ob_df_scrval(ctypes.byref(self.dsh.c), _p(self.df_sp_scrval))
        self.max_df_scrval = self.df_sp_scrval.max()
        eta = SHELL_SCRTOL2 / self.max_df_scrval
        am = self.sh.am
        pairs = []
        for M in range(nsh):
            for N in range(M, nsh):
                if self.sp_scrval[M * nsh + N] > eta:
                    mn, nm = am[M] * 5 + am[N], am[N] * 5 + am[M]   # CMS_Simint.c:308-312
                    pairs.append((M, N) if mn > nm else (N, M))
        pairs.sort()
        self.uniq_sp = np.array(pairs, dtype=np.int32).reshape(-1, 2)

    # TinySCF_prepare_sparsity (TinySCF.c:228-280)
    def prepare_sparsity(self):
        n = self.nbf
        eta = SHELL_SCRTOL2 / self.max_df_scrval
        keep = self.bf_pair_scrval.reshape(n, n) > eta
        self.bf_pair_mask = -np.ones((n, n), dtype=np.int32)
        self.bf_pair_mask[keep] = np.arange(int(keep.sum()), dtype=np.int32)
        self.bf_pair_j = np.nonzero(keep)[1].astype(np.int32)
        self.bf_mask_displs = np.concatenate([[0], np.cumsum(keep.sum(axis=1))]).astype(np.int32)
        self.bf_pair_diag = self.bf_pair_mask[np.arange(n), np.arange(n)].copy()
        self.nnz = int(self.bf_mask_displs[-1])

    # TinySCF_D2Cocc (TinySCF.c:282-322), including its quirks: the pivot is
    # ignored and the Cholesky diagonal is dropped for the first n_occ rows.
    @staticmethod
    def D2Cocc(D, n_occ):
        n = D.shape[0]
        chol, piv, rank, info = lapack.dpstrf(np.array(D, order="F"), tol=1e-12, lower=1)
        chol = np.array(chol)
        if rank < n_occ:
            chol[:, rank:n_occ] = 0.0
        C = np.zeros((n, n_occ))
        for i in range(min(n_occ, n)):
            C[i, :i] = chol[i, :i]
        C[n_occ:, :] = chol[n_occ:, :n_occ]
        return C

    # TinySCF_get_initial_guess (TinySCF.c:324-364)
    def get_initial_guess(self):
        n = self.nbf
        D = np.zeros((n, n))
        for a, el in enumerate(self.mol["sym"]):
            s, e = self.sh.atom_bf[a]
            nf = sum(ncart(l) for (l, _, _) in self.basis[el])
            D[s:e, s:e] = load_sad(self.bas_fname, el, nf)
        R = 1.0
        if self.charge != 0 and self.electron != 0:
            R = (self.electron - self.charge) / self.electron
        self.D = D * (R * 0.5)
        self.Cocc = self.D2Cocc(self.D, self.n_occ)

    # TinySCF_build_DF_tensor (build_DF_tensor.c:256-287)
    def build_DF_tensor(self):
        naux = self.naux
        self.pqA = np.zeros((self.nnz, naux))
        ul = np.ascontiguousarray(self.uniq_sp[:, 0])
        ur = np.ascontiguousarray(self.uniq_sp[:, 1])
        lib().ob_3center(ctypes.byref(self.sh.c), ctypes.byref(self.dsh.c), _p(ul), _p(ur), len(ul),
                         _p(self.sp_scrval), _p(self.df_sp_scrval), ctypes.c_double(SHELL_SCRTOL2),
                         _p(np.ascontiguousarray(self.bf_pair_mask)), _p(self.pqA))
        self.Jpq = np.zeros((naux, naux))
        lib().ob_2center(ctypes.byref(self.dsh.c), _p(self.df_sp_scrval), ctypes.c_double(SHELL_SCRTOL2), _p(self.Jpq))
        w, U = np.linalg.eigh(self.Jpq)                       # calc_inverse_sqrt_Jpq, :205-237
        self.Jpq_invsqrt = (U * (1.0 / np.sqrt(w))) @ U.T
        self.df_tensor = self.pqA @ self.Jpq_invsqrt          # generate_df_tensor, :240-254

    # build_J_mat (build_Fock.c:37-130): screened upper entries stay zero.
    def build_J(self, D):
        n, B = self.nbf, self.df_tensor
        rows = np.repeat(np.arange(n), np.diff(self.bf_mask_displs))
        cols = self.bf_pair_j
        up = cols >= rows
        w = np.where(cols[up] == rows[up], 1.0, 2.0) * D[rows[up], cols[up]]
        t = w @ B[up]
        J = np.zeros((n, n))
        J[rows[up], cols[up]] = B[up] @ t
        iu = np.triu_indices(n, 1)
        J[(iu[1], iu[0])] = J[iu]                             # symmetrize, build_Fock.c:369-379
        return J

    # build_K_mat_Cocc (build_Fock.c:244-347): T(i,s,P) = sum_j C(j,s) B(ij,P), K = T T^T.
    def build_K(self, Cocc):
        n, naux, no = self.nbf, self.naux, Cocc.shape[1]
        T = np.zeros((n, no, naux))
        for i in range(n):
            s, e = self.bf_mask_displs[i], self.bf_mask_displs[i + 1]
            T[i] = Cocc[self.bf_pair_j[s:e]].T @ self.df_tensor[s:e]
        T2 = T.reshape(n, no * naux)
        K = T2 @ T2.T
        iu = np.triu_indices(n, 1)
        K[(iu[1], iu[0])] = K[iu]
        return K

    # TinySCF_build_FockMat (build_Fock.c:349-396)
    def build_FockMat(self):
        self.J = self.build_J(self.D)
        self.K = self.build_K(self.Cocc)
        self.F = self.H + 2.0 * self.J - self.K

    # TinySCF_calc_energy (TinySCF.c:367-376)
    def calc_energy(self):
        self.HF_energy = float(np.sum(self.D * (self.F + self.H)))

    # TinySCF_DIIS (DIIS.c:12-123), commutator DIIS with its replacement policy.
    def DIIS(self, it):
        X, F = self.X, self.F
        if it <= 1:
            self.F = X.T @ F @ X
            return
        if self.diis_len < self.max_diis:
            idx = self.diis_len
            self.diis_len += 1
        else:
            idx = self.bmax_id
        FDS = F @ self.D @ self.S
        Rn = X.T @ (FDS - FDS.T) @ X
        self.R[idx] = Rn
        L = self.diis_len
        dots = np.array([float(np.dot(Rn.ravel(), self.R[j].ravel())) for j in range(L)])
        self.B[idx, :L] = dots
        self.B[:L, idx] = dots
        for i in range(L):
            if self.B[i, i] > self.bmax:
                self.bmax, self.bmax_id = self.B[i, i], i
        Fo = X.T @ F @ X
        self.F0[idx] = Fo
        rhs = np.zeros(L + 1)
        rhs[L] = -1.0
        c = np.linalg.solve(self.B[:L + 1, :L + 1], rhs)
        self.F = np.tensordot(c[:L], self.F0[:L], axes=1)

    # quickSort_eigval (build_density.c:12-35), including its index-swap slip.
    @staticmethod
    def quickSort_eigval(ev, idx, l, r):
        i, j = l, r
        mid = ev[(i + j) // 2]
        while i <= j:
            while ev[i] < mid:
                i += 1
            while ev[j] > mid:
                j -= 1
            if i <= j:
                idx[i] = idx[j]
                idx[j] = idx[i]
                ev[i], ev[j] = ev[j], ev[i]
                i += 1
                j -= 1
        if i < r:
            OracleSCF.quickSort_eigval(ev, idx, i, r)
        if j > l:
            OracleSCF.quickSort_eigval(ev, idx, l, j)

    # TinySCF_build_DenMat (build_density.c:37-69)
    def build_DenMat(self):
        w, C0 = np.linalg.eigh(self.F)
        C = self.X @ C0
        idx = list(range(self.nbf))
        ev = list(w)
        self.quickSort_eigval(ev, idx, 0, self.nbf - 1)
        self.eigval = np.array(ev)
        self.Cocc = np.ascontiguousarray(C[:, idx[:self.n_occ]])
        self.D = self.Cocc @ self.Cocc.T

    def setup(self):
        """main.c:28-40 in order."""
        self.compute_Hcore_Ovlp_mat()
        self.compute_sq_Schwarz_scrvals()
        self.prepare_sparsity()
        self.get_initial_guess()
        self.build_DF_tensor()

    # TinySCF_do_SCF (TinySCF.c:378-435)
    def do_SCF(self, callback=None):
        self.energies = []
        prev, delta, it = 0.0, 223.0, 0
        while it < self.niters and delta >= ENE_TOL:
            self.build_FockMat()
            self.calc_energy()
            delta = abs(self.HF_energy - prev)
            prev = self.HF_energy
            if callback is not None:
                callback(it, self)
            self.DIIS(it)
            self.build_DenMat()
            self.energies.append(self.HF_energy + self.nuc_energy)
            if it == 0:
                delta = 223.0
            it += 1
        self.iter = it
        return self.energies
