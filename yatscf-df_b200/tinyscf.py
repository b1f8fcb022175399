"""Python binding of the B200 TinySCF engine (libtinyscf_b200.so) via ctypes.

Mirrors the reference's TinySCF C API (huanghua1994/YATSCF-DF, TinySCF.h:107-138,
build_DF_tensor.h:6, build_Fock.h:6, build_density.h:6-8, DIIS.h:6) one call per
function, in main.c's order, plus the engine's status-returning extensions
(include/tinyscf_b200.h). Every call goes through the C ABI; there is no Python
or CPU fallback: if the shared library or a CUDA device is missing, the calls
raise.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libtinyscf_b200.so")

MAX_DIIS = 10
TIMERS = ["HCORE", "SCHWARZ", "GUESS", "3C", "2C", "INVSQRT", "DFGEMM", "J", "K_HT", "K_SYRK",
          "FOCK", "DIIS", "DENSITY", "ITER", "SCF", "K_MIXED", "FINAL", "K_HALF", "K_GEMM"]
K_FP64, K_MIXED = 0, 1
DENSITY_EIG, DENSITY_REFINE = 0, 1
GUESS_SAD, GUESS_LEARNED, GUESS_SAD_PROJECTED = 0, 1, 2
GUESS_DIN, GUESS_MAXF = 128, 15
GUESS_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "guess_weights.bin")
STATUS = {0: "success", 1: "CUDA error", 2: "cannot open input file", 3: "invalid input",
          4: "unsupported input", 5: "device allocation failed", 6: "numerical failure",
          7: "call out of order"}


class TinySCFStruct(ctypes.Structure):
    """struct TinySCF_struct of include/TinySCF.h, field for field."""
    _fields_ = [
        ("basis", ctypes.c_void_p), ("df_basis", ctypes.c_void_p),
        ("natoms", ctypes.c_int), ("nshells", ctypes.c_int),
        ("nbasfuncs", ctypes.c_int), ("n_occ", ctypes.c_int),
        ("charge", ctypes.c_int), ("electron", ctypes.c_int),
        ("df_nbf", ctypes.c_int), ("df_nshells", ctypes.c_int),
        ("nshellpairs", ctypes.c_int), ("num_uniq_sp", ctypes.c_int),
        ("mat_size", ctypes.c_int), ("max_dim", ctypes.c_int),
        ("niters", ctypes.c_int), ("iter", ctypes.c_int),
        ("nuc_energy", ctypes.c_double), ("HF_energy", ctypes.c_double), ("ene_tol", ctypes.c_double),
        ("shell_scrtol2", ctypes.c_double), ("max_scrval", ctypes.c_double), ("max_df_scrval", ctypes.c_double),
        ("sp_scrval", ctypes.POINTER(ctypes.c_double)), ("bf_pair_scrval", ctypes.POINTER(ctypes.c_double)),
        ("uniq_sp_lid", ctypes.POINTER(ctypes.c_int)), ("uniq_sp_rid", ctypes.POINTER(ctypes.c_int)),
        ("df_sp_scrval", ctypes.POINTER(ctypes.c_double)),
        ("bf_pair_mask", ctypes.POINTER(ctypes.c_int)), ("bf_pair_j", ctypes.POINTER(ctypes.c_int)),
        ("bf_pair_diag", ctypes.POINTER(ctypes.c_int)), ("bf_mask_displs", ctypes.POINTER(ctypes.c_int)),
        ("num_bf_pair_scr", ctypes.c_int),
        ("shell_bf_sind", ctypes.POINTER(ctypes.c_int)), ("shell_bf_num", ctypes.POINTER(ctypes.c_int)),
        ("df_shell_bf_sind", ctypes.POINTER(ctypes.c_int)), ("df_shell_bf_num", ctypes.POINTER(ctypes.c_int)),
        ("Hcore_mat", ctypes.POINTER(ctypes.c_double)), ("S_mat", ctypes.POINTER(ctypes.c_double)),
        ("F_mat", ctypes.POINTER(ctypes.c_double)), ("D_mat", ctypes.POINTER(ctypes.c_double)),
        ("J_mat", ctypes.POINTER(ctypes.c_double)), ("K_mat", ctypes.POINTER(ctypes.c_double)),
        ("X_mat", ctypes.POINTER(ctypes.c_double)),
        ("Cocc_mat", ctypes.POINTER(ctypes.c_double)), ("eigval", ctypes.POINTER(ctypes.c_double)),
        ("ev_idx", ctypes.POINTER(ctypes.c_int)), ("tmp_mat", ctypes.POINTER(ctypes.c_double)),
        ("DIIS_len", ctypes.c_int), ("DIIS_bmax_id", ctypes.c_int), ("DIIS_bmax", ctypes.c_double),
        ("max_diis", ctypes.c_int),
        ("mem_size", ctypes.c_double), ("init_time", ctypes.c_double),
        ("S_Hcore_time", ctypes.c_double), ("shell_scr_time", ctypes.c_double),
        ("status", ctypes.c_int), ("device", ctypes.c_int), ("verbose", ctypes.c_int),
        ("dev", ctypes.c_void_p),
    ]


TinySCF_t = ctypes.POINTER(TinySCFStruct)
_lib = None


def load_library(path=LIBPATH):
    """Load libtinyscf_b200.so and declare every entry point's signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("libtinyscf_b200.so is not built (%s); run __graft_entry__.build()" % path)
    lib = ctypes.CDLL(path)
    T = TinySCF_t
    cp, dp, ip = ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int
    fp = ctypes.POINTER(ctypes.c_float)
    sig = {
        "TinySCF_alloc": ([], T),
        "TinySCF_status_string": ([ip], ctypes.c_char_p),
        "TinySCF_struct_size": ([], ctypes.c_size_t),
        "TinySCF_init_status": ([T, cp, cp, cp, ip], ip),
        "TinySCF_compute_Hcore_Ovlp_mat_status": ([T], ip),
        "TinySCF_compute_sq_Schwarz_scrvals_status": ([T], ip),
        "TinySCF_prepare_sparsity_status": ([T], ip),
        "TinySCF_get_initial_guess_status": ([T], ip),
        "TinySCF_build_DF_tensor_status": ([T], ip),
        "TinySCF_build_FockMat_status": ([T], ip),
        "TinySCF_DIIS_status": ([T], ip),
        "TinySCF_build_DenMat_status": ([T], ip),
        "TinySCF_do_SCF_status": ([T], ip),
        "TinySCF_free_status": ([T], ip),
        "TinySCF_set_density": ([T, dp, dp], ip),
        "TinySCF_set_fock": ([T, dp, ip], ip),
        "TinySCF_sync_host": ([T], ip),
        "TinySCF_get_df_tensor": ([T, dp], ip),
        "TinySCF_get_timings": ([T, dp, ip], ip),
        "TinySCF_get_timing_stats": ([T, dp, ctypes.POINTER(ctypes.c_longlong), ip], ip),
        "TinySCF_reset_timing_stats": ([T], ip),
        "TinySCF_get_counters": ([T, ctypes.POINTER(ctypes.c_longlong), ip], ip),
        "TinySCF_reset_scf": ([T], ip),
        "TinySCF_set_k_precision": ([T, ip], ip),
        "TinySCF_set_density_solver": ([T, ip], ip),
        "TinySCF_set_graph": ([T, ip], ip),
        "TinySCF_set_guess": ([T, ip, ctypes.c_char_p], ip),
        "TinySCF_batch_create": ([ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(T), ip], ip),
        "TinySCF_batch_do_SCF": ([ctypes.c_void_p], ip),
        "TinySCF_batch_stats": ([ctypes.c_void_p, dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)],
                                ip),
        "TinySCF_batch_free": ([ctypes.c_void_p], ip),
        "TinySCF_batch_phase_ms": ([ctypes.c_void_p, dp, ip], ip),
        "TinySCF_set_autotune": ([ip], ip),
        "TinySCF_device_memory": ([ip, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)], ip),
        "TinySCF_autotune_report": ([ctypes.c_char_p, ip], ip),
        "TinySCF_guess_used": ([T], ip),
        "TinySCF_guess_dataset": ([T, dp, fp, fp, ctypes.POINTER(ctypes.c_int), ctypes.c_longlong], ctypes.c_longlong),
        "TinySCF_guess_train": ([fp, fp, ctypes.POINTER(ctypes.c_int), ctypes.c_longlong, ip, ip, ctypes.c_float,
                                 ctypes.c_uint, ctypes.c_char_p, fp], ip),
        "TinySCF_guess_mlp_grad": ([ip, ip, ip, fp, fp, fp, ip, fp, fp], ip),
        "TinySCF_guess_rotation": ([ctypes.POINTER(ctypes.c_int), ip, dp, dp], ip),
        "TinySCF_guess_pairs": ([ip, ctypes.POINTER(ctypes.c_int), dp, ctypes.POINTER(ctypes.c_int),
                                 ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                 ctypes.POINTER(ctypes.c_int), dp, ctypes.POINTER(ctypes.c_float),
                                 ctypes.c_longlong], ctypes.c_longlong),
        "quickSort_eigval": ([dp, ctypes.POINTER(ctypes.c_int), ip, ip], None),
        "TinySCF_eigh": ([ip, ip, dp, dp, dp], ip),
        "TinySCF_syrk_int8": ([ip, ip, ctypes.c_longlong, dp, dp], ip),
        "TinySCF_trim_memory": ([ip], ip),
        "TinySCF_kmix_wait_probe": ([T, ctypes.c_longlong, ctypes.POINTER(ctypes.c_int)], ip),
        "TinySCF_set_aux_slice": ([T, ip, ip], ip),
        "TinySCF_set_JK": ([T, dp, dp], ip),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


class TinySCFError(RuntimeError):
    pass


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def guess_train(feat, target, types, path, epochs=40, batch=512, lr=2e-3, seed=0):
    """Train the guess networks on the GPU (the engine's kernels); returns the per-type final MSE."""
    lib = load_library()
    feat = np.ascontiguousarray(feat, dtype=np.float32)
    target = np.ascontiguousarray(target, dtype=np.float32)
    types = np.ascontiguousarray(types, dtype=np.int32)
    loss = np.zeros(5, dtype=np.float32)
    rc = lib.TinySCF_guess_train(_fptr(feat), _fptr(target), types.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                 len(types), epochs, batch, lr, seed, path.encode(), _fptr(loss))
    if rc:
        raise TinySCFError("guess_train: " + STATUS.get(rc, str(rc)))
    return loss


def guess_mlp_grad(params, X, T, din, hid, dout):
    """(loss, gradient) of one guess MLP computed by the training kernels."""
    lib = load_library()
    params = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    g = np.zeros_like(params)
    loss = np.zeros(1, dtype=np.float32)
    rc = lib.TinySCF_guess_mlp_grad(din, hid, dout, _fptr(params), _fptr(X), _fptr(T), X.shape[0], _fptr(g),
                                    _fptr(loss))
    if rc:
        raise TinySCFError("guess_mlp_grad: " + STATUS.get(rc, str(rc)))
    return float(loss[0]), g


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class TinySCF:
    """One engine instance (one molecule) on one GPU."""

    def __init__(self, bas_fname, df_bas_fname, xyz_fname, niters=30, verbose=0, max_diis=MAX_DIIS, device=None):
        self.lib = load_library()
        self.t = self.lib.TinySCF_alloc()
        old = os.environ.get("TINYSCF_VERBOSE")
        olddev = os.environ.get("TINYSCF_DEVICE")
        os.environ["TINYSCF_VERBOSE"] = str(int(verbose))
        if device is not None:
            os.environ["TINYSCF_DEVICE"] = str(int(device))
        try:
            rc = self.lib.TinySCF_init_status(self.t, bas_fname.encode(), df_bas_fname.encode(),
                                              xyz_fname.encode(), int(niters))
        finally:
            for k, v in (("TINYSCF_VERBOSE", old), ("TINYSCF_DEVICE", olddev)):
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        if rc:
            self.lib.TinySCF_free_status(self.t)
            self.t = None
            raise TinySCFError("init_TinySCF: " + STATUS.get(rc, str(rc)))
        self.s.max_diis = int(max_diis)

    @property
    def s(self):
        return self.t.contents

    def _call(self, name):
        rc = getattr(self.lib, name + "_status")(self.t)
        if rc:
            raise TinySCFError("%s: %s" % (name, STATUS.get(rc, str(rc))))

    # --- the reference's API, main.c:28-46 order
    def compute_Hcore_Ovlp_mat(self):
        self._call("TinySCF_compute_Hcore_Ovlp_mat")

    def compute_sq_Schwarz_scrvals(self):
        self._call("TinySCF_compute_sq_Schwarz_scrvals")

    def prepare_sparsity(self):
        self._call("TinySCF_prepare_sparsity")

    def get_initial_guess(self):
        self._call("TinySCF_get_initial_guess")

    def build_DF_tensor(self):
        self._call("TinySCF_build_DF_tensor")

    def build_FockMat(self):
        self._call("TinySCF_build_FockMat")

    def DIIS(self):
        self._call("TinySCF_DIIS")

    def build_DenMat(self):
        self._call("TinySCF_build_DenMat")

    def do_SCF(self):
        self._call("TinySCF_do_SCF")

    def setup(self, guess=None):
        """main.c's set-up sequence; guess selects the initial guess (default: SAD)."""
        self.compute_Hcore_Ovlp_mat()
        self.compute_sq_Schwarz_scrvals()
        self.prepare_sparsity()
        if guess is not None:
            self.set_guess(guess)
        self.get_initial_guess()
        self.build_DF_tensor()

    # --- extensions
    def set_density(self, D, Cocc=None):
        D = np.ascontiguousarray(D, dtype=np.float64)
        C = None if Cocc is None else np.ascontiguousarray(Cocc, dtype=np.float64)
        rc = self.lib.TinySCF_set_density(self.t, _dptr(D), None if C is None else _dptr(C))
        if rc:
            raise TinySCFError("set_density: " + STATUS.get(rc, str(rc)))

    def set_fock(self, F, orthogonal=False):
        F = np.ascontiguousarray(F, dtype=np.float64)
        rc = self.lib.TinySCF_set_fock(self.t, _dptr(F), int(bool(orthogonal)))
        if rc:
            raise TinySCFError("set_fock: " + STATUS.get(rc, str(rc)))

    def sync_host(self):
        rc = self.lib.TinySCF_sync_host(self.t)
        if rc:
            raise TinySCFError("sync_host: " + STATUS.get(rc, str(rc)))

    def df_tensor(self):
        out = np.empty((self.s.num_bf_pair_scr, self.s.df_nbf))
        rc = self.lib.TinySCF_get_df_tensor(self.t, _dptr(out))
        if rc:
            raise TinySCFError("get_df_tensor: " + STATUS.get(rc, str(rc)))
        return out

    def set_k_precision(self, mode):
        """K_FP64 (the reference's arithmetic) or K_MIXED (tensor-core incremental K, final FP64 build)."""
        rc = self.lib.TinySCF_set_k_precision(self.t, int(mode))
        if rc:
            raise TinySCFError("set_k_precision: " + STATUS.get(rc, str(rc)))

    def set_density_solver(self, mode):
        """DENSITY_EIG (full eigensolve every iteration, the reference's) or DENSITY_REFINE."""
        rc = self.lib.TinySCF_set_density_solver(self.t, int(mode))
        if rc:
            raise TinySCFError("set_density_solver: " + STATUS.get(rc, str(rc)))

    def set_graph(self, on):
        """Run SCF iterations from the DIIS start as CUDA-graph launches."""
        rc = self.lib.TinySCF_set_graph(self.t, int(bool(on)))
        if rc:
            raise TinySCFError("set_graph: " + STATUS.get(rc, str(rc)))

    def set_guess(self, mode, weights=None):
        """GUESS_SAD (the reference's) or GUESS_LEARNED (weights file; default: the packaged one)."""
        if mode == GUESS_LEARNED and weights is None:
            weights = GUESS_WEIGHTS
        rc = self.lib.TinySCF_set_guess(self.t, int(mode), None if weights is None else weights.encode())
        if rc:
            raise TinySCFError("set_guess: " + STATUS.get(rc, str(rc)))

    def guess_used(self):
        return int(self.lib.TinySCF_guess_used(self.t))

    def guess_dataset(self, D):
        """(features [n,128], local target blocks [n,225], block types [n]) for density D."""
        D = np.ascontiguousarray(D, dtype=np.float64)
        n = self.lib.TinySCF_guess_dataset(self.t, _dptr(D), None, None, None, 0)
        if n < 0:
            raise TinySCFError("guess_dataset: " + STATUS.get(-n, str(-n)))
        feat = np.zeros((n, GUESS_DIN), dtype=np.float32)
        tgt = np.zeros((n, GUESS_MAXF * GUESS_MAXF), dtype=np.float32)
        typ = np.zeros(n, dtype=np.int32)
        got = self.lib.TinySCF_guess_dataset(self.t, _dptr(D), _fptr(feat), _fptr(tgt),
                                            typ.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n)
        if got != n:
            raise TinySCFError("guess_dataset: %d" % got)
        return feat, tgt, typ

    def set_aux_slice(self, p0, p1):
        """Hold and use only the DF tensor's aux columns [p0, p1) (before build_DF_tensor)."""
        rc = self.lib.TinySCF_set_aux_slice(self.t, int(p0), int(p1))
        if rc:
            raise TinySCFError("set_aux_slice: " + STATUS.get(rc, str(rc)))

    def set_JK(self, J, K):
        """Set the (reduced) J and K and recompute F and the energy."""
        J = np.ascontiguousarray(J, dtype=np.float64)
        K = np.ascontiguousarray(K, dtype=np.float64)
        rc = self.lib.TinySCF_set_JK(self.t, _dptr(J), _dptr(K))
        if rc:
            raise TinySCFError("set_JK: " + STATUS.get(rc, str(rc)))

    def kmix_wait_probe(self, wait_cycles):
        """Code recorded by the tensor-core G GEMM kernel when its waits are run
        out on purpose (wait_cycles clock cycles, no copies issued); 0 if none gave up."""
        code = ctypes.c_int(0)
        rc = self.lib.TinySCF_kmix_wait_probe(self.t, int(wait_cycles), ctypes.byref(code))
        if rc:
            raise TinySCFError("kmix_wait_probe: " + STATUS.get(rc, str(rc)))
        return code.value

    def reset_scf(self):
        rc = self.lib.TinySCF_reset_scf(self.t)
        if rc:
            raise TinySCFError("reset_scf: " + STATUS.get(rc, str(rc)))

    def timing_stats(self):
        """{phase: (total ms, number of timed calls)} since the last reset_timing_stats()."""
        ms = np.zeros(len(TIMERS))
        cnt = (ctypes.c_longlong * len(TIMERS))()
        self.lib.TinySCF_get_timing_stats(self.t, _dptr(ms), cnt, len(TIMERS))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(TIMERS)}

    def reset_timing_stats(self):
        self.lib.TinySCF_reset_timing_stats(self.t)

    def counters(self):
        """(engine kernel launches in this process, bytes host->device, bytes device->host,
        full eigensolves, subspace refinement steps, 3-centre (shell pair, aux shell) tuples,
        restarts from the SAD guess by the divergence guard, K = T T^T products run on the
        integer tensor cores)."""
        out = (ctypes.c_longlong * 8)()
        self.lib.TinySCF_get_counters(self.t, out, 8)
        return tuple(int(v) for v in out)

    def timings(self):
        ms = np.zeros(len(TIMERS))
        self.lib.TinySCF_get_timings(self.t, _dptr(ms), len(TIMERS))
        return dict(zip(TIMERS, ms))

    # --- host mirrors as numpy copies
    def _mat(self, name, shape):
        p = getattr(self.s, name)
        n = int(np.prod(shape))
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(shape).copy()

    def mat(self, name):
        n = self.s.nbasfuncs
        if name == "Cocc_mat":
            return self._mat(name, (n, self.s.n_occ))
        if name == "eigval":
            return self._mat(name, (n,))
        return self._mat(name, (n, n))

    def csr(self):
        n = self.s.nbasfuncs
        nnz = self.s.num_bf_pair_scr
        return (self._mat("bf_pair_mask", (n, n)), self._mat("bf_pair_j", (nnz,)),
                self._mat("bf_mask_displs", (n + 1,)))

    @property
    def energy(self):
        return self.s.HF_energy + self.s.nuc_energy

    def free(self):
        if self.t is not None:
            self.lib.TinySCF_free_status(self.t)
            self.t = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class TinySCFBatch:
    """Batched SCF over engines that have been set up (TinySCF.setup()); every
    SCF phase is one launch over all molecules still iterating."""

    def __init__(self, engines):
        self.lib = load_library()
        self.engines = list(engines)
        arr = (TinySCF_t * len(self.engines))(*[e.t for e in self.engines])
        self.b = ctypes.c_void_p()
        rc = self.lib.TinySCF_batch_create(ctypes.byref(self.b), arr, len(self.engines))
        if rc:
            raise TinySCFError("batch_create: " + STATUS.get(rc, str(rc)))

    def do_SCF(self):
        rc = self.lib.TinySCF_batch_do_SCF(self.b)
        if rc:
            raise TinySCFError("batch_do_SCF: " + STATUS.get(rc, str(rc)))

    def stats(self):
        """(device ms of the last batched SCF, batched iterations, kernel launches)."""
        ms = ctypes.c_double()
        it = ctypes.c_int()
        nl = ctypes.c_longlong()
        self.lib.TinySCF_batch_stats(self.b, ctypes.byref(ms), ctypes.byref(it), ctypes.byref(nl))
        return ms.value, it.value, nl.value

    def phase_ms(self):
        """{phase: device ms} of the last batched SCF."""
        ms = np.zeros(6)
        self.lib.TinySCF_batch_phase_ms(self.b, _dptr(ms), 6)
        return dict(zip(("J", "K", "FOCK", "DIIS", "DENSITY", "FINAL"), (float(v) for v in ms)))

    def free(self):
        if self.b:
            self.lib.TinySCF_batch_free(self.b)
            self.b = None


def autotune_report():
    """The autotuner's choices so far (text, one line per tuned shape)."""
    lib = load_library()
    n = lib.TinySCF_autotune_report(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib.TinySCF_autotune_report(buf, n + 1)
    return buf.value.decode()


def set_autotune(on):
    load_library().TinySCF_set_autotune(int(bool(on)))


def eigh(A, device=0):
    """(w, V) of a symmetric matrix from the engine's device eigensolver:
    eigenvalues ascending, V[k] the k-th eigenvector."""
    lib = load_library()
    A = np.ascontiguousarray(A, dtype=np.float64)
    n = A.shape[0]
    w = np.zeros(n)
    V = np.zeros((n, n))
    rc = lib.TinySCF_eigh(int(device), n, _dptr(A), _dptr(w), _dptr(V))
    if rc:
        raise TinySCFError("eigh: " + STATUS.get(rc, str(rc)))
    return w, V


def trim_memory(device=0):
    """Return the memory that freed engines left in the device's pool."""
    rc = load_library().TinySCF_trim_memory(int(device))
    if rc:
        raise TinySCFError("trim_memory: " + STATUS.get(rc, str(rc)))


def syrk_int8(T, device=0):
    """K = T T^T (FP64 accuracy) from the engine's integer-tensor-core product."""
    lib = load_library()
    T = np.ascontiguousarray(T, dtype=np.float64)
    n, q = T.shape
    K = np.zeros((n, n))
    rc = lib.TinySCF_syrk_int8(int(device), n, ctypes.c_longlong(q), _dptr(T), _dptr(K))
    if rc:
        raise TinySCFError("syrk_int8: " + STATUS.get(rc, str(rc)))
    return K


def device_memory(device=0):
    """(free bytes, total bytes) of a CUDA device."""
    lib = load_library()
    f, t = ctypes.c_longlong(), ctypes.c_longlong()
    rc = lib.TinySCF_device_memory(int(device), ctypes.byref(f), ctypes.byref(t))
    if rc:
        raise TinySCFError("device_memory: " + STATUS.get(rc, str(rc)))
    return f.value, t.value


def guess_pairs(elem, xyz_bohr, shell_am):
    """The learned guess's pair blocks (host code, no GPU): elem (0-based element
    indices), xyz_bohr (natoms x 3), shell_am (one list of shell angular momenta
    per atom). Returns dict(ab [n,2], type [n], frame [n,3,3], feat [n,128])."""
    lib = load_library()
    ci = ctypes.POINTER(ctypes.c_int)
    el = np.ascontiguousarray(elem, dtype=np.int32)
    xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64)
    ns = np.ascontiguousarray([len(s) for s in shell_am], dtype=np.int32)
    am = np.ascontiguousarray([l for s in shell_am for l in s], dtype=np.int32)
    args = (len(el), el.ctypes.data_as(ci), _dptr(xyz), ns.ctypes.data_as(ci), am.ctypes.data_as(ci))
    n = lib.TinySCF_guess_pairs(*args, None, None, None, None, 0)
    if n < 0:
        raise TinySCFError("guess_pairs: " + STATUS.get(-n, str(-n)))
    ab = np.zeros((n, 2), dtype=np.int32)
    ty = np.zeros(n, dtype=np.int32)
    fr = np.zeros((n, 3, 3))
    ft = np.zeros((n, GUESS_DIN), dtype=np.float32)
    m = lib.TinySCF_guess_pairs(*args, ab.ctypes.data_as(ci), ty.ctypes.data_as(ci), _dptr(fr),
                                ft.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n)
    if m != n:
        raise TinySCFError("guess_pairs: " + STATUS.get(-m, str(m)))
    return dict(ab=ab, type=ty, frame=fr, feat=ft)


def guess_rotation(shell_am, Q):
    """M with phi_molecule = M phi_local for one atom's Cartesian shells (x_m = Q^T x_l)."""
    lib = load_library()
    am = np.ascontiguousarray(shell_am, dtype=np.int32)
    Q = np.ascontiguousarray(Q, dtype=np.float64)
    nf = int(sum((l + 1) * (l + 2) // 2 for l in am))
    M = np.zeros((nf, nf))
    rc = lib.TinySCF_guess_rotation(am.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(am), _dptr(Q), _dptr(M))
    if rc:
        raise TinySCFError("guess_rotation: " + STATUS.get(rc, str(rc)))
    return M
