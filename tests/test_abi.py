"""The C-ABI library loads without a GPU, exports every entry point declared
in include/*.h, and its struct layout matches the Python mirror."""
import ctypes
import glob
import os
import re

import pytest

from conftest import REPO
import tinyscf

HEADERS = sorted(glob.glob(os.path.join(REPO, "include", "*.h")))


def declared_symbols():
    names = set()
    for h in HEADERS:
        for m in re.finditer(r"^TINYSCF_API\s+[\w\s\*]+?\b(\w+)\s*\(", open(h).read(), flags=re.M):
            names.add(m.group(1))
    return names


def test_headers_declare_the_reference_api():
    names = declared_symbols()
    reference_api = {"init_TinySCF", "free_TinySCF", "TinySCF_init_batch_dgemm_arrays",
                     "TinySCF_free_batch_dgemm_arrays", "TinySCF_compute_Hcore_Ovlp_mat",
                     "TinySCF_compute_sq_Schwarz_scrvals", "TinySCF_prepare_sparsity", "TinySCF_get_initial_guess",
                     "TinySCF_do_SCF", "TinySCF_build_DF_tensor", "TinySCF_build_FockMat", "TinySCF_build_DenMat",
                     "quickSort_eigval", "TinySCF_DIIS"}
    assert reference_api <= names


def test_library_exports_every_declared_symbol():
    lib = tinyscf.load_library()
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layout_matches_mirror():
    lib = tinyscf.load_library()
    assert lib.TinySCF_struct_size() == ctypes.sizeof(tinyscf.TinySCFStruct)


def test_status_strings_and_host_helper():
    lib = tinyscf.load_library()
    assert lib.TinySCF_status_string(0) == b"success"
    assert lib.TinySCF_status_string(7) == b"call out of order"
    # quickSort_eigval keeps the reference's behaviour (build_density.c:12-35)
    ev = (ctypes.c_double * 4)(1.0, 2.0, 2.0, 3.0)
    idx = (ctypes.c_int * 4)(0, 1, 2, 3)
    lib.quickSort_eigval(ev, idx, 0, 3)
    assert list(ev) == [1.0, 2.0, 2.0, 3.0]
    assert list(idx) != [0, 1, 2, 3]


def test_no_device_fails_loudly_without_gpu():
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import tinyscf\n"
            "try:\n    tinyscf.TinySCF(%r, %r, %r)\nexcept tinyscf.TinySCFError as e:\n    print('ERR', e)\n"
            % (os.path.join(REPO, "yatscf-df_b200"), os.path.join(REPO, "tests/golden/data/cc-pvdz/cc-pvdz.gbs"),
               os.path.join(REPO, "tests/golden/data/cc-pVDZ-RI/cc-pVDZ-RI.gbs"),
               os.path.join(REPO, "tests/golden/data/water.xyz")))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         env=dict(os.environ, CUDA_VISIBLE_DEVICES=""), timeout=120)
    assert "ERR init_TinySCF: CUDA error" in out.stdout, out.stdout + out.stderr


def test_bad_inputs_return_status():
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import tinyscf\n"
            "try:\n    tinyscf.TinySCF('/nonexistent.gbs', 'x', 'y')\nexcept tinyscf.TinySCFError as e:\n    print('ERR', e)\n"
            % os.path.join(REPO, "yatscf-df_b200"))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert "ERR init_TinySCF: cannot open input file" in out.stdout, out.stdout + out.stderr
