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


def _init_message(bas, dfbas, xyz):
    """init_TinySCF's outcome in a child process with no visible GPU: parse
    errors come back before any CUDA call; input that parses ends at the
    missing device."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import tinyscf\n"
            "try:\n    tinyscf.TinySCF(%r, %r, %r)\nexcept tinyscf.TinySCFError as e:\n    print('ERR', e)\n"
            % (os.path.join(REPO, "yatscf-df_b200"), str(bas), str(dfbas), str(xyz)))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         env=dict(os.environ, CUDA_VISIBLE_DEVICES=""), timeout=120)
    return out.stdout + out.stderr


BAS = os.path.join(REPO, "tests/golden/data/cc-pvdz/cc-pvdz.gbs")
DFBAS = os.path.join(REPO, "tests/golden/data/cc-pVDZ-RI/cc-pVDZ-RI.gbs")
WATER = "3\n0\nO 0.0 0.0 0.1173\nH 0.0 0.7572 -0.4692\nH 0.0 -0.7572 -0.4692\n"


@pytest.mark.parametrize("xyz", [
    "3\n0\nO 0.0 0.0 nan\nH 0.0 0.7572 -0.4692\nH 0.0 -0.7572 -0.4692\n",     # non-finite coordinate
    "3\n0\nO 0.0 0.0 0.0\nH 0.0 0.0 0.0\nH 0.0 -0.7572 -0.4692\n",            # coincident nuclei
    "3\n0\nO 0.0 0.0 0.1173\nH 0.0 0.7572\nH 0.0 -0.7572 -0.4692\n",         # missing coordinate
    "4\n0\nO 0.0 0.0 0.1173\nH 0.0 0.7572 -0.4692\nH 0.0 -0.7572 -0.4692\n",  # fewer atoms than declared
    "3\n0\nO 0.0 0.0 0.1173\nXx 0.0 0.7572 -0.4692\nH 0.0 -0.7572 -0.4692\n", # unknown element
])
def test_bad_geometry_is_invalid_input(tmp_path, xyz):
    f = tmp_path / "m.xyz"
    f.write_text(xyz)
    assert "ERR init_TinySCF: invalid input" in _init_message(BAS, DFBAS, f)


def _edit_first_primitive(tmp_path, fn):
    """The orbital basis with the first primitive row of the first shell edited by fn."""
    lines = open(BAS).read().splitlines()
    for k, L in enumerate(lines):
        parts = L.split()
        if k > 0 and len(parts) >= 2 and parts[0] == "S" and parts[1].isdigit():
            lines[k + 1] = fn(lines[k + 1])
            break
    f = tmp_path / "b.gbs"
    f.write_text("\n".join(lines) + "\n")
    return f


@pytest.mark.parametrize("edit", [
    lambda r: r.split()[0],                                 # coefficient missing
    lambda r: "-" + r.split()[0] + " " + r.split()[1],      # negative exponent
    lambda r: r.split()[0] + " inf",                        # non-finite coefficient
])
def test_bad_basis_row_is_invalid_input(tmp_path, edit):
    m = tmp_path / "w.xyz"
    m.write_text(WATER)
    assert "ERR init_TinySCF: invalid input" in _init_message(_edit_first_primitive(tmp_path, edit), DFBAS, m)


def test_fortran_exponents_parse(tmp_path):
    """1.234D+01 reads as 1.234E+01: such a basis gets past parsing (and then
    stops at the missing device), where a misread row would be invalid input."""
    m = tmp_path / "w.xyz"
    m.write_text(WATER)

    def to_fortran(r):
        e, c = r.split()[:2]
        return "%.10EAND%.10E" % (float(e), float(c))

    f = _edit_first_primitive(tmp_path, lambda r: to_fortran(r).replace("E", "D").replace("AND", "  "))
    assert "D+" in f.read_text() or "D-" in f.read_text()
    assert "ERR init_TinySCF: CUDA error" in _init_message(f, DFBAS, m)
    assert "ERR init_TinySCF: CUDA error" in _init_message(BAS, DFBAS, m)
