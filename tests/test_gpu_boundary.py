"""The drop-in boundary as a C caller sees it: the reference's own main.c
(main.c:24-46: init_TinySCF ... TinySCF_do_SCF, free_TinySCF), compiled
unchanged against include/ and linked to libtinyscf_b200.so by
`make -C oracle ref` (oracle/_ref/main_on_engine), solves water and prints
the reference's per-iteration energy lines; the last one must be the
reference's converged energy."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import BAS, DFBAS, GOLDEN, REPO, xyz

pytestmark = pytest.mark.gpu

EXE = os.path.join(REPO, "oracle", "_ref", "main_on_engine")


@pytest.mark.skipif(not os.path.exists(EXE), reason="main.c was not compiled (no reference checkout at build time)")
def test_reference_main_runs_on_the_engine():
    gold = np.load(os.path.join(GOLDEN, "water_ref.npz"))
    out = subprocess.run([EXE, BAS, DFBAS, xyz("water"), "30"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    energies = [float(m) for m in re.findall(r"\* Energy = (-?\d+\.\d+)", out.stdout)]
    assert len(energies) == len(gold["energies"])
    assert abs(energies[-1] - float(gold["energies"][-1])) < 1e-9
