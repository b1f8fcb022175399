import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "yatscf-df_b200")
ORACLE = os.path.join(REPO, "oracle")
GOLDEN = os.path.join(REPO, "tests", "golden")
DATA = os.path.join(GOLDEN, "data")
BAS = os.path.join(DATA, "cc-pvdz", "cc-pvdz.gbs")
DFBAS = os.path.join(DATA, "cc-pVDZ-RI", "cc-pVDZ-RI.gbs")

for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine through its C ABI")


def xyz(name):
    return os.path.join(DATA, name + ".xyz")
