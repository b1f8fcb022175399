"""The benchmark's reference arm on the CPU: `bench.py --impl reference` runs
the reference's own C sources (oracle/_ref/ref_bench) and prints one JSON line
in the contract's shape; under a multi-rank launch only rank 0 works."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO

REF_BENCH = os.path.join(REPO, "oracle", "_ref", "ref_bench")


def _run(extra_env=None):
    env = dict(os.environ, **(extra_env or {}))
    res = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--config", "water",
                          "--steps", "2", "--warmup", "1"], env=env, capture_output=True, text=True, timeout=300,
                         cwd=REPO)
    assert res.returncode == 0, res.stderr[-2000:]
    return [line for line in res.stdout.splitlines() if line.strip()]


@pytest.mark.skipif(not os.path.exists(REF_BENCH), reason="oracle/_ref not built (needs the reference sources)")
def test_reference_arm_line():
    lines = _run()
    assert len(lines) == 1, lines
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "SCF time-to-converge at 1e-8 Eh" and d["unit"] == "s"
    assert d["higher_is_better"] is False and d["steps"] == 2 and d["warmup"] == 1
    assert d["value"] > 0 and abs(d["ms_per_step"] - 1e3 * d["value"]) < 1e-9 * max(1.0, d["ms_per_step"])
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the reference's converged energy at 1e-8 Eh against the golden run at the reference's own tolerance
    gold = np.load(os.path.join(REPO, "tests", "golden", "water_ref.npz"))["energies"][-1]
    assert abs(d["config"]["sample_energy"] - gold) < 1e-7


@pytest.mark.skipif(not os.path.exists(REF_BENCH), reason="oracle/_ref not built (needs the reference sources)")
def test_reference_arm_other_ranks_exit_quietly():
    assert _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []
