"""bench.py's JSON line for our arm, assembled on the CPU from a stand-in
engine module (fixed timings and counters; no GPU, nothing measured): every
key the benchmark contract asks for is present with the right type, and the
derived figures follow from the engine's numbers."""
import json
import os
import subprocess
import sys

from conftest import REPO

_SCRIPT = r"""
import sys, types
sys.path.insert(0, sys.argv[1])
TIMERS = ["HCORE", "SCHWARZ", "GUESS", "3C", "2C", "INVSQRT", "DFGEMM", "J", "K_HT", "K_SYRK", "FOCK", "DIIS",
          "DENSITY", "ITER", "SCF", "K_MIXED", "FINAL", "K_HALF", "K_GEMM"]
fake = types.ModuleType("tinyscf")
fake.K_FP64, fake.K_MIXED, fake.DENSITY_EIG, fake.DENSITY_REFINE = 0, 1, 0, 1
fake.GUESS_SAD, fake.GUESS_LEARNED, fake.GUESS_SAD_PROJECTED = 0, 1, 2
fake.load_library = lambda: None


class Struct:
    nbasfuncs, n_occ, df_nbf, num_bf_pair_scr, iter = 1010, 161, 3870, 243254, 8


class Engine:
    def __init__(self, *a, **k):
        self.s, self.energy, self.g = Struct(), -1562.6, 0
        self.mixed = False
    def setup(self, guess=None): pass
    def timings(self): return {k: (2.0 if k == "GUESS" else 100.0) for k in TIMERS}
    def set_k_precision(self, m): self.mixed = m == 1
    def set_density_solver(self, m): pass
    def set_graph(self, on): pass
    def set_guess(self, m, w=None): self.g = m
    def reset_scf(self): pass
    def do_SCF(self): pass
    def reset_timing_stats(self): pass
    def counters(self): return [1000, 8 << 20, 100 << 20, 1, 16, 12345]
    def timing_stats(self): return {k: (4.0 * 45, 45) for k in TIMERS}
    def guess_used(self): return self.g
    def build_FockMat(self): pass
    def mat(self, name):
        import numpy as np
        return np.zeros((1010, 1010))
    def free(self): pass


fake.TinySCF = Engine
sys.modules["tinyscf"] = fake
import bench
bench.ClockSampler = type("Clocks", (), {"__init__": lambda s, i: None, "start": lambda s: None,
                          "stop": lambda s: {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": []}})
args = types.SimpleNamespace(gpus=1, steps=5, warmup=3, impl="ours", config="c40h82", ene_tol=1e-8, e2e_steps=1,
                             no_cpu_baseline=True, precision="mixed", no_graph=False)
bench.run_ours(args, 0, 1, 0)
"""


def test_bench_line_has_the_contract_keys():
    res = subprocess.run([sys.executable, "-c", _SCRIPT, REPO], capture_output=True, text=True, timeout=300,
                         cwd=REPO)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [line for line in res.stdout.splitlines() if line.strip()]
    assert len(lines) == 1, lines
    d = json.loads(lines[0])
    for k, t in (("metric", str), ("value", float), ("unit", str), ("n_gpus", int), ("steps", int),
                 ("warmup", int), ("ms_per_step", float), ("higher_is_better", bool), ("scaling", str),
                 ("dtype", str), ("data", str), ("config", dict), ("roofline", dict), ("e2e", dict),
                 ("gpu_launches", int), ("clocks", dict)):
        assert isinstance(d[k], t), (k, d.get(k))
    assert d["vs_baseline"] is None and d["higher_is_better"] is False
    assert d["steps"] == 5 and d["warmup"] == 3 and d["n_gpus"] == 1 and d["scaling"] == "weak"
    # one solve = GUESS (2 ms) + SCF (100 ms) device time
    assert abs(d["ms_per_step"] - 102.0) < 1e-9 and abs(d["value"] - 0.102) < 1e-12
    assert d["config"]["workload"].startswith("c40h82")
    r = d["roofline"]
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in r, k
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    # k_gemm: 2 nbf^2 n_occ naux flops per 4 ms build
    assert abs(r["achieved"] - 2.0 * 1010 ** 2 * 161 * 3870 / 4e-3 / 1e12) < 1e-6 * r["achieved"]
    e = d["e2e"]
    assert set(e) == {"value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"}
    assert e["h2d_bytes_per_step"] == 8 << 20 and e["d2h_bytes_per_step"] == 100 << 20
    assert d["gpu_launches"] == 0   # the stand-in's launch counter does not move
    assert set(d["clocks"]) >= {"sm_mhz", "sm_max_mhz", "reasons"}
    assert d["config"]["e2e_split"]["setup_device_ms"]["DFGEMM"] == 100.0
    # errors against the reference's own results (tests/golden/c40h82_ref.npz) are stated
    v = d["config"]["errors_vs_reference"]
    for k in ("J_it0_maxabs", "K_it0_maxabs", "E_it0", "E_mixed_minus_reference_limit",
              "E_plain_minus_reference_limit", "reference_limit"):
        assert isinstance(v[k], float), k
    assert abs(v["E_mixed_minus_reference_limit"] - (-1562.6 - v["reference_limit"])) < 1e-9
