"""bench.py's CPU pieces (no device): the reference arm's JSON line for one short step, the workload
builder, and the config-0 helper with stand-in solvers."""

from __future__ import annotations

import json
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_its_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "solves/s" and line["value"] > 0
    for key in ("metric", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling", "dtype",
                "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    import bench

    assert line["config"] == bench.bench_config(4096)  # the same config our arm prints
    assert line["e2e"] == {"value": line["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_workload_and_config0_helper():
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    import bench
    from am1gpu import _abi

    mols = bench.workload(6)
    assert len(mols) == 6 and all(len(m) == 4 and m[1].shape == (len(m[0]), 3) for m in mols)

    class Solver:  # stands in for am1gpu.native and the oracle module: only .scf is called
        def __init__(self, hof):
            self.hof, self.calls = hof, 0

        def scf(self, numbers, xyz_bohr, want_matrices=True):
            self.calls += 1
            assert len(numbers) == 96 and not want_matrices  # the 32-water cluster
            return {"iterations": 10, "heat_of_formation_kcal": self.hof}

    gpu, oracle = Solver(-1893.9), Solver(-1893.9 + 1e-9)
    r = bench.config0_block(gpu, _abi, oracle, reps=3)
    assert gpu.calls == 4 and oracle.calls == 1  # a warm-up call, then the timed ones
    assert r["iterations"] == 10 and abs(r["abs_dHf_kcal_vs_oracle"] - 1e-9) < 1e-12
    assert r["published_reference_cpu_s"] == 0.27 and r["gpu_scf_s"] >= 0.0 and r["oracle_threads"] == 1


def test_stratified_cpu_sample_has_the_batch_size_mix():
    # both arms time the CPU on the same 64 molecules; their orbital counts follow the batch's, so
    # the CPU's cost per molecule (about n^3) on the sample is its cost on the batch
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    import numpy as np

    import bench

    mols = bench.workload(4096)
    nao = np.array([int(np.sum(np.where(m[0] == 1, 1, 4))) for m in mols], dtype=float)
    idx = bench.stratified_sample(mols)
    assert len(idx) == bench.CPU_SAMPLE == len(set(idx))
    s = nao[idx]
    assert abs(s.mean() / nao.mean() - 1) < 0.02
    assert abs((s ** 3).mean() / (nao ** 3).mean() - 1) < 0.05
    assert bench.stratified_sample(mols) == idx  # deterministic
