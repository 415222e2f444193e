"""The FP64 purification step and the commutator with their operands copied by the tensor memory
accelerator (k_sp2_step_tma, k_commutator_tma: TMA boxes and an mbarrier pipeline) against the same
products copied with cp.async (AM1GPU_SP2_TMA=0: k_sp2_step16, k_commutator16), on a B200.

Both runs use the same MMAs in the same order.  The tensor-map kernels read the second operand by
rows (B = M^T for a symmetric M), so an operand that is symmetric only to rounding (the Fock matrix
and the first iterate built from it) can move the last bits, and two SCF runs whose roundings differ
stop at slightly different points of the same convergence test: the bars are 1e-7 kcal/mol on the heat
of formation and 1e-8 on the density (a tenth of the oracle's bar, and the oracle's bar), and the
iteration counts agree within one.  The batch mixes even orders (the tensor-map kernels) with odd ones (radicals: the 8-byte
cp.async kernels)."""

from __future__ import annotations

import json
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SCRIPT = textwrap.dedent(f"""
    import sys, json
    sys.path[:0] = [{str(ROOT / 'am1-rs_b200')!r}, {str(ROOT / 'oracle')!r}]
    import numpy as np
    from am1gpu import native, workloads as W, _abi
    rng = np.random.default_rng(17)
    mols = [W.alkane(n, rng) for n in (2, 9, 20, 33, 40)] + [W.water_cluster(k, rng) for k in (4, 11, 37, 64)]
    batch = [(m.numbers, _abi.angstrom_to_bohr(m.xyz), 0.0, 1) for m in mols]
    for n in (5, 17):
        r = W.alkane(n, rng, radical=True)
        batch.append((r.numbers, _abi.angstrom_to_bohr(r.xyz), 0.0, 2))
    status, res = native.scf_batch(batch, want_matrices=True)
    out = {{"status": [int(s) for s in status],
           "hof": [r["heat_of_formation_kcal"] for r in res],
           "iters": [int(r["iterations"]) for r in res],
           "nao": [int(r["density"].shape[0]) for r in res]}}
    np.save(sys.argv[1], np.concatenate([r["density"].ravel() for r in res]))
    print(json.dumps(out))
""")


def _run(tmp_path, tma: bool):
    f = tmp_path / "tma_run.py"
    f.write_text(SCRIPT)
    dens = tmp_path / ("dens_tma.npy" if tma else "dens_cp.npy")
    env = dict(os.environ, AM1GPU_SP2_TMA="1" if tma else "0")
    r = subprocess.run([sys.executable, str(f), str(dens)], env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1]), np.load(dens)


def test_tensor_map_products_match_cp_async_products(tmp_path):
    a, pa = _run(tmp_path, True)
    b, pb = _run(tmp_path, False)
    assert all(s == 0 for s in a["status"]) and all(s == 0 for s in b["status"])
    assert a["nao"] == b["nao"]
    assert any(n % 2 == 0 for n in a["nao"]) and any(n % 2 == 1 for n in a["nao"])
    assert np.max(np.abs(np.array(a["hof"]) - np.array(b["hof"]))) < 1e-7
    assert np.max(np.abs(pa - pb)) < 1e-8
    assert np.max(np.abs(np.array(a["iters"]) - np.array(b["iters"]))) <= 1
