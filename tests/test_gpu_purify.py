"""The purification step alone (am1gpu_density_purify) at the three product precisions of the
batched SCF, against the exact projector from numpy's eigendecomposition, on a B200.

The matrices have an AM1-like spectrum: occupied eigenvalues in [-40, -12] eV, virtual ones in
[1, 10] eV, random eigenvectors.  Bars on max |P - P_exact|: 1e-10 for the FP64 tensor-core
products and for the FP64 products from 7-bit digit planes on tcgen05's integer path; 1e-4 for
FP32-accurate products on tcgen05 (TF32 operands split in two, FP32 accumulation) and at least ten
times closer than TF32 products; 5e-2 for TF32 products, on mma.sync or in one tcgen05 pass (whose
error is within a factor of 4 of the mma.sync kernel's: the same TF32 iterates, another summation
order).  The trace is n_occ * weight in every case
(the reduced-precision runs are rescaled to it).
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fock_like(n, nocc, seed):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    ev = np.r_[rng.uniform(-40.0, -12.0, nocc), rng.uniform(1.0, 10.0, n - nocc)]
    f = (q * ev) @ q.T
    f = 0.5 * (f + f.T)
    w, v = np.linalg.eigh(f)
    return f, 2.0 * v[:, :nocc] @ v[:, :nocc].T


@pytest.mark.parametrize("n", [5, 64, 127, 128, 129, 200, 300, 448])
def test_purification_precisions_against_the_exact_projector(gpu, n):
    nocc = max(1, (2 * n) // 3)
    f, p_exact = _fock_like(n, nocc, n)
    err = {}
    for prec in ("fp64", "fp64_digits", "fp32_tcgen05", "tf32", "tf32_tcgen05"):
        p, steps = gpu.density_purify(f, nocc, 2.0, prec)
        assert 0 < steps <= 100
        assert abs(np.trace(p) - 2.0 * nocc) < 1e-6 * nocc, prec
        assert np.max(np.abs(p - p.T)) == 0.0, prec  # mirrored: exactly symmetric
        err[prec] = float(np.max(np.abs(p - p_exact)))
    assert err["fp64"] < 1e-10, err
    assert err["fp64_digits"] < 1e-10, err
    assert err["fp32_tcgen05"] < 1e-4, err
    assert err["tf32"] < 5e-2, err
    assert err["tf32_tcgen05"] < 5e-2, err
    assert err["tf32_tcgen05"] < 4.0 * err["tf32"] and err["tf32"] < 4.0 * err["tf32_tcgen05"], err
    assert err["fp32_tcgen05"] < 0.1 * err["tf32"], err


def test_purification_refuses_bad_input(gpu):
    from am1gpu import _abi

    f = np.eye(10)
    f[3, 2] = np.nan
    with pytest.raises(gpu.Am1GpuError) as e:
        gpu.density_purify(f, 3)
    assert e.value.code == _abi.LINALG
    with pytest.raises(gpu.Am1GpuError) as e:
        gpu.density_purify(np.eye(449), 3)
    assert e.value.code == _abi.INVALID_INPUT


def test_scf_with_digit_plane_products_matches_oracle(tmp_path):
    # the whole batched SCF with every FP64 purification product from digit planes on the integer
    # tensor cores (AM1GPU_FP64_DIGITS=1): the oracle's bars, as for the FP64 tensor-core products
    import subprocess
    import sys
    import textwrap

    from conftest import ROOT

    script = textwrap.dedent(f"""
        import sys
        sys.path[:0] = [{str(ROOT / 'am1-rs_b200')!r}, {str(ROOT / 'oracle')!r}]
        import numpy as np
        from am1gpu import native, workloads as W, _abi
        import oracle
        rng = np.random.default_rng(91)
        mols = [W.alkane(n, rng) for n in (1, 6, 23, 40)] + [W.water_cluster(k, rng) for k in (3, 30, 64)]
        batch = [(m.numbers, _abi.angstrom_to_bohr(m.xyz), 0.0, 1) for m in mols]
        r = W.alkane(11, rng, radical=True)
        batch.append((r.numbers, _abi.angstrom_to_bohr(r.xyz), 0.0, 2))
        status, res = native.scf_batch(batch, want_matrices=True)
        assert all(s == 0 for s in status), status
        for (z, xyz, q, mult), g in zip(batch, res):
            o = oracle.scf(z, xyz, q, mult)
            assert abs(g["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < 1e-6
            assert np.max(np.abs(g["charges"] - o["charges"])) < 1e-7
            assert np.max(np.abs(g["density"] - o["density"])) < 1e-8
            assert abs(g["iterations"] - o["iterations"]) <= 1
        print("ok")
    """)
    f = tmp_path / "digits.py"
    f.write_text(script)
    env = dict(__import__("os").environ, AM1GPU_FP64_DIGITS="1")
    r = subprocess.run([sys.executable, str(f)], env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr
