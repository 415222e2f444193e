"""The mixed-precision batched path on a B200: TF32 purification in the early SCF iterations,
FP64 for the rest (integrals, Fock build, commutator, DIIS and energies are FP64 throughout).
Its results are compared with the FP64 batched path and the oracle, for AM1 and RM1, RHF and UHF."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# the bar for the mixed path against FP64 (kcal/mol); its final iterations are FP64, so the
# results agree far below it.  Charges and densities of two SCF runs that stop at the same
# convergence test (|dE| < 1e-8 eV, RMS dP < 1e-7) on different trajectories agree to about 1e-6.
DHF_BAR = 1e-4
Q_TOL = 1e-5


def _mols(seed):
    from am1gpu import workloads as W, _abi

    rng = np.random.default_rng(seed)
    out = []
    for n in (1, 4, 9, 17, 30):
        a = W.alkane(n, rng)
        out.append((a.numbers, _abi.angstrom_to_bohr(a.xyz), 0.0, 1))
    for k in (2, 7, 16, 40):
        w = W.water_cluster(k, rng)
        out.append((w.numbers, _abi.angstrom_to_bohr(w.xyz), 0.0, 1))
    for n in (2, 5, 12):
        r = W.alkane(n, rng, radical=True)
        out.append((r.numbers, _abi.angstrom_to_bohr(r.xyz), 0.0, 2))
    return out


@pytest.mark.parametrize("method", ["am1", "rm1"])
def test_mixed_matches_fp64_and_oracle(gpu, oracle, method):
    mols = _mols(31)
    s64, r64 = gpu.scf_batch(mols, want_matrices=True, method=method)
    smx, rmx = gpu.scf_batch(mols, want_matrices=True, method=method, precision="mixed")
    st = gpu.last_call_stats()
    assert st["lowp_purification_steps"] > 0 and st["purification_steps"] > 0
    assert all(s == 0 for s in s64) and all(s == 0 for s in smx), (s64, smx)
    for i, (a, b) in enumerate(zip(r64, rmx)):
        assert a["converged"] and b["converged"]
        assert abs(a["heat_of_formation_kcal"] - b["heat_of_formation_kcal"]) < DHF_BAR, i
        assert np.max(np.abs(a["charges"] - b["charges"])) < Q_TOL, i
        assert np.max(np.abs(a["density"] - b["density"])) < Q_TOL, i
    for i in (0, 6, 10):
        z, x, q, mult = mols[i]
        o = oracle.scf(z, x, q, mult, method=method, want_matrices=False)
        assert abs(rmx[i]["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < DHF_BAR


@pytest.mark.parametrize("kernel", [0, 1, 2])
def test_mixed_with_each_reduced_precision_kernel(tmp_path, kernel):
    # AM1GPU_LOWP_TC forces the kernel of the TF32 phase (0 mma.sync TF32, 1 tcgen05 3xTF32, 2 tcgen05
    # in one TF32 pass) instead of the autotuner's choice; every one must give the FP64 results
    import subprocess
    import sys
    import textwrap

    from conftest import ROOT

    script = textwrap.dedent(f"""
        import sys
        sys.path[:0] = [{str(ROOT / 'am1-rs_b200')!r}, {str(ROOT / 'tests')!r}]
        import numpy as np
        from am1gpu import native
        from test_gpu_mixed import _mols, DHF_BAR, Q_TOL
        mols = _mols(43)
        s64, r64 = native.scf_batch(mols, want_matrices=True)
        smx, rmx = native.scf_batch(mols, want_matrices=True, precision="mixed")
        st = native.last_call_stats()
        assert st["lowp_purification_steps"] > 0, st
        assert all(x == 0 for x in s64) and all(x == 0 for x in smx), (s64, smx)
        for a, b in zip(r64, rmx):
            assert abs(a["heat_of_formation_kcal"] - b["heat_of_formation_kcal"]) < DHF_BAR
            assert np.max(np.abs(a["charges"] - b["charges"])) < Q_TOL
            assert np.max(np.abs(a["density"] - b["density"])) < Q_TOL
        print("ok")
    """)
    f = tmp_path / "lowp.py"
    f.write_text(script)
    env = dict(__import__("os").environ, AM1GPU_LOWP_TC=str(kernel))
    r = subprocess.run([sys.executable, str(f)], env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr


def test_autotuner_reports_three_kernels(gpu):
    gpu.scf_batch(_mols(5)[:4], precision="mixed")
    tab = gpu.lowp_tuning()
    tuned = [v for v in tab.values() if v["kernel"] is not None]
    assert tuned
    for v in tuned:
        assert v["kernel"] in gpu.LOWP_KERNELS
        assert all(t > 0.0 for t in v["ms"].values())
        assert v["ms"][v["kernel"]] == min(v["ms"].values())


def test_mixed_large_molecule(gpu):
    # 540 orbitals: TF32 purification on the large-matrix path too
    from am1gpu import workloads as W, _abi

    m = W.water_cluster(90, np.random.default_rng(7))
    mol = [(m.numbers, _abi.angstrom_to_bohr(m.xyz), 0.0, 1)]
    _, a = gpu.scf_batch(mol, want_matrices=False)
    s, b = gpu.scf_batch(mol, want_matrices=False, precision="mixed")
    assert s[0] == 0 and b[0]["converged"]
    assert abs(a[0]["heat_of_formation_kcal"] - b[0]["heat_of_formation_kcal"]) < DHF_BAR
    assert np.max(np.abs(a[0]["mo_energies"] - b[0]["mo_energies"])) < 1e-5


def test_plain_path_stays_fp64(gpu):
    from am1gpu import _abi

    z, x, q, m = _mols(32)[7]
    gpu.scf(z, x, q, m, precision="mixed", want_matrices=False)
    assert gpu.last_call_stats()["lowp_purification_steps"] == 0


def test_large_radicals_stay_fp64_on_the_mixed_path(gpu):
    # requests 58497, 77601 and 85316 of the serving stream (100 000 requests, seed 2): alkyl
    # radicals of 595-1021 orbitals that a TF32 start left unconverged; open shells above 448
    # orbitals now run FP64 on the mixed path, beside closed shells that take TF32
    from am1gpu import workloads as W, _abi

    rng = np.random.default_rng(58497)
    rad = W.alkane(170, rng, radical=True)  # 1021 orbitals
    clo = W.water_cluster(90, rng)          # 540 orbitals, closed shell
    mols = [(rad.numbers, _abi.angstrom_to_bohr(rad.xyz), 0.0, 2), (clo.numbers, _abi.angstrom_to_bohr(clo.xyz), 0.0, 1)]
    s64, r64 = gpu.scf_batch(mols, want_matrices=False)
    smx, rmx = gpu.scf_batch(mols, want_matrices=False, precision="mixed")
    st = gpu.last_call_stats()
    assert all(x == 0 for x in s64) and all(x == 0 for x in smx), (s64, smx)
    assert st["lowp_purification_steps"] > 0  # the closed shell still took TF32 steps
    assert r64[0]["iterations"] == rmx[0]["iterations"]  # the radical ran FP64 throughout
    assert abs(r64[0]["heat_of_formation_kcal"] - rmx[0]["heat_of_formation_kcal"]) < 1e-9
    assert abs(r64[1]["heat_of_formation_kcal"] - rmx[1]["heat_of_formation_kcal"]) < DHF_BAR
