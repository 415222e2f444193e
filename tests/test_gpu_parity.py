"""Parity of the CUDA path (through the C ABI) with the CPU oracle, on a B200.

Tolerances are the bars for the plain FP64 path: heat of formation within 1e-6 kcal/mol,
Mulliken charges within 1e-7 e, density within 1e-8 max-abs, dipole within 1e-6 D; operators
(H_core, Fock) within 1e-10 eV, eigenvalues within 1e-10 relative.  Eigenvectors are compared through
sign- and rotation-invariant quantities (reconstruction, density), as the reference's own tests do.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import atoms_to_arrays

pytestmark = pytest.mark.gpu

HOF_TOL = 1e-6      # kcal/mol
Q_TOL = 1e-7        # e
P_TOL = 1e-8        # max |dP|
MU_TOL = 1e-6       # Debye, each Cartesian component of the dipole
OP_TOL = 1e-10      # eV, operator elements


def _golden_molecules(ref_values):
    out = []
    for c in ref_values["auxiliary_integral_impact"]["cases"]:
        out.append((c["name"], *atoms_to_arrays(c["atoms"])))
    out.append(("formaldehyde", *atoms_to_arrays(ref_values["scf_formaldehyde"]["atoms"])))
    return out


def _compare_scf(g, o, tag):
    assert g["status"] == o["status"] == 0, (tag, g.get("error"), o.get("error"))
    assert g["converged"] and o["converged"], tag
    assert abs(g["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < HOF_TOL, (tag, g["heat_of_formation_kcal"], o["heat_of_formation_kcal"])
    assert np.max(np.abs(g["charges"] - o["charges"])) < Q_TOL, tag
    if "density" in g and "density" in o:
        assert np.max(np.abs(g["density"] - o["density"])) < P_TOL, (tag, np.max(np.abs(g["density"] - o["density"])))
    # point-charge plus s-p hybrid dipole (src/scf.rs:410-427)
    dmu = np.max(np.abs(np.array(g["dipole_debye"]) - np.array(o["dipole_debye"])))
    assert dmu < MU_TOL, (tag, dmu)
    assert abs(g["dipole_magnitude"] - o["dipole_magnitude"]) < MU_TOL, tag
    assert abs(g["iterations"] - o["iterations"]) <= 1, (tag, g["iterations"], o["iterations"])


@pytest.mark.parametrize("n", [1, 2, 3, 5, 17, 64, 100, 113, 161, 200, 257, 330, 400])
def test_symmetric_eigen(gpu, oracle, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n))
    a = a + a.T
    w, v = gpu.eigh(a)
    wo, _ = oracle.eigh(a)
    scale = max(1.0, np.max(np.abs(wo)))
    assert np.all(np.diff(w) >= 0)
    assert np.max(np.abs(w - wo)) < 1e-10 * scale
    assert np.max(np.abs(v.T @ v - np.eye(n))) < 1e-11 * max(1, n)
    assert np.max(np.abs(v @ np.diag(w) @ v.T - a)) < 1e-11 * scale * max(1, n)


def test_symmetric_eigen_known_answers(gpu):
    # src/linalg.rs:479-519
    w, v = gpu.eigh(np.array([[2.0, 1.0], [1.0, 2.0]]))
    assert abs(w[0] - 1) < 1e-10 and abs(w[1] - 3) < 1e-10
    a = np.array([[4.0, 1.0, 2.0], [1.0, 3.0, 0.0], [2.0, 0.0, 1.0]])
    w, v = gpu.eigh(a)
    assert np.max(np.abs(v @ np.diag(w) @ v.T - a)) < 1e-9


def test_symmetric_eigen_refuses_non_finite(gpu):
    # src/linalg.rs:292-304
    a = np.eye(4)
    a[2, 1] = np.nan
    with pytest.raises(gpu.Am1GpuError) as e:
        gpu.eigh(a)
    assert e.value.code == 5


def test_core_hamiltonian(gpu, oracle, ref_values):
    from am1gpu import workloads as W, _abi

    mols = _golden_molecules(ref_values)
    w = W.water_cluster(5, np.random.default_rng(11))
    mols.append(("water5", w.numbers, _abi.angstrom_to_bohr(w.xyz)))
    a = W.alkane(6, np.random.default_rng(12))
    mols.append(("hexane", a.numbers, _abi.angstrom_to_bohr(a.xyz)))
    for name, z, xyz in mols:
        h, e = gpu.build_core(z, xyz)
        ho, eo = oracle.build_core(z, xyz)
        assert np.max(np.abs(h - ho)) < OP_TOL, (name, np.max(np.abs(h - ho)))
        assert abs(e - eo) < 1e-9 * max(1.0, abs(eo)), name


def test_fock_build(gpu, oracle, ref_values):
    rng = np.random.default_rng(3)
    for name, z, xyz in _golden_molecules(ref_values):
        h, _ = oracle.build_core(z, xyz)
        n = h.shape[0]
        p = rng.standard_normal((n, n)) * 0.3
        p = p + p.T
        ps = rng.standard_normal((n, n)) * 0.2
        ps = ps + ps.T
        for pt, pspin, sc in ((p, p, 0.5), (p, ps, 1.0)):
            f = gpu.build_fock(z, xyz, pt, pspin, sc)
            fo = oracle.build_fock(z, xyz, pt, pspin, sc)
            assert np.max(np.abs(f - fo)) < OP_TOL, (name, sc, np.max(np.abs(f - fo)))


def test_scf_golden_molecules(gpu, oracle, ref_values):
    for name, z, xyz in _golden_molecules(ref_values):
        g = gpu.scf(z, xyz)
        o = oracle.scf(z, xyz)
        _compare_scf(g, o, name)


def test_scf_recorded_heats_of_formation(gpu, ref_values):
    # tests/auxiliary_integral_impact.rs:22-80 through the GPU path
    for c in ref_values["auxiliary_integral_impact"]["cases"]:
        z, xyz = atoms_to_arrays(c["atoms"])
        g = gpu.scf(z, xyz)
        assert abs(g["heat_of_formation_kcal"] - c["hof_kcal"]) < 6e-5, c["name"]


@pytest.mark.parametrize("method,tag", [("am1", "AM1_CO2"), ("rm1", "RM1_CO2")])
def test_co2_spectrum(gpu, ref_values, method, tag):
    # tests/mopac_reference.rs: all 12 orbital energies (two degenerate pairs) and the carbon charge
    from am1gpu import _abi

    ref = ref_values["mopac_co2"][tag]
    tol = ref_values["mopac_co2"]["tolerance"]
    b = ref["bond"]
    g = gpu.scf([6, 8, 8], _abi.angstrom_to_bohr([[0, 0, 0], [b, 0, 0], [-b, 0, 0]]), method=method)
    assert g["converged"]
    assert np.max(np.abs(g["mo_energies"] - np.array(ref["orbital_energies"]))) < tol["orbital"]
    assert abs(g["charges"][0] - ref["charge_carbon"]) < tol["charge"]


def test_water_dipole_band(gpu, ref_values):
    # src/scf.rs:1298-1312: water's AM1 dipole is 1.86 +- 0.15 D, and lies in the molecular plane
    w = ref_values["scf_water"]
    z, xyz = atoms_to_arrays(w["atoms"])
    g = gpu.scf(z, xyz)
    mu = np.array(g["dipole_debye"])
    assert abs(g["dipole_magnitude"] - w["dipole_debye"]) < w["dipole_tol"], g["dipole_magnitude"]
    assert abs(np.linalg.norm(mu) - g["dipole_magnitude"]) < 1e-12
    normal = np.cross(xyz[1] - xyz[0], xyz[2] - xyz[0])
    assert abs(np.dot(mu, normal)) < 1e-10 * np.linalg.norm(normal)


def test_uhf_radical_and_forced_references(gpu, oracle, ref_values):
    m = ref_values["scf_methyl_radical"]
    z, xyz = atoms_to_arrays(m["atoms"])
    g = gpu.scf(z, xyz, multiplicity=2)
    o = oracle.scf(z, xyz, multiplicity=2)
    _compare_scf(g, o, "CH3 doublet")
    assert g["unrestricted"]
    assert abs(np.trace(g["spin_density"]) - 1.0) < 1e-6
    assert np.max(np.abs(g["spin_density"] - o["spin_density"])) < P_TOL
    zw, xw = atoms_to_arrays(ref_values["scf_water"]["atoms"])
    rhf = gpu.scf(zw, xw, reference="rhf")
    uhf = gpu.scf(zw, xw, reference="uhf")
    auto = gpu.scf(zw, xw)
    assert abs(uhf["energy_ev"] - rhf["energy_ev"]) < 1e-6
    assert abs(auto["energy_ev"] - rhf["energy_ev"]) < 1e-12
    # restricted open shell is refused (src/scf.rs:1442-1460)
    r = gpu.scf(z, xyz, multiplicity=2, reference="rhf")
    assert r["status"] == 1


def test_accelerators(gpu, oracle, ref_values):
    # src/scf.rs:1344-1369 on the GPU path, each against the oracle's same accelerator
    z, xyz = atoms_to_arrays(ref_values["scf_formaldehyde"]["atoms"])
    res = {}
    for acc in ("adiis_cdiis", "cdiis", "none"):
        g = gpu.scf(z, xyz, accelerator=acc, max_scf=500)
        o = oracle.scf(z, xyz, accelerator=acc, max_scf=500)
        _compare_scf(g, o, acc)
        res[acc] = g
    assert abs(res["adiis_cdiis"]["energy_ev"] - res["none"]["energy_ev"]) < 1e-6
    assert res["adiis_cdiis"]["iterations"] < res["none"]["iterations"]


def test_error_codes(gpu):
    from am1gpu import _abi

    r = gpu.scf([2, 1], [[0, 0, 0], [1.4, 0, 0]])
    assert r["status"] == _abi.ELEMENT_NOT_PARAMETERIZED
    # more than 8192 orbitals: refused before any device work
    big = np.zeros((2049, 3))
    big[:, 0] = 2.9 * np.arange(2049)
    r = gpu.scf(np.full(2049, 6), big, want_matrices=False)
    assert r["status"] == _abi.UNSUPPORTED
    r = gpu.scf([8, 1, 1], [[0, 0, 0], [1.8, 0, 0], [-0.45, 1.75, 0]], multiplicity=2)
    assert r["status"] == _abi.INVALID_INPUT
    r = gpu.scf([8, 1, 1], [[0, 0, 0], [1.8, 0, 0], [-0.45, 1.75, 0]], max_scf=2)
    assert r["status"] == _abi.SCF_NOT_CONVERGED and r["iterations"] == 2 and np.isfinite(r["residual"])


def test_water32_cluster(gpu, oracle):
    from am1gpu import workloads as W, _abi

    m = W.water32_cluster()
    xyz = _abi.angstrom_to_bohr(m.xyz)
    g = gpu.scf(m.numbers, xyz)
    o = oracle.scf(m.numbers, xyz)
    _compare_scf(g, o, "water32_cluster")


def test_batch_matches_oracle_and_solo(gpu, oracle):
    from am1gpu import workloads as W, _abi

    rng = np.random.default_rng(21)
    mols = []
    for n in (1, 2, 3, 7, 12, 19):
        a = W.alkane(n, rng)
        mols.append((a.numbers, _abi.angstrom_to_bohr(a.xyz), 0.0, 1))
    for k in (1, 2, 4, 9, 20, 33):
        w = W.water_cluster(k, rng)
        mols.append((w.numbers, _abi.angstrom_to_bohr(w.xyz), 0.0, 1))
    for n in (1, 3, 6):
        r = W.alkane(n, rng, radical=True)
        mols.append((r.numbers, _abi.angstrom_to_bohr(r.xyz), 0.0, 2))
    status, res = gpu.scf_batch(mols, want_matrices=True)
    assert all(s == 0 for s in status), status
    for i, (z, xyz, q, mult) in enumerate(mols):
        o = oracle.scf(z, xyz, q, mult)
        _compare_scf(res[i], o, f"batch[{i}]")
        solo = gpu.scf(z, xyz, q, mult)
        # same alone and in the mix, bit for bit (no sum of a molecule depends on its batch)
        assert solo["heat_of_formation_kcal"] == res[i]["heat_of_formation_kcal"]
        assert np.array_equal(solo["density"], res[i]["density"])


def _largest_config1_molecules():
    """The largest molecules of the 4096-molecule benchmark's size range: C30H62, C40H82 (242
    orbitals), water clusters of 43, 50 and 64 monomers (258, 300 and 384 orbitals, past the
    256-orbital cut-over of the on-chip kernels) and the C40H81 radical (UHF, 241 orbitals)."""
    from am1gpu import workloads as W, _abi

    rng = np.random.default_rng(31)
    mols = []
    for n in (30, 40):
        a = W.alkane(n, rng)
        mols.append((f"C{n}H{2 * n + 2}", a.numbers, _abi.angstrom_to_bohr(a.xyz), 1))
    for k in (43, 50, 64):
        w = W.water_cluster(k, rng)
        mols.append((f"(H2O){k}", w.numbers, _abi.angstrom_to_bohr(w.xyz), 1))
    r = W.alkane(40, rng, radical=True)
    mols.append(("C40H81 radical", r.numbers, _abi.angstrom_to_bohr(r.xyz), 2))
    return mols


def test_largest_batch_molecules_match_oracle(gpu, oracle):
    mols = _largest_config1_molecules()
    for name, z, xyz, mult in mols:
        g = gpu.scf(z, xyz, 0.0, mult)
        o = oracle.scf(z, xyz, 0.0, mult)
        _compare_scf(g, o, name)
        assert np.max(np.abs(g["mo_energies"] - o["mo_energies"])) < 1e-7, name
        if mult == 2:
            assert g["unrestricted"]
            assert np.max(np.abs(g["spin_density"] - o["spin_density"])) < P_TOL, name
            assert np.max(np.abs(g["beta_energies"] - o["beta_energies"])) < 1e-7, name
    # the same molecules in one batch: every result equal to its solo run, bit for bit
    status, res = gpu.scf_batch([(z, xyz, 0.0, mult) for _, z, xyz, mult in mols], want_matrices=True)
    assert all(s == 0 for s in status), status
    for (name, z, xyz, mult), r in zip(mols, res):
        solo = gpu.scf(z, xyz, 0.0, mult)
        assert solo["heat_of_formation_kcal"] == r["heat_of_formation_kcal"], name
        assert np.array_equal(solo["density"], r["density"]), name
        assert solo["dipole_debye"] == r["dipole_debye"], name


def test_orbital_energies_match_oracle(gpu, oracle, ref_values):
    # mo_energies are the eigenvalues of the last extrapolated Fock matrix (src/scf.rs:654-689)
    for name, z, xyz in _golden_molecules(ref_values):
        g = gpu.scf(z, xyz)
        o = oracle.scf(z, xyz)
        assert np.max(np.abs(g["mo_energies"] - o["mo_energies"])) < 1e-7, name
        assert abs(g["homo_ev"] - o["homo_ev"]) < 1e-7 and abs(g["lumo_ev"] - o["lumo_ev"]) < 1e-7, name


def test_mo_coefficients_reproduce_the_density(gpu, ref_values):
    # columns are MOs (src/scf.rs:200-240); P = 2 C_occ C_occ^T (RHF), P = Ca Ca^T + Cb Cb^T (UHF)
    for name, z, xyz in _golden_molecules(ref_values)[:3]:
        g = gpu.scf(z, xyz)
        c = g["mo_coeff"]
        k = g["n_occ"]
        assert np.max(np.abs(c.T @ c - np.eye(c.shape[0]))) < 1e-10, name
        assert np.max(np.abs(2.0 * c[:, :k] @ c[:, :k].T - g["density"])) < 1e-8, name
    m = ref_values["scf_methyl_radical"]
    z, xyz = atoms_to_arrays(m["atoms"])
    g = gpu.scf(z, xyz, multiplicity=2)
    ca, cb = g["mo_coeff"], g["beta_coeff"]
    pa = ca[:, : g["n_occ"]] @ ca[:, : g["n_occ"]].T
    pb = cb[:, : g["n_occ_beta"]] @ cb[:, : g["n_occ_beta"]].T
    assert np.max(np.abs(pa + pb - g["density"])) < 1e-8
    assert np.max(np.abs(pa - pb - g["spin_density"])) < 1e-8


def test_eigensolver_density_path(tmp_path):
    # AM1GPU_DENSITY=jacobi forms P from eigenvectors every iteration instead of purification;
    # both paths must land on the oracle's answer
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
        rng = np.random.default_rng(5)
        mols = [W.alkane(n, rng) for n in (2, 9)] + [W.water_cluster(k, rng) for k in (3, 22)]
        for m in mols:
            xyz = _abi.angstrom_to_bohr(m.xyz)
            g = native.scf(m.numbers, xyz)
            o = oracle.scf(m.numbers, xyz)
            assert g["status"] == 0, g.get("error")
            assert abs(g["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < 1e-6
            assert np.max(np.abs(g["density"] - o["density"])) < 1e-8
        print("ok")
    """)
    f = tmp_path / "jac.py"
    f.write_text(script)
    env = dict(__import__("os").environ, AM1GPU_DENSITY="jacobi")
    r = subprocess.run([sys.executable, str(f)], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr


def test_symmetric_eigen_batch(gpu):
    # many small blocks in one call, as the divide-and-conquer subsystems are
    # (src/divide_conquer.rs:587-617); each equals its solo am1gpu_symmetric_eigen, bit for bit
    rng = np.random.default_rng(44)
    sizes = [1, 2, 3, 7, 16, 33, 64, 100, 150, 200, 257, 320, 448, 5, 90]
    mats = []
    for n in sizes:
        a = rng.standard_normal((n, n))
        mats.append(a + a.T)
    b = rng.standard_normal((600, 600))  # past the cluster Jacobi: the large-matrix path, after the batch
    sizes.append(600)
    mats.append(b + b.T)
    mats.append(np.array([[1.0, np.nan], [np.nan, 1.0]]))  # refused alone, the rest still solved
    status, out = gpu.eigh_batch(mats)
    from am1gpu import _abi

    assert status[-1] == _abi.LINALG and all(s == 0 for s in status[:-1]), status
    for a, (w, v), n in zip(mats, out, sizes):
        assert np.max(np.abs(w - np.linalg.eigvalsh(a))) < 1e-10 * max(1.0, np.max(np.abs(w)))
        assert np.max(np.abs(v @ np.diag(w) @ v.T - a)) < 1e-9
        w1, v1 = gpu.eigh(a)
        assert np.array_equal(w1, w) and np.array_equal(v1, v)


def test_caller_parameter_set(gpu, oracle, ref_values):
    # run_am1(molecule, params, options) takes any &Am1Parameters (src/scf.rs:294; the elements map
    # is public and Am1Parameters::from_csv builds custom sets, src/params.rs:61-70,139): a custom
    # set must change the GPU result exactly as it changes the oracle's
    import ctypes

    from am1gpu import native, workloads as W, _abi

    std = native.Am1Parameters.for_method("am1")
    mols = _golden_molecules(ref_values)
    a = W.alkane(6, np.random.default_rng(12))
    mols.append(("hexane", a.numbers, _abi.angstrom_to_bohr(a.xyz)))
    # the built-in set passed explicitly: the default call, bit for bit
    for name, z, xyz in mols:
        d = gpu.scf(z, xyz)
        e = gpu.scf(z, xyz, params=std)
        assert d["heat_of_formation_kcal"] == e["heat_of_formation_kcal"], name
        assert np.array_equal(d["density"], e["density"]), name
    # carbon U_ss + 0.1 eV, and a derived field (hydrogen rho0 x 1.01), which is used as given
    mod = std.copy()
    mod.elements[6]["u_ss"] += 0.1
    mod.elements[1]["rho0"] *= 1.01
    for name, z, xyz in mols:
        g = gpu.scf(z, xyz, params=mod)
        o = oracle.scf(z, xyz, params=mod)
        _compare_scf(g, o, name)
        assert abs(g["heat_of_formation_kcal"] - gpu.scf(z, xyz)["heat_of_formation_kcal"]) > 1e-3, name
    # the set's method is the calculation's: the built-in RM1 set equals method="rm1"
    z, xyz = mols[0][1], mols[0][2]
    r1 = gpu.scf(z, xyz, params=native.Am1Parameters.for_method("rm1"))
    r2 = gpu.scf(z, xyz, method="rm1")
    assert r1["heat_of_formation_kcal"] == r2["heat_of_formation_kcal"]
    # batched and gradient calls take the set too; each batch result equals its solo run
    batch = [(z, xyz, 0.0, 1) for _, z, xyz in mols]
    status, res = gpu.scf_batch(batch, want_matrices=True, params=mod)
    assert all(s == 0 for s in status), status
    for (name, z, xyz), r in zip(mols, res):
        solo = gpu.scf(z, xyz, params=mod)
        assert r["heat_of_formation_kcal"] == solo["heat_of_formation_kcal"], name
    gst, gres = gpu.gradient_batch(batch, params=mod)
    gst0, gres0 = gpu.gradient_batch(batch)
    assert all(s == 0 for s in gst)
    for r, r0 in zip(gres, gres0):
        assert np.max(np.abs(r["gradient"].sum(axis=0))) < 1e-8  # translation invariance
        assert np.max(np.abs(r["gradient"] - r0["gradient"])) > 1e-6  # the set is used
    # an element the set lacks, and malformed sets
    no_o = native.Am1Parameters({k: v for k, v in std.elements.items() if k != 8}, "am1")
    w = gpu.scf(*atoms_to_arrays(ref_values["scf_water"]["atoms"]), params=no_o)
    assert w["status"] == _abi.ELEMENT_NOT_PARAMETERIZED and "Z=8" in w["error"]
    mb = _abi.MolBuffers(*atoms_to_arrays(ref_values["scf_water"]["atoms"]))
    rb = _abi.ResultBuffers(3, 6, False)
    o = _abi.default_options()
    twice = (_abi.Element * 2)(_abi.element_from_dict(std.elements[1]), _abi.element_from_dict(std.elements[1]))
    t = _abi.ParamTable(method=0, count=2, elements=twice)
    rc = _abi.lib().am1gpu_scf_params(ctypes.byref(mb.mol), ctypes.byref(t), ctypes.byref(o), ctypes.byref(rb.res))
    assert rc == _abi.INVALID_INPUT and b"twice" in _abi.lib().am1gpu_last_error()
    bad = std.copy()
    bad.elements[8]["g_ss"] = float("nan")
    w = gpu.scf(*atoms_to_arrays(ref_values["scf_water"]["atoms"]), params=bad)
    assert w["status"] == _abi.INVALID_INPUT


def test_captured_solve_equals_host_driven_loop(gpu):
    # The SCF loop as one CUDA graph launch (device-side WHILE loops) must give the host-driven
    # loop's results bit for bit: phase timing forces the host-driven loop, so the same calls are
    # made with timing on and off.  A resident batch reuses its graph across runs.
    from am1gpu import workloads as W, _abi

    rng = np.random.default_rng(77)
    mols = []
    for n in (1, 4, 13, 30):
        a = W.alkane(n, rng)
        mols.append((a.numbers, _abi.angstrom_to_bohr(a.xyz), 0.0, 1))
    for k in (2, 11, 40):
        w = W.water_cluster(k, rng)
        mols.append((w.numbers, _abi.angstrom_to_bohr(w.xyz), 0.0, 1))
    r = W.alkane(7, rng, radical=True)
    mols.append((r.numbers, _abi.angstrom_to_bohr(r.xyz), 0.0, 2))
    try:
        gpu.set_timing(True)
        st_e, res_e = gpu.scf_batch(mols, want_matrices=True)
        assert gpu.last_call_stats()["graph_launches"] == 0
        solo_e = gpu.scf(*mols[3][:2])
        gpu.set_timing(False)
        st_g, res_g = gpu.scf_batch(mols, want_matrices=True)
        stats = gpu.last_call_stats()
        assert stats["graph_launches"] == 1 and stats["scf_cycles"] == max(x["iterations"] for x in res_g)
        solo_g = gpu.scf(*mols[3][:2])
        assert gpu.last_call_stats()["graph_launches"] == 1
    finally:
        gpu.set_timing(False)
    assert st_e == st_g and all(s == 0 for s in st_g)
    for a, b in zip(res_e, res_g):
        assert a["heat_of_formation_kcal"] == b["heat_of_formation_kcal"] and a["iterations"] == b["iterations"]
        assert np.array_equal(a["density"], b["density"]) and np.array_equal(a["charges"], b["charges"])
    assert solo_e["heat_of_formation_kcal"] == solo_g["heat_of_formation_kcal"]
    rb = gpu.ResidentBatch(mols)
    try:
        for _ in range(2):
            rb.run()
            assert rb.stats()["graph_launches"] == 1
            st, res = rb.results()
            assert [x["heat_of_formation_kcal"] for x in res] == [x["heat_of_formation_kcal"] for x in res_g]
    finally:
        rb.close()
