"""Closed-form nuclear gradient on a B200 (am1gpu_gradient), checked against the oracle.

Two checks, as the reference checks its own closed_form_gradient (tests/rm1.rs:195-219 compares
it with a central finite difference of the SCF energy, step 1e-4 Bohr, to 5e-5 eV/Bohr):
  * against central differences of the oracle's energy at the GPU's converged density held
    fixed, E(R; P) = 1/2 sum P (H(R) + F(R; P)) + E_cc(R) (the Hellmann-Feynman gradient is
    exactly its derivative), to 2e-6 eV/Bohr;
  * against central differences of the oracle's full SCF energy, to the reference's 5e-5.
Plus translation and rotation invariance and batch/solo agreement.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

A2B = 1.0 / 0.529167


def _mol(atoms):
    z = np.array([a[0] for a in atoms], dtype=np.int32)
    x = np.array([a[1:] for a in atoms], dtype=np.float64) * A2B
    return z, x


# (name, Z, xyz Bohr, multiplicity, method): slightly distorted geometries, so no component
# of the gradient vanishes by symmetry
MOLS = [
    ("water", *_mol([(8, 0.0, 0.0, 0.11), (1, 0.77, 0.0, -0.47), (1, -0.74, 0.05, -0.49)]), 1, "am1"),
    ("formaldehyde", *_mol([(6, 0.0, 0.0, 0.0), (8, 0.0, 0.02, 1.23), (1, 0.93, 0.0, -0.56), (1, -0.95, 0.04, -0.55)]), 1, "am1"),
    ("methyl radical", *_mol([(6, 0.0, 0.0, 0.02), (1, 1.08, 0.0, 0.0), (1, -0.55, 0.93, 0.0), (1, -0.53, -0.95, 0.05)]), 2, "am1"),
    ("methanol rm1", *_mol([(6, -0.05, 0.0, 0.0), (8, 1.41, 0.02, 0.0), (1, 1.72, 0.9, 0.1), (1, -0.44, 1.02, 0.05),
                            (1, -0.42, -0.52, 0.89), (1, -0.40, -0.5, -0.9)]), 1, "rm1"),
]


def fixed_density_energy(O, z, xyz, P, S, method):
    """The oracle's total energy at positions xyz with the density held at P (spin density S
    for UHF, None for RHF): 1/2 sum P H + 1/2 sum_sigma P^sigma F^sigma + E_cc."""
    h, ecc = O.build_core(z, xyz, method)
    if S is None:
        f = O.build_fock(z, xyz, P, P, 0.5, method)
        return 0.5 * float(np.sum(P * (h + f))) + ecc
    pa, pb = 0.5 * (P + S), 0.5 * (P - S)
    fa = O.build_fock(z, xyz, P, pa, 1.0, method)
    fb = O.build_fock(z, xyz, P, pb, 1.0, method)
    return 0.5 * float(np.sum(P * h) + np.sum(pa * fa) + np.sum(pb * fb)) + ecc


def fd_gradient(energy, xyz, step=1e-4):
    g = np.zeros_like(xyz)
    for a in range(xyz.shape[0]):
        for k in range(3):
            xp, xm = xyz.copy(), xyz.copy()
            xp[a, k] += step
            xm[a, k] -= step
            g[a, k] = (energy(xp) - energy(xm)) / (2.0 * step)
    return g


@pytest.mark.parametrize("case", MOLS, ids=[m[0] for m in MOLS])
def test_gradient_matches_fixed_density_differences(gpu, oracle, case):
    name, z, xyz, mult, method = case
    g = gpu.scf_gradient(z, xyz, 0.0, mult, method=method)
    assert g["status"] == 0 and g["converged"]
    s = gpu.scf(z, xyz, 0.0, mult, method=method, want_matrices=True)  # the same converged density
    assert s["energy_ev"] == g["energy_ev"]
    P, S = s["density"], s.get("spin_density")
    ref = fd_gradient(lambda X: fixed_density_energy(oracle, z, X, P, S, method), xyz)
    assert np.max(np.abs(g["gradient"] - ref)) < 2e-6, (name, g["gradient"], ref)
    np.testing.assert_allclose(g["forces"], -g["gradient"])
    # translation invariance holds at any fixed density; rotation invariance only at the
    # self-consistent one (the density's p blocks do not turn with the frame), so the net torque
    # is as small as the SCF convergence makes it
    assert np.max(np.abs(g["gradient"].sum(axis=0))) < 1e-8
    torque = np.cross(xyz, g["gradient"]).sum(axis=0)
    assert np.max(np.abs(torque)) < 1e-5


@pytest.mark.parametrize("case", [MOLS[0], MOLS[3]], ids=["water", "methanol rm1"])
def test_gradient_matches_scf_differences(gpu, oracle, case):
    # the reference's own bar for its closed-form gradient (tests/rm1.rs:195-219)
    name, z, xyz, mult, method = case
    g = gpu.scf_gradient(z, xyz, 0.0, mult, method=method)
    ref = fd_gradient(lambda X: oracle.scf(z, X, 0.0, mult, method=method, want_matrices=False)["energy_ev"], xyz)
    assert np.max(np.abs(g["gradient"] - ref)) < 5e-5, (name, g["gradient"], ref)


def test_gradient_batch_matches_solo(gpu):
    from am1gpu import workloads as W, _abi

    rng = np.random.default_rng(12)
    mols = [(m[1], m[2], 0.0, m[3]) for m in MOLS if m[4] == "am1"]
    for n in (3, 8):
        a = W.alkane(n, rng)
        mols.append((a.numbers, _abi.angstrom_to_bohr(a.xyz), 0.0, 1))
    w = W.water_cluster(6, rng)
    mols.append((w.numbers, _abi.angstrom_to_bohr(w.xyz), 0.0, 1))
    status, res = gpu.gradient_batch(mols)
    assert all(s == 0 for s in status), status
    for m, r in zip(mols, res):
        solo = gpu.scf_gradient(*m)
        assert np.max(np.abs(solo["gradient"] - r["gradient"])) < 1e-9
        assert np.max(np.abs(r["gradient"].sum(axis=0))) < 1e-8


def test_front_end_gradient_dictionary(gpu):
    # am1_rs.native.gradient's dictionary (src/python.rs:201-277): Angstrom in, Hartree/Bohr and
    # eV/Angstrom out, with the SCF properties
    import numpy as np

    from am1gpu import _abi

    name, z, xyz, mult, method = MOLS[1]
    d = gpu.gradient(z, xyz * 0.529167, method=method)
    g = gpu.scf_gradient(z, xyz, method=method)["gradient"]
    assert set(d) >= {"energy_hartree", "energy_ev", "heat_of_formation_kcal", "gradient_hartree_per_bohr",
                      "gradient_ev_per_angstrom", "charges", "dipole_debye", "converged", "method",
                      "max_gradient_hartree_per_bohr"}
    np.testing.assert_allclose(np.array(d["gradient_hartree_per_bohr"]), g * _abi.EV_TO_HARTREE, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(np.array(d["gradient_ev_per_angstrom"]), g * _abi.ANGSTROM_TO_BOHR, rtol=1e-12, atol=1e-12)
    assert d["method"] == "AM1" or d["method"].lower() == "am1"
