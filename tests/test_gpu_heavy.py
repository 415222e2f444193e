"""Elements with valence shells n >= 4 (Zn, Ge, As, Se, Br, Sb, Te, I, Hg) on a B200: their Slater
overlaps come from the prolate-spheroidal quadrature (src/overlap_numeric.rs), in the SCF and,
differentiated through the quadrature, in the gradient."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

A2B = 1.0 / 0.529167
# Z, bond length to H (Angstrom, near the covalent-radius sum)
HEAVY = [(30, 1.54), (32, 1.53), (33, 1.52), (34, 1.46), (35, 1.41), (51, 1.70), (52, 1.66), (53, 1.61), (80, 1.74)]


def _hydride(z, bond):
    d = np.array([0.6, -0.3, 0.74])
    d = d / np.linalg.norm(d) * bond
    return np.array([z, 1], dtype=np.int32), np.array([[0.0, 0.0, 0.0], d]) * A2B


def _mult(z, oracle, method="am1"):
    zv = oracle.element(z, method)["core_charge"] + 1.0
    return 1 if int(round(zv)) % 2 == 0 else 2


@pytest.mark.parametrize("z,bond", HEAVY, ids=[str(h[0]) for h in HEAVY])
def test_heavy_hydride_matches_oracle(gpu, oracle, z, bond):
    zz, x = _hydride(z, bond)
    mult = _mult(z, oracle)
    g = gpu.scf(zz, x, 0.0, mult, want_matrices=True)
    o = oracle.scf(zz, x, 0.0, mult, want_matrices=True)
    assert g["status"] == 0 and o["status"] == 0 and g["converged"]
    assert abs(g["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < 1e-6
    assert np.max(np.abs(g["charges"] - o["charges"])) < 1e-7
    # Ge, As, Se, Sb and Te hydrides half-fill a degenerate pi pair: the SCF occupies one
    # direction perpendicular to the bond, and which one is arbitrary (the two solutions differ by a
    # rotation about the bond axis, with the same energy and charges).  Quantities invariant under
    # that rotation are compared: the spectrum of the density and the orbital energies.
    np.testing.assert_allclose(np.linalg.eigvalsh(g["density"]), np.linalg.eigvalsh(o["density"]), atol=1e-8)
    if z not in (32, 33, 34, 51, 52):
        assert np.max(np.abs(g["density"] - o["density"])) < 1e-8
    assert np.max(np.abs(g["mo_energies"] - o["mo_energies"])) < 1e-7


@pytest.mark.parametrize("method", ["am1", "rm1"])
def test_halomethanes_batch_matches_oracle(gpu, oracle, method):
    # CH3Br and CH3I (RM1 covers Br and I) with a methane beside them in one batch
    mols = []
    for hal, b in ((35, 1.94), (53, 2.14)):
        z = np.array([6, hal, 1, 1, 1], dtype=np.int32)
        x = np.array([[0.0, 0.0, 0.0], [b, 0.02, 0.0], [-0.36, 1.03, 0.0], [-0.36, -0.51, 0.89], [-0.37, -0.51, -0.90]]) * A2B
        mols.append((z, x, 0.0, 1))
    mols.append((np.array([6, 1, 1, 1, 1], dtype=np.int32),
                 np.array([[0, 0, 0], [0.63, 0.63, 0.63], [-0.63, -0.63, 0.63], [-0.63, 0.63, -0.63], [0.63, -0.63, -0.63]]) * A2B, 0.0, 1))
    status, res = gpu.scf_batch(mols, method=method)
    assert all(s == 0 for s in status), status
    for (z, x, q, m), g in zip(mols, res):
        o = oracle.scf(z, x, q, m, method=method, want_matrices=False)
        assert abs(g["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < 1e-6
        assert np.max(np.abs(g["charges"] - o["charges"])) < 1e-7


@pytest.mark.parametrize("z,bond", [(35, 1.41), (53, 1.61), (80, 1.74)], ids=["HBr", "HI", "HgH"])
def test_heavy_gradient_through_the_quadrature(gpu, oracle, z, bond):
    from test_gpu_gradient import fd_gradient, fixed_density_energy

    zz, x = _hydride(z, bond)
    mult = _mult(z, oracle)
    g = gpu.scf_gradient(zz, x, 0.0, mult)
    s = gpu.scf(zz, x, 0.0, mult, want_matrices=True)
    ref = fd_gradient(lambda X: fixed_density_energy(oracle, zz, X, s["density"], s.get("spin_density"), "am1"), x)
    assert np.max(np.abs(g["gradient"] - ref)) < 2e-6, (g["gradient"], ref)
