"""The C ABI library loads and exports every entry point include/am1gpu.h declares (CPU only:
no compute call is made here)."""

from __future__ import annotations

import ctypes
import re

from conftest import ROOT


def _declared():
    text = (ROOT / "include" / "am1gpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(am1gpu_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = _declared()
    for required in ("am1gpu_scf", "am1gpu_scf_batch", "am1gpu_build_core", "am1gpu_build_fock",
                     "am1gpu_symmetric_eigen", "am1gpu_basis_size", "am1gpu_default_options",
                     "am1gpu_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from am1gpu import _abi

    assert _abi.LIB_PATH.exists(), "build libam1gpu.so first (__graft_entry__.build())"
    dll = ctypes.CDLL(str(_abi.LIB_PATH))
    for name in _declared():
        assert hasattr(dll, name), name
    # the ctypes signature table covers the header
    assert set(_declared()) <= set(_abi.SIGNATURES)


def test_default_options_match_the_reference():
    # Am1Options::default(), src/scf.rs:174-197; am1gpu_default_options needs no device
    from am1gpu import _abi

    o = _abi.default_options()
    assert (o.max_scf, o.use_diis, o.accelerator, o.reference, o.method) == (200, 1, 2, 0, 0)
    assert (o.e_tol, o.p_tol, o.adiis_switch) == (1e-8, 1e-7, 0.1)


def test_basis_size_without_a_device():
    from am1gpu import native

    assert native._nao([8, 1, 1], "am1") == 6
    assert native._nao([6, 6, 1, 1, 1, 1, 1, 1], "am1") == 14
    try:
        native._nao([2], "am1")
    except native.Am1GpuError as e:
        assert e.code == 2
    else:
        raise AssertionError("helium must be refused")


def test_constants_are_the_reference_dictionary():
    # am1_rs.native.constants (src/python.rs:2514-2539) over src/constants.rs:13-32 and src/ir.rs:73-76
    from am1gpu import native

    c = native.constants()
    assert set(c) == {"hartree_to_ev", "ev_to_hartree", "angstrom_to_bohr", "bohr_to_angstrom", "ev_to_kcal",
                      "kcal_to_ev", "au_dipole_to_debye", "ir_intensity_km_per_mol", "e_to_debye_per_angstrom"}
    assert (c["hartree_to_ev"], c["bohr_to_angstrom"], c["ev_to_kcal"]) == (27.21, 0.529167, 23.061)
    assert c["ev_to_hartree"] == 1.0 / 27.21 and c["angstrom_to_bohr"] == 1.0 / 0.529167 and c["kcal_to_ev"] == 1.0 / 23.061
    assert c["au_dipole_to_debye"] == 2.541746473 and c["ir_intensity_km_per_mol"] == 42.2561
    assert c["e_to_debye_per_angstrom"] == 2.541746473 * (1.0 / 0.529167)


def test_parameter_sets_without_a_device():
    # Am1Parameters (src/params.rs:61-263) through am1gpu_element_params / am1gpu_derive_element,
    # which need no device: the built-in records equal the oracle's derivation, and a CSV written
    # from them parses back (Am1Parameters::from_csv) to the same records bit for bit
    import oracle as O

    from am1gpu import native

    for method in ("am1", "rm1"):
        ps = native.Am1Parameters.for_method(method)
        assert 1 in ps.elements and 6 in ps.elements and 8 in ps.elements
        for z, e in ps.elements.items():
            o = O.element(z, method)
            for f in ("u_ss", "u_pp", "zeta_s", "zeta_p", "beta_s", "beta_p", "g_ss", "g_sp", "g_pp", "g_p2", "h_sp",
                      "alpha", "core_charge", "eheat_ev", "e_isol", "dd", "qq", "rho0", "rho1", "rho2"):
                assert e[f] == o[f], (method, z, f)
            assert (e["n"], e["n_orb"], len(e["gauss"])) == (o["n"], o["norb"], o["ngauss"])
        names = ["N", "U_ss", "U_pp", "zeta_s", "zeta_p", "beta_s", "beta_p", "g_ss", "g_sp", "g_pp", "g_p2", "h_sp",
                 "alpha"] + [f"Gaussian{k}_{x}" for k in range(1, 5) for x in ("K", "L", "M")]
        rows = ["# provenance line", ", ".join(n.replace("_s", " _s") if n == "zeta_s" else n for n in names)]
        for z, e in sorted(ps.elements.items()):
            g = list(e["gauss"]) + [(0.0, 0.0, 0.0)] * (4 - len(e["gauss"]))
            vals = [z] + [e[f.lower() if f.startswith("U_") else f] for f in names[1:13]] + [x for t in g for x in t]
            rows.append(",".join(repr(float(v)) for v in vals))
        rows.append("99,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0")  # not parameterized: skipped
        back = native.Am1Parameters.from_csv("\n".join(rows), method)
        assert back.elements == ps.elements
    try:
        native.Am1Parameters.for_method("am1").element(2)
    except native.Am1GpuError as err:
        assert err.code == 2
    else:
        raise AssertionError("helium must be refused")
