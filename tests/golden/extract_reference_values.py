"""Extract the reference's own recorded values for the SCF hot path into reference_values.json.

am1-rs cannot be compiled here (no cargo), so its golden vectors are taken from its test files,
read as text:

* ``tests/auxiliary_integral_impact.rs`` ``CASES``: five molecules, XYZ inline, heats of
  formation recorded to four decimals (the test asserts < 0.01 kcal/mol);
* ``tests/mopac_reference.rs`` ``AM1_CO2`` / ``RM1_CO2``: MOPAC 22's shipped CO2 outputs
  (heat of formation at C-O = 1.16 A, optimized bond, carbon charge, 12 orbital energies) and
  the per-observable tolerances of that file;
* ``src/params.rs`` test ``loads_core_elements``: carbon's U_ss and g_ss;
* ``src/scf.rs`` tests: the water geometry with its heat-of-formation / dipole bands and the
  methyl-radical geometry.

Usage: python extract_reference_values.py REFERENCE_ROOT   (the am1-rs source tree)
"""

from __future__ import annotations

import json
import pathlib
import re
import sys

HERE = pathlib.Path(__file__).resolve().parent


def parse_xyz_literal(s: str):
    s = s.replace("\\\n", "").replace("\\n", "\n")
    lines = [l.strip() for l in s.split("\n")]
    n = int(lines[0])
    atoms = []
    for l in lines[2 : 2 + n]:
        sym, x, y, z = l.split()[:4]
        atoms.append([sym, float(x), float(y), float(z)])
    return atoms


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: python extract_reference_values.py REFERENCE_ROOT")
    root = pathlib.Path(sys.argv[1])
    out: dict = {"source": "ss0832/am1-rs 0.2.3 test files (see extract_reference_values.py)"}

    aux = (root / "tests/auxiliary_integral_impact.rs").read_text()
    body = aux[aux.index("const CASES"):aux.index("];", aux.index("const CASES"))]
    cases = []
    for m in re.finditer(r'\(\s*"([^"]+)",\s*"((?:[^"\\]|\\.|\\\n)*)",\s*(-?[0-9.]+),\s*\)', body, re.S):
        name, xyz, hof = m.group(1), m.group(2), float(m.group(3))
        cases.append({"name": name, "atoms": parse_xyz_literal(xyz), "hof_kcal": hof})
    assert len(cases) == 5, cases
    out["auxiliary_integral_impact"] = {
        "file": "tests/auxiliary_integral_impact.rs",
        "tolerance_kcal": 0.01,
        "recorded_decimals": 4,
        "cases": cases,
    }

    mop = (root / "tests/mopac_reference.rs").read_text()
    refs = {}
    for tag in ("AM1_CO2", "RM1_CO2"):
        blk = mop[mop.index(f"const {tag}"):]
        blk = blk[: blk.index("};")]

        def f(key):
            return float(re.search(rf"{key}:\s*(-?[0-9.]+)", blk).group(1))

        orb = re.search(r"orbital_energies:\s*&\[(.*?)\]", blk, re.S).group(1)
        refs[tag] = {
            "hof_at_input": f("hof_at_input"),
            "hof_optimized": f("hof_optimized"),
            "bond": f("bond"),
            "ionization": f("ionization"),
            "charge_carbon": f("charge_carbon"),
            "orbital_energies": [float(x) for x in re.findall(r"-?[0-9]+\.[0-9]+", orb)],
        }
    tol = {}
    tol["hof_kcal"] = float(re.search(r"HOF_TOLERANCE_KCAL: f64 = ([0-9.]+)", mop).group(1))
    for key in ("CHARGE", "DIPOLE", "IONIZATION", "ORBITAL", "BOND"):
        tol[key.lower()] = float(re.search(rf"pub const {key}: f64 = ([0-9.e-]+)", mop).group(1))
    out["mopac_co2"] = {"file": "tests/mopac_reference.rs", "input_bond_angstrom": 1.16, "tolerance": tol, **refs}

    params = (root / "src/params.rs").read_text()
    out["carbon_params"] = {
        "file": "src/params.rs",
        "u_ss": float(re.search(r"c\.u_ss - \((-?[0-9.]+)\)", params).group(1)),
        "g_ss": float(re.search(r"c\.g_ss - ([0-9.]+)", params).group(1)),
        "n_gauss": int(re.search(r"c\.gauss\.len\(\), (\d+)", params).group(1)),
    }

    scf = (root / "src/scf.rs").read_text()
    wblk = scf[scf.index("fn water_heat_of_formation"):]
    wxyz = re.search(r'"(3\\nwater\\n[^"]+)"', wblk).group(1)
    out["scf_water"] = {
        "file": "src/scf.rs",
        "atoms": parse_xyz_literal(wxyz),
        "hof_kcal": -59.24,
        "hof_tol": float(re.search(r"\(-59\.24\)\)\.abs\(\) < ([0-9.]+)", wblk).group(1)),
        "dipole_debye": 1.86,
        "dipole_tol": float(re.search(r"\(r\.dipole_magnitude - 1\.86\)\.abs\(\) < ([0-9.]+)", wblk).group(1)),
    }
    mblk = scf[scf.index("fn methyl_radical_uhf"):]
    mxyz = re.search(r'"(4\\nmethyl\\n[^"]+)"', mblk).group(1)
    out["scf_methyl_radical"] = {
        "file": "src/scf.rs",
        "atoms": parse_xyz_literal(mxyz),
        "multiplicity": 2,
        "hof_kcal": 32.0,
        "hof_tol": 6.0,
        "spin_tol": 1.0e-6,
    }
    fblk = scf[scf.index("fn accelerators_agree_on_energy"):]
    fxyz = re.search(r'"(4\\nformaldehyde\\n[^"]+)"', fblk).group(1)
    out["scf_formaldehyde"] = {"file": "src/scf.rs", "atoms": parse_xyz_literal(fxyz), "energy_tol_ev": 1.0e-6}

    (HERE / "reference_values.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", HERE / "reference_values.json")


if __name__ == "__main__":
    main()
