"""Regenerate ``nddo_param_table.h`` from the reference's published parameter tables.

The AM1 and RM1 element parameters are published scientific constants (Dewar, Zoebisch,
Healy & Stewart, JACS 107, 3902 (1985); Rocha, Freire, Simas & Stewart, J. Comput. Chem.
27, 1101 (2006)).  am1-rs ships them as ``src/data/am1_parameters.csv`` and
``src/data/rm1_parameters.csv`` and reads them in ``src/params.rs:139-263``; the per-element
facts (valence principal quantum number, neutral-atom s/p occupations, atomic heats of
formation) are in ``src/data_tables.rs:53-89``.

This script reads those files as text and writes the numbers, untouched (every literal is
emitted exactly as it is spelled in the source so both sides parse the same decimal), into
a C header used by the CUDA library and by the CPU oracle.  Only elements the reference keeps
are written: ``src/params.rs:186-188`` drops a row whose ``U_ss`` and ``beta_s`` are both 0.

Usage:  python gen_param_table.py REFERENCE_ROOT   (the am1-rs source tree, which holds src/data/*.csv)
"""

from __future__ import annotations

import pathlib
import re
import sys

HERE = pathlib.Path(__file__).resolve().parent
OUT = HERE / "nddo_param_table.h"

RAW_COLS = [
    "U_ss", "U_pp", "zeta_s", "zeta_p", "beta_s", "beta_p", "g_ss", "g_sp", "g_pp", "g_p2",
    "h_sp", "alpha",
]
GAUSS_COLS = [f"Gaussian{i}_{k}" for i in range(1, 5) for k in "KLM"]


def _csv_rows(path: pathlib.Path):
    lines = [l for l in path.read_text().splitlines() if not l.lstrip().startswith("#")]
    header = [c.strip().replace(" ", "") for c in lines[0].split(",")]
    rows = []
    for line in lines[1:]:
        if not line.strip():
            continue
        toks = [t.strip() for t in line.split(",")]
        rows.append(dict(zip(header, toks)))
    return rows


def _num(tok: str) -> float:
    try:
        return float(tok)
    except ValueError:
        return 0.0


def _lit(tok: str) -> str:
    """C literal for a CSV token, spelled as in the source (parses to the same double)."""
    v = _num(tok)
    if v == 0.0:
        return "0.0"
    t = tok.strip()
    if re.fullmatch(r"[-+]?\d+", t):
        t += ".0"
    return t


def _rust_array(text: str, name: str) -> list[str]:
    m = re.search(rf"pub const {name}: \[[^\]]+\] = \[(.*?)\];", text, re.S)
    if not m:
        raise SystemExit(f"array {name} not found")
    body = re.sub(r"//[^\n]*", "", m.group(1))
    return [t.strip() for t in body.split(",") if t.strip()]


def _table(name: str, rows) -> list[str]:
    out = [f"static const nddo_raw_element {name}[] = {{"]
    for r in rows:
        if _num(r["U_ss"]) == 0.0 and _num(r["beta_s"]) == 0.0:
            continue
        z = int(_num(r["N"]))
        vals = ", ".join(_lit(r[c]) for c in RAW_COLS)
        g = ", ".join(_lit(r[c]) for c in GAUSS_COLS)
        out.append(f"    {{{z}, {{{vals}}}, {{{g}}}}},  /* {r['sym']} */")
    out.append("};")
    return out


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: python gen_param_table.py REFERENCE_ROOT")
    root = pathlib.Path(sys.argv[1])
    am1 = _csv_rows(root / "src/data/am1_parameters.csv")
    rm1 = _csv_rows(root / "src/data/rm1_parameters.csv")
    tables = (root / "src/data_tables.rs").read_text()
    qn = _rust_array(tables, "QN")
    ns = _rust_array(tables, "N_S")
    npp = _rust_array(tables, "N_P")
    eheat = _rust_array(tables, "EHEAT_KCAL")
    assert len(qn) == len(ns) == len(npp) == len(eheat) == 87

    lines = [
        "/* Generated by gen_param_table.py -- do not edit by hand.",
        " *",
        " * Raw AM1 / RM1 element parameters (eV, Bohr^-1, Angstrom^-1 for the core-core",
        " * Gaussians) and per-element facts, exactly as the reference am1-rs 0.2.3 tabulates",
        " * them (src/data/am1_parameters.csv, src/data/rm1_parameters.csv,",
        " * src/data_tables.rs).  Published scientific constants; the derived multipole",
        " * quantities (dd, qq, rho0..rho2, e_isol) are computed by the code that includes this.",
        " */",
        "#ifndef NDDO_PARAM_TABLE_H",
        "#define NDDO_PARAM_TABLE_H",
        "",
        "/* raw[] order: U_ss U_pp zeta_s zeta_p beta_s beta_p g_ss g_sp g_pp g_p2 h_sp alpha;",
        " * gauss[] order: K1 L1 M1 K2 L2 M2 K3 L3 M3 K4 L4 M4. */",
        "typedef struct { int z; double raw[12]; double gauss[12]; } nddo_raw_element;",
        "",
        "#define NDDO_MAX_Z 86",
        "",
        "/* valence principal quantum number by Z */",
        "static const int NDDO_QN[87] = {" + ", ".join(qn) + "};",
        "/* neutral-atom valence s and p occupations by Z */",
        "static const double NDDO_NS[87] = {" + ", ".join(ns) + "};",
        "static const double NDDO_NP[87] = {" + ", ".join(npp) + "};",
        "/* experimental atomic heats of formation, kcal/mol, by Z */",
        "static const double NDDO_EHEAT_KCAL[87] = {" + ", ".join(eheat) + "};",
        "",
    ]
    lines += _table("NDDO_AM1_RAW", am1)
    lines.append("")
    lines += _table("NDDO_RM1_RAW", rm1)
    lines += ["", "#endif", ""]
    OUT.write_text("\n".join(lines))
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
