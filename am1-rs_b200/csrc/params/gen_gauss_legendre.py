"""Write ``gauss_legendre.h``: the Gauss-Legendre rules on [-1, 1] of orders 48 (xi) and 40 (eta)
that the numerical Slater overlap integrates with (the orders of src/overlap_numeric.rs:124-126).

Nodes and weights come from numpy.polynomial.legendre.leggauss (the Golub-Welsch eigenvalue
method, refined by Newton steps), written with 17 significant digits so the header reproduces
the doubles exactly.  Usage: python gen_gauss_legendre.py
"""

from __future__ import annotations

import pathlib

import numpy as np

ORDERS = {"XI": 48, "ETA": 40}


def main() -> None:
    out = ["// Generated by gen_gauss_legendre.py: Gauss-Legendre rules on [-1, 1] for the numerical",
           "// Slater overlap (orders of src/overlap_numeric.rs:124-126).  Device constants, one copy per",
           "// translation unit.", "#pragma once", ""]
    for name, n in ORDERS.items():
        x, w = np.polynomial.legendre.leggauss(n)
        out.append(f"constexpr int kGl{name.capitalize()}N = {n};")
        out.append(f"static __constant__ double kGl{name.capitalize()}X[{n}] = {{" + ", ".join(f"{v:.17g}" for v in x) + "};")
        out.append(f"static __constant__ double kGl{name.capitalize()}W[{n}] = {{" + ", ".join(f"{v:.17g}" for v in w) + "};")
        out.append("")
    pathlib.Path(__file__).with_name("gauss_legendre.h").write_text("\n".join(out))


if __name__ == "__main__":
    main()
