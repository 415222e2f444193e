"""FP64 against mixed precision on the batched path: speed and the error of every molecule.

The mixed path (``precision="mixed"``) purifies the density with TF32 tensor-core products in a
molecule's early SCF iterations and switches to FP64 once its RMS density change is below 1e-3;
integrals, Fock build, commutator, extrapolation and energies are FP64 throughout, and the SCF
converges on FP64 iterations.  This module measures what that buys and costs:

    python -m am1gpu.precision_report                      # 4096 molecules + 512 UHF radicals, AM1 and RM1
    python -m am1gpu.precision_report --workload large     # 1024 waters, 6144 orbitals

One JSON line per (workload, method): device time of both paths, SCF iterations, and per
molecule |dHf| (kcal/mol), max |dq| (Mulliken, e) and max |dP| (density, on a sample) of the
mixed result against the FP64 one.
"""

from __future__ import annotations

import argparse
import json

import numpy as np


def _solve(mols, **opts):
    from . import native

    native.set_timing(True)
    native.scf_batch(mols[: min(64, len(mols))], **opts)  # grow the workspace outside the measurement
    status, res = native.scf_batch(mols, **opts)
    return status, res, native.last_call_stats()


def compare(mols, method: str = "am1", density_sample: int = 128) -> dict:
    """Solve ``mols`` ((numbers, xyz_bohr, charge, multiplicity) tuples) on both paths."""
    s64, r64, st64 = _solve(mols, method=method)
    smx, rmx, stmx = _solve(mols, method=method, precision="mixed")
    dhf = np.array([abs(a["heat_of_formation_kcal"] - b["heat_of_formation_kcal"]) for a, b in zip(r64, rmx)])
    dq = np.array([float(np.max(np.abs(a["charges"] - b["charges"]))) for a, b in zip(r64, rmx)])
    idx = list(range(0, len(mols), max(1, len(mols) // density_sample)))
    sub = [mols[i] for i in idx]
    _, a, _ = _solve(sub, method=method, want_matrices=True)
    _, b, _ = _solve(sub, method=method, want_matrices=True, precision="mixed")
    dp = max(float(np.max(np.abs(x["density"] - y["density"]))) for x, y in zip(a, b))
    it64 = np.array([r["iterations"] for r in r64])
    itmx = np.array([r["iterations"] for r in rmx])
    out = {
        "method": method,
        "molecules": len(mols),
        "uhf": int(sum(1 for m in mols if m[3] > 1)),
        "failed": {"fp64": int(sum(1 for s in s64 if s != 0)), "mixed": int(sum(1 for s in smx if s != 0))},
        "device_ms": {"fp64": st64["device_ms"], "mixed": stmx["device_ms"]},
        "solves_per_s": {"fp64": len(mols) / st64["device_ms"] * 1e3, "mixed": len(mols) / stmx["device_ms"] * 1e3},
        "scf_iterations_mean": {"fp64": float(it64.mean()), "mixed": float(itmx.mean())},
        "purification_products": {"fp64": st64["purification_steps"], "mixed_fp64": stmx["purification_steps"],
                                  "mixed_tf32": stmx["lowp_purification_steps"]},
        "dHf_kcal": {"max": float(dhf.max()), "p99": float(np.percentile(dhf, 99)), "median": float(np.median(dhf))},
        "dq_max": float(dq.max()),
        "dP_max": dp,
        "dP_sample": len(sub),
        "bar_dHf_kcal": 1e-4,
    }
    if len(mols) == 1:  # one molecule: its time per SCF iteration
        out["ms_per_scf_iteration"] = {"fp64": st64["device_ms"] / int(it64[0]), "mixed": stmx["device_ms"] / int(itmx[0])}
    return out


def _main():
    from . import _abi, native, workloads as W

    ap = argparse.ArgumentParser(description="FP64 against mixed precision on the batched path")
    ap.add_argument("--workload", choices=["batch", "large"], default="batch")
    ap.add_argument("--methods", default="am1,rm1")
    args = ap.parse_args()
    native.ensure_loaded()
    if args.workload == "batch":
        ms = W.alkane_water_radical_batch()
        name = "4096 molecules (2048 alkanes n~U{1..40}, 2048 water clusters k~U{1..64}, seed 1) + 512 UHF alkyl radicals"
    else:
        ms = [W.water1024_cluster()]
        name = "1024 H2O, 3072 atoms, 6144 orbitals, seed 3"
    mols = [(m.numbers, _abi.angstrom_to_bohr(m.xyz), m.charge, m.multiplicity) for m in ms]
    for method in args.methods.split(","):
        out = {"workload": name, **compare(mols, method, density_sample=128 if len(mols) > 1 else 1)}
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    _main()
