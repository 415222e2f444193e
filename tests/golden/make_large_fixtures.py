"""Oracle results for the largest water clusters, recorded once as a fixture.

The CPU oracle needs minutes to an hour for these molecules (3072 and 6144 orbitals), far more
than a test may take, so this script runs it once, on every host thread (``oracle.set_threads``;
the results do not depend on the thread count), and writes ``large_oracle.json`` beside it.
``tests/test_gpu_large.py`` regenerates each geometry from the same seeded generator, checks
its coordinate digest against the one recorded here, and compares the GPU's FP64 result.

    python tests/golden/make_large_fixtures.py [name ...]

Names: water512_cluster (8x8x8 grid, seed 30, 3072 orbitals: the blocked reduction's size
range) and water1024_cluster (the 1024-water benchmark molecule, seed 3, 6144 orbitals).
"""

from __future__ import annotations

import hashlib
import json
import os
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
for p in (ROOT / "am1-rs_b200", ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

from am1gpu import _abi, workloads as W  # noqa: E402

OUT = HERE / "large_oracle.json"


def molecules() -> dict:
    return {
        "water512_cluster": lambda: W.water_cluster(512, np.random.default_rng(30), grid=(8, 8, 8)),
        "water1024_cluster": W.water1024_cluster,
    }


def xyz_digest(xyz_bohr: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(xyz_bohr, dtype=np.float64).tobytes()).hexdigest()


def main(names: list[str]) -> None:
    import oracle

    oracle.set_threads(os.cpu_count() or 1)
    data = json.loads(OUT.read_text()) if OUT.exists() else {}
    gens = molecules()
    for name in names or list(gens):
        m = gens[name]()
        xyz = _abi.angstrom_to_bohr(m.xyz)
        t0 = time.time()
        o = oracle.scf(m.numbers, xyz, want_matrices=False)
        dt = time.time() - t0
        assert o["status"] == 0 and o["converged"], o.get("error")
        data[name] = {
            "natoms": int(m.natoms),
            "nao": int(o["nao"]),
            "xyz_bohr_sha256": xyz_digest(xyz),
            "heat_of_formation_kcal": o["heat_of_formation_kcal"],
            "energy_ev": o["energy_ev"],
            "electronic_ev": o["electronic_ev"],
            "core_ev": o["core_ev"],
            "iterations": o["iterations"],
            "homo_ev": o["homo_ev"],
            "lumo_ev": o["lumo_ev"],
            "dipole_debye": o["dipole_debye"],
            "charges": [float(x) for x in o["charges"]],
            "oracle_seconds": round(dt, 1),
            "oracle_threads": os.cpu_count(),
        }
        OUT.write_text(json.dumps(data, indent=1) + "\n")
        print(f"{name}: n={o['nao']} dHf={o['heat_of_formation_kcal']:.9f} kcal/mol, {o['iterations']} iterations, "
              f"{dt:.0f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
