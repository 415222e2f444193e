"""Shared fixtures.  Tests marked ``gpu`` need a B200 and call the library through its C ABI;
everything else runs on the CPU (oracle against the reference's recorded values, host logic,
the ABI's symbol table)."""

from __future__ import annotations

import json
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
for p in (ROOT / "am1-rs_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libam1gpu.so")
    config.addinivalue_line("markers", "slow: long-running")


SYMBOL_Z = {"H": 1, "C": 6, "N": 7, "O": 8, "F": 9, "Cl": 17, "S": 16, "P": 15}


def atoms_to_arrays(atoms):
    """[[sym, x, y, z], ...] (Angstrom) -> (Z int32, xyz Bohr) exactly as the reference converts."""
    from am1gpu import _abi

    z = np.array([SYMBOL_Z[a[0]] for a in atoms], dtype=np.int32)
    xyz = np.array([a[1:4] for a in atoms], dtype=np.float64)
    return z, _abi.angstrom_to_bohr(xyz)


@pytest.fixture(scope="session")
def ref_values():
    return json.loads((GOLDEN / "reference_values.json").read_text())


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def gpu():
    """The library, on a machine with a CUDA device; the test fails (not skips) if the
    library cannot be loaded there, so a GPU run never passes on a missing extension."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from am1gpu import native

    native.ensure_loaded()
    return native
