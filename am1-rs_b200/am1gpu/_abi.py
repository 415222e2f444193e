"""ctypes mirror of ``include/am1gpu.h`` and the loader for ``libam1gpu.so``.

The structs here are the C ABI's, field for field; see the header for the meaning of each.
The library is built in-tree (``am1-rs_b200/csrc/build/libam1gpu.so``); there is no fallback:
if the library cannot be loaded, :func:`lib` raises.
"""

from __future__ import annotations

import ctypes
import os
import pathlib
import threading

import numpy as np

PKG_ROOT = pathlib.Path(__file__).resolve().parent.parent  # am1-rs_b200/
LIB_PATH = PKG_ROOT / "csrc" / "build" / "libam1gpu.so"

# enum am1gpu_status (mirrors Am1Error, src/error.rs:13-93)
OK = 0
INVALID_INPUT = 1
ELEMENT_NOT_PARAMETERIZED = 2
SCF_NOT_CONVERGED = 3
SCF_DIVERGED = 4
LINALG = 5
UNSUPPORTED = 6
DEVICE_ERROR = 7

STATUS_NAMES = {
    OK: "OK",
    INVALID_INPUT: "INVALID_INPUT",
    ELEMENT_NOT_PARAMETERIZED: "ELEMENT_NOT_PARAMETERIZED",
    SCF_NOT_CONVERGED: "SCF_NOT_CONVERGED",
    SCF_DIVERGED: "SCF_DIVERGED",
    LINALG: "LINALG",
    UNSUPPORTED: "UNSUPPORTED",
    DEVICE_ERROR: "DEVICE_ERROR",
}

REF = {"auto": 0, "rhf": 1, "uhf": 2}
ACCEL = {"none": 0, "cdiis": 1, "adiis_cdiis": 2}
METHOD = {"am1": 0, "rm1": 1}
PRECISION = {"fp64": 0, "mixed": 1}

# MOPAC7 constants the reference uses (src/constants.rs:13-25)
AM1_EV = 27.21
AM1_A0 = 0.529167
ANGSTROM_TO_BOHR = 1.0 / AM1_A0
EV_TO_KCAL = 23.061
EV_TO_HARTREE = 1.0 / AM1_EV
AU_DIPOLE_TO_DEBYE = 2.541746473  # src/constants.rs:32

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class Options(ctypes.Structure):
    _fields_ = [
        ("reference", ctypes.c_int32),
        ("method", ctypes.c_int32),
        ("max_scf", ctypes.c_int32),
        ("use_diis", ctypes.c_int32),
        ("accelerator", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("e_tol", ctypes.c_double),
        ("p_tol", ctypes.c_double),
        ("adiis_switch", ctypes.c_double),
    ]


class Molecule(ctypes.Structure):
    _fields_ = [
        ("natoms", ctypes.c_int32),
        ("multiplicity", ctypes.c_int32),
        ("charge", ctypes.c_double),
        ("z", _ip),
        ("xyz_bohr", _dp),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("electronic_ev", ctypes.c_double),
        ("core_ev", ctypes.c_double),
        ("total_ev", ctypes.c_double),
        ("heat_of_formation_kcal", ctypes.c_double),
        ("dipole_debye", ctypes.c_double * 3),
        ("dipole_magnitude", ctypes.c_double),
        ("homo_ev", ctypes.c_double),
        ("lumo_ev", ctypes.c_double),
        ("homo_beta_ev", ctypes.c_double),
        ("lumo_beta_ev", ctypes.c_double),
        ("residual", ctypes.c_double),
        ("nao", ctypes.c_int32),
        ("n_occ", ctypes.c_int32),
        ("n_occ_beta", ctypes.c_int32),
        ("iterations", ctypes.c_int32),
        ("converged", ctypes.c_int32),
        ("unrestricted", ctypes.c_int32),
        ("charges", _dp),
        ("density", _dp),
        ("spin_density", _dp),
        ("mo_energies", _dp),
        ("mo_coeff", _dp),
        ("beta_energies", _dp),
        ("beta_coeff", _dp),
    ]


# am1gpu_element: Am1Element (src/params.rs:24-55), field for field
ELEMENT_SCALARS = ["u_ss", "u_pp", "zeta_s", "zeta_p", "beta_s", "beta_p", "g_ss", "g_sp", "g_pp", "g_p2", "h_sp", "alpha"]
ELEMENT_DERIVED = ["core_charge", "eheat_ev", "e_isol", "dd", "qq", "rho0", "rho1", "rho2"]


class Element(ctypes.Structure):
    _fields_ = (
        [("z", ctypes.c_int32), ("n", ctypes.c_int32), ("n_orb", ctypes.c_int32), ("n_gauss", ctypes.c_int32)]
        + [(f, ctypes.c_double) for f in ELEMENT_SCALARS]
        + [("gauss_k", ctypes.c_double * 4), ("gauss_l", ctypes.c_double * 4), ("gauss_m", ctypes.c_double * 4)]
        + [(f, ctypes.c_double) for f in ELEMENT_DERIVED]
    )


class ParamTable(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int32), ("count", ctypes.c_int32), ("elements", ctypes.POINTER(Element))]


def element_to_dict(e: Element) -> dict:
    d = {"z": e.z, "n": e.n, "n_orb": e.n_orb}
    for f in ELEMENT_SCALARS + ELEMENT_DERIVED:
        d[f] = getattr(e, f)
    d["gauss"] = [(e.gauss_k[k], e.gauss_l[k], e.gauss_m[k]) for k in range(e.n_gauss)]
    return d


def element_from_dict(d: dict) -> Element:
    g = list(d.get("gauss", []))
    if len(g) > 4:
        raise ValueError(f"element {d['z']}: at most 4 core-core Gaussians")
    e = Element(z=int(d["z"]), n=int(d["n"]), n_orb=int(d["n_orb"]), n_gauss=len(g))
    for f in ELEMENT_SCALARS + ELEMENT_DERIVED:
        setattr(e, f, float(d[f]))
    for k, (kk, ll, mm) in enumerate(g):
        e.gauss_k[k], e.gauss_l[k], e.gauss_m[k] = float(kk), float(ll), float(mm)
    return e


class ParamBuffers:
    """Keeps the element array behind an ``am1gpu_param_table`` alive."""

    def __init__(self, elements: dict, method: int):
        recs = [element_from_dict(elements[z]) for z in sorted(elements)]
        self.arr = (Element * max(1, len(recs)))(*recs)
        self.table = ParamTable(method=int(method), count=len(recs), elements=self.arr)


class CallStats(ctypes.Structure):
    _fields_ = [
        ("device_ms", ctypes.c_double),
        ("phase_ms", ctypes.c_double * 8),
        ("phase_launches", ctypes.c_int64 * 8),
        ("kernel_launches", ctypes.c_int64),
        ("h2d_bytes", ctypes.c_int64),
        ("d2h_bytes", ctypes.c_int64),
        ("scf_cycles", ctypes.c_int32),
        ("eigen_fallbacks", ctypes.c_int32),
        ("purification_steps", ctypes.c_double),
        ("purification_flops", ctypes.c_double),
        ("purification_bytes", ctypes.c_double),
        ("lowp_purification_steps", ctypes.c_double),
        ("lowp_purification_flops", ctypes.c_double),
        ("graph_launches", ctypes.c_int64),
    ]


PHASES = ["basis+core", "scf:fock", "scf:commutator", "scf:accel", "scf:eigen", "eigen:inner", "scf:density", "final"]

_bp = ctypes.c_void_p

# Every function the header declares, with its ctypes signature.
SIGNATURES = {
    "am1gpu_default_options": (None, [ctypes.POINTER(Options)]),
    "am1gpu_basis_size": (ctypes.c_int, [ctypes.c_int32, _ip, ctypes.c_int32, _ip]),
    "am1gpu_scf": (ctypes.c_int, [ctypes.POINTER(Molecule), ctypes.POINTER(Options), ctypes.POINTER(Result)]),
    "am1gpu_scf_batch": (
        ctypes.c_int,
        [ctypes.c_int32, ctypes.POINTER(Molecule), ctypes.POINTER(Options), ctypes.POINTER(Result), _ip],
    ),
    "am1gpu_gradient": (
        ctypes.c_int,
        [ctypes.POINTER(Molecule), ctypes.POINTER(Options), ctypes.POINTER(Result), ctypes.POINTER(ctypes.c_double)],
    ),
    "am1gpu_gradient_batch": (
        ctypes.c_int,
        [ctypes.c_int32, ctypes.POINTER(Molecule), ctypes.POINTER(Options), ctypes.POINTER(Result),
         ctypes.POINTER(ctypes.POINTER(ctypes.c_double)), _ip],
    ),
    "am1gpu_element_params": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(Element)]),
    "am1gpu_derive_element": (ctypes.c_int, [ctypes.c_int32, _dp, _dp, ctypes.POINTER(Element)]),
    "am1gpu_scf_params": (
        ctypes.c_int,
        [ctypes.POINTER(Molecule), ctypes.POINTER(ParamTable), ctypes.POINTER(Options), ctypes.POINTER(Result)],
    ),
    "am1gpu_scf_batch_params": (
        ctypes.c_int,
        [ctypes.c_int32, ctypes.POINTER(Molecule), ctypes.POINTER(ParamTable), ctypes.POINTER(Options),
         ctypes.POINTER(Result), _ip],
    ),
    "am1gpu_gradient_batch_params": (
        ctypes.c_int,
        [ctypes.c_int32, ctypes.POINTER(Molecule), ctypes.POINTER(ParamTable), ctypes.POINTER(Options),
         ctypes.POINTER(Result), ctypes.POINTER(ctypes.POINTER(ctypes.c_double)), _ip],
    ),
    "am1gpu_build_core": (ctypes.c_int, [ctypes.POINTER(Molecule), ctypes.c_int32, _dp, _dp]),
    "am1gpu_build_fock": (
        ctypes.c_int,
        [ctypes.POINTER(Molecule), ctypes.c_int32, _dp, _dp, ctypes.c_double, _dp],
    ),
    "am1gpu_g_matrix_batch": (ctypes.c_int, [ctypes.POINTER(Molecule), ctypes.c_int32, ctypes.c_int32, _dp, _dp]),
    "am1gpu_symmetric_eigen": (ctypes.c_int, [ctypes.c_int32, _dp, _dp, _dp]),
    "am1gpu_symmetric_eigenvalues": (ctypes.c_int, [ctypes.c_int32, _dp, _dp]),
    "am1gpu_lowp_tuning": (ctypes.c_int, [_ip, ctypes.POINTER(ctypes.c_float)]),
    "am1gpu_density_purify": (ctypes.c_int, [ctypes.c_int32, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_int32, _dp, _ip]),
    "am1gpu_set_stream_priority": (ctypes.c_int, [ctypes.c_int32]),
    "am1gpu_symmetric_eigen_batch": (
        ctypes.c_int,
        [ctypes.c_int32, _ip, ctypes.POINTER(_dp), ctypes.POINTER(_dp), ctypes.POINTER(_dp), _ip],
    ),
    "am1gpu_last_error": (ctypes.c_char_p, []),
    "am1gpu_symmetric_eigen_noalloc": (ctypes.c_int, [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p]),
    "am1gpu_batch_create": (
        ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(Molecule), ctypes.POINTER(Options), ctypes.POINTER(_bp)]),
    "am1gpu_batch_run": (ctypes.c_int, [_bp]),
    "am1gpu_batch_results": (ctypes.c_int, [_bp, ctypes.POINTER(Result), _ip]),
    "am1gpu_batch_destroy": (None, [_bp]),
    "am1gpu_set_timing": (None, [ctypes.c_int32]),
    "am1gpu_last_call_stats": (ctypes.c_int, [ctypes.POINTER(CallStats)]),
    "am1gpu_batch_stats": (ctypes.c_int, [_bp, ctypes.POINTER(CallStats)]),
}


def stats_dict(st: CallStats) -> dict:
    return {
        "device_ms": st.device_ms,
        "phase_ms": dict(zip(PHASES, list(st.phase_ms))),
        "phase_launches": dict(zip(PHASES, list(st.phase_launches))),
        "kernel_launches": int(st.kernel_launches),
        "h2d_bytes": int(st.h2d_bytes),
        "d2h_bytes": int(st.d2h_bytes),
        "scf_cycles": int(st.scf_cycles),
        "eigen_fallbacks": int(st.eigen_fallbacks),
        "purification_steps": float(st.purification_steps),
        "purification_flops": float(st.purification_flops),
        "purification_bytes": float(st.purification_bytes),
        "lowp_purification_steps": float(st.lowp_purification_steps),
        "lowp_purification_flops": float(st.lowp_purification_flops),
        "graph_launches": int(st.graph_launches),
    }

_lib = None
_lock = threading.Lock()


def bind(dll: ctypes.CDLL, signatures: dict, prefix_from: str = "am1gpu_", prefix_to: str = "am1gpu_"):
    for name, (res, args) in signatures.items():
        fn = getattr(dll, name.replace(prefix_from, prefix_to, 1))
        fn.restype = res
        fn.argtypes = args
    return dll


def lib() -> ctypes.CDLL:
    """The loaded ``libam1gpu.so``.  Raises if it has not been built: no fallback exists."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                path = os.environ.get("AM1GPU_LIB", str(LIB_PATH))
                if not pathlib.Path(path).exists():
                    raise RuntimeError(
                        f"libam1gpu.so not found at {path}; build it with "
                        "`python -c 'import __graft_entry__ as g; g.build()'` (there is no CPU fallback)"
                    )
                _lib = bind(ctypes.CDLL(path), SIGNATURES)
    return _lib


def default_options(**kw) -> Options:
    o = Options()
    lib().am1gpu_default_options(ctypes.byref(o))
    return apply_options(o, **kw)


def plain_default_options(**kw) -> Options:
    """Am1Options::default() (src/scf.rs:174-197) without touching the library."""
    o = Options(reference=0, method=0, max_scf=200, use_diis=1, accelerator=2, precision=0,
                e_tol=1.0e-8, p_tol=1.0e-7, adiis_switch=0.1)
    return apply_options(o, **kw)


def apply_options(o: Options, reference=None, method=None, max_scf=None, use_diis=None,
                  accelerator=None, precision=None, e_tol=None, p_tol=None, adiis_switch=None) -> Options:
    if reference is not None:
        o.reference = REF[reference] if isinstance(reference, str) else int(reference)
    if method is not None:
        o.method = METHOD[method.lower()] if isinstance(method, str) else int(method)
    if max_scf is not None:
        o.max_scf = int(max_scf)
    if use_diis is not None:
        o.use_diis = int(bool(use_diis))
    if accelerator is not None:
        o.accelerator = ACCEL[accelerator] if isinstance(accelerator, str) else int(accelerator)
    if precision is not None:
        o.precision = PRECISION[precision] if isinstance(precision, str) else int(precision)
    if e_tol is not None:
        o.e_tol = float(e_tol)
    if p_tol is not None:
        o.p_tol = float(p_tol)
    if adiis_switch is not None:
        o.adiis_switch = float(adiis_switch)
    return o


class MolBuffers:
    """Keeps the numpy arrays behind an ``am1gpu_molecule`` alive."""

    def __init__(self, numbers, xyz_bohr, charge=0.0, multiplicity=1):
        self.z = np.ascontiguousarray(np.asarray(numbers, dtype=np.int32).reshape(-1))
        self.xyz = np.ascontiguousarray(np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3))
        if self.xyz.shape[0] != self.z.shape[0]:
            raise ValueError("numbers and positions length mismatch")
        self.mol = Molecule(
            natoms=self.z.shape[0],
            multiplicity=int(multiplicity),
            charge=float(charge),
            z=self.z.ctypes.data_as(_ip),
            xyz_bohr=self.xyz.ctypes.data_as(_dp),
        )


def angstrom_to_bohr(positions) -> np.ndarray:
    """Positions in Angstrom -> Bohr exactly as the reference converts (``* ANGSTROM_TO_BOHR``)."""
    return np.asarray(positions, dtype=np.float64).reshape(-1, 3) * ANGSTROM_TO_BOHR


class ResultBuffers:
    """Caller-owned output arrays for one ``am1gpu_result``."""

    def __init__(self, natoms: int, nao: int, want_matrices: bool = True, unrestricted: bool = True):
        self.charges = np.zeros(natoms)
        self.mo_energies = np.zeros(nao)
        self.density = np.zeros((nao, nao)) if want_matrices else None
        self.mo_coeff = np.zeros((nao, nao)) if want_matrices else None
        self.spin_density = np.zeros((nao, nao)) if (want_matrices and unrestricted) else None
        self.beta_energies = np.zeros(nao) if unrestricted else None
        self.beta_coeff = np.zeros((nao, nao)) if (want_matrices and unrestricted) else None
        self.res = Result()
        for name in ("charges", "density", "spin_density", "mo_energies", "mo_coeff", "beta_energies", "beta_coeff"):
            arr = getattr(self, name)
            setattr(self.res, name, arr.ctypes.data_as(_dp) if arr is not None else None)
