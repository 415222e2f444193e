"""ctypes wrapper of the CPU oracle (``oracle/build/liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` (to check its results)
and by ``bench.py``'s CPU-baseline leg.  The oracle restates am1-rs's SCF on the CPU in FP64
(see ``am1_oracle.cpp``); it shares the C structs of ``include/am1gpu.h`` with the library so
one ctypes layout describes both.
"""

from __future__ import annotations

import ctypes
import pathlib
import subprocess
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
if str(ROOT / "am1-rs_b200") not in sys.path:
    sys.path.insert(0, str(ROOT / "am1-rs_b200"))

from am1gpu import _abi  # noqa: E402

LIB_PATH = HERE / "build" / "liboracle.so"

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)

_SIGS = {
    "oracle_scf": (ctypes.c_int, [ctypes.POINTER(_abi.Molecule), ctypes.POINTER(_abi.Options), ctypes.POINTER(_abi.Result)]),
    "oracle_scf_batch": (
        ctypes.c_int,
        [ctypes.c_int, ctypes.POINTER(_abi.Molecule), ctypes.POINTER(_abi.Options), ctypes.POINTER(_abi.Result),
         ctypes.POINTER(ctypes.c_int), ctypes.c_int],
    ),
    "oracle_build_core": (ctypes.c_int, [ctypes.POINTER(_abi.Molecule), ctypes.c_int, _dp, _dp]),
    "oracle_build_fock": (ctypes.c_int, [ctypes.POINTER(_abi.Molecule), ctypes.c_int, _dp, _dp, ctypes.c_double, _dp]),
    "oracle_symmetric_eigen": (ctypes.c_int, [ctypes.c_int, _dp, _dp, _dp]),
    "oracle_element": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _dp]),
    "oracle_pair_block": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.POINTER(ctypes.c_int), _dp, _dp, _dp]),
    "oracle_bintgs": (None, [ctypes.c_double, _dp]),
    "oracle_local_overlaps": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp]),
    "oracle_last_error": (ctypes.c_char_p, []),
    "oracle_set_threads": (None, [ctypes.c_int]),
    "oracle_scf_params": (ctypes.c_int, [ctypes.POINTER(_abi.Molecule), ctypes.POINTER(_abi.ParamTable),
                                         ctypes.POINTER(_abi.Options), ctypes.POINTER(_abi.Result)]),
}

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        dll = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(dll, name)
            fn.restype = res
            fn.argtypes = args
        _lib = dll
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def result_dict(rb: "_abi.ResultBuffers", rc: int, natoms: int) -> dict:
    r = rb.res
    out = {
        "status": rc,
        "electronic_ev": r.electronic_ev,
        "core_ev": r.core_ev,
        "energy_ev": r.total_ev,
        "heat_of_formation_kcal": r.heat_of_formation_kcal,
        "dipole_debye": list(r.dipole_debye),
        "dipole_magnitude": r.dipole_magnitude,
        "homo_ev": r.homo_ev,
        "lumo_ev": r.lumo_ev,
        "homo_beta_ev": r.homo_beta_ev,
        "lumo_beta_ev": r.lumo_beta_ev,
        "residual": r.residual,
        "nao": r.nao,
        "n_occ": r.n_occ,
        "n_occ_beta": r.n_occ_beta,
        "iterations": r.iterations,
        "converged": bool(r.converged),
        "unrestricted": bool(r.unrestricted),
        "charges": rb.charges.copy(),
        "mo_energies": rb.mo_energies.copy(),
    }
    if rb.density is not None:
        out["density"] = rb.density.copy()
        out["mo_coeff"] = rb.mo_coeff.copy()
    if r.unrestricted and rb.beta_energies is not None:
        out["beta_energies"] = rb.beta_energies.copy()
        if rb.spin_density is not None:
            out["spin_density"] = rb.spin_density.copy()
            out["beta_coeff"] = rb.beta_coeff.copy()
    return out


def nao_of(numbers, method="am1") -> int:
    m = _abi.METHOD[method]
    tot = 0
    out = np.zeros(23)
    for z in np.asarray(numbers).reshape(-1):
        rc = lib().oracle_element(m, int(z), _p(out))
        if rc:
            raise ValueError(f"element {z} not parameterized")
        tot += int(out[1])
    return tot


def set_threads(nthreads: int) -> None:
    """Host threads for the O(n^3) loops inside one molecule's SCF (default 1).  Every element
    is summed in the same order whatever the count, so results are the same bit for bit."""
    lib().oracle_set_threads(int(nthreads))


def scf(numbers, xyz_bohr, charge=0.0, multiplicity=1, want_matrices=True, params=None, **opts) -> dict:
    """params: an optional am1gpu.native.Am1Parameters (elements as given, its method applies)."""
    mb = _abi.MolBuffers(numbers, xyz_bohr, charge, multiplicity)
    o = _abi.plain_default_options(**opts)
    if params is None:
        nao = nao_of(numbers, opts.get("method", "am1"))
    else:
        nao = int(sum(params.elements[int(z)]["n_orb"] for z in np.asarray(numbers).reshape(-1)))
    rb = _abi.ResultBuffers(mb.z.shape[0], nao, want_matrices)
    if params is None:
        rc = lib().oracle_scf(ctypes.byref(mb.mol), ctypes.byref(o), ctypes.byref(rb.res))
    else:
        pb = _abi.ParamBuffers(params.elements, _abi.METHOD[params.method])
        rc = lib().oracle_scf_params(ctypes.byref(mb.mol), ctypes.byref(pb.table), ctypes.byref(o), ctypes.byref(rb.res))
    d = result_dict(rb, rc, mb.z.shape[0])
    if rc:
        d["error"] = lib().oracle_last_error().decode()
    return d


def scf_batch(mols, nthreads=1, want_matrices=False, **opts):
    """mols: list of (numbers, xyz_bohr, charge, multiplicity).  Returns (status, results)."""
    mbs = [_abi.MolBuffers(*m) for m in mols]
    o = _abi.plain_default_options(**opts)
    arr = (_abi.Molecule * len(mbs))(*[m.mol for m in mbs])
    rbs = [_abi.ResultBuffers(m.z.shape[0], nao_of(m.z, opts.get("method", "am1")), want_matrices) for m in mbs]
    res = (_abi.Result * len(rbs))(*[r.res for r in rbs])
    status = (ctypes.c_int * len(mbs))()
    lib().oracle_scf_batch(len(mbs), arr, ctypes.byref(o), res, status, int(nthreads))
    out = []
    for i, rb in enumerate(rbs):
        rb.res = res[i]
        out.append(result_dict(rb, status[i], mbs[i].z.shape[0]))
    return list(status), out


def build_core(numbers, xyz_bohr, method="am1"):
    mb = _abi.MolBuffers(numbers, xyz_bohr)
    nao = nao_of(numbers, method)
    h = np.zeros((nao, nao))
    e = ctypes.c_double()
    rc = lib().oracle_build_core(ctypes.byref(mb.mol), _abi.METHOD[method], _p(h), ctypes.byref(e))
    if rc:
        raise RuntimeError(lib().oracle_last_error().decode())
    return h, e.value


def build_fock(numbers, xyz_bohr, p_tot, p_spin, spin_scale, method="am1"):
    mb = _abi.MolBuffers(numbers, xyz_bohr)
    pt = np.ascontiguousarray(p_tot, dtype=np.float64)
    ps = np.ascontiguousarray(p_spin, dtype=np.float64)
    f = np.zeros_like(pt)
    rc = lib().oracle_build_fock(ctypes.byref(mb.mol), _abi.METHOD[method], _p(pt), _p(ps), float(spin_scale), _p(f))
    if rc:
        raise RuntimeError(lib().oracle_last_error().decode())
    return f


def eigh(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    w = np.zeros(n)
    v = np.zeros((n, n))
    rc = lib().oracle_symmetric_eigen(n, _p(a), _p(w), _p(v))
    if rc:
        raise RuntimeError(lib().oracle_last_error().decode())
    return w, v


ELEMENT_FIELDS = ["n", "norb", "u_ss", "u_pp", "zeta_s", "zeta_p", "beta_s", "beta_p", "g_ss", "g_sp", "g_pp",
                  "g_p2", "h_sp", "alpha", "core_charge", "eheat_ev", "e_isol", "dd", "qq", "rho0", "rho1",
                  "rho2", "ngauss"]


def element(z, method="am1") -> dict:
    out = np.zeros(23)
    rc = lib().oracle_element(_abi.METHOD[method], int(z), _p(out))
    if rc:
        raise ValueError(f"Z={z} not parameterized by {method}")
    return dict(zip(ELEMENT_FIELDS, out.tolist()))


def pair_block(za, zb, dvec, method="am1"):
    dv = np.ascontiguousarray(dvec, dtype=np.float64)
    w = np.zeros(100)
    e1b = np.zeros(16)
    e2a = np.zeros(16)
    s = np.zeros(16)
    wc = ctypes.c_int()
    rc = lib().oracle_pair_block(_abi.METHOD[method], int(za), int(zb), _p(dv), _p(w), ctypes.byref(wc), _p(e1b), _p(e2a), _p(s))
    if rc:
        raise ValueError("pair not supported")
    nrow = 10 if wc.value == 10 else (10 if element(za, method)["norb"] == 4 else 1)
    return {
        "w": w[: nrow * wc.value].reshape(nrow, wc.value),
        "e1b": e1b.reshape(4, 4),
        "e2a": e2a.reshape(4, 4),
        "s": s.reshape(4, 4),
    }


def local_overlaps(za, zb, r, numeric=False, method="am1"):
    """The five local-frame overlaps (s111, s211, s121, s221, s222) of the pair at distance r
    (Bohr); numeric=True forces the prolate-spheroidal quadrature."""
    out = np.zeros(5)
    rc = lib().oracle_local_overlaps(_abi.METHOD[method], int(za), int(zb), float(r), 1 if numeric else 0, _p(out))
    if rc:
        raise RuntimeError(f"oracle_local_overlaps: {rc}")
    return out


def bintgs(x):
    out = np.zeros(13)
    lib().oracle_bintgs(float(x), _p(out))
    return out
