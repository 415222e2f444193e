"""Python surface of the B200 library, mirroring am1-rs's ``am1_rs.native`` (python/am1_rs/native.py).

``single_point`` and ``orbitals`` take the reference's arguments (atomic numbers, positions in
Angstrom, charge, multiplicity, reference, method) and return the same dictionary keys
(src/python.rs:147-199, 1911-1975); errors raise ``ValueError`` as the reference's binding does
(src/python.rs:27-29).  Every call goes through ``libam1gpu.so``'s C ABI; there is no CPU path.
``scf`` / ``scf_batch`` expose the full result (density, orbitals) for one molecule or a batch,
positions in Bohr.
"""

from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import _abi

_dp = ctypes.POINTER(ctypes.c_double)


class Am1GpuError(ValueError):
    """An am1-rs error (``Am1Error``) reported by the library; ``code`` is the ``am1gpu_status``."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def ensure_loaded() -> ctypes.CDLL:
    """Load the library (raises if it is missing)."""
    return _abi.lib()


def _check(rc: int, allow_not_converged: bool = False):
    if rc == _abi.OK or (allow_not_converged and rc == _abi.SCF_NOT_CONVERGED):
        return
    raise Am1GpuError(rc, _abi.lib().am1gpu_last_error().decode() or _abi.STATUS_NAMES.get(rc, str(rc)))


def _nao(numbers, method) -> int:
    z = np.ascontiguousarray(np.asarray(numbers, dtype=np.int32).reshape(-1))
    out = ctypes.c_int32()
    rc = _abi.lib().am1gpu_basis_size(z.shape[0], z.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                      _abi.METHOD[method.lower()], ctypes.byref(out))
    _check(rc)
    return out.value


class Am1Parameters:
    """A parameter set, as the reference's ``Am1Parameters`` (src/params.rs:61-70): ``elements``
    maps Z to a dict of ``Am1Element``'s fields (src/params.rs:24-55; ``gauss`` is the list of
    (K, L, M) triples) and ``method`` names the parameterization ("am1" or "rm1"), which is the
    method of every calculation run with the set.  Entries may be edited or replaced; the
    calculation uses them as given (no field is re-derived)."""

    def __init__(self, elements: dict, method: str = "am1"):
        self.elements = {int(z): dict(e) for z, e in elements.items()}
        self.method = method.lower()
        if self.method not in _abi.METHOD:
            raise ValueError(f"unknown method {method!r}")

    @classmethod
    def for_method(cls, method: str = "am1") -> "Am1Parameters":
        """The built-in set (Am1Parameters::for_method, src/params.rs:88-90)."""
        m = _abi.METHOD[method.lower()]
        els = {}
        e = _abi.Element()
        for z in range(1, 87):
            if _abi.lib().am1gpu_element_params(m, z, ctypes.byref(e)) == _abi.OK:
                els[z] = _abi.element_to_dict(e)
        return cls(els, method)

    standard = for_method

    @classmethod
    def from_csv(cls, text: str, method: str = "am1") -> "Am1Parameters":
        """Am1Parameters::from_csv (src/params.rs:139-263): '#' lines skipped, the first other line
        is the header (names with spaces removed), a cell that does not parse reads 0, rows with
        U_ss = beta_s = 0 are skipped; each row is derived by ``am1gpu_derive_element``."""
        lines = [ln for ln in text.splitlines() if not ln.lstrip().startswith("#")]
        if not lines:
            raise ValueError("empty parameter CSV")
        cols = [c.strip().replace(" ", "") for c in lines[0].split(",")]

        def col(name):
            if name not in cols:
                raise ValueError(f"missing parameter column {name}")
            return cols.index(name)

        raw_cols = [col(n) for n in ("U_ss", "U_pp", "zeta_s", "zeta_p", "beta_s", "beta_p", "g_ss", "g_sp", "g_pp",
                                     "g_p2", "h_sp", "alpha")]
        gcols = [col(f"Gaussian{k}_{x}") for k in range(1, 5) for x in ("K", "L", "M")]
        cn = col("N")

        def num(cell):
            try:
                return float(cell.strip())
            except ValueError:
                return 0.0

        els = {}
        for line in lines[1:]:
            line = line.strip()
            if not line:
                continue
            f = [num(c) for c in line.split(",")]
            z = int(f[cn])
            if f[raw_cols[0]] == 0.0 and f[raw_cols[4]] == 0.0:
                continue
            raw = (ctypes.c_double * 12)(*[f[c] for c in raw_cols])
            gauss = (ctypes.c_double * 12)(*[f[c] for c in gcols])
            e = _abi.Element()
            _check(_abi.lib().am1gpu_derive_element(z, raw, gauss, ctypes.byref(e)))
            els[z] = _abi.element_to_dict(e)
        if not els:
            raise ValueError("no AM1 elements parsed from parameter table")
        return cls(els, method)

    def element(self, z: int) -> dict:
        if int(z) not in self.elements:
            raise Am1GpuError(_abi.ELEMENT_NOT_PARAMETERIZED, f"{self.method.upper()} has no parameters for element Z={z}")
        return self.elements[int(z)]

    def copy(self) -> "Am1Parameters":
        return Am1Parameters({z: dict(e, gauss=list(e["gauss"])) for z, e in self.elements.items()}, self.method)

    def buffers(self) -> _abi.ParamBuffers:
        return _abi.ParamBuffers(self.elements, _abi.METHOD[self.method])

    def nao(self, numbers) -> int:
        return int(sum(self.element(int(z))["n_orb"] for z in np.asarray(numbers).reshape(-1)))


def _result_dict(rb: _abi.ResultBuffers, rc: int, want_matrices: bool) -> dict:
    r = rb.res
    d = {
        "status": rc,
        "energy_ev": r.total_ev,
        "energy_hartree": r.total_ev * _abi.EV_TO_HARTREE,
        "electronic_ev": r.electronic_ev,
        "core_ev": r.core_ev,
        "heat_of_formation_kcal": r.heat_of_formation_kcal,
        "charges": rb.charges.copy(),
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
        "mo_energies": rb.mo_energies.copy(),
    }
    if want_matrices:
        d["density"] = rb.density.copy()
        d["mo_coeff"] = rb.mo_coeff.copy()
        if r.unrestricted:
            d["spin_density"] = rb.spin_density.copy()
            d["beta_energies"] = rb.beta_energies.copy()
            d["beta_coeff"] = rb.beta_coeff.copy()
    elif r.unrestricted and rb.beta_energies is not None:
        d["beta_energies"] = rb.beta_energies.copy()
    return d


def _nao_for(numbers, method, params):
    """AOs of a molecule under a method's built-in set or a caller's set (0 when an element is
    missing: the library reports that error itself)."""
    z = np.asarray(numbers).reshape(-1)
    if not z.size:
        return 0
    try:
        return params.nao(z) if params is not None else _nao(z, method)
    except Am1GpuError:
        return 0


def scf(numbers, xyz_bohr, charge=0.0, multiplicity=1, want_matrices=True, raise_on_error=False, params=None,
        **opts) -> dict:
    """One molecule through ``am1gpu_scf`` (the plain FP64 drop-in), or ``am1gpu_scf_params`` with
    ``params`` (an :class:`Am1Parameters`, whose method then applies).  Positions in Bohr."""
    mb = _abi.MolBuffers(numbers, xyz_bohr, charge, multiplicity)
    o = _abi.default_options(**opts)
    method = opts.get("method", "am1")
    nao = _nao_for(mb.z, method, params)
    if nao == 0 and mb.z.size:
        want_matrices = False
    rb = _abi.ResultBuffers(mb.z.shape[0], nao, want_matrices)
    if params is None:
        rc = _abi.lib().am1gpu_scf(ctypes.byref(mb.mol), ctypes.byref(o), ctypes.byref(rb.res))
    else:
        pb = params.buffers()
        rc = _abi.lib().am1gpu_scf_params(ctypes.byref(mb.mol), ctypes.byref(pb.table), ctypes.byref(o), ctypes.byref(rb.res))
    if raise_on_error:
        _check(rc, allow_not_converged=False)
    d = _result_dict(rb, rc, want_matrices)
    if rc:
        d["error"] = _abi.lib().am1gpu_last_error().decode()
    return d


class Batch:
    """Host buffers of one batched call; reusable across calls with the same molecules."""

    def __init__(self, mols, method="am1", want_matrices=False, params=None):
        self.mbs = [_abi.MolBuffers(*m) for m in mols]
        self.arr = (_abi.Molecule * len(self.mbs))(*[m.mol for m in self.mbs])
        if params is None:
            naos = [_nao(m.z, method) if m.z.size else 0 for m in self.mbs]
        else:
            naos = [_nao_for(m.z, method, params) for m in self.mbs]
        self.rbs = [_abi.ResultBuffers(m.z.shape[0], nao, want_matrices and (nao > 0 or not m.z.size),
                                       unrestricted=(m.mol.multiplicity > 1)) for m, nao in zip(self.mbs, naos)]
        self.res = (_abi.Result * len(self.rbs))(*[r.res for r in self.rbs])
        self.status = (ctypes.c_int32 * len(self.mbs))()
        self.want_matrices = want_matrices
        self.params = params
        self.pbuf = params.buffers() if params is not None else None

    def run(self, **opts) -> int:
        o = _abi.default_options(**opts)
        if self.pbuf is not None:
            return _abi.lib().am1gpu_scf_batch_params(len(self.mbs), self.arr, ctypes.byref(self.pbuf.table), ctypes.byref(o),
                                                      self.res, self.status)
        return _abi.lib().am1gpu_scf_batch(len(self.mbs), self.arr, ctypes.byref(o), self.res, self.status)

    def results(self) -> list[dict]:
        out = []
        for i, rb in enumerate(self.rbs):
            rb.res = self.res[i]
            out.append(_result_dict(rb, int(self.status[i]), self.want_matrices and rb.density is not None))
        return out


def scf_gradient(numbers, xyz_bohr, charge=0.0, multiplicity=1, **opts) -> dict:
    """SCF plus the closed-form nuclear gradient through ``am1gpu_gradient`` (positions in Bohr).
    Returns the SCF result dict with ``gradient`` (natoms x 3, eV/Bohr) and ``forces``."""
    mb = _abi.MolBuffers(numbers, xyz_bohr, charge, multiplicity)
    o = _abi.default_options(**opts)
    nao = _nao(mb.z, opts.get("method", "am1")) if mb.z.size else 0
    rb = _abi.ResultBuffers(mb.z.shape[0], nao, False)
    g = np.zeros((mb.z.shape[0], 3))
    rc = _abi.lib().am1gpu_gradient(ctypes.byref(mb.mol), ctypes.byref(o), ctypes.byref(rb.res),
                                    g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    d = _result_dict(rb, rc, False)
    if rc:
        d["error"] = _abi.lib().am1gpu_last_error().decode()
    d["gradient"] = g
    d["forces"] = -g
    return d


def gradient_batch(mols, params=None, **opts):
    """Batched ``am1gpu_gradient_batch`` (``am1gpu_gradient_batch_params`` with ``params``):
    (status list, result dicts with ``gradient``)."""
    b = Batch(mols, opts.get("method", "am1"), False, params=params)
    gs = [np.zeros((m.z.shape[0], 3)) for m in b.mbs]
    ptrs = (ctypes.POINTER(ctypes.c_double) * len(gs))(*[g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for g in gs])
    o = _abi.default_options(**opts)
    if b.pbuf is not None:
        _abi.lib().am1gpu_gradient_batch_params(len(b.mbs), b.arr, ctypes.byref(b.pbuf.table), ctypes.byref(o), b.res, ptrs,
                                                b.status)
    else:
        _abi.lib().am1gpu_gradient_batch(len(b.mbs), b.arr, ctypes.byref(o), b.res, ptrs, b.status)
    res = b.results()
    for r, g in zip(res, gs):
        r["gradient"] = g
        r["forces"] = -g
    return list(b.status), res


def last_call_stats() -> dict:
    st = _abi.CallStats()
    _check(_abi.lib().am1gpu_last_call_stats(ctypes.byref(st)))
    return _abi.stats_dict(st)


def set_stream_priority(priority: int) -> None:
    """CUDA priority of this host thread's stream (0 default, negative higher)."""
    _check(_abi.lib().am1gpu_set_stream_priority(int(priority)))


def set_timing(enable: bool) -> None:
    _abi.lib().am1gpu_set_timing(1 if enable else 0)


class ResidentBatch:
    """``am1gpu_batch_*``: molecules uploaded once, the SCF re-run on device-resident inputs."""

    def __init__(self, mols, method="am1", want_matrices=False, **opts):
        self.host = Batch(mols, method, want_matrices)
        self.opts = _abi.default_options(method=method, **opts)
        self.handle = ctypes.c_void_p()
        _check(_abi.lib().am1gpu_batch_create(len(self.host.mbs), self.host.arr, ctypes.byref(self.opts),
                                              ctypes.byref(self.handle)))

    def run(self) -> None:
        _check(_abi.lib().am1gpu_batch_run(self.handle))

    def stats(self) -> dict:
        st = _abi.CallStats()
        _check(_abi.lib().am1gpu_batch_stats(self.handle, ctypes.byref(st)))
        return _abi.stats_dict(st)

    def results(self) -> tuple[list[int], list[dict]]:
        _abi.lib().am1gpu_batch_results(self.handle, self.host.res, self.host.status)
        return list(self.host.status), self.host.results()

    def close(self) -> None:
        if self.handle:
            _abi.lib().am1gpu_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scf_batch(mols, want_matrices=False, params=None, **opts):
    """Batched solve.  ``mols``: sequence of (numbers, xyz_bohr, charge, multiplicity); ``params``
    an optional :class:`Am1Parameters`.  Returns (status list, result dicts)."""
    b = Batch(mols, opts.get("method", "am1"), want_matrices, params=params)
    b.run(**opts)
    return list(b.status), b.results()


def build_core(numbers, xyz_bohr, method="am1"):
    mb = _abi.MolBuffers(numbers, xyz_bohr)
    nao = _nao(mb.z, method)
    h = np.zeros((nao, nao))
    e = ctypes.c_double()
    _check(_abi.lib().am1gpu_build_core(ctypes.byref(mb.mol), _abi.METHOD[method], h.ctypes.data_as(_dp), ctypes.byref(e)))
    return h, e.value


def build_fock(numbers, xyz_bohr, p_tot, p_spin, spin_scale, method="am1"):
    mb = _abi.MolBuffers(numbers, xyz_bohr)
    pt = np.ascontiguousarray(p_tot, dtype=np.float64)
    ps = np.ascontiguousarray(p_spin, dtype=np.float64)
    f = np.zeros_like(pt)
    _check(_abi.lib().am1gpu_build_fock(ctypes.byref(mb.mol), _abi.METHOD[method], pt.ctypes.data_as(_dp),
                                        ps.ctypes.data_as(_dp), float(spin_scale), f.ctypes.data_as(_dp)))
    return f


def g_matrix_batch(numbers, xyz_bohr, densities, method="am1"):
    """G(P) = J(P) - K(P/2) for a stack of densities (nrhs x nao x nao), ``am1gpu_g_matrix_batch``."""
    mb = _abi.MolBuffers(numbers, xyz_bohr)
    d = np.ascontiguousarray(densities, dtype=np.float64)
    g = np.zeros_like(d)
    _check(_abi.lib().am1gpu_g_matrix_batch(ctypes.byref(mb.mol), _abi.METHOD[method], int(d.shape[0]), d.ctypes.data_as(_dp),
                                            g.ctypes.data_as(_dp)))
    return g


PURIFY_PRECISION = {"fp64": 0, "fp32_tcgen05": 1, "tf32": 2, "fp64_digits": 3, "tf32_tcgen05": 4}


def density_purify(f, n_occ, weight=2.0, precision="fp64"):
    """P = weight * projector onto the n_occ lowest eigenvectors of symmetric f (n <= 448), by
    purification at one of the batched path's product precisions (``am1gpu_density_purify``).
    Returns (P, number of products)."""
    a = np.ascontiguousarray(f, dtype=np.float64)
    p = np.zeros_like(a)
    steps = ctypes.c_int32()
    _check(_abi.lib().am1gpu_density_purify(a.shape[0], a.ctypes.data_as(_dp), float(n_occ), float(weight),
                                            PURIFY_PRECISION[precision], p.ctypes.data_as(_dp), ctypes.byref(steps)))
    return p, steps.value


LOWP_KERNELS = ("mma.sync tf32", "tcgen05 3xtf32", "tcgen05 tf32")


def lowp_tuning() -> dict:
    """The autotuner's choice of reduced-precision purification kernel per size class on this device
    (``am1gpu_lowp_tuning``): {class: {"kernel": one of LOWP_KERNELS or None, "ms": {kernel: ms}}}."""
    choice = (ctypes.c_int32 * 4)()
    ms = (ctypes.c_float * 12)()
    _check(_abi.lib().am1gpu_lowp_tuning(choice, ms))
    names = ["n<=128", "n<=256", "n<=384", "n>384"]
    return {names[c]: {"kernel": LOWP_KERNELS[choice[c]] if choice[c] >= 0 else None,
                       "ms": {k: ms[3 * c + i] for i, k in enumerate(LOWP_KERNELS)}} for c in range(4)}


def eigvalsh(a):
    """Ascending eigenvalues of a symmetric matrix (up to 8192 rows), ``am1gpu_symmetric_eigenvalues``."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    w = np.zeros(a.shape[0])
    _check(_abi.lib().am1gpu_symmetric_eigenvalues(a.shape[0], a.ctypes.data_as(_dp), w.ctypes.data_as(_dp)))
    return w


def eigh_batch(mats):
    """Eigendecompositions of a list of symmetric matrices in one ``am1gpu_symmetric_eigen_batch``
    call: (status list, [(eigenvalues, eigenvector columns)])."""
    ms = [np.ascontiguousarray(m, dtype=np.float64) for m in mats]
    ns = (ctypes.c_int32 * len(ms))(*[m.shape[0] for m in ms])
    ws = [np.zeros(m.shape[0]) for m in ms]
    vs = [np.zeros_like(m) for m in ms]
    arr = lambda xs: (_dp * len(xs))(*[x.ctypes.data_as(_dp) for x in xs])
    st = (ctypes.c_int32 * len(ms))()
    _abi.lib().am1gpu_symmetric_eigen_batch(len(ms), ns, arr(ms), arr(ws), arr(vs), st)
    return list(st), list(zip(ws, vs))


def eigh(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    w = np.zeros(n)
    v = np.zeros((n, n))
    _check(_abi.lib().am1gpu_symmetric_eigen(n, a.ctypes.data_as(_dp), w.ctypes.data_as(_dp), v.ctypes.data_as(_dp)))
    return w, v


# ---------------------------------------------------------------------------------------
# The reference's Python entry points (positions in Angstrom)
# ---------------------------------------------------------------------------------------
def _prep(numbers, positions):
    z = np.asarray(numbers, dtype=np.int32).reshape(-1)
    xyz = _abi.angstrom_to_bohr(np.asarray(positions, dtype=float).reshape(len(z), 3))
    return z, xyz


def _reference_name(reference: str) -> str:
    r = reference.strip().lower()
    if r in ("auto", ""):
        return "auto"
    if r in ("rhf", "r", "restricted"):
        return "rhf"
    if r in ("uhf", "u", "unrestricted"):
        return "uhf"
    raise ValueError(f"invalid reference '{reference}': expected 'auto', 'rhf', or 'uhf'")


def _method_name(method: str) -> str:
    m = method.strip().lower()
    if m not in _abi.METHOD:
        raise ValueError(f"unknown method `{m}`; expected one of: am1, rm1")
    return m


def constants() -> dict:
    """The unit constants of the path; the dictionary of am1_rs.native.constants (src/python.rs:2514-2539):
    MOPAC7's Hartree and Bohr (src/constants.rs:13-32), the kcal/mol factor, the dipole unit, and the two
    factors of the infrared chain (src/ir.rs:73-76)."""
    return {
        "hartree_to_ev": _abi.AM1_EV,
        "ev_to_hartree": _abi.EV_TO_HARTREE,
        "angstrom_to_bohr": _abi.ANGSTROM_TO_BOHR,
        "bohr_to_angstrom": _abi.AM1_A0,
        "ev_to_kcal": _abi.EV_TO_KCAL,
        "kcal_to_ev": 1.0 / _abi.EV_TO_KCAL,
        "au_dipole_to_debye": _abi.AU_DIPOLE_TO_DEBYE,
        "ir_intensity_km_per_mol": 42.2561,
        "e_to_debye_per_angstrom": _abi.AU_DIPOLE_TO_DEBYE * _abi.ANGSTROM_TO_BOHR,
    }


def single_point(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1,
                 reference: str = "auto", method: str = "am1", electric_field=None) -> dict:
    """Single-point energy and properties; the dictionary of am1_rs.native.single_point."""
    if electric_field is not None:
        raise ValueError("electric_field is not supported on the GPU path")
    z, xyz = _prep(numbers, positions)
    m = _method_name(method)
    r = scf(z, xyz, charge, multiplicity, want_matrices=False, reference=_reference_name(reference), method=m)
    _check(r["status"])
    return {
        "method": m,
        "energy_hartree": r["energy_hartree"],
        "energy_ev": r["energy_ev"],
        "heat_of_formation_kcal": r["heat_of_formation_kcal"],
        "electronic_ev": r["electronic_ev"],
        "core_ev": r["core_ev"],
        "charges": [float(x) for x in r["charges"]],
        "dipole_debye": r["dipole_debye"],
        "dipole_magnitude": r["dipole_magnitude"],
        "homo_ev": None if np.isnan(r["homo_ev"]) else r["homo_ev"],
        "lumo_ev": None if np.isnan(r["lumo_ev"]) else r["lumo_ev"],
        "homo_beta_ev": None if np.isnan(r["homo_beta_ev"]) else r["homo_beta_ev"],
        "lumo_beta_ev": None if np.isnan(r["lumo_beta_ev"]) else r["lumo_beta_ev"],
        "field_nuclear_ev": 0.0,
        "converged": r["converged"],
        "iterations": r["iterations"],
        "unrestricted": r["unrestricted"],
    }


def gradient(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1,
             reference: str = "auto", method: str = "am1", electric_field=None) -> dict:
    """Energy and closed-form nuclear gradient; the dictionary of am1_rs.native.gradient
    (src/python.rs:201-277): positions in Angstrom, the gradient in Hartree/Bohr and eV/Angstrom
    (forces = -gradient), with the SCF properties of the same run."""
    if electric_field is not None:
        raise ValueError("electric_field is not supported on the GPU path")
    z, xyz = _prep(numbers, positions)
    m = _method_name(method)
    r = scf_gradient(z, xyz, charge, multiplicity, reference=_reference_name(reference), method=m)
    _check(r["status"])
    g = r["gradient"]
    return {
        "energy_hartree": r["energy_hartree"],
        "energy_ev": r["energy_ev"],
        "heat_of_formation_kcal": r["heat_of_formation_kcal"],
        "electronic_ev": r["electronic_ev"],
        "core_ev": r["core_ev"],
        "homo_ev": None if np.isnan(r["homo_ev"]) else r["homo_ev"],
        "lumo_ev": None if np.isnan(r["lumo_ev"]) else r["lumo_ev"],
        "gradient_hartree_per_bohr": (g * _abi.EV_TO_HARTREE).tolist(),
        "gradient_ev_per_angstrom": (g * _abi.ANGSTROM_TO_BOHR).tolist(),
        "charges": [float(x) for x in r["charges"]],
        "dipole_debye": r["dipole_debye"],
        "dipole_magnitude": r["dipole_magnitude"],
        "max_gradient_hartree_per_bohr": float(np.max(np.abs(g))) * _abi.EV_TO_HARTREE if g.size else 0.0,
        "converged": r["converged"],
        "iterations": r["iterations"],
        "unrestricted": r["unrestricted"],
        "method": m,
    }


def orbitals(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1,
             reference: str = "auto", method: str = "am1", electric_field=None) -> dict:
    """Orbital energies and coefficients; the dictionary of am1_rs.native.orbitals."""
    if electric_field is not None:
        raise ValueError("electric_field is not supported on the GPU path")
    z, xyz = _prep(numbers, positions)
    m = _method_name(method)
    r = scf(z, xyz, charge, multiplicity, want_matrices=True, reference=_reference_name(reference), method=m)
    _check(r["status"])
    labels = []
    for ia, zz in enumerate(z):
        labels += [(ia, "s")] if zz == 1 else [(ia, "s"), (ia, "px"), (ia, "py"), (ia, "pz")]
    d = {
        "energies_hartree": [e * _abi.EV_TO_HARTREE for e in r["mo_energies"]],
        "energies_ev": list(r["mo_energies"]),
        "coefficients": r["mo_coeff"].tolist(),
        "n_occupied": r["n_occ"],
        "homo_ev": None if np.isnan(r["homo_ev"]) else r["homo_ev"],
        "lumo_ev": None if np.isnan(r["lumo_ev"]) else r["lumo_ev"],
        "unrestricted": r["unrestricted"],
        "ao_labels": labels,
    }
    if r["unrestricted"]:
        d.update({
            "beta_energies_hartree": [e * _abi.EV_TO_HARTREE for e in r["beta_energies"]],
            "beta_energies_ev": list(r["beta_energies"]),
            "beta_coefficients": r["beta_coeff"].tolist(),
            "beta_n_occupied": r["n_occ_beta"],
            "homo_beta_ev": None if np.isnan(r["homo_beta_ev"]) else r["homo_beta_ev"],
            "lumo_beta_ev": None if np.isnan(r["lumo_beta_ev"]) else r["lumo_beta_ev"],
        })
    return d
