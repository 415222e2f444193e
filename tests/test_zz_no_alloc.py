"""The allocation-free eigensolver entry point, am1gpu_symmetric_eigen_noalloc.

Some callers cannot let a library allocate device memory -- they run beside a framework that
owns the whole device memory pool, or in a real-time loop, or only hold device buffers handed to
them -- so this entry point takes device pointers for its input and outputs and keeps its
scratch in a fixed array inside the library.  Here its results are checked, through the C ABI,
against the existing (allocating) am1gpu_symmetric_eigen on the same matrices, on two calls in a
row (the second call must not see anything left over from the first), and the device's free
memory is checked to stay the same across calls.  The file is named to be
collected last, so a run that stops at its first failure has run every other test before it.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EIG_TOL = 1e-10  # relative, as the other eigensolver parity tests


def _noalloc(lib, torch, a: np.ndarray):
    n = a.shape[0]
    da = torch.from_numpy(np.ascontiguousarray(a)).to("cuda")
    dw = torch.empty(n, dtype=torch.float64, device="cuda")
    dv = torch.empty((n, n), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.am1gpu_symmetric_eigen_noalloc(n, ctypes.c_void_p(da.data_ptr()), ctypes.c_void_p(dw.data_ptr()),
                                            ctypes.c_void_p(dv.data_ptr()), ctypes.c_void_p(stream))
    return rc, dw.cpu().numpy(), dv.cpu().numpy()


def _check_against_allocating(native, w, v, a):
    wr, vr = native.eigh(a)
    scale = max(1.0, float(np.max(np.abs(wr))))
    assert np.max(np.abs(w - wr)) < EIG_TOL * scale
    # distinct eigenvalues: each eigenvector agrees up to sign
    overlap = np.abs(np.sum(v * vr, axis=0))
    assert np.max(np.abs(overlap - 1.0)) < 1e-8
    assert np.max(np.abs(v @ np.diag(w) @ v.T - a)) < 1e-11 * scale * a.shape[0]


def test_noalloc_eigensolver_matches_the_allocating_one(gpu):
    import torch

    from am1gpu import _abi

    lib = _abi.lib()
    rng = np.random.default_rng(2024)
    mats = []
    for n in (77, 128):  # two calls in a row, different sizes
        m = rng.standard_normal((n, n))
        mats.append(m + m.T)
    for a in mats:
        rc, w, v = _noalloc(lib, torch, a)
        assert rc == 0, lib.am1gpu_last_error().decode()
        _check_against_allocating(gpu, w, v, a)
    # the same matrix again after a larger one: the shared scratch keeps nothing that matters
    rc, w, v = _noalloc(lib, torch, mats[0])
    assert rc == 0
    _check_against_allocating(gpu, w, v, mats[0])


def test_noalloc_eigensolver_refuses_what_it_cannot_hold(gpu):
    import torch

    from am1gpu import _abi

    lib = _abi.lib()
    a = np.eye(129)
    rc, _, _ = _noalloc(lib, torch, a)
    assert rc == _abi.INVALID_INPUT and "128" in lib.am1gpu_last_error().decode()
    b = np.eye(8)
    b[3, 1] = np.nan
    rc, _, _ = _noalloc(lib, torch, b)
    assert rc == _abi.LINALG


def test_noalloc_eigensolver_allocates_no_device_memory(gpu):
    # the property the entry point exists for: after one warm call (which loads the kernels and
    # fetches the scratch address), further calls -- here from a host thread the library has not
    # seen, so no per-thread workspace exists for it -- leave the device's free memory unchanged
    import threading

    import torch

    from am1gpu import _abi

    lib = _abi.lib()
    n = 100
    rng = np.random.default_rng(99)
    m = rng.standard_normal((n, n))
    a = m + m.T
    da = torch.from_numpy(a).to("cuda")
    dw = torch.empty(n, dtype=torch.float64, device="cuda")
    dv = torch.empty((n, n), dtype=torch.float64, device="cuda")
    args = (n, ctypes.c_void_p(da.data_ptr()), ctypes.c_void_p(dw.data_ptr()), ctypes.c_void_p(dv.data_ptr()), None)
    assert lib.am1gpu_symmetric_eigen_noalloc(*args) == 0
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    codes = []

    def worker():
        for _ in range(3):
            codes.append(lib.am1gpu_symmetric_eigen_noalloc(*args))

    t = threading.Thread(target=worker)
    t.start()
    t.join()
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert codes == [0, 0, 0], lib.am1gpu_last_error().decode()
    assert free_after == free_before, (free_before, free_after)
    _check_against_allocating(gpu, dw.cpu().numpy(), dv.cpu().numpy(), a)
