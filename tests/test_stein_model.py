"""A NumPy emulation of the large-matrix eigenvector path (csrc/k_stein.cu, driven by
symmetric_eigen_large in csrc/driver.cu), buffer for buffer: the reduction's reflector rows in W,
inverse iteration with the kernels' flat [component][vector] layout and their per-thread branches
(vectorised over the threads), the cluster Gram-Schmidt through the vector-major scratch, and the
compact-WY back-transformation through the same flat pointers, leading dimensions and zero-filled
tile loads as the k_dgemm launches.  Every flat index is checked against its buffer's length.  The
result must be an orthonormal eigenbasis (CPU only, no device)."""

from __future__ import annotations

import numpy as np
import pytest

EPS = 2.220446049250313e-16
ORTOL = 1e-4  # kSteinOrtol
NB = 64  # kWyNb
M64 = (1 << 64) - 1


def reduce_store(a):
    """Householder reduction (the unblocked kernels' conventions); row s of W holds v_s (cols > s)."""
    W = a.astype(np.float64).copy()
    n = W.shape[0]
    d = np.zeros(n)
    e = np.zeros(n)
    for s in range(n - 2):
        x = W[s, s + 1:].copy()
        alpha = np.sqrt(x @ x)
        sg = 1.0 if x[0] >= 0 else -1.0
        beta = 0.0 if alpha == 0 else 1.0 / (alpha * (alpha + abs(x[0])))
        v = x.copy()
        if alpha != 0:
            v[0] = x[0] + sg * alpha
        d[s] = W[s, s]
        e[s] = 0.0 if alpha == 0 else -sg * alpha
        r = slice(s + 1, n)
        p = beta * (W[r, r] @ v)
        w = p - 0.5 * beta * (p @ v) * v
        W[r, r] -= np.outer(v, w) + np.outer(w, v)
        W[s, s + 1:] = v
    if n >= 2:
        d[n - 2] = W[n - 2, n - 2]
        e[n - 2] = W[n - 2, n - 1]
    d[n - 1] = W[n - 1, n - 1]
    return W.ravel(), d, e


def start_vectors(n):
    i = np.arange(n, dtype=object)[:, None]
    k = np.arange(n, dtype=object)[None, :]
    h = (i * 0x9E3779B97F4A7C15 + k * 0xBF58476D1CE4E5B9 + 1) & M64
    h = h ^ (h >> 31)
    h = (h * 0x94D049BB133111EB) & M64
    h = h ^ (h >> 29)
    return ((h >> 11).astype(np.float64) * 2.0 ** -53) * 2.0 - 1.0


class Buf:
    """A flat device buffer whose reads and writes are bounds-checked."""

    def __init__(self, size):
        self.a = np.full(size, np.nan)

    def get(self, idx):
        idx = np.asarray(idx)
        assert idx.min() >= 0 and idx.max() < self.a.size, "out of range"
        return self.a[idx]

    def put(self, idx, val):
        idx = np.asarray(idx)
        assert idx.min() >= 0 and idx.max() < self.a.size, "out of range"
        self.a[idx] = val


def stein_prep(d, e, eps):
    n = d.size
    r = np.abs(d) + np.r_[0.0, np.abs(e[: n - 1])] + np.r_[np.abs(e[: n - 1]), 0.0]
    tn = r.max() if n else 0.0
    if not tn > 0:
        tn = 1.0
    ortol, pert = ORTOL * tn, 10 * EPS * tn
    shift = np.zeros(n)
    cl = np.zeros(n, dtype=int)
    cl_list = []
    prev = eps[0]
    shift[0] = prev
    for k in range(1, n):
        sh = eps[k]
        if eps[k] - eps[k - 1] <= ortol:
            cl[k] = cl[k - 1]
            if cl[k] == k - 1:
                cl_list.append(cl[k])
            sh = max(eps[k], prev + pert)
        else:
            cl[k] = k
        shift[k] = sh
        prev = sh
    return tn, EPS * tn, shift, cl, cl_list


def stein_solve(d, e, shift, Z, U, scale, floor_, first, n, last=False, tn=1.0):
    """k_stein_solve, every thread k at once.  Returns the growth-test flags of the last solve
    (True where a vector falls below sqrt(0.1 / n) / (n eps ||T||))."""
    nn = n * n
    k = np.arange(n)
    lam = shift
    sc = np.ones(n) if first else scale
    st = start_vectors(n) if first else None

    def rhs(i):
        return st[i] if first else Z.get(i * n + k) * sc

    cd = d[0] - lam
    cs = np.full(n, e[0] if n > 1 else 0.0)
    y = rhs(0)
    for i in range(n - 1):
        c = np.full(n, e[i])
        a1 = d[i + 1] - lam
        b1 = np.full(n, e[i + 1] if i + 2 < n else 0.0)
        yn = rhs(i + 1)
        o = i * n + k
        keep = np.abs(cd) >= np.abs(c)
        cd = np.where(keep & (cd == 0.0), floor_, cd)
        with np.errstate(divide="ignore", invalid="ignore"):
            m = np.where(keep, c / cd, cd / c)
        U.put(o, np.where(keep, cd, c))
        U.put(nn + o, np.where(keep, cs, a1))
        U.put(2 * nn + o, np.where(keep, 0.0, b1))
        Z.put(o, np.where(keep, y, yn))
        y, cd, cs = (np.where(keep, yn - m * y, y - m * yn), np.where(keep, a1 - m * cs, cs - m * a1),
                     np.where(keep, b1, -m * b1))
    cd = np.where(cd == 0.0, floor_, cd)
    x1 = y / cd
    x2 = np.zeros(n)
    Z.put((n - 1) * n + k, x1)
    for i in range(n - 2, -1, -1):
        o = i * n + k
        x = (Z.get(o) - U.get(nn + o) * x1 - U.get(2 * nn + o) * x2) / U.get(o)
        Z.put(o, x)
        x2, x1 = x1, x
    nrm = np.sqrt(np.sum(Z.a[: nn].reshape(n, n) ** 2, axis=0))
    assert np.all(nrm > 0) and np.all(np.isfinite(nrm))
    scale[:] = 1.0 / nrm
    if not last:
        return np.zeros(n, dtype=bool)
    return nrm * (n * EPS * tn) < np.sqrt(0.1 / n)


def stein_orth(Z, Zt, cl, cl_list, scale, n):
    for k0 in cl_list:
        m = 1
        while k0 + m < n and cl[k0 + m] == k0:
            m += 1
        i = np.repeat(np.arange(n), m)
        l = np.tile(np.arange(m), n)
        Zt.put(k0 * n + l * n + i, Z.get(i * n + k0 + l) * scale[k0 + l])
        for j in range(m):
            xi = k0 * n + j * n + np.arange(n)
            for _ in range(2 if j > 0 else 0):
                dl = np.array([Zt.get(k0 * n + q * n + np.arange(n)) @ Zt.get(xi) for q in range(j)])
                t = Zt.get(xi)
                for q in range(j):
                    t = t - dl[q] * Zt.get(k0 * n + q * n + np.arange(n))
                Zt.put(xi, t)
            x = Zt.get(xi)
            mx = np.max(np.abs(x))
            assert mx > 0
            Zt.put(xi, x * ((1 / mx) / np.sqrt(np.sum((x / mx) ** 2))))
        Z.put(i * n + k0 + l, Zt.get(k0 * n + l * n + i))
        scale[k0:k0 + m] = 1.0


def dgemm(A, a0, lda, sA, B, b0, ldb, sB, C, c0, ldc, sC, M, N, K, sub, batch):
    """k_dgemm: zero-filled loads (row < M, k < K, col < N), the epilogue writes row < M, col < N."""
    for z in range(batch):
        if M <= 0 or N <= 0:
            continue
        ri = np.arange(M)[:, None]
        ki = np.arange(K)[None, :]
        Am = A.get(a0 + z * sA + ri * lda + ki) if K else np.zeros((M, 0))
        kj = np.arange(K)[:, None]
        cj = np.arange(N)[None, :]
        Bm = B.get(b0 + z * sB + kj * ldb + cj) if K else np.zeros((0, N))
        cidx = c0 + z * sC + np.arange(M)[:, None] * ldc + np.arange(N)[None, :]
        prod = Am @ Bm
        C.put(cidx, C.get(cidx) - prod if sub else prod)


def eigen_large(a):
    Wf, d, e = reduce_store(a)
    return back_transform_emulated(Wf.reshape(a.shape), d, e)


def back_transform_emulated(Wm, d, e):
    """Everything after the reduction: Wm's row s holds v_s (columns > s), d and e the tridiagonal."""
    n = Wm.shape[0]
    nn = n * n
    nref = n - 2
    P = -(-nref // NB) * NB
    nblk = P // NB
    W = Buf(nn)
    W.a[:] = Wm.ravel()
    eps = np.linalg.eigvalsh(np.diag(d) + np.diag(e[: n - 1], 1) + np.diag(e[: n - 1], -1))
    tn, floor_, shift, cl, cl_list = stein_prep(d, e, eps)
    Z = Buf(nn)
    Ubuf = Buf(3 * max(nn, P * n))
    Zt = Buf(nn)
    scale = np.ones(n)
    for it in range(4):
        bad = stein_solve(d, e, shift, Z, Ubuf, scale, floor_, it == 0, n, last=it == 3, tn=tn)
        stein_orth(Z, Zt, cl, cl_list, scale, n)
    assert not bad.any(), "growth test failed on an accurate spectrum"
    Z.a[:nn] = (Z.a[:nn].reshape(n, n) * scale[None, :]).ravel()
    # back-transformation: Vt | V | Uw share the factor storage
    U = Ubuf
    vt0, v0, uw0 = 0, P * n, P * n + n * P
    s_idx = np.arange(P)[:, None]
    c_idx = np.arange(n)[None, :]
    vals = np.where((s_idx < nref) & (c_idx > s_idx), W.get(np.minimum(s_idx, n - 1) * n + c_idx), 0.0)
    U.put(vt0 + s_idx * n + c_idx, vals)
    U.put(v0 + c_idx * P + s_idx, vals)
    S = Buf(2 * nblk * NB * NB)
    t0 = nblk * NB * NB
    blk, panel = NB * NB, NB * n
    dgemm(U, vt0, n, panel, U, v0, P, NB, S, 0, NB, blk, NB, NB, n, 0, nblk)
    for b in range(nblk):  # k_wy_tfactor
        k = b * NB
        m = min(NB, nref - k)
        T = np.zeros((NB, NB))
        Sb = S.get(b * blk + np.arange(blk)).reshape(NB, NB)
        for j in range(m):
            s = k + j
            es, v1 = abs(e[s]), abs(W.get(s * n + s + 1))
            beta = 0.0 if es == 0 or v1 == 0 else 1.0 / (es * v1)
            T[:j, j] = -beta * np.array([T[r, r:j] @ Sb[r:j, j] for r in range(j)]) if j else T[:j, j]
            T[j, j] = beta
        S.put(t0 + b * blk + np.arange(blk), T.ravel())
    dgemm(S, t0, NB, blk, U, vt0, n, panel, U, uw0, n, panel, NB, n, NB, 0, nblk)
    Y = Buf(NB * n)
    for b in range(nblk - 1, -1, -1):
        k = b * NB
        dgemm(U, uw0 + b * panel + k, n, 0, Z, k * n, n, 0, Y, 0, n, 0, NB, n, n - k, 0, 1)
        dgemm(U, v0 + k * P + k, P, 0, Y, 0, n, 0, Z, k * n, n, 0, n - k, n, NB, 1, 1)
    return eps, Z.a[:nn].reshape(n, n)


def _check(a, tol=1e-12):
    n = a.shape[0]
    w, v = eigen_large(a)
    scale = max(np.max(np.abs(a)), 1e-300)
    assert np.max(np.abs(a @ v - v * w)) / scale < tol * max(1, n / 100)
    assert np.max(np.abs(v.T @ v - np.eye(n))) < tol * max(1, n / 100)
    assert np.max(np.abs(w - np.linalg.eigvalsh(a))) / scale < 1e-13 * n


@pytest.mark.parametrize("n", [3, 4, 37, 66, 130, 131, 200])
def test_emulated_path_random(n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n))
    _check(a + a.T)


def test_emulated_path_degenerate_and_split():
    rng = np.random.default_rng(7)
    n = 140
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    _check(q @ np.diag(np.repeat(rng.standard_normal(35), 4)) @ q.T)   # four-fold eigenvalues
    _check(q @ np.diag(np.r_[np.zeros(70), rng.standard_normal(70)]) @ q.T)  # a 70-fold zero
    ev = np.sort(rng.standard_normal(n))
    ev[20:30] = ev[20] + 1e-9 * np.arange(10)  # ten eigenvalues within 1e-8
    _check(q @ np.diag(ev) @ q.T)
    b = rng.standard_normal((65, 65))
    a = np.zeros((130, 130))
    a[:65, :65] = a[65:, 65:] = b + b.T  # two identical blocks: T splits, every eigenvalue double
    _check(a)
    _check(np.diag(np.arange(70.0)))
    _check(np.zeros((67, 67)))


def test_growth_test_flags_a_shift_that_is_no_eigenvalue():
    # the last solve's growth test (bit 4 of counts[1], LINALG): with the exact eigenvalues every
    # vector passes; a shift halfway between two eigenvalues gives a growth of about 2 / gap, far
    # below the threshold, and only that vector is flagged
    rng = np.random.default_rng(5)
    n = 90
    a = rng.standard_normal((n, n))
    Wf, d, e = reduce_store(a + a.T)
    eps = np.linalg.eigvalsh(np.diag(d) + np.diag(e[: n - 1], 1) + np.diag(e[: n - 1], -1))
    tn, floor_, shift, cl, cl_list = stein_prep(d, e, eps)
    bad_k = 40
    shift = shift.copy()
    shift[bad_k] = 0.5 * (eps[bad_k] + eps[bad_k + 1])
    Z, U, Zt, scale = Buf(n * n), Buf(3 * n * n), Buf(n * n), np.ones(n)
    for it in range(4):
        bad = stein_solve(d, e, shift, Z, U, scale, floor_, it == 0, n, last=it == 3, tn=tn)
        stein_orth(Z, Zt, cl, cl_list, scale, n)
    assert bad[bad_k] and bad.sum() == 1
