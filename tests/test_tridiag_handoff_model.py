"""CPU models of two ways the batch reuses work (no device):

* the hand-off of k_tridiag (csrc/k_eigvals.cu) and its job chain (csrc/driver.cu): a Householder
  reduction in the kernel's lazy form (update s - 1 applied to row s, then to the trailing rows while
  A v_s is formed) stops after `stop` reflectors and writes the trailing block with its last update
  applied; a fresh reduction of that block, continuing at d[stop], e[stop], must give a tridiagonal with
  the matrix's eigenvalues.  The chain of cluster sizes (C -> C/2 -> ... -> 1, each hand-off at the
  largest order C/2 CTAs hold) is restated from tridiag_smem_bytes and checked to fit at every level;
* the spectral interval of the purification reused from the previous SCF iteration (k_sp2_bounds in
  csrc/k_sp2.cu): an interval holding the spectrum of A, widened by ||E||_F on both sides, holds the
  spectrum of A + E (Weyl)."""

from __future__ import annotations

import numpy as np
import pytest

TRI_WARPS, TRI_THREADS = 16, 512
BUDGET = 232448 - 1024  # the 227 KB opt-in shared memory less the kernel's static share


def tridiag_smem_bytes(n: int, C: int) -> int:
    rows = (n + C - 1) // C
    return 8 * (rows * n + 5 * n + 2 + TRI_WARPS + TRI_THREADS)


def cluster_max(C: int) -> int:
    m = 2
    while tridiag_smem_bytes(m + 1, C) <= BUDGET:
        m += 1
    return m


def tridiag_cluster(n: int) -> int:
    for C in (1, 2, 4, 8, 16):
        if tridiag_smem_bytes(n, C) <= BUDGET:
            return C
    return 0


def chain(n: int):
    """[(order, CTAs)] of the job and its continuations, as the driver builds them."""
    C = tridiag_cluster(n)
    out = [(n, C)]
    cur = n
    while C > 1:
        m = cluster_max(C // 2)
        if m < 8 or m >= cur:
            break
        out.append((m, C // 2))
        cur, C = m, C // 2
    return out


def lazy_tridiag(a: np.ndarray, stop: int | None = None):
    """d, e of the reduction, or (d[:stop], e[:stop], trailing block) when it stops after `stop` reflectors."""
    A = a.copy()
    n = A.shape[0]
    d, e = np.zeros(n), np.zeros(max(n - 1, 0))
    v, w = np.zeros(n), np.zeros(n)
    for s in range(n - 1):
        A[s, s:] -= v[s] * w[s:] + w[s] * v[s:]
        x = A[s, s + 1 :].copy()
        alpha = np.sqrt(x @ x)
        sg = 1.0 if x[0] >= 0.0 else -1.0
        d[s] = A[s, s]
        e[s] = 0.0 if alpha == 0.0 else -sg * alpha
        if s + 2 >= n:  # the last 2 x 2 block, read as it stands (k_tridiag's tail)
            e[s] = x[0]
            A[n - 1, n - 1] -= 2.0 * v[n - 1] * w[n - 1]
            d[n - 1] = A[n - 1, n - 1]
            break
        beta = 0.0 if alpha == 0.0 else 1.0 / (alpha * (alpha + abs(x[0])))
        vn = np.zeros(n)
        vn[s + 1 :] = x
        if alpha != 0.0:
            vn[s + 1] = x[0] + sg * alpha
        A[s + 1 :, s + 1 :] -= np.outer(v[s + 1 :], w[s + 1 :]) + np.outer(w[s + 1 :], v[s + 1 :])
        p = np.zeros(n)
        p[s + 1 :] = beta * (A[s + 1 :, s + 1 :] @ vn[s + 1 :])
        kk = 0.5 * beta * (p[s + 1 :] @ vn[s + 1 :])
        v, w = vn, p - kk * vn
        if stop is not None and s + 1 == stop:
            T = A[stop:, stop:] - np.outer(v[stop:], w[stop:]) - np.outer(w[stop:], v[stop:])
            return d[:stop], e[:stop], T
    return d, e


def tridiagonal_eigs(d, e):
    return np.linalg.eigvalsh(np.diag(d) + np.diag(e[: len(d) - 1], 1) + np.diag(e[: len(d) - 1], -1))


@pytest.mark.parametrize("n,stops", [(12, [3]), (40, [25]), (60, [10, 20, 20]), (90, [30, 20, 15])])
def test_handed_off_reduction_keeps_the_spectrum(n, stops):
    rng = np.random.default_rng(n)
    m = rng.standard_normal((n, n))
    a = m + m.T
    d_all, e_all = [], []
    block = a
    for st in stops:  # a chain of hand-offs, each continuing on the block the previous one wrote
        d, e, block = lazy_tridiag(block, st)
        d_all.append(d)
        e_all.append(e)
    d, e = lazy_tridiag(block)
    d = np.concatenate(d_all + [d])
    e = np.concatenate(e_all + [e])
    assert d.shape == (n,) and e.shape == (n - 1,)
    ref = np.linalg.eigvalsh(a)
    assert np.max(np.abs(tridiagonal_eigs(d, e) - ref)) < 1e-12 * np.max(np.abs(ref)) * n


def test_handoff_chain_fits_every_level():
    assert [cluster_max(C) for C in (1, 2, 4, 8)] == [166, 232, 326, 456]
    for n in range(2, 632):
        ch = chain(n)
        assert ch[0] == (n, tridiag_cluster(n))
        for order, C in ch:
            assert tridiag_smem_bytes(order, C) <= BUDGET
        for (n1, c1), (n2, c2) in zip(ch, ch[1:]):
            assert c2 == c1 // 2 and n2 < n1 and n1 - n2 >= 1
        if ch[0][1] > 1:  # every cluster job ends on one CTA
            assert ch[-1][1] == 1
    assert chain(384) == [(384, 8), (326, 4), (232, 2), (166, 1)]


def test_widened_interval_holds_the_moved_spectrum():
    rng = np.random.default_rng(5)
    for n in (10, 60, 200):
        m = rng.standard_normal((n, n))
        a = m + m.T
        ev = np.linalg.eigvalsh(a)
        lo, hi = ev[0] - 1e-3, ev[-1] + 1e-3
        for scale in (1e-6, 1e-3, 1e-1):
            p = rng.standard_normal((n, n)) * scale
            E = p + p.T
            delta = np.linalg.norm(E)  # Frobenius, the sum of the rows' squared differences
            ev2 = np.linalg.eigvalsh(a + E)
            assert lo - delta <= ev2[0] and ev2[-1] <= hi + delta
