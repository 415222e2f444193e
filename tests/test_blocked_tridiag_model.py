"""A NumPy model of the blocked Householder reduction of k_tridiag_panel / k_tridiag_syr2k
(csrc/k_eigvals.cu), step for step: per column the corrected column x, the reflector, p and w
against the trailing matrix as it stood at the panel's start, then one rank-2B update per panel.
The model's tridiagonal must have the matrix's eigenvalues, and the reflectors it leaves in the rows of
the working copy (as k_tridiag_panel writes them) must back-transform the tridiagonal's eigenvectors into
the matrix's (CPU only, no device)."""

from __future__ import annotations

import numpy as np
import pytest


def blocked_tridiag(a: np.ndarray, B: int, keep: bool = False):
    """d, e (and, with keep, the working copy whose row c holds reflector v_c in columns > c)."""
    A = a.copy()
    n = A.shape[0]
    d = np.zeros(n)
    e = np.zeros(max(n - 1, 0))
    k = 0
    while k < n - 1:
        bw = min(B, n - 1 - k)
        V = np.zeros((n, B))
        W = np.zeros((n, B))
        for j in range(bw):
            c = k + j
            # column c with the panel's earlier updates: x_i = A_ic - sum_l (V_il W_cl + W_il V_cl)
            x = A[c:, c] - V[c:, :j] @ W[c, :j] - W[c:, :j] @ V[c, :j]
            d[c] = x[0]
            if c + 2 > n - 1:  # the last 2 x 2 block
                e[c] = x[1]
                d[n - 1] = A[n - 1, n - 1] - 2.0 * V[n - 1, :j] @ W[n - 1, :j]
                break
            xs = x[1:]
            alpha = np.sqrt(xs @ xs)
            sg = 1.0 if xs[0] >= 0.0 else -1.0
            beta = 0.0 if alpha == 0.0 else 1.0 / (alpha * (alpha + abs(xs[0])))
            v = xs.copy()
            v[0] += sg * alpha
            # p = beta (A v - V (W^T v) - W (V^T v)) over rows and columns > c, A as at the panel start
            r = slice(c + 1, n)
            p = beta * (A[r, r] @ v - V[r, :j] @ (W[r, :j].T @ v) - W[r, :j] @ (V[r, :j].T @ v))
            kk = 0.5 * beta * (p @ v)
            V[r, j] = v
            W[r, j] = p - kk * v
            A[c, c + 1:] = v  # row c is never read again
            e[c] = 0.0 if alpha == 0.0 else -sg * alpha
        if k + bw < n - 1:  # the trailing update, rank 2B
            t = slice(k + B, n)
            A[t, t] -= V[t] @ W[t].T + W[t] @ V[t].T
        k += B
    if n == 1:
        d[0] = A[0, 0]
    return (d, e, A) if keep else (d, e)


@pytest.mark.parametrize("n,B", [(2, 32), (3, 32), (33, 32), (64, 32), (97, 32), (150, 8), (200, 32)])
def test_blocked_model_keeps_the_spectrum(n, B):
    rng = np.random.default_rng(n * 7 + B)
    a = rng.standard_normal((n, n))
    a = a + a.T
    d, e = blocked_tridiag(a, B)
    t = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    assert np.max(np.abs(np.linalg.eigvalsh(t) - np.linalg.eigvalsh(a))) < 1e-10 * max(1.0, np.max(np.abs(a)))


def test_blocked_model_equals_the_unblocked_reduction():
    # one column per panel (B = 1) is the plain Householder sequence; any panel width gives the same
    # tridiagonal (the rank-2 updates only regroup)
    rng = np.random.default_rng(5)
    a = rng.standard_normal((70, 70))
    a = a + a.T
    d1, e1 = blocked_tridiag(a, 1)
    d32, e32 = blocked_tridiag(a, 32)
    assert np.max(np.abs(d1 - d32)) < 1e-11 and np.max(np.abs(e1 - e32)) < 1e-11


@pytest.mark.parametrize("n,B", [(66, 32), (131, 32), (200, 8)])
def test_blocked_reflectors_back_transform(n, B):
    from test_stein_model import back_transform_emulated

    rng = np.random.default_rng(n + B)
    a = rng.standard_normal((n, n))
    a = a + a.T
    d, e, Wk = blocked_tridiag(a, B, keep=True)
    w, v = back_transform_emulated(Wk, d, np.r_[e, 0.0])
    assert np.max(np.abs(a @ v - v * w)) < 1e-12 * np.max(np.abs(w))
    assert np.max(np.abs(v.T @ v - np.eye(n))) < 1e-12
