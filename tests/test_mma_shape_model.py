"""A CPU model of which 16x8 MMA blocks the TMA-fed purification and commutator tiles issue
(dg_quarter_on / dg_quarter_shape / dt_ktile_shape in csrc/dmma_gemm.cuh), checked exhaustively:

* every element an epilogue keeps lies in an issued block -- the purification step keeps r <= c < n of
  each upper-triangle 64x64 tile (k_sp2.cu, sp2_step_epilogue), the commutator r < c < n
  (k_scf.cu, commutator_body) -- so skipping the others changes no kept element;
* over the 4096-molecule benchmark's sizes the issued MMAs come to about 1.10 times the algorithmic
  n^3 flops per symmetric product (1.28 with whole quarters only).

CPU only, no device."""

from __future__ import annotations

import numpy as np
import pytest

TILE = 64


def quarter_on(m0: int, n0: int, n: int, diag_tile: bool, warp: int) -> bool:
    wr, wc = (warp >> 1) * 32, (warp & 1) * 32
    return m0 + wr < n and n0 + wc < n and not (diag_tile and wr > wc)


def quarter_shape(m0: int, n0: int, n: int, diag_tile: bool, warp: int):
    """(mi, nj, dg) of dg_quarter_shape, or None when the warp issues no MMAs."""
    if not quarter_on(m0, n0, n, diag_tile, warp):
        return None
    r0, c0 = m0 + (warp >> 1) * 32, n0 + (warp & 1) * 32
    mi = min(2, (n - r0 + 15) // 16)
    nj = min(4, (n - c0 + 7) // 8)
    dg = 1 if (diag_tile and r0 - m0 == c0 - n0 and mi == 2) else 0
    return mi, nj, dg


def issued_blocks(shape):
    """(i, j) MMA blocks of dt_ktile<MI, NJ, DG>: rows 16 i .. 16 i + 15, columns 8 j .. 8 j + 7."""
    mi, nj, dg = shape
    return [(i, j) for i in range(mi) for j in range(nj) if not (dg and i == 1 and j < 2)]


def coverage(n: int):
    """Boolean n x n map of the elements some issued block computes, and the issued block count."""
    cov = np.zeros((n + 64, n + 64), dtype=bool)
    blocks = 0
    T = (n + TILE - 1) // TILE
    for tm in range(T):
        for tn in range(tm, T):
            m0, n0 = tm * TILE, tn * TILE
            for warp in range(4):
                shp = quarter_shape(m0, n0, n, tm == tn, warp)
                if shp is None:
                    continue
                r0, c0 = m0 + (warp >> 1) * 32, n0 + (warp & 1) * 32
                for i, j in issued_blocks(shp):
                    cov[r0 + 16 * i : r0 + 16 * i + 16, c0 + 8 * j : c0 + 8 * j + 8] = True
                    blocks += 1
    return cov[:n, :n], blocks


@pytest.mark.parametrize("n", list(range(1, 140)) + [150, 161, 192, 198, 200, 241, 242, 256, 257, 300, 330, 384, 400, 448])
def test_issued_blocks_hold_every_kept_element(n):
    cov, _ = coverage(n)
    r, c = np.indices((n, n))
    assert np.all(cov[r <= c]), n  # the purification keeps r <= c (the commutator's r < c is a subset)
    # the skipped blocks hold no element the epilogues keep: everything missing lies below the diagonal
    assert not np.any(~cov & (r <= c))


def test_issued_mma_work_over_the_benchmark_sizes():
    # sizes from the distribution of bench.py's 4096-molecule batch: 2048 alkanes C_k H_2k+2 (6 k + 2
    # orbitals, k ~ U{1..40}) and 2048 water clusters of k ~ U{1..64} monomers (6 k orbitals)
    rng = np.random.default_rng(1)
    ns = [6 * int(k) + 2 for k in rng.integers(1, 41, 2048)] + [6 * int(k) for k in rng.integers(1, 65, 2048)]
    alg = sum(n**3 for n in ns)
    issued = 0
    quarters = 0
    for n in set(ns):
        cnt = ns.count(n)
        _, blocks = coverage(n)
        k8 = (n + 7) // 8 * 8  # the k-loop runs to n rounded up to 8 (the second half of the last k-tile is skipped)
        issued += cnt * blocks * 16 * 8 * k8 * 2  # upper-triangle outputs only, like the n^3 count
        b = (n + 31) // 32
        quarters += cnt * b * (b + 1) // 2 * 32 * 32 * ((n + 15) // 16 * 16) * 2
    assert 1.05 < issued / alg < 1.12, issued / alg
    assert 1.2 < quarters / alg < 1.35, quarters / alg
