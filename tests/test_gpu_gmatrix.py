"""Batched two-electron matrices G(P) = J(P) - K(P/2) on a B200 (am1gpu_g_matrix_batch), the
CPHF response kernel of the reference (build_g_matrix, src/fock.rs:556-575), against the oracle's
Fock build at the same densities minus its H_core."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method", ["am1", "rm1"])
def test_g_matrix_batch_matches_oracle(gpu, oracle, method):
    from am1gpu import workloads as W, _abi

    rng = np.random.default_rng(17)
    m = W.alkane(3, rng)
    w = W.water_cluster(2, rng)
    z = np.concatenate([m.numbers, w.numbers])
    xyz = _abi.angstrom_to_bohr(np.concatenate([m.xyz, w.xyz + np.array([6.0, 0.0, 0.0])]))
    n = oracle.nao_of(z, method)
    nrhs = 70  # more than one chunk of copies
    d = rng.standard_normal((nrhs, n, n)) * 0.1
    d = d + d.transpose(0, 2, 1)  # response densities are symmetric
    g = gpu.g_matrix_batch(z, xyz, d, method=method)
    h, _ = oracle.build_core(z, xyz, method)
    for r in (0, 1, 33, 63, 64, 69):
        ref = oracle.build_fock(z, xyz, d[r], d[r], 0.5, method) - h
        assert np.max(np.abs(g[r] - ref)) < 1e-9, r
    # linear in P: G(a P1 + b P2) = a G(P1) + b G(P2)
    lin = gpu.g_matrix_batch(z, xyz, (2.0 * d[0] - 0.5 * d[1])[None], method=method)[0]
    assert np.max(np.abs(lin - (2.0 * g[0] - 0.5 * g[1]))) < 1e-9
