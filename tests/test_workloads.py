"""The seeded synthetic workloads: sizes, determinism, geometry sanity (CPU only)."""

from __future__ import annotations

import numpy as np

from am1gpu import workloads as W


def test_water32_cluster_shape():
    m = W.water32_cluster()
    assert m.natoms == 96 and m.nao() == 192
    assert int(np.sum(m.numbers == 8)) == 32
    # O-H bonds of every monomer are 0.9572 A
    for k in range(32):
        o, h1, h2 = m.xyz[3 * k: 3 * k + 3]
        assert abs(np.linalg.norm(h1 - o) - 0.9572) < 1e-12
        assert abs(np.linalg.norm(h2 - o) - 0.9572) < 1e-12


def test_alkane_water_batch_is_deterministic_and_sized():
    a = W.alkane_water_batch(n_alkanes=16, n_waters=16)
    b = W.alkane_water_batch(n_alkanes=16, n_waters=16)
    assert len(a) == 32
    for x, y in zip(a, b):
        assert np.array_equal(x.numbers, y.numbers) and np.array_equal(x.xyz, y.xyz)
    for m in a[:16]:
        n = m.tags["n"]
        assert m.natoms == 3 * n + 2 and m.nao() == 6 * n + 2
    for m in a[16:]:
        k = m.tags["k"]
        assert m.natoms == 3 * k and m.nao() == 6 * k


def test_alkane_geometry():
    rng = np.random.default_rng(0)
    for n in (1, 2, 5):
        m = W.alkane(n, rng, jitter=0.0)
        c = m.xyz[:n]
        h = m.xyz[n:]
        assert len(h) == 2 * n + 2
        d = np.linalg.norm(h[:, None] - c[None], axis=-1).min(1)
        assert np.allclose(d, 1.09)
        if n > 1:
            assert np.allclose(np.linalg.norm(np.diff(c, axis=0), axis=1), 1.54)
        assert W.min_contact(m) > 1.0
    r = W.alkane(4, rng, radical=True)
    assert r.multiplicity == 2 and r.natoms == 13


def test_serving_stream():
    reqs = W.serving_stream(n_requests=200)
    t = np.array([r.arrival_s for r in reqs])
    assert np.all(np.diff(t) > 0)
    uhf = sum(r.mol.multiplicity == 2 for r in reqs)
    assert 5 <= uhf <= 40
