"""The serving loop on a B200: requests arriving while batches run on several worker streams
give the same results as the molecule solved alone, bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_stream_results_equal_solo_runs(gpu):
    from am1gpu import serve, workloads as W, _abi

    reqs = [r for r in W.serving_stream(400, rate=1000.0, seed=5) if r.mol.numbers.size <= 150][:120]
    assert len(reqs) >= 60 and any(r.mol.multiplicity > 1 for r in reqs)
    with serve.ScfServer(workers=3, budget_bytes=8 << 30, small_lane=64, small_workers=2) as srv:
        m0 = reqs[0].mol
        srv.submit(m0.numbers, _abi.angstrom_to_bohr(m0.xyz), m0.charge, m0.multiplicity).result()  # workers up
        out, wall = serve.run_stream(reqs, srv)
        stats = srv.stats
    assert stats.solved == len(reqs) + 1 and stats.batches >= 3
    for rq, (status, r, lat) in zip(reqs, out):
        m = rq.mol
        assert status == 0 and r["converged"]
        solo = gpu.scf(m.numbers, _abi.angstrom_to_bohr(m.xyz), m.charge, m.multiplicity, want_matrices=False)
        # every sum of a molecule runs in an order fixed by that molecule alone: bit for bit
        assert solo["heat_of_formation_kcal"] == r["heat_of_formation_kcal"]
        assert np.array_equal(solo["charges"], r["charges"])
        assert solo["iterations"] == r["iterations"]
        assert lat > 0
