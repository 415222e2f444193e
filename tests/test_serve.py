"""The serving loop's scheduling (am1gpu.serve), on CPU with a stand-in solver."""

from __future__ import annotations

import threading
import time

import numpy as np
import pytest

from am1gpu import serve


def _mol(k):
    # water-like stand-in: k heavy atoms, 2k hydrogens (coordinates unused by the stand-in)
    z = np.array([8] * k + [1] * (2 * k), dtype=np.int32)
    return z, np.zeros((z.size, 3))


class _Recorder:
    """A solver that records the batches it sees, how many run at once, and returns each
    molecule's atom count as its result."""

    def __init__(self, delay=0.01, fail=False):
        self.delay, self.fail = delay, fail
        self.lock = threading.Lock()
        self.batches, self.running, self.max_running = [], 0, 0

    def __call__(self, mols):
        with self.lock:
            self.running += 1
            self.max_running = max(self.max_running, self.running)
            self.batches.append(len(mols))
        try:
            time.sleep(self.delay)
            if self.fail:
                raise RuntimeError("device error")
            return [0] * len(mols), [{"natoms": int(m[0].size)} for m in mols]
        finally:
            with self.lock:
                self.running -= 1


def test_every_request_gets_its_own_result_and_batches_overlap():
    rec = _Recorder(delay=0.02)
    with serve.ScfServer(workers=3, budget_bytes=1 << 40, solve=rec) as srv:
        futs = []
        for i in range(300):
            z, x = _mol(1 + i % 17)
            futs.append((z.size, srv.submit(z, x)))
            if i % 25 == 0:
                time.sleep(0.005)  # arrivals while batches run
        for natoms, f in futs:
            s, r = f.result(timeout=30)
            assert s == 0 and r["natoms"] == natoms
    assert sum(rec.batches) == 300
    assert len(rec.batches) > 3          # requests arriving later were admitted into new batches
    assert rec.max_running >= 2          # batches overlapped
    assert srv.stats.max_concurrent_batches <= 3


def test_memory_budget_is_respected():
    rec = _Recorder(delay=0.01)
    cost = serve.device_bytes(*_mol(10)[:1])
    with serve.ScfServer(workers=2, budget_bytes=6 * cost, solve=rec) as srv:
        futs = [srv.submit(*_mol(10)) for _ in range(40)]
        for f in futs:
            f.result(timeout=30)
        assert srv.stats.max_in_flight_bytes <= 6 * cost
        assert max(rec.batches) <= 3  # one worker's share of the budget


def test_oversized_request_runs_alone():
    rec = _Recorder(delay=0.0)
    small = serve.device_bytes(*_mol(2)[:1])
    with serve.ScfServer(workers=2, budget_bytes=small, solve=rec) as srv:
        big = srv.submit(*_mol(40))
        s, r = big.result(timeout=30)
        assert s == 0 and r["natoms"] == 120


def test_solver_failure_reaches_every_request_of_the_batch():
    with serve.ScfServer(workers=1, budget_bytes=1 << 40, solve=_Recorder(fail=True)) as srv:
        futs = [srv.submit(*_mol(3)) for _ in range(5)]
        for f in futs:
            with pytest.raises(RuntimeError):
                f.result(timeout=30)


def test_device_bytes_grows_with_size_and_spin():
    a = serve.device_bytes(np.array([8, 1, 1]))
    b = serve.device_bytes(np.array([8, 1, 1] * 10))
    assert b > 50 * a / 10
    assert serve.device_bytes(np.array([6, 1, 1, 1]), multiplicity=2) > serve.device_bytes(np.array([6, 1, 1, 1]))


def test_no_request_is_lost_when_closing_with_a_queue():
    rec = _Recorder(delay=0.005)
    srv = serve.ScfServer(workers=2, budget_bytes=1 << 40, max_batch=4, solve=rec)
    futs = [srv.submit(*_mol(2)) for _ in range(50)]
    srv.close()
    assert all(f.done() and f.result()[0] == 0 for f in futs)
    assert max(rec.batches) <= 4
    with pytest.raises(RuntimeError):
        srv.submit(*_mol(1))


def test_small_lane_does_not_wait_behind_large_molecules():
    # a solver whose time grows with the largest molecule of its batch: with a lane for small
    # requests, they finish while the large batch is still running
    done = {}

    def solve(mols):
        big = max(int(m[0].size) for m in mols)
        time.sleep(0.6 if big > 60 else 0.01)
        return [0] * len(mols), [{"natoms": int(m[0].size)} for m in mols]

    with serve.ScfServer(workers=1, budget_bytes=1 << 40, solve=solve, small_lane=100, small_workers=1) as srv:
        large = srv.submit(*_mol(40))  # 160 + 80 orbitals: the large lane
        time.sleep(0.05)
        t = time.perf_counter()
        small = [srv.submit(*_mol(3)) for _ in range(5)]  # 18 orbitals each
        for f in small:
            f.result(timeout=30)
        done["small"] = time.perf_counter() - t
        assert not large.done()  # still running
        assert large.result(timeout=30)[1]["natoms"] == 120
    assert done["small"] < 0.4


def test_orbital_count():
    assert serve.orbitals(np.array([8, 1, 1])) == 6
    assert serve.orbitals(np.array([6, 6, 1, 1, 1, 1, 1, 1])) == 14


def test_a_failing_lane_start_does_not_stop_the_lane():
    rec = _Recorder(delay=0.0)

    def boom(lane):
        raise RuntimeError("no device")

    with serve.ScfServer(workers=1, budget_bytes=1 << 40, solve=rec, small_lane=100, small_workers=1,
                         on_worker_start=boom) as srv:
        futs = [srv.submit(*_mol(2)), srv.submit(*_mol(40))]  # one per lane
        assert all(f.result(timeout=30)[0] == 0 for f in futs)
