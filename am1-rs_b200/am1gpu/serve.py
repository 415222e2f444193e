"""Serving: a continuous-batching request loop over the batched SCF.

Requests (one molecule each) arrive at any time.  ``ScfServer`` keeps ``workers`` host threads;
each owns a CUDA stream and a device workspace inside libam1gpu (the library keeps both per host
thread).  A free worker takes every pending request that fits the device-memory budget, in
arrival order, and solves them as one batch (``am1gpu_scf_batch``).  Requests that arrive while
batches are on the GPU wait only for the next free worker, and up to ``workers`` batches run at
the same time on the device, so the work of different batches overlaps there.  Inside a batch
every molecule keeps its own SCF trajectory and convergence test and retires in place, so a
result is the same whether the molecule was solved alone or in any mix (tested).

With ``small_lane`` set, requests of at most that many orbitals go to a lane of their own, served
by ``small_workers`` further threads: a small molecule then waits for other small ones, not behind a
batch of 1000-orbital molecules (the lanes share the device, each batch on its own stream, and the
small lane's streams have the higher CUDA priority).

The budget is a fraction of the free device memory when the server starts; each request is
charged an estimate of its device footprint (the per-channel matrix slots, the packed DIIS
histories and the integral store).  The library's per-thread device pool only grows, so one
batch is also capped at ``budget / workers``: the pools of all workers together stay inside the
budget.  A request larger than that share still runs, alone, once nothing else is in flight.

Run as a module for the serving workload (open-loop Poisson arrivals, sizes log-uniform on
[3, 600] atoms, RHF:UHF = 9:1): ``python -m am1gpu.serve --requests 20000 --rate 2000``.
"""

from __future__ import annotations

import collections
import concurrent.futures
import json
import threading
import time
from dataclasses import dataclass, field

import numpy as np


def orbitals(numbers) -> int:
    """Valence orbitals of a molecule (4 per heavy atom, 1 per hydrogen)."""
    z = np.asarray(numbers)
    return int(4 * np.count_nonzero(z != 1) + np.count_nonzero(z == 1))


def device_bytes(numbers, multiplicity: int = 1) -> int:
    """Device memory one molecule occupies inside a batch (an estimate, in bytes)."""
    z = np.asarray(numbers)
    h = int(np.count_nonzero(z != 1))
    H = int(z.size) - h
    n = 4 * h + H
    nch = 2 if multiplicity > 1 else 1
    slots = n * n * (1 + 6 * nch)                   # H_core + six matrix slots per channel
    hist = nch * 8 * (3 * n * (n + 1) // 2)         # packed F, e, D histories, depth 8
    store = 100 * h * (h - 1) // 2 + 10 * h * H + H * (H - 1) // 2
    return 8 * (slots + hist + store) + 4096


@dataclass
class _Pending:
    mol: tuple
    cost: int
    future: concurrent.futures.Future
    t_submit: float


@dataclass
class ServerStats:
    batches: int = 0
    solved: int = 0
    largest_batch: int = 0
    max_in_flight_bytes: int = 0
    max_concurrent_batches: int = 0
    batch_sizes: list = field(default_factory=list)


class ScfServer:
    """Continuous-batching SCF service.

    ``solve(mols) -> (status list, result dicts)`` defaults to the library's batched call; any
    callable with that signature can stand in (the CPU tests use one).
    """

    def __init__(self, workers: int = 3, max_batch: int = 2048, budget_bytes: int | None = None,
                 budget_fraction: float = 0.7, solve=None, small_lane: int | None = None, small_workers: int = 2,
                 on_worker_start=None, **opts):
        self._lane_start = None
        if solve is None:
            from . import native

            def solve(mols, _o=opts):
                return native.scf_batch(mols, want_matrices=False, **_o)

            # the small-request lane's streams go first on the SMs
            self._lane_start = lambda lane: native.set_stream_priority(-1 if lane == 1 else 0)
        if on_worker_start is not None:  # called in each worker thread with its lane (0 large, 1 small)
            self._lane_start = on_worker_start
        self._solve = solve
        if budget_bytes is None:
            budget_bytes = int(budget_fraction * _free_device_bytes())
        self.budget = int(budget_bytes)
        self.small_lane = small_lane
        lanes = [0] * int(workers) + ([1] * int(small_workers) if small_lane is not None else [])
        self.share = self.budget // max(1, len(lanes))
        self.max_batch = int(max_batch)
        self._queues: list[collections.deque[_Pending]] = [collections.deque(), collections.deque()]
        self._cv = threading.Condition()
        self._in_flight = 0
        self._running_batches = 0
        self._closed = False
        self.stats = ServerStats()
        self._threads = [threading.Thread(target=self._worker, args=(lane,), name=f"scf-worker-{i}", daemon=True)
                         for i, lane in enumerate(lanes)]
        for t in self._threads:
            t.start()

    def submit(self, numbers, xyz_bohr, charge: float = 0.0, multiplicity: int = 1) -> concurrent.futures.Future:
        """Queue one molecule (positions in Bohr); the future resolves to (status, result dict)."""
        fut: concurrent.futures.Future = concurrent.futures.Future()
        p = _Pending((np.asarray(numbers, dtype=np.int32), np.asarray(xyz_bohr, dtype=np.float64), float(charge), int(multiplicity)),
                     device_bytes(numbers, multiplicity), fut, time.perf_counter())
        lane = 1 if self.small_lane is not None and orbitals(numbers) <= self.small_lane else 0
        with self._cv:
            if self._closed:
                raise RuntimeError("server closed")
            self._queues[lane].append(p)
            self._cv.notify_all()
        return fut

    def close(self, wait: bool = True) -> None:
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        if wait:
            for t in self._threads:
                t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- scheduling --------------------------------------------------------------------------
    def _take(self, lane: int) -> list[_Pending]:
        """The lane's pending requests that fit the budget, in arrival order (lock held)."""
        q = self._queues[lane]
        batch: list[_Pending] = []
        room = min(self.budget - self._in_flight, self.share)
        while q and len(batch) < self.max_batch:
            p = q[0]
            if p.cost > room and (batch or self._in_flight > 0):
                break  # wait for memory to free up
            batch.append(q.popleft())
            room -= p.cost
        return batch

    def _worker(self, lane: int) -> None:
        if self._lane_start is not None:
            try:
                self._lane_start(lane)
            except Exception:  # the priority only orders the work; the lane still serves without it
                pass
        while True:
            with self._cv:
                while True:
                    batch = self._take(lane)
                    if batch or (self._closed and not self._queues[lane]):
                        break
                    self._cv.wait()
                if not batch:
                    return
                cost = sum(p.cost for p in batch)
                self._in_flight += cost
                self._running_batches += 1
                st = self.stats
                st.batches += 1
                st.batch_sizes.append(len(batch))
                st.largest_batch = max(st.largest_batch, len(batch))
                st.max_in_flight_bytes = max(st.max_in_flight_bytes, self._in_flight)
                st.max_concurrent_batches = max(st.max_concurrent_batches, self._running_batches)
            try:
                status, results = self._solve([p.mol for p in batch])
                for p, s, r in zip(batch, status, results):
                    p.future.set_result((int(s), r))
            except BaseException as exc:  # the whole batch failed: every request sees the error
                for p in batch:
                    if not p.future.done():
                        p.future.set_exception(exc)
            finally:
                with self._cv:
                    self._in_flight -= cost
                    self._running_batches -= 1
                    self.stats.solved += len(batch)
                    self._cv.notify_all()


def _free_device_bytes() -> int:
    try:
        import torch

        if torch.cuda.is_available():
            return int(torch.cuda.mem_get_info()[0])
    except Exception:
        pass
    return 16 << 30


def run_stream(requests, server: ScfServer, time_scale: float = 1.0):
    """Feed requests (objects with ``arrival_s`` and ``mol``) at their arrival times; returns
    per-request (status, result, latency_s) and the wall time from the first arrival to the last
    completion."""
    from . import _abi

    t0 = time.perf_counter()
    futs = []
    for rq in requests:
        delay = t0 + rq.arrival_s * time_scale - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        m = rq.mol
        f = server.submit(m.numbers, _abi.angstrom_to_bohr(m.xyz), m.charge, m.multiplicity)
        f.t_arrive = time.perf_counter()
        f.add_done_callback(lambda fut: setattr(fut, "t_done", time.perf_counter()))
        futs.append(f)
    out = []
    for f in futs:
        s, r = f.result()
        out.append((s, r, f.t_done - f.t_arrive))
    wall = max(f.t_done for f in futs) - t0
    return out, wall


def _pct(lat_s):
    if not lat_s:
        return None
    a = np.array(lat_s) * 1e3
    return {"n": int(a.size), "p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99))}


def _main():
    import argparse

    from . import native, workloads as W

    ap = argparse.ArgumentParser(description="serving workload: open-loop Poisson stream of SCF requests")
    ap.add_argument("--requests", type=int, default=20000)
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--workers", type=int, default=3)
    ap.add_argument("--plain-sample", type=int, default=32)
    ap.add_argument("--small-lane", type=int, default=None,
                    help="orbital count up to which requests get their own lane (and --small-workers threads)")
    ap.add_argument("--small-workers", type=int, default=2)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                    help="arithmetic of the batched solves (mixed: TF32 purification in the early iterations)")
    args = ap.parse_args()
    reqs = W.serving_stream(args.requests, args.rate, seed=2)
    from . import _abi

    native.ensure_loaded()
    with ScfServer(workers=args.workers, precision=args.precision, small_lane=args.small_lane,
                   small_workers=args.small_workers) as srv:
        # warm every worker's workspace once
        warm = [srv.submit(r.mol.numbers, _abi.angstrom_to_bohr(r.mol.xyz), r.mol.charge, r.mol.multiplicity) for r in reqs[:64]]
        for f in warm:
            f.result()
        out, wall = run_stream(reqs, srv)
        stats = srv.stats
    lat = np.array([o[2] for o in out]) * 1e3
    ok = sum(1 for o in out if o[0] == 0)
    # plain path: one am1gpu_scf call per molecule on a sample
    t = time.perf_counter()
    for r in reqs[: args.plain_sample]:
        native.scf(r.mol.numbers, _abi.angstrom_to_bohr(r.mol.xyz), r.mol.charge, r.mol.multiplicity, want_matrices=False)
    plain = args.plain_sample / (time.perf_counter() - t)
    line = {
        "workload": f"{args.requests} requests, Poisson arrivals at {args.rate:g}/s, sizes log-uniform on [3, 600] atoms, "
                    "RHF:UHF = 9:1, seed 2 (alkanes, alkane radicals, water clusters)",
        "solves_per_s": len(out) / wall, "offered_per_s": args.rate, "ok": ok, "failed": len(out) - ok,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
        "plain_solves_per_s": plain, "batches": stats.batches, "mean_batch": float(np.mean(stats.batch_sizes)),
        "largest_batch": stats.largest_batch, "max_concurrent_batches": stats.max_concurrent_batches,
        "max_in_flight_gb": stats.max_in_flight_bytes / 1e9, "workers": args.workers, "precision": args.precision,
        "small_lane": args.small_lane, "small_workers": args.small_workers if args.small_lane is not None else 0,
        "latency_ms_small": _pct([o[2] for o, r in zip(out, reqs) if args.small_lane is not None and orbitals(r.mol.numbers) <= args.small_lane]),
        "latency_ms_large": _pct([o[2] for o, r in zip(out, reqs) if args.small_lane is not None and orbitals(r.mol.numbers) > args.small_lane]),
    }
    print(json.dumps(line))


if __name__ == "__main__":
    _main()
