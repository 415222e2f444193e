"""Two ranks over gloo on the CPU: partition, per-rank solve, gather (CPU only).

The per-rank solver here is the CPU oracle; on GPUs the same helper drives the batched
library on each rank.  The multi-rank result must equal the single-process one.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import torch.multiprocessing as mp

from am1gpu import parallel


def _mols():
    from am1gpu import workloads as W, _abi

    rng = np.random.default_rng(9)
    mols = [W.alkane(n, rng) for n in (1, 3, 5, 2)] + [W.water_cluster(k, rng) for k in (1, 2, 4)]
    return [(m.numbers, _abi.angstrom_to_bohr(m.xyz), 0.0, 1) for m in mols]


def _oracle_solve(batch):
    import oracle

    _, res = oracle.scf_batch(batch, nthreads=1)
    return [(r["status"], r["heat_of_formation_kcal"], r["iterations"]) for r in res]


def _worker(rank, world, port, out_path):
    import sys

    import torch.distributed as dist

    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (os.path.join(root, "am1-rs_b200"), os.path.join(root, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        res = parallel.solve_sharded(_mols(), _oracle_solve, dist)
        if rank == 0:
            import json

            with open(out_path, "w") as f:
                json.dump(res, f)
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_partition_balances_and_covers():
    costs = [5.0, 1.0, 1.0, 1.0, 4.0, 3.0, 3.0]
    parts = parallel.partition(costs, 2)
    assert sorted(i for p in parts for i in p) == list(range(7))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert abs(loads[0] - loads[1]) <= 2.0


def test_two_ranks_gloo_match_one(tmp_path):
    out = tmp_path / "res.json"
    mp.start_processes(_worker, args=(2, _free_port(), str(out)), nprocs=2, join=True, start_method="spawn")
    import json

    two = [tuple(x) for x in json.loads(out.read_text())]
    one = [tuple(x) for x in parallel.solve_sharded(_mols(), _oracle_solve, None)]
    assert len(two) == len(one) == 7
    for a, b in zip(two, one):
        assert a[0] == b[0] == 0
        assert abs(a[1] - b[1]) < 1e-9 and a[2] == b[2]
