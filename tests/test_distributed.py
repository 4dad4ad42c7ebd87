"""Multi-process (world size 2, gloo, CPU) tests of the ensemble sharding across ranks.

Each rank runs its share with a CPU runner built on the oracle (the GPU runner is the batched
engine, covered by tests/test_batch.py); rank 0 gathers and checks that every job's series and
final lattice equal a single-process run, whichever rank ran it.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pyising_b200.distributed import job_cost, partition


def test_partition_balances_and_covers():
    costs = [10, 1, 7, 7, 3, 3, 2, 8, 1, 5]
    for world in (1, 2, 3, 4):
        plan = partition(costs, world)
        assert sorted(i for p in plan for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in plan]
        assert max(loads) - min(loads) <= max(costs)
        assert plan == partition(costs, world)  # deterministic
    with pytest.raises(ValueError):
        partition(costs, 0)


def test_job_cost_weights_packed_words():
    from pyising_b200.ensemble import Job

    a = Job((64, 128), 0.4, 10, init="cold")
    b = Job((64, 128), 0.4, 10, variant="msc", init="cold")
    assert job_cost(a) == 4 * job_cost(b) == 64 * 128 * 10


def _jobs():
    from pyising_b200.ensemble import Job

    return [Job((16, 24), 0.42, 6, seed=2**40 + 7, measure_every=2, keep_lattice=True),
            Job((8, 8, 16), 0.22, 5, seed=3, algorithm="heatbath", measure_every=1,
                keep_lattice=True),
            Job((32, 128), 0.44, 7, seed=11, variant="msc", measure_every=7, keep_lattice=True),
            Job((64, 32), 0.3, 9, seed=5, measure_every=3, keep_lattice=True, init="cold"),
            Job((16, 16), 0.5, 4, seed=8, keep_lattice=True)]


def oracle_runner(jobs):
    """CPU stand-in for the GPU batch: the oracle, one job at a time."""
    import oracle
    from pyising_b200.ensemble import Result

    out = []
    for j in jobs:
        init = j.init
        if isinstance(init, str) and init == "hot":
            init = oracle.random_lattice(j.shape, j.seed)
        sim = oracle.create(j.variant, shape=j.shape, beta=j.beta, seed=j.seed,
                            algorithm=j.algorithm, init=init)
        sim.t = j.t0
        series = sim.sweep(j.sweeps, measure_every=j.measure_every)
        out.append(Result(series if series is not None else np.zeros((0, 2), np.int64),
                          sim.get_lattice()))
    return out


def _worker(rank, world, port, queue):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pyising_b200.distributed import run_sharded

        res = run_sharded(_jobs(), runner=oracle_runner, gather_to=0)
        allres = run_sharded(_jobs(), runner=oracle_runner, gather_to=None)
        if rank == 0:
            queue.put(("gather", [(r.series, r.lattice) for r in res]))
        else:
            assert res is None
        queue.put((f"all{rank}", [(r.series, r.lattice) for r in allres]))
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_ensemble_world2_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(3))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = [(r.series, r.lattice) for r in oracle_runner(_jobs())]
    for key in ("gather", "all0", "all1"):
        assert len(got[key]) == len(want)
        for (s, lat), (ws, wl) in zip(got[key], want, strict=True):
            np.testing.assert_array_equal(s, ws)
            np.testing.assert_array_equal(lat, wl)
