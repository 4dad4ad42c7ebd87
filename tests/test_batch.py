"""Batched ensembles and serving: every lattice run in a batch (or through the server, mixed
with others that arrive while it runs) is bit-identical to the same job run alone with the
single-lattice kernels, and to the oracle.  Exact integer comparison throughout."""

from __future__ import annotations

import threading
import time

import numpy as np
import pytest
from conftest import golden, unpack_lattice

pytestmark = pytest.mark.gpu

BETA_C_2D = 0.44068679350977147


def solo(job, oracle_mod):
    """The job alone: single-lattice kernels (and the oracle for small lattices)."""
    from pyising_b200.backend import B200Int8, B200MultiSpin

    cls = B200MultiSpin if job.variant == "msc" else B200Int8
    init = job.init
    sim = cls(job.shape, job.beta, seed=job.seed, algorithm=job.algorithm,
              init=init if isinstance(init, np.ndarray) else ("cold" if init == "cold" else
                                                              ("philox" if init == "philox"
                                                               else "hot")))
    sim.t = job.t0
    sim.table = job.table
    sim._upload_table()
    if job.measure_every:
        series = sim.sweep_measured(job.sweeps, job.measure_every)
    else:
        sim.sweep(job.sweeps)
        series = np.zeros((0, 2), np.int64)
    return series, sim.get_lattice()


def mixed_jobs():
    from pyising_b200.ensemble import Job

    rng = np.random.default_rng(3)
    jobs = [
        Job((64, 64), 1 / 2.3, 40, seed=1, measure_every=10, keep_lattice=True),
        Job((128, 256), BETA_C_2D, 25, seed=2**40 + 5, measure_every=5, keep_lattice=True),
        Job((16, 24), 0.42, 30, seed=3, algorithm="heatbath", measure_every=3, keep_lattice=True),
        Job((8, 8, 16), 0.22, 17, seed=4, algorithm="heatbath", measure_every=4,
            keep_lattice=True),
        Job((16, 16, 32), 0.2216, 22, seed=5, measure_every=11, keep_lattice=True),
        Job((128, 128), BETA_C_2D, 33, seed=6, variant="msc", measure_every=3, keep_lattice=True),
        Job((64, 384), 0.3, 12, seed=7, variant="msc", keep_lattice=True),
        Job((40, 1032), 0.4, 9, seed=8, measure_every=2, keep_lattice=True, init="cold"),
        Job((32, 64), 0.35, 15, seed=9, t0=2**32 - 4, measure_every=5, keep_lattice=True),
        Job((256, 512), 0.41, 21, seed=10, variant="msc", init="philox", measure_every=7,
            keep_lattice=True),
        Job((32, 32, 32), 0.23, 14, seed=11, algorithm="heatbath", init="philox",
            measure_every=7, keep_lattice=True),
        Job((24, 48), -0.3, 8, seed=12, algorithm="heatbath", keep_lattice=True),  # generic rule
        Job((32, 64), 0.4, 0, seed=13, keep_lattice=True),  # zero sweeps
    ]
    for k in range(6):  # a few random 2D int8 lattices of uneven size
        L = int(rng.choice([8, 16, 24, 32, 48, 64, 96]))
        jobs.append(Job((L, 2 * L), float(rng.uniform(0.3, 0.5)), int(rng.integers(1, 30)),
                        seed=100 + k, measure_every=int(rng.integers(0, 4)), keep_lattice=True))
    return jobs


def test_device_seeded_start_matches_oracle(oracle_mod):
    from pyising_b200.backend import B200Int8, B200MultiSpin

    for cls, shape in ((B200Int8, (16, 24)), (B200Int8, (6, 8, 16)), (B200MultiSpin, (16, 256)),
                       (B200Int8, (16, 256))):
        sim = cls(shape, 0.4, seed=2**40 + 77, init="philox")
        np.testing.assert_array_equal(sim.get_lattice(), oracle_mod.philox_start(shape, 2**40 + 77))
    lat = oracle_mod.philox_start((64, 64), 9)
    assert abs(lat.mean()) < 0.05


def test_ensemble_members_equal_solo_runs(oracle_mod):
    from pyising_b200.ensemble import Ensemble

    jobs = mixed_jobs()
    with Ensemble(memory_budget=1 << 30) as ens:
        ids = [ens.add(j) for j in jobs]
        ens.run()
        for jid, job in zip(ids, jobs, strict=True):
            assert ens.status(jid) == ("done", job.sweeps)
            res = ens.result(jid)
            want_series, want_lat = solo(job, oracle_mod)
            np.testing.assert_array_equal(res.series, want_series, err_msg=str(job))
            np.testing.assert_array_equal(res.lattice, want_lat, err_msg=str(job))
            ens.release(jid)


def test_run_counts_half_sweeps_with_graph_chunks(oracle_mod):
    """run(k) advances exactly k half-sweeps, also while the batch replays graph chunks of many
    sweeps (a chunk that does not fit the k left is not replayed), and a run split into pieces
    gives the results of the job alone."""
    from pyising_b200.ensemble import Ensemble, Job

    jobs = [Job((64, 64), BETA_C_2D, 120, seed=s, measure_every=10, keep_lattice=True)
            for s in range(3)]
    with Ensemble(memory_budget=1 << 30) as ens:
        ens.set_knob("graph_chunk", 8)
        ids = [ens.add(j) for j in jobs]
        assert ens.run(2) == 2
        assert all(ens.status(i) == ("active", 1) for i in ids)
        assert ens.run(37) == 37  # ends between the two colours of a sweep
        assert all(ens.status(i) == ("active", 19) for i in ids)
        assert ens.run(70) == 70
        assert all(ens.status(i) == ("active", 54) for i in ids)
        ens.run()
        for jid, job in zip(ids, jobs, strict=True):
            assert ens.status(jid) == ("done", job.sweeps)
            want_series, want_lat = solo(job, oracle_mod)
            res = ens.result(jid)
            np.testing.assert_array_equal(res.series, want_series)
            np.testing.assert_array_equal(res.lattice, want_lat)


def test_ensemble_small_budget_admits_in_turns(oracle_mod):
    """A budget that holds about two lattices at a time: jobs wait and join at later sweep
    boundaries, and the results are unchanged."""
    from pyising_b200.ensemble import Ensemble, Job

    jobs = [Job((64, 128), 0.3 + 0.02 * k, 10 + 3 * k, seed=k, measure_every=5,
                keep_lattice=True) for k in range(6)]
    per_job = 64 * 128 + (jobs[-1].n_measurements) * 16
    with Ensemble(memory_budget=2 * per_job + 100) as ens:
        ids = [ens.add(j) for j in jobs]
        states = [ens.status(i)[0] for i in ids]
        assert states.count("pending") == 6
        ens.run()
        for jid, job in zip(ids, jobs, strict=True):
            res = ens.result(jid)
            want_series, want_lat = solo(job, oracle_mod)
            np.testing.assert_array_equal(res.series, want_series)
            np.testing.assert_array_equal(res.lattice, want_lat)


def test_ensemble_rejects_job_over_budget():
    from pyising_b200.ensemble import Ensemble, Job

    with Ensemble(memory_budget=1000) as ens:
        with pytest.raises(MemoryError):
            ens.add(Job((64, 64), 0.4, 5))


def test_ensemble_golden_c4_members():
    """The seeded 96-lattice draw's small members (L <= 128), against the reference's runs."""
    from pyising_b200.ensemble import Ensemble, Job

    g = golden("c4_batch.npz")
    with Ensemble(memory_budget=1 << 30) as ens:
        ids = {}
        for i in g["picked"]:
            i = int(i)
            L = 2 ** int(g["ks"][i])
            ids[i] = ens.add(Job((L, L), 1.0 / float(g["Ts"][i]), 500, seed=i, measure_every=10,
                                 keep_lattice=True))
        ens.run()
        for i, jid in ids.items():
            L = 2 ** int(g["ks"][i])
            res = ens.result(jid)
            np.testing.assert_array_equal(res.series, g[f"series{i}"])
            np.testing.assert_array_equal(res.lattice, unpack_lattice(g[f"final{i}"], (L, L)))


def test_server_mixed_arrivals_equal_solo_runs(oracle_mod):
    """Jobs arrive from two threads while others run; each result equals its solo run."""
    from pyising_b200.ensemble import Server

    jobs = mixed_jobs()
    ids: dict[int, object] = {}
    lock = threading.Lock()
    with Server(memory_budget=1 << 28) as srv:
        def feeder(part):
            for j in part:
                jid = srv.submit(j)
                with lock:
                    ids[jid] = j
                time.sleep(0.002)

        threads = [threading.Thread(target=feeder, args=(jobs[k::2],)) for k in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for jid, job in ids.items():
            assert srv.wait(jid, timeout=120) == "done"
            res = srv.result(jid)
            assert res.latency_s is not None and res.latency_s >= 0
            want_series, want_lat = solo(job, oracle_mod)
            np.testing.assert_array_equal(res.series, want_series, err_msg=str(job))
            np.testing.assert_array_equal(res.lattice, want_lat, err_msg=str(job))
            srv.release(jid)
        st = srv.status()
        assert st["active"] == 0 and st["pending"] == 0


def test_server_job_alone_and_in_the_mix_agree():
    """The same job through the server alone and while a large mix runs."""
    from pyising_b200.ensemble import Job, Server

    probe = Job((256, 256), BETA_C_2D, 200, seed=42, measure_every=10, keep_lattice=True,
                init="philox")
    with Server(memory_budget=1 << 30) as srv:
        a = srv.submit(probe)
        srv.wait(a)
        alone = srv.result(a)
        filler = [srv.submit(Job((512, 512), 0.4 + 0.001 * k, 300, seed=k, init="philox",
                                 variant="msc" if k % 2 else "int8")) for k in range(8)]
        b = srv.submit(probe)
        srv.wait(b)
        mixed = srv.result(b)
        for f in filler:
            srv.wait(f)
    np.testing.assert_array_equal(alone.series, mixed.series)
    np.testing.assert_array_equal(alone.lattice, mixed.lattice)


def test_run_sharded_single_process_uses_the_batch(oracle_mod):
    """World size 1: the default runner is the batched engine on this GPU."""
    from pyising_b200.distributed import run_sharded

    jobs = mixed_jobs()[:6]
    res = run_sharded(jobs)
    for r, job in zip(res, jobs, strict=True):
        want_series, want_lat = solo(job, oracle_mod)
        np.testing.assert_array_equal(r.series, want_series)
        np.testing.assert_array_equal(r.lattice, want_lat)
