"""The benched configurations at their full sizes against the oracle, word for word.

The reference checks its backends by running the same seeded job on two implementations and
comparing the spins exactly (tests/test_backends.py:22-51, src/pyising/validate.py:69-93).  The
jobs here are the ones bench.py times, unchanged, through the product API (single-lattice
handles, and the batched engine for the ensemble); the oracle runs the same jobs on every host
thread.  All results are integers, so every comparison is exact.

* msc 2D Metropolis 16384^2 at T_c, seed 7, hot start, 1000 sweeps (the headline): final colour
  arrays and (M, E); plus the series every 100 sweeps.
* int8 3D heat bath 256^3, beta 0.221654626, cold start, 2000 sweeps with (M, E) every 10: the
  200-point series and the final lattice.
* int8 2D at 16384^2 (Metropolis), 8192^2 (heat bath) and 4096 x 4104 (rows padded to 16
  bytes): the (M, E) series every 10 sweeps and the final colour arrays.
* The 96-lattice ensemble (L = 2^k, k ~ U{6..12}, T ~ U[2.0, 2.6], seed = index, hot starts,
  5000 sweeps, (M, E) every 10) through the batched engine: every member's 500-point series
  and final lattice (the oracle's vectorised int8 half-sweep keeps its 1.4e12 updates to
  about two minutes on 16 host threads).
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BETA_C_2D = 0.44068679350977147
BETA_3D = 0.221654626


def test_headline_msc_16384_1000_sweeps(oracle_mod):
    from pyising_b200.backend import B200MultiSpin

    shape = (16384, 16384)
    sim = B200MultiSpin(shape, BETA_C_2D, seed=7, init="hot")
    st = sim.state()
    series = sim.sweep_measured(1000, 100)
    ref = oracle_mod.OracleMultiSpin(shape, BETA_C_2D, seed=7, init="cold")
    # copies: the oracle sweeps its arrays in place, and the unmeasured run below starts from st
    ref.w = [np.array(st["c0"], copy=True), np.array(st["c1"], copy=True)]
    ref_series = ref.sweep(1000, measure_every=100)
    np.testing.assert_array_equal(series, ref_series)
    w0, w1 = sim.colour_arrays()
    np.testing.assert_array_equal(w0, ref.w[0])
    np.testing.assert_array_equal(w1, ref.w[1])
    assert sim.observables_int() == ref.observables_int()
    # the unmeasured sweep loop (the bench step) gives the same lattice
    plain = B200MultiSpin.from_state(st)
    plain.sweep(1000)
    p0, p1 = plain.colour_arrays()
    np.testing.assert_array_equal(p0, ref.w[0])
    np.testing.assert_array_equal(p1, ref.w[1])


def test_int8_3d_256_heatbath_2000_sweeps(oracle_mod):
    from pyising_b200.backend import B200Int8

    shape = (256, 256, 256)
    sim = B200Int8(shape, BETA_3D, seed=0, algorithm="heatbath", init="cold")
    series = sim.sweep_measured(2000, 10)
    ref = oracle_mod.OracleInt8(shape, BETA_3D, seed=0, algorithm="heatbath", init="cold")
    ref_series = ref.sweep(2000, measure_every=10)
    assert series.shape == (200, 2)
    np.testing.assert_array_equal(series, ref_series)
    c0, c1 = sim.colour_arrays()
    np.testing.assert_array_equal(c0, ref.c[0])
    np.testing.assert_array_equal(c1, ref.c[1])


def _run_batched(jobs):
    from pyising_b200.ensemble import Ensemble

    with Ensemble() as ens:
        ids = [ens.add(j) for j in jobs]
        ens.run()
        return [ens.result(i) for i in ids]


def test_ensemble_of_96_lattices_against_the_oracle(oracle_mod):
    import dataclasses

    from bench import c4_jobs

    jobs = [dataclasses.replace(j, keep_lattice=True) for j in c4_jobs()]
    assert len(jobs) == 96
    for job, res in zip(jobs, _run_batched(jobs), strict=True):
        assert res.series.shape == (500, 2)
        ref = oracle_mod.OracleInt8(job.shape, job.beta, seed=job.seed, init=job.init)
        np.testing.assert_array_equal(res.series, ref.sweep(5000, measure_every=10),
                                      err_msg=f"L={job.shape[0]} seed={job.seed}")
        np.testing.assert_array_equal(res.lattice, ref.get_lattice())


@pytest.mark.parametrize("shape,algorithm,beta,sweeps", [
    ((16384, 16384), "metropolis", BETA_C_2D, 60),   # the band schedule's longest bands
    ((8192, 8192), "heatbath", 0.42, 60),
    ((4096, 4104), "metropolis", 0.4, 100),          # rows padded to 16 bytes (2052 sites)
], ids=str)
def test_int8_2d_large_lattices(oracle_mod, shape, algorithm, beta, sweeps):
    """The plain int8 2D kernels on lattices of the served stream's largest sizes and the
    headline's, hot start, against the oracle: the (M, E) series every 10 sweeps and the final
    colour arrays."""
    from pyising_b200.backend import B200Int8

    lat = oracle_mod.random_lattice(shape, 5)
    sim = B200Int8(shape, beta, seed=2**36 + 11, algorithm=algorithm, init=lat)
    ref = oracle_mod.OracleInt8(shape, beta, seed=2**36 + 11, algorithm=algorithm, init=lat)
    np.testing.assert_array_equal(sim.sweep_measured(sweeps, 10),
                                  ref.sweep(sweeps, measure_every=10))
    c0, c1 = sim.colour_arrays()
    np.testing.assert_array_equal(c0, ref.c[0])
    np.testing.assert_array_equal(c1, ref.c[1])
