"""Sweep schedules (per-half-sweep launches, replayed graphs, one persistent cooperative launch)
give identical results, and the persistent schedule's bounded waits turn a stalled band into an
error status instead of a hang.  The stalled band is a host-selected test hook: the band simply
stops publishing its progress, its neighbours' waits expire after ~0.3 s, every CTA returns, and
the host reads the error word; nothing faults and the context stays usable."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
from conftest import golden, unpack_lattice

pytestmark = pytest.mark.gpu

BETA_C_2D = 0.44068679350977147


@pytest.mark.parametrize("shape,algorithm,beta", [
    ((64, 64), "metropolis", BETA_C_2D),
    ((100, 264), "metropolis", 0.41),   # ragged bands, padded rows
    ((6, 32), "heatbath", 0.42),        # fewer rows than SMs
    ((512, 1024), "heatbath", 0.44),
    ((48, 96), "heatbath", -0.3),       # non-monotone table: lookup rule
    ((32, 64), "heatbath", 0.42),       # temporal tiles: Ly = 2 bands + halo
    ((16, 2048), "metropolis", 0.44),   # temporal tiles: Ly = the smallest allowed
])
def test_schedules_match_oracle(oracle_mod, shape, algorithm, beta):
    from pyising_b200.backend import B200Int8

    lat = oracle_mod.random_lattice(shape, 12)
    ref = oracle_mod.OracleInt8(shape, beta, seed=2**40 + 9, algorithm=algorithm, init=lat)
    want = ref.sweep(40, measure_every=5)
    ref.sweep(11)
    for schedule in ("launches", "graphs", "persistent", "temporal", "auto"):
        sim = B200Int8(shape, beta, seed=2**40 + 9, algorithm=algorithm, init=lat)
        sim.set_schedule(schedule)
        np.testing.assert_array_equal(sim.sweep_measured(40, 5), want, err_msg=schedule)
        sim.sweep(11)
        np.testing.assert_array_equal(sim.get_lattice(), ref.get_lattice(), err_msg=schedule)


@pytest.mark.parametrize("shape,algorithm,beta", [
    ((2048, 2048), "metropolis", BETA_C_2D),  # 256 bands: more CTAs than one wave holds
    ((2400, 256), "heatbath", 0.42),
], ids=str)
def test_temporal_tiles_read_and_write_separate_arrays(oracle_mod, shape, algorithm, beta):
    """A temporal launch reads one pair of colour arrays and writes the other (a CTA's halo rows
    are other CTAs' bands, rewritten in the same launch): with more bands than resident CTAs,
    and with odd and even numbers of launches between measurements, the oracle's results."""
    from pyising_b200.backend import B200Int8

    lat = oracle_mod.random_lattice(shape, 8)
    ref = oracle_mod.OracleInt8(shape, beta, seed=2**33 + 1, algorithm=algorithm, init=lat)
    sim = B200Int8(shape, beta, seed=2**33 + 1, algorithm=algorithm, init=lat)
    sim.set_schedule("temporal")
    for n in (6, 8, 2, 3):  # 3, 4, 1 launches and one launch plus a single sweep
        sim.sweep(n)
        ref.sweep(n)
        np.testing.assert_array_equal(sim.get_lattice(), ref.get_lattice(), err_msg=str(n))
    np.testing.assert_array_equal(sim.sweep_measured(21, 7), ref.sweep(21, measure_every=7))
    np.testing.assert_array_equal(sim.get_lattice(), ref.get_lattice())


def test_temporal_c1_golden():
    """C1 on the temporally blocked schedule (two sweeps per launch between measurements)."""
    from pyising_b200.backend import B200Int8

    g = golden("c1_int8_L1024.npz")
    sim = B200Int8((1024, 1024), float(g["beta"]), seed=1, init="hot")
    sim.set_schedule("temporal")
    np.testing.assert_array_equal(sim.sweep_measured(1000, 100), g["series"])
    np.testing.assert_array_equal(sim.get_lattice(), unpack_lattice(g["final"], (1024, 1024)))
    sim2 = B200Int8((1024, 1024), float(g["beta"]), seed=1, init="hot")
    sim2.set_schedule("temporal")
    sim2.sweep(999)  # odd count: a graph chunk tail and one single sweep
    sim2.sweep(1)
    np.testing.assert_array_equal(sim2.get_lattice(), unpack_lattice(g["final"], (1024, 1024)))


def test_persistent_c1_golden():
    """C1 (1024^2 int8 Metropolis, beta_c, seed 1, hot, 1000 sweeps) on the persistent path."""
    from pyising_b200.backend import B200Int8

    g = golden("c1_int8_L1024.npz")
    sim = B200Int8((1024, 1024), float(g["beta"]), seed=1, init="hot")
    sim.set_schedule("persistent")
    np.testing.assert_array_equal(sim.sweep_measured(1000, 100), g["series"])
    np.testing.assert_array_equal(sim.get_lattice(), unpack_lattice(g["final"], (1024, 1024)))


def test_bounded_wait_selftest():
    from pyising_b200._lib import check, lib

    flag = ctypes.c_int(0)
    check(lib().ising_selftest_bounded_wait(0, ctypes.byref(flag)), "selftest")
    assert flag.value == 1


def test_stalled_band_reports_timeout_and_context_survives(oracle_mod):
    from pyising_b200._lib import DeviceTimeout
    from pyising_b200.backend import B200Int8

    shape = (128, 128)
    lat = oracle_mod.random_lattice(shape, 4)
    sim = B200Int8(shape, 0.4, seed=5, init=lat)
    sim.set_schedule("persistent", test_mute_band=1)
    sim.sweep(20)
    with pytest.raises(DeviceTimeout):
        sim.synchronize()
    # the same handle and context keep working
    sim.set_schedule("persistent")
    sim.set_lattice(lat)
    sim.t = 0
    sim.sweep(20)
    ref = oracle_mod.OracleInt8(shape, 0.4, seed=5, init=lat)
    ref.sweep(20)
    np.testing.assert_array_equal(sim.get_lattice(), ref.get_lattice())
