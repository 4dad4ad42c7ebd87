"""Every msc schedule (range and strip, each intake depth and register bound) against the
oracle: the same spins, series and observables bit for bit, on lattices whose rows hold 32,
64 or 96 words (strips) and on narrower ones (where the automatic choice is the range
schedule)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KNOB_MSC_KERNEL = 9


# (4800, 4096): bands of 3 rows, so the two-row steps and a final single row both run
@pytest.mark.parametrize("shape", [(64, 4096), (34, 8192), (16, 12288), (128, 1024),
                                   (4800, 4096)], ids=str)
@pytest.mark.parametrize("kernel", [0, 1, 2, 3, 4, 5, 6, 7])
def test_msc_schedules_match_the_oracle(oracle_mod, shape, kernel):
    from pyising_b200._lib import check, lib
    from pyising_b200.backend import B200MultiSpin
    from pyising_b200.lattice import random_lattice

    lat = random_lattice(shape, 3)
    beta = 0.44
    sim = B200MultiSpin(shape, beta, seed=2**35 + 17, init=lat)
    check(lib().ising_set_knob(sim._h, KNOB_MSC_KERNEL, kernel), "set_knob")
    ref = oracle_mod.OracleMultiSpin(shape, beta, seed=2**35 + 17, init=lat)
    np.testing.assert_array_equal(sim.sweep_measured(12, 3), ref.sweep(12, measure_every=3))
    sim.sweep(5)
    ref.sweep(5)
    w0, w1 = sim.colour_arrays()
    np.testing.assert_array_equal(w0, ref.w[0])
    np.testing.assert_array_equal(w1, ref.w[1])
    assert sim.observables_int() == ref.observables_int()


def test_msc_kernel_knob_range():
    from pyising_b200._lib import check, lib
    from pyising_b200.backend import B200MultiSpin

    sim = B200MultiSpin((16, 256), 0.4, init="cold")
    for bad in (-1, 8):
        with pytest.raises(ValueError):
            check(lib().ising_set_knob(sim._h, KNOB_MSC_KERNEL, bad), "set_knob")
