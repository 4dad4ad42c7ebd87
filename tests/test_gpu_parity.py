"""Parity of the CUDA path with the oracle: bit-identical spins, exact integer observables.

Every simulation here runs through the C ABI of libising_b200.so (pyising_b200.backend) and is
compared with the CPU oracle (oracle/) on the same seeded inputs and with the golden fixtures
the pyising reference produced (tests/golden).  Cases follow the reference's own tests
(tests/test_backends.py:22-80, tests/test_lattice.py:75-99) plus the layout and rule edge
cases of this implementation (chunk widths 4/8/16, 3D, non-monotone tables, 64-bit seeds,
sweep counters that wrap at 2^32).
"""

from __future__ import annotations

import numpy as np
import pytest
from conftest import golden, unpack_lattice
from test_oracle_golden import int8_cases, msc_cases

pytestmark = pytest.mark.gpu

BETA_C_2D = 0.44068679350977147


@pytest.fixture(scope="module")
def B():
    from pyising_b200 import backend

    return backend


# ------------------------------------------------------------------- generator ------------
def test_device_philox_known_answers(oracle_mod):
    from pyising_b200._lib import philox_range

    g = golden("philox.npz")
    for ctr, key, exp in zip(g["kat_ctr"], g["kat_key"], g["kat_out"], strict=True):
        out = philox_range(int(ctr[0]), 1, int(ctr[1]), int(ctr[2]), int(ctr[3]), int(key[0]),
                           int(key[1]))
        assert tuple(int(x) for x in out[0]) == tuple(int(x) for x in exp)
    out = philox_range(0xFFFFFF00, 4096, 77, 1, 5, 0xDEADBEEF, 0x12345678)
    ref = oracle_mod.philox_range(0xFFFFFF00, 4096, 77, 1, 5, 0xDEADBEEF, 0x12345678)
    np.testing.assert_array_equal(out, ref)


# ---------------------------------------------------------------- golden cases ------------
@pytest.mark.parametrize("case", int8_cases(), ids=lambda c: f"{c['shape']}-{c['algorithm']}")
def test_int8_identity_golden(B, oracle_mod, case):
    lat = oracle_mod.random_lattice(case["shape"], case["init_seed"])
    sim = B.B200Int8(case["shape"], case["beta"], seed=case["seed"],
                     algorithm=case["algorithm"], init=lat)
    sim.sweep(case["sweeps"])
    got = sim.get_lattice()
    np.testing.assert_array_equal(got, case["final"])
    M, E = oracle_mod.energy_magnetization(case["final"])
    assert sim.observables_int() == (M, E)
    m, e = sim.observables()
    assert m == pytest.approx(M / got.size) and e == pytest.approx(E / got.size)


@pytest.mark.parametrize("case", msc_cases(), ids=lambda c: f"{c['shape']}")
def test_msc_identity_golden(B, oracle_mod, case):
    lat = oracle_mod.random_lattice(case["shape"], case["init_seed"])
    sim = B.B200MultiSpin(case["shape"], case["beta"], seed=case["seed"], init=lat)
    sim.sweep(case["sweeps"])
    np.testing.assert_array_equal(sim.get_lattice(), case["final"])
    assert sim.observables_int() == oracle_mod.energy_magnetization(case["final"])


@pytest.mark.parametrize("variant", ["int8", "msc"])
def test_set_beta_and_split_sweeps(B, variant):
    cls = B.B200Int8 if variant == "int8" else B.B200MultiSpin
    g = golden(f"{variant}_cases.npz")
    from pyising_b200.lattice import random_lattice

    lat = random_lattice((128, 128), 1)
    a = cls((128, 128), 0.3, seed=3, init=lat)
    b = cls((128, 128), 0.3, seed=3, init=lat)
    a.sweep(2)
    a.set_beta(0.5)
    a.sweep(3)
    b.sweep(2)
    b.set_beta(0.5)
    b.sweep(1)
    b.sweep(2)
    np.testing.assert_array_equal(a.get_lattice(), b.get_lattice())
    np.testing.assert_array_equal(a.get_lattice(), unpack_lattice(g["set_beta_final"], (128, 128)))


@pytest.mark.parametrize("variant", ["int8", "msc"])
def test_hot_and_cold_starts(B, oracle_mod, variant):
    cls = B.B200Int8 if variant == "int8" else B.B200MultiSpin
    shape = (128, 128)
    cold = cls(shape, 0.5, init="cold")
    assert cold.observables() == pytest.approx((1.0, -2.0))
    np.testing.assert_array_equal(cold.get_lattice(), np.ones(shape, np.int8))
    hot = cls(shape, 0.5, seed=17, init="hot")
    m, e = hot.observables()
    assert abs(m) < 0.05 and abs(e) < 0.05
    # the hot start is pyising's NumPy one, so it is bit-identical to the oracle's
    np.testing.assert_array_equal(hot.get_lattice(), oracle_mod.random_lattice(shape, 17))


# ------------------------------------------------------------------ random cases ----------
INT8_SHAPES = [(16, 24), (8, 8, 16), (64, 32), (6, 8), (4, 6, 8), (2, 8), (10, 40), (32, 96),
               (12, 10, 24), (128, 256), (16, 16, 64), (40, 1032)]


@pytest.mark.parametrize("shape", INT8_SHAPES, ids=str)
@pytest.mark.parametrize("algorithm", ["metropolis", "heatbath"])
def test_int8_random_vs_oracle(B, oracle_mod, shape, algorithm):
    beta = 0.44 if len(shape) == 2 else 0.23
    seed = (2**63 + 12345) if algorithm == "heatbath" else 2**40 + 99
    lat = oracle_mod.random_lattice(shape, 11)
    sim = B.B200Int8(shape, beta, seed=seed, algorithm=algorithm, init=lat)
    ref = oracle_mod.OracleInt8(shape, beta, seed=seed, algorithm=algorithm, init=lat)
    sim.sweep(3)
    ref.sweep(3)
    series = sim.sweep_measured(6, 2)
    want = ref.sweep(6, measure_every=2)
    np.testing.assert_array_equal(series, want)
    np.testing.assert_array_equal(sim.get_lattice(), ref.get_lattice())
    assert sim.observables_int() == ref.observables_int()


@pytest.mark.parametrize("shape", [(128, 128), (64, 384), (2, 128), (6, 256), (130, 1152),
                                   (256, 4096)], ids=str)
@pytest.mark.parametrize("beta", [0.0, 0.2, BETA_C_2D, 1.5])
def test_msc_random_vs_oracle(B, oracle_mod, shape, beta):
    lat = oracle_mod.random_lattice(shape, 3)
    sim = B.B200MultiSpin(shape, beta, seed=2**33 + 5, init=lat)
    ref = oracle_mod.OracleMultiSpin(shape, beta, seed=2**33 + 5, init=lat)
    sim.sweep(2)
    ref.sweep(2)
    series = sim.sweep_measured(4, 2)
    want = ref.sweep(4, measure_every=2)
    np.testing.assert_array_equal(series, want)
    np.testing.assert_array_equal(sim.get_lattice(), ref.get_lattice())


def test_msc_equals_int8_at_beta_zero(B, oracle_mod):
    """tests/test_lattice.py:91-99 of the reference: at beta = 0 every spin flips."""
    lat = oracle_mod.random_lattice((16, 128), 4)
    a = B.B200MultiSpin((16, 128), 0.0, seed=5, init=lat)
    b = B.B200Int8((16, 128), 0.0, seed=5, init=lat)
    a.sweep(1)
    b.sweep(1)
    np.testing.assert_array_equal(a.get_lattice(), b.get_lattice())
    np.testing.assert_array_equal(a.get_lattice(), -lat)


@pytest.mark.parametrize("algorithm,beta", [("heatbath", -0.3), ("metropolis", -0.3)])
def test_negative_beta_tables(B, oracle_mod, algorithm, beta):
    """Antiferromagnetic tables: heat bath becomes non-monotone (generic rule)."""
    shape = (16, 32)
    lat = oracle_mod.random_lattice(shape, 8)
    sim = B.B200Int8(shape, beta, seed=9, algorithm=algorithm, init=lat)
    ref = oracle_mod.OracleInt8(shape, beta, seed=9, algorithm=algorithm, init=lat)
    sim.sweep(4)
    ref.sweep(4)
    np.testing.assert_array_equal(sim.get_lattice(), ref.get_lattice())


@pytest.mark.parametrize("shape", [(16, 32), (8, 8, 16)], ids=str)
@pytest.mark.parametrize("algorithm", ["metropolis", "heatbath"])
def test_arbitrary_tables_use_generic_rule(B, oracle_mod, shape, algorithm):
    """A custom non-monotone table (through the table hook) still matches the oracle."""
    lat = oracle_mod.random_lattice(shape, 2)
    n = 2 * len(shape) + 1
    table = np.array([(0x9E3779B9 * (i + 3)) & 0xFFFFFFFF for i in range(n)], np.uint32)
    sim = B.B200Int8(shape, 0.3, seed=4, algorithm=algorithm, init=lat)
    ref = oracle_mod.OracleInt8(shape, 0.3, seed=4, algorithm=algorithm, init=lat)
    sim.table = table
    sim._upload_table()
    ref.table = table.copy()
    sim.sweep(3)
    ref.sweep(3)
    np.testing.assert_array_equal(sim.get_lattice(), ref.get_lattice())


def test_sweep_counter_wraps_at_2_32(B, oracle_mod):
    """Philox counter word 1 is the sweep counter truncated to 32 bits (philox.py:37)."""
    shape = (32, 64)
    lat = oracle_mod.random_lattice(shape, 1)
    for cls, ocls in ((B.B200Int8, oracle_mod.OracleInt8),
                      (B.B200MultiSpin, None)):
        if ocls is None:
            shape2 = (32, 128)
            lat2 = oracle_mod.random_lattice(shape2, 1)
            sim = cls(shape2, 0.4, seed=1, init=lat2)
            ref = oracle_mod.OracleMultiSpin(shape2, 0.4, seed=1, init=lat2)
        else:
            sim = cls(shape, 0.4, seed=1, init=lat)
            ref = ocls(shape, 0.4, seed=1, init=lat)
        sim.t = ref.t = 2**32 - 2
        sim.sweep(4)
        ref.sweep(4)
        np.testing.assert_array_equal(sim.get_lattice(), ref.get_lattice())


def test_half_sweep_hook_matches_sweep(B, oracle_mod):
    shape = (8, 8, 16)
    lat = oracle_mod.random_lattice(shape, 6)
    a = B.B200Int8(shape, 0.25, seed=2, init=lat)
    b = B.B200Int8(shape, 0.25, seed=2, init=lat)
    a.sweep(3)
    from pyising_b200.base import IsingSimulation

    IsingSimulation.sweep(b, 3)  # the ABC's Python loop over the _half_sweep hook
    assert a.t == b.t == 3
    np.testing.assert_array_equal(a.get_lattice(), b.get_lattice())


def test_layout_transfers_match_oracle(B, oracle_mod):
    for shape in [(16, 24), (8, 8, 16), (6, 10, 8)]:
        lat = oracle_mod.random_lattice(shape, 5)
        sim = B.B200Int8(shape, 0.3, init=lat)
        c0, c1 = sim.colour_arrays()
        r0, r1 = oracle_mod.to_compressed(lat)
        np.testing.assert_array_equal(c0, r0)
        np.testing.assert_array_equal(c1, r1)
        np.testing.assert_array_equal(sim.get_lattice(), lat)
    for shape in [(16, 128), (6, 384)]:
        lat = oracle_mod.random_lattice(shape, 5)
        sim = B.B200MultiSpin(shape, 0.3, init=lat)
        w0, w1 = sim.colour_arrays()
        r0, r1 = oracle_mod.to_compressed(lat)
        np.testing.assert_array_equal(w0, oracle_mod.pack_bits(r0))
        np.testing.assert_array_equal(w1, oracle_mod.pack_bits(r1))
        np.testing.assert_array_equal(sim.get_lattice(), lat)


def test_checkpoint_resume_is_bit_exact(B, oracle_mod):
    shape = (64, 256)
    for cls in (B.B200Int8, B.B200MultiSpin):
        lat = oracle_mod.random_lattice(shape, 7)
        a = cls(shape, 0.41, seed=5, init=lat)
        a.sweep(3)
        st = a.state()
        a.sweep(4)
        b = cls.from_state(st)
        b.sweep(4)
        assert a.t == b.t == 7
        np.testing.assert_array_equal(a.get_lattice(), b.get_lattice())


def test_colour_arrays_into_caller_buffers(B, oracle_mod):
    shape = (24, 1032)  # int8 rows padded on the device: host rows stay 516 bytes
    for cls, sh in ((B.B200Int8, shape), (B.B200MultiSpin, (32, 256))):
        lat = oracle_mod.random_lattice(sh, 9)
        sim = cls(sh, 0.4, seed=3, init=lat)
        sim.sweep(5)
        want = sim.colour_arrays()
        out = (np.empty_like(want[0]), np.empty_like(want[1]))
        got = sim.colour_arrays(out)
        assert got[0] is out[0] and got[1] is out[1]
        np.testing.assert_array_equal(out[0], want[0])
        np.testing.assert_array_equal(out[1], want[1])
        with pytest.raises(ValueError):
            sim.colour_arrays((out[0][:, :-1].copy(), out[1]))
        # in-place upload of contiguous arrays, and of strided ones (copied)
        sim.load_colour_arrays(out[0], out[1])
        np.testing.assert_array_equal(sim.colour_arrays()[0], want[0])
        wide = np.zeros((want[1].shape[0], 2 * want[1].shape[1]), want[1].dtype)
        wide[:, ::2] = want[1]
        sim.load_colour_arrays(want[0], wide[:, ::2])
        np.testing.assert_array_equal(sim.colour_arrays()[1], want[1])


def test_msc_calls_per_word_diagnostic(B, oracle_mod):
    shape = (256, 1024)
    lat = oracle_mod.random_lattice(shape, 1)
    sim = B.B200MultiSpin(shape, BETA_C_2D, seed=1, init=lat)
    ref = oracle_mod.OracleMultiSpin(shape, BETA_C_2D, seed=1, init=lat)
    mean = sim.philox_calls_per_word(2)
    ref.sweep(2)
    assert mean == pytest.approx(ref.calls / (4 * 256 * 8))
    assert sim.philox_calls_per_word(1, warp=True) >= mean * 0.9
    ref.sweep(1)  # the diagnostic advances the lattice like sweep()
    np.testing.assert_array_equal(sim.get_lattice(), ref.get_lattice())


# ------------------------------------------------------------- config parity ---------------
def test_c1_int8_L1024_1000_sweeps(B, oracle_mod):
    """C1: 1024^2 int8 Metropolis, beta_c, seed 1, NumPy hot start, 1000 sweeps."""
    g = golden("c1_int8_L1024.npz")
    shape = (1024, 1024)
    sim = B.B200Int8(shape, float(g["beta"]), seed=1, init="hot")
    series = sim.sweep_measured(1000, 100)
    np.testing.assert_array_equal(series, g["series"])
    np.testing.assert_array_equal(sim.get_lattice(), unpack_lattice(g["final"], shape))


@pytest.mark.parametrize("L", [1024, 2048])
def test_c2_msc_parity_shapes(B, L):
    g = golden("c2_msc.npz")
    shape = (L, L)
    sim = B.B200MultiSpin(shape, float(g["beta"]), seed=7, init="hot")
    sim.sweep(int(g[f"sweeps{L}"]))
    assert sim.observables_int() == tuple(int(x) for x in g[f"me{L}"])
    np.testing.assert_array_equal(sim.get_lattice(), unpack_lattice(g[f"final{L}"], shape))


def test_c3_int8_3d_L64_heatbath(B):
    g = golden("c3_int8_3d_L64.npz")
    shape = (64, 64, 64)
    sim = B.B200Int8(shape, float(g["beta"]), seed=0, algorithm="heatbath", init="cold")
    series = sim.sweep_measured(2000, 10)
    np.testing.assert_array_equal(series, g["series"])
    np.testing.assert_array_equal(sim.get_lattice(), unpack_lattice(g["final"], shape))


def test_c2_full_size_properties(B, oracle_mod):
    """msc L=16384 (the bench workload): the fused series equals the standalone reduction,
    split sweeps equal one call, and a sampled row band matches the oracle run on the same
    full lattice for one sweep."""
    shape = (16384, 16384)
    a = B.B200MultiSpin(shape, BETA_C_2D, seed=7, init="hot")
    st = a.state()
    series = a.sweep_measured(4, 2)
    assert tuple(series[-1]) == a.observables_int()
    b = B.B200MultiSpin.from_state(st)
    b.sweep(1)
    b.sweep(3)
    assert b.observables_int() == a.observables_int()
    wa, wb = a.colour_arrays(), b.colour_arrays()
    np.testing.assert_array_equal(wa[0], wb[0])
    np.testing.assert_array_equal(wa[1], wb[1])
    # one sweep of the full lattice on the oracle (multi-threaded C), compared word for word
    c = B.B200MultiSpin.from_state(st)
    c.sweep(1)
    ref = oracle_mod.OracleMultiSpin(shape, BETA_C_2D, seed=7, init="cold")
    ref.w = [np.ascontiguousarray(st["c0"]), np.ascontiguousarray(st["c1"])]
    ref.sweep(1)
    w0, w1 = c.colour_arrays()
    np.testing.assert_array_equal(w0, ref.w[0])
    np.testing.assert_array_equal(w1, ref.w[1])


@pytest.mark.parametrize("variant", ["int8", "msc"])
def test_handles_reusing_pooled_memory_start_clean(B, variant):
    """Handles take their arrays from a pool that keeps freed memory: a handle created on memory
    another handle left (other spins, other measurements) gives exactly the results of the first
    handle of that configuration."""
    cls = B.B200Int8 if variant == "int8" else B.B200MultiSpin
    shape = (256, 256)

    def run(seed, every):
        sim = cls(shape, 0.44, seed=seed, init="hot")
        series = sim.sweep_measured(40, every)
        out = (series, sim.get_lattice(), sim.observables_int())
        del sim
        return out

    first = run(5, 4)
    for other in range(3):  # dirty the pooled memory with other lattices and series
        run(100 + other, 1 + other)
    again = run(5, 4)
    np.testing.assert_array_equal(first[0], again[0])
    np.testing.assert_array_equal(first[1], again[1])
    assert first[2] == again[2]
