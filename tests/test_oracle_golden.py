"""Pin the CPU oracle to the reference: every golden vector in tests/golden was produced by the
pyising reference itself (tests/golden/make_golden.py).  CPU only."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import golden, unpack_lattice

BETA_C_2D = 0.44068679350977147


def int8_cases():
    g = golden("int8_cases.npz")
    out = []
    for i in range(int(g["n_cases"])):
        c = g[f"case{i}"]
        ndim = int(c[0])
        shape = tuple(int(x) for x in c[1:1 + ndim])
        beta, seed, sweeps, init_seed, alg = g[f"meta{i}"]
        out.append(dict(shape=shape, beta=float(beta), seed=int(seed), sweeps=int(sweeps),
                        init_seed=int(init_seed),
                        algorithm="metropolis" if alg == 0 else "heatbath",
                        final=unpack_lattice(g[f"final{i}"], shape)))
    return out


def msc_cases():
    g = golden("msc_cases.npz")
    out = []
    for i in range(int(g["n_cases"])):
        shape = tuple(int(x) for x in g[f"case{i}"])
        beta, seed, sweeps, init_seed = g[f"meta{i}"]
        out.append(dict(shape=shape, beta=float(beta), seed=int(seed), sweeps=int(sweeps),
                        init_seed=int(init_seed), final=unpack_lattice(g[f"final{i}"], shape)))
    return out


def test_philox_known_answers(oracle_mod):
    g = golden("philox.npz")
    assert len(g["kat_out"]) == 3
    for ctr, key, exp in zip(g["kat_ctr"], g["kat_key"], g["kat_out"], strict=True):
        assert oracle_mod.philox4x32(ctr, key) == tuple(int(x) for x in exp)
    for ctr, key, exp in zip(g["rnd_ctr"], g["rnd_key"], g["rnd_out"], strict=True):
        assert oracle_mod.philox4x32(ctr, key) == tuple(int(x) for x in exp)


def test_streams(oracle_mod):
    g = golden("streams.npz")
    assert oracle_mod.split_seed(2**40 + 3) == tuple(int(x) for x in g["split_seed"])
    np.testing.assert_array_equal(oracle_mod.site_uniforms(64, 5, 1, 2**40 + 3),
                                  g["site_uniforms"])
    for lp in range(3):
        a, b = oracle_mod.word_randoms(16, 3, 0, 12345, lp)
        np.testing.assert_array_equal(a, g["word_randoms"][lp, 0])
        np.testing.assert_array_equal(b, g["word_randoms"][lp, 1])


def test_threshold_tables(oracle_mod):
    from pyising_b200.lattice import threshold_table

    g = golden("tables.npz")
    for (beta, ndim, alg), exp in zip(g["cases"], g["tables"], strict=True):
        ndim = int(ndim)
        name = "metropolis" if alg == 0 else "heatbath"
        want = exp[: 2 * ndim + 1].astype(np.uint32)
        np.testing.assert_array_equal(oracle_mod.threshold_table(beta, ndim, name), want)
        np.testing.assert_array_equal(oracle_mod.threshold_table_py(beta, ndim, name), want)
        # the product's host table (pyising_b200.lattice) is pinned by the same vectors
        np.testing.assert_array_equal(threshold_table(beta, ndim, name), want)


@pytest.fixture(params=["plain", "avx512"])
def int8_path(request, oracle_mod):
    """Both int8 half-sweeps of the oracle: the plain restatement and its AVX-512 variant (where
    the host has AVX-512), each pinned to the same golden vectors."""
    if request.param == "avx512":
        oracle_mod.set_fast(True)
        if not oracle_mod.fast_active():
            pytest.skip("no AVX-512 on this host")
    else:
        oracle_mod.set_fast(False)
    yield request.param
    oracle_mod.set_fast(True)


@pytest.mark.parametrize("case", int8_cases(), ids=lambda c: f"{c['shape']}-{c['algorithm']}")
def test_int8_identity_cases(oracle_mod, int8_path, case):
    lat = oracle_mod.random_lattice(case["shape"], case["init_seed"])
    sim = oracle_mod.OracleInt8(case["shape"], case["beta"], seed=case["seed"],
                                algorithm=case["algorithm"], init=lat)
    sim.sweep(case["sweeps"])
    np.testing.assert_array_equal(sim.get_lattice(), case["final"])


def test_int8_set_beta_split(oracle_mod, int8_path):
    g = golden("int8_cases.npz")
    lat = oracle_mod.random_lattice((128, 128), 1)
    a = oracle_mod.OracleInt8((128, 128), 0.3, seed=3, init=lat)
    a.sweep(2)
    a.set_beta(0.5)
    a.sweep(1)
    a.sweep(2)
    np.testing.assert_array_equal(a.get_lattice(), unpack_lattice(g["set_beta_final"], (128, 128)))


@pytest.mark.parametrize("case", msc_cases(), ids=lambda c: f"{c['shape']}")
def test_msc_identity_cases(oracle_mod, case):
    lat = oracle_mod.random_lattice(case["shape"], case["init_seed"])
    sim = oracle_mod.OracleMultiSpin(case["shape"], case["beta"], seed=case["seed"], init=lat)
    sim.sweep(case["sweeps"])
    np.testing.assert_array_equal(sim.get_lattice(), case["final"])


def test_msc_set_beta_split(oracle_mod):
    g = golden("msc_cases.npz")
    lat = oracle_mod.random_lattice((128, 128), 1)
    a = oracle_mod.OracleMultiSpin((128, 128), 0.3, seed=3, init=lat)
    a.sweep(2)
    a.set_beta(0.5)
    a.sweep(3)
    np.testing.assert_array_equal(a.get_lattice(), unpack_lattice(g["set_beta_final"], (128, 128)))


def test_layout_roundtrips(oracle_mod):
    for shape in [(8, 16), (6, 8), (4, 6, 8), (16, 256)]:
        lat = oracle_mod.random_lattice(shape, 1)
        c0, c1 = oracle_mod.to_compressed(lat)
        np.testing.assert_array_equal(oracle_mod.from_compressed(c0, c1, shape), lat)
        if c0.shape[1] % 64 == 0:
            np.testing.assert_array_equal(oracle_mod.unpack_bits(oracle_mod.pack_bits(c0)), c0)


def test_observables_definitions(oracle_mod):
    for shape in [(16, 24), (8, 8, 16), (32, 256)]:
        lat = oracle_mod.random_lattice(shape, 3)
        sim = oracle_mod.OracleInt8(shape, 0.4, init=lat)
        assert sim.observables_int() == oracle_mod.energy_magnetization(lat)
        if len(shape) == 2 and shape[1] % 128 == 0:
            msc = oracle_mod.OracleMultiSpin(shape, 0.4, init=lat)
            assert msc.observables_int() == oracle_mod.energy_magnetization(lat)
    cold = oracle_mod.OracleMultiSpin((16, 128), 0.5, init="cold")
    assert cold.observables() == (1.0, -2.0)


def test_c1_int8_L1024(oracle_mod, int8_path):
    """1024^2 int8 Metropolis at beta_c, seed 1, hot start, 1000 sweeps (the reference: 33 s)."""
    g = golden("c1_int8_L1024.npz")
    shape = (1024, 1024)
    sim = oracle_mod.OracleInt8(shape, float(g["beta"]), seed=1,
                                init=oracle_mod.random_lattice(shape, 1))
    for k in range(10):
        sim.sweep(100)
        assert sim.observables_int() == tuple(int(x) for x in g["series"][k])
    np.testing.assert_array_equal(sim.get_lattice(), unpack_lattice(g["final"], shape))


@pytest.mark.parametrize("L", [1024, 2048])
def test_c2_msc(oracle_mod, L):
    g = golden("c2_msc.npz")
    shape = (L, L)
    sim = oracle_mod.OracleMultiSpin(shape, float(g["beta"]), seed=7,
                                     init=oracle_mod.random_lattice(shape, 7))
    sim.sweep(int(g[f"sweeps{L}"]))
    assert sim.observables_int() == tuple(int(x) for x in g[f"me{L}"])
    np.testing.assert_array_equal(sim.get_lattice(), unpack_lattice(g[f"final{L}"], shape))


def test_c3_int8_3d_L64(oracle_mod, int8_path):
    g = golden("c3_int8_3d_L64.npz")
    shape = (64, 64, 64)
    sim = oracle_mod.OracleInt8(shape, float(g["beta"]), seed=0, algorithm="heatbath",
                                init="cold")
    series = sim.sweep(2000, measure_every=10)
    np.testing.assert_array_equal(series, g["series"])
    np.testing.assert_array_equal(sim.get_lattice(), unpack_lattice(g["final"], shape))


def test_c4_ensemble_members(oracle_mod, int8_path):
    g = golden("c4_batch.npz")
    for i in g["picked"]:
        i = int(i)
        L = 2 ** int(g["ks"][i])
        sim = oracle_mod.OracleInt8((L, L), 1.0 / float(g["Ts"][i]), seed=i,
                                    init=oracle_mod.random_lattice((L, L), i))
        series = sim.sweep(500, measure_every=10)
        np.testing.assert_array_equal(series, g[f"series{i}"])
        np.testing.assert_array_equal(sim.get_lattice(), unpack_lattice(g[f"final{i}"], (L, L)))


def test_avx512_half_sweep_equals_the_plain_one(oracle_mod):
    """Random shapes (rows whose length is not a multiple of 4 sites or of 64, 3D, tiny), both
    rules, negative beta: the two int8 paths give the same spins and series."""
    if not oracle_mod.fast_active():
        pytest.skip("no AVX-512 on this host")
    rng = np.random.default_rng(11)
    cases = [((6, 10), "metropolis", 0.3), ((34, 258), "metropolis", -0.3),
             ((128, 250), "heatbath", -0.2), ((10, 6, 22), "heatbath", 0.25),
             ((12, 14, 18), "metropolis", 0.22), ((2, 2), "metropolis", 1.0)]
    cases += [((2 * int(rng.integers(1, 40)), 2 * int(rng.integers(1, 90))),
               ["metropolis", "heatbath"][i % 2], float(rng.uniform(-0.5, 0.9)))
              for i in range(10)]
    try:
        for shape, alg, beta in cases:
            lat = oracle_mod.random_lattice(shape, 5)
            out = []
            for fast in (False, True):
                oracle_mod.set_fast(fast)
                sim = oracle_mod.OracleInt8(shape, beta, seed=2**40 + 9, algorithm=alg, init=lat)
                out.append((sim.sweep(9, measure_every=3), sim.get_lattice()))
            np.testing.assert_array_equal(out[0][0], out[1][0], err_msg=str(shape))
            np.testing.assert_array_equal(out[0][1], out[1][1], err_msg=str(shape))
    finally:
        oracle_mod.set_fast(True)


def test_beta_c_constant():
    from pyising_b200.lattice import BETA_C_2D as b

    g = golden("c1_int8_L1024.npz")
    assert b == float(g["beta"]) == BETA_C_2D
