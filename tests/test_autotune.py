"""The autotuner of the launch knobs (pyising_b200.autotune).

Every knob value of the search space must give bit-identical spins and exact observables (the
random numbers depend only on site, sweep and colour), so the GPU test runs each value against
the oracle; the tuner itself must write a cache entry that new simulations of the same shape
pick up.  The cache logic is tested on the CPU.
"""

from __future__ import annotations

import json

import numpy as np
import pytest

from pyising_b200 import autotune


# ------------------------------------------------------------------------- CPU --------------
@pytest.mark.parametrize("variant,shape", [("int8", (64, 64)), ("int8", (16, 16, 40)),
                                           ("int8", (24, 1032)), ("msc", (128, 256)),
                                           ("msc", (64, 4096))])
def test_search_space_starts_at_the_defaults(variant, shape):
    space = autotune.search_space(variant, shape)
    for name, values in space.items():
        assert values[0] == autotune.DEFAULTS[name]
        assert len(set(values)) == len(values)
    if variant == "int8":
        lh = shape[-1] // 2
        assert (8 in space["chunk_width"]) == (lh % 8 == 0)
        assert ("persistent" in space["schedule"]) == (len(shape) == 2)
        assert "msc_waves" not in space
    else:
        assert "band" not in space and "chunk_width" not in space
        assert (7 in space["msc_kernel"]) == (shape[-1] % 4096 == 0)


def test_cache_round_trip(tmp_path):
    path = tmp_path / "tune.json"
    k = autotune.key("NVIDIA B200 sm_100 148 SMs", "int8", "metropolis", (1024, 1024))
    assert k == "NVIDIA B200 sm_100 148 SMs|int8|metropolis|1024x1024"
    assert autotune.lookup(k, path) is None
    cfg = {"band": 4, "chunk_width": 16, "blocks_per_sm": 8, "schedule": "auto",
           "graph_chunk": 32}
    autotune.save_entry(k, {"config": cfg, "flips_per_ns": 1.0}, path)
    assert autotune.lookup(k, path) == cfg
    autotune.save_entry("other", {"config": {"band": 1}}, path)
    data = json.loads(path.read_text())
    assert set(data) == {k, "other"} and data[k]["config"] == cfg
    path.write_text("not json")
    assert autotune.load_cache(tmp_path / "missing.json") == {}


# ------------------------------------------------------------------------- GPU --------------
CASES = [
    ("int8", (64, 256), "metropolis", 0.44),
    ("int8", (24, 1032), "metropolis", 0.44),  # padded rows, chunk width 8 not allowed
    ("int8", (24, 48), "heatbath", 0.42),
    ("int8", (16, 16, 32), "heatbath", 0.22),
    ("msc", (128, 256), "metropolis", 0.44),
    ("msc", (40, 4096), "metropolis", 0.44),  # 32-word rows: the strip schedules too
]


@pytest.mark.gpu
@pytest.mark.parametrize("variant,shape,algorithm,beta", CASES, ids=lambda x: str(x))
def test_every_knob_value_gives_identical_results(oracle_mod, variant, shape, algorithm, beta):
    from pyising_b200.backend import B200Int8, B200MultiSpin

    cls = B200MultiSpin if variant == "msc" else B200Int8
    ocls = oracle_mod.OracleMultiSpin if variant == "msc" else oracle_mod.OracleInt8
    seed = 2**33 + 5
    lat = oracle_mod.random_lattice(shape, 3)
    ref = ocls(shape, beta, seed=seed, algorithm=algorithm, init=lat)
    ref.sweep(70)
    want_series = ref.sweep(20, measure_every=5)
    want = ref.get_lattice()
    for name, values in autotune.search_space(variant, shape, algorithm).items():
        for v in values:
            sim = cls(shape, beta, seed=seed, algorithm=algorithm, init=lat)
            autotune.apply(sim, {name: v})
            sim.sweep(70)  # graph chunks and direct launches
            series = sim.sweep_measured(20, 5)
            np.testing.assert_array_equal(series, want_series, err_msg=f"{name}={v}")
            np.testing.assert_array_equal(sim.get_lattice(), want, err_msg=f"{name}={v}")


@pytest.mark.gpu
def test_tune_writes_the_cache_and_new_simulations_use_it(tmp_path, monkeypatch):
    from pyising_b200.backend import B200Int8

    monkeypatch.setenv("PYISING_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    res = autotune.tune("int8", (256, 256), target_ms=2.0, reps=1)
    space = autotune.search_space("int8", (256, 256))
    assert set(res["config"]) == set(space)
    for name, v in res["config"].items():
        assert v in space[name]
    assert res["flips_per_ns"] >= res["default_flips_per_ns"] > 0
    k = autotune.key(autotune.device_name(0), "int8", "metropolis", (256, 256))
    assert autotune.lookup(k) == res["config"]
    sim = B200Int8((256, 256), 0.44, seed=1, init="cold")
    cur = autotune.current(sim)
    for name, v in cur.items():
        assert v == res["config"][name]


@pytest.mark.gpu
def test_invalid_knob_values_are_rejected():
    from pyising_b200.backend import B200Int8, B200MultiSpin

    sim = B200Int8((24, 1032), 0.44, seed=1, init="cold")  # Lx/2 = 516: no 8-byte chunks
    with pytest.raises(ValueError):
        autotune.apply(sim, {"band": -1})
    with pytest.raises(ValueError):
        autotune.apply(sim, {"blocks_per_sm": 0})
    from pyising_b200._lib import lib

    assert lib().ising_set_knob(sim._h, autotune.KNOBS["chunk_width"], 8) == 1
    msc = B200MultiSpin((128, 256), 0.44, seed=1, init="cold")
    assert lib().ising_set_knob(msc._h, autotune.KNOBS["band"], 4) == 1


@pytest.mark.gpu
def test_batch_knobs_give_identical_results():
    from pyising_b200.backend import B200Int8, B200MultiSpin
    from pyising_b200.ensemble import Ensemble, Job

    jobs = [Job((40, 1032), 0.44, 30, seed=1, measure_every=5, init="philox"),
            Job((64, 64), 0.40, 40, seed=2, measure_every=10, init="philox"),
            Job((16, 24, 32), 0.22, 25, seed=3, algorithm="heatbath", measure_every=5,
                init="philox"),
            Job((128, 256), 0.44, 30, seed=4, variant="msc", measure_every=5, init="philox")]
    solo = []
    for j in jobs:
        cls = B200MultiSpin if j.variant == "msc" else B200Int8
        sim = cls(j.shape, j.beta, seed=j.seed, algorithm=j.algorithm, init="philox")
        solo.append(sim.sweep_measured(j.sweeps, j.measure_every))
    for cfg in [{"band": 1, "graph_chunk": 0}, {"band": 2, "items_per_slot": 1},
                {"band": 16, "items_per_slot": 12, "graph_chunk": 1}, {"graph_chunk": 4}]:
        with Ensemble() as ens:
            for name, v in cfg.items():
                ens.set_knob(name, v)
                assert ens.get_knob(name) == v
            ids = [ens.add(j) for j in jobs]
            ens.run()
            for i, want in zip(ids, solo, strict=True):
                np.testing.assert_array_equal(ens.result(i).series, want, err_msg=str(cfg))
    with Ensemble() as ens, pytest.raises(ValueError):
        ens.set_knob("band", 0)
