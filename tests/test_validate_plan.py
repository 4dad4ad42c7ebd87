"""The validation suite (pyising_b200.validate, after src/pyising/validate.py) and the benchmark
plan in the reference's run-record schema (pyising_b200.plan, after bench/run.py).

CPU: every job the QUICK and FULL settings build is a valid lattice of the backend, and the plan
covers the reference's CUDA C rows.  GPU: the QUICK suite runs (a few seconds, deterministic
seeds) and lands within the tolerances; one plan row has every field of the reference's schema.
"""

from __future__ import annotations

import pytest

from pyising_b200 import plan, validate
from pyising_b200.ensemble import Job


@pytest.mark.parametrize("cfg", [validate.QUICK, validate.FULL], ids=["quick", "full"])
def test_settings_build_valid_jobs(cfg):
    for T in cfg["T2"]:
        for variant in ("int8", "msc"):
            Job((cfg["L2"],) * 2, 1.0 / T, 10, variant=variant, measure_every=cfg["every"])
    for dim in (2, 3):
        for L in cfg[f"binder{dim}_L"]:
            Job((L,) * dim, 0.3, 10, measure_every=cfg[f"binder{dim}_every"])
    Job((cfg["L3"],) * 3, 0.2, 10, algorithm="heatbath", measure_every=cfg["every"])
    assert len(cfg["binder2_L"]) >= 2 and len(cfg["binder3_L"]) >= 2


def test_plan_covers_the_reference_rows():
    rows = {(v, d, a) for _, v, d, _, a in plan.PLAN_FULL}
    assert rows == {("int8", 2, "metropolis"), ("msc", 2, "metropolis"), ("int8", 2, "heatbath"),
                    ("int8", 3, "metropolis"), ("int8", 3, "heatbath")}
    for _, variant, _, sizes, _ in plan.PLAN_FULL:
        for L in sizes:
            assert L % (128 if variant == "msc" else 8) == 0
    assert plan.dram_bytes("msc", 2, 16384, "metropolis") > 0


@pytest.mark.gpu
def test_quick_validation_suite():
    res = validate.run(quick=True, out=None, log=lambda *a: None)
    s = res["summary"]
    assert s["e_max_abs_z"] < 4.5
    assert s["m_max_abs_err_vs_yang_away_from_Tc"] < 0.01
    assert s["Tc2d_rel_error"] < 0.02
    assert s["Tc3d_rel_error"] < 0.02
    assert s["e3d_max_abs_z_metropolis_vs_heatbath"] < 4.5


@pytest.mark.gpu
def test_plan_run_record_schema():
    res = plan.run([("b200", "int8", 2, [256], "metropolis"), ("b200", "msc", 2, [256],
                                                                "metropolis")],
                   repeats=1, min_time=0.01, log=lambda *a: None)
    keys = {"backend", "variant", "algorithm", "size", "dim", "dtype", "metric", "value",
            "repeats", "median", "min", "max", "sweeps_per_repeat", "bytes_per_unit",
            "effective_GBs", "pct_copy_bw", "pct_spec_bw", "flops_per_unit", "pct_peak_flops",
            "memory_ceiling_flips_per_ns", "philox_calls_per_update", "rng_ceiling_flips_per_ns",
            "pct_roofline", "temperature", "final_m", "final_e", "notes"}
    assert len(res["runs"]) == 2
    for r in res["runs"]:
        assert keys <= set(r)
        assert r["value"] > 0 and 0 < r["pct_roofline"] <= 100
    assert res["ceiling"]["philox_calls_per_ns"] > 0
