"""The reference's benchmark plan (bench/run.py) for this backend, in the same JSON schema.

    python -m pyising_b200.plan --quick|--full [--out b200-plan.json] [--repeats 5]

Each run record has the fields of the reference's (bench/run.py:209-226): flips/ns median, min
and max over repeats of a run sized to at least ``min_time`` seconds (bench/run.py:121-142),
effective bandwidth at 3 B (int8) or 3/8 B (packed) per update, % of the copy bandwidth, the
memory and Philox ceilings and % of the lower one, plus ``dram_bytes_per_launch`` where an ncu
summary of that kernel and size is committed under profiles/.

Differences from the reference's plan: lattices start from the device seeded start (not a host
NumPy hot start, which for the largest sizes would need the whole lattice in host memory), and
the "max" sizes (largest lattice that fits the free device memory) are left out.
"""

from __future__ import annotations

import argparse
import datetime as dt
import json
import math
import platform
import statistics
import time
from pathlib import Path

from ._lib import philox_rate
from .backend import B200Int8, B200MultiSpin
from .physics import BETA_C_2D, BETA_C_3D

FULL_2D = [1024, 2048, 4096, 8192, 16384, 32768, 65536]
FULL_MSC = [1024, 2048, 4096, 8192, 16384, 32768, 65536, 131072]
FULL_3D = [64, 128, 256, 512, 1024]
# backend, variant, dim, sizes, algorithm (bench/run.py:37-63, the cupy-cuda-c rows)
PLAN_FULL = [
    ("b200", "int8", 2, FULL_2D, "metropolis"),
    ("b200", "msc", 2, FULL_MSC, "metropolis"),
    ("b200", "int8", 2, [16384], "heatbath"),
    ("b200", "int8", 3, FULL_3D, "metropolis"),
    ("b200", "int8", 3, [256], "heatbath"),
]
PLAN_QUICK = [
    ("b200", "int8", 2, [1024, 4096], "metropolis"),
    ("b200", "msc", 2, [1024, 8192], "metropolis"),
    ("b200", "int8", 3, [128], "metropolis"),
]
SPEC_BANDWIDTH_GBS = 7700.0  # B200 (HGX) HBM3e

ROOT = Path(__file__).resolve().parent.parent
# ncu summaries (profiles/<kernel>_<workload>.md) that match a plan row
PROFILES = {("int8", 2, 16384, "metropolis"): "int8_half_kernel_int8_16384.md",
            ("msc", 2, 16384, "metropolis"): "msc_strip_kernel_msc16384.md",
            ("int8", 3, 256, "heatbath"): "int8_half_kernel_int8_3d_256_heatbath.md"}


def ceilings() -> dict:
    """Copy bandwidth (MEASURED_PEAKS.json of this machine when present, else a 1 GiB device
    copy timed here) and the measured Philox4x32-10 rate."""
    bw, source = None, "measured here"
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        bw, source = float(json.loads(p.read_text())["hbm_gbs"]), "MEASURED_PEAKS.json"
    if bw is None:
        import torch

        a = torch.empty(1 << 30, dtype=torch.uint8, device="cuda")
        b = torch.empty_like(a)
        best = math.inf
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            b.copy_(a)
            e.record()
            e.synchronize()
            best = min(best, s.elapsed_time(e))
        bw = 2 * a.numel() / (best * 1e-3) / 1e9
    return {"copy_bandwidth_GBs": round(bw, 1), "copy_bandwidth_source": source,
            "spec_bandwidth_GBs": SPEC_BANDWIDTH_GBS,
            "philox_calls_per_ns": round(philox_rate(0, 512, 5), 2)}


def dram_bytes(variant: str, dim: int, L: int, algorithm: str) -> float | None:
    name = PROFILES.get((variant, dim, L, algorithm))
    if not name or not (ROOT / "profiles" / name).exists():
        return None
    for line in (ROOT / "profiles" / name).read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch"):
            return float(line.split("=")[1].split()[0])
    return None


def time_one(cls, shape, algorithm: str, beta: float, repeats: int, min_time: float) -> dict:
    """Warm up, size the run to >= min_time s, return median/min/max flips/ns (wall clock
    around synchronised sweeps, as bench/run.py:121-142)."""
    sim = cls(shape, beta, seed=12345, algorithm=algorithm, init="philox")
    sim.sweep(2)
    sim.synchronize()
    t0 = time.perf_counter()
    sim.sweep(1)
    sim.synchronize()
    t1 = time.perf_counter() - t0
    n = max(1, math.ceil(min_time / max(t1, 1e-6)))
    sim.sweep(min(n, 5))
    sim.synchronize()
    rates = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        sim.sweep(n)
        sim.synchronize()
        rates.append(n * sim.n_spins / (time.perf_counter() - t0) / 1e9)
    calls = sim.philox_calls_per_word(2, warp=False) if cls is B200MultiSpin else None
    m, e = sim.observables()
    del sim
    return {"median": statistics.median(rates), "min": min(rates), "max": max(rates),
            "sweeps_per_repeat": n, "m": m, "e": e, "calls_per_word": calls}


def run(plan, repeats: int, min_time: float, log=print) -> dict:
    t_start = time.time()
    ceil = ceilings()
    bw, ph = ceil["copy_bandwidth_GBs"], ceil["philox_calls_per_ns"]
    runs = []
    for backend, variant, dim, sizes, algorithm in plan:
        cls = B200MultiSpin if variant == "msc" else B200Int8
        beta = BETA_C_2D if dim == 2 else BETA_C_3D
        for L in sizes:
            shape = (int(L),) * dim
            r = time_one(cls, shape, algorithm, beta, repeats, min_time)
            bpu = cls.bytes_per_update
            eff = r["median"] * bpu
            calls = (r["calls_per_word"] / 64.0) if variant == "msc" else 0.25
            rng = ph / calls
            run = {
                "backend": backend, "variant": variant, "algorithm": algorithm,
                "size": list(shape), "dim": dim,
                "dtype": "uint64-packed-1bit" if variant == "msc" else "int8",
                "metric": "flips/ns", "value": round(r["median"], 3), "repeats": repeats,
                "median": round(r["median"], 3), "min": round(r["min"], 3),
                "max": round(r["max"], 3), "sweeps_per_repeat": r["sweeps_per_repeat"],
                "bytes_per_unit": bpu, "effective_GBs": round(eff, 2),
                "pct_copy_bw": round(100 * eff / bw, 2),
                "pct_spec_bw": round(100 * eff / SPEC_BANDWIDTH_GBS, 2),
                "flops_per_unit": None, "pct_peak_flops": None,
                "memory_ceiling_flips_per_ns": round(bw / bpu, 1),
                "philox_calls_per_update": round(calls, 5),
                "rng_ceiling_flips_per_ns": round(rng, 1),
                "pct_roofline": round(100 * r["median"] / min(bw / bpu, rng), 2),
                "temperature": 1.0 / beta, "final_m": r["m"], "final_e": r["e"],
                "dram_bytes_per_launch": dram_bytes(variant, dim, int(L), algorithm),
                "notes": f"{algorithm}, T=Tc, device seeded start",
            }
            runs.append(run)
            log(f"{backend}/{variant:<5} {algorithm[:5]} {str(shape):>22}: "
                f"{run['median']:9.2f} flips/ns [{run['min']:.2f}, {run['max']:.2f}] "
                f"{run['pct_copy_bw']:6.1f}% copy BW {run['pct_roofline']:6.1f}% roofline "
                f"({time.time() - t_start:5.0f} s)")
    return {"machine": machine_info(), "ceiling": ceil, "runs": runs,
            "seconds": round(time.time() - t_start, 1)}


def machine_info() -> dict:
    from .autotune import device_name

    return {"gpu": device_name(0), "python": platform.python_version(),
            "date": dt.datetime.now(dt.timezone.utc).isoformat(timespec="seconds")}


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    g = ap.add_mutually_exclusive_group(required=True)
    g.add_argument("--quick", action="store_true")
    g.add_argument("--full", action="store_true")
    ap.add_argument("--out", default="b200-plan.json")
    ap.add_argument("--repeats", type=int, default=5)
    args = ap.parse_args(argv)
    plan = PLAN_QUICK if args.quick else PLAN_FULL
    res = run(plan, 3 if args.quick else args.repeats, 0.1 if args.quick else 0.5)
    res["mode"] = "quick" if args.quick else "full"
    Path(args.out).write_text(json.dumps(res, indent=1))
    print(f"wrote {args.out} in {res['seconds']} s")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
