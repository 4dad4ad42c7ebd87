"""Benchmark of the pyising sweep hot path on B200: one JSON line on stdout (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload msc16384|int8_1024|int8_3d_256] [--no-extras]
    python bench.py --profile-case CASE L SWEEPS   (one small case for ncu; no JSON line)

Headline workload (one "step" = one whole job of the config): 2D multi-spin-coded Metropolis,
L = 16384 (64 spins per uint64, 16384 x 128 words per colour), periodic, T = T_c, hot start
seed 7 (pyising's NumPy hot start), 1000 sweeps.  ``value`` is flips/ns (attempted spin updates
per ns) with the lattice resident in HBM; ``e2e`` is the same job through the public Python API
with the lattice uploaded from and downloaded to host memory inside the timed region.
The L2 cache (126 MB) is flushed between steps by writing a 256 MiB buffer; within a step the
32 MiB lattice stays L2-resident, which is part of the workload.

Under torchrun (N > 1) every rank runs its own replica (seed 7 + rank; no collective on the data
path): ``value`` is the flips of all ranks / the slowest rank's time ("scaling": "weak").

``--impl reference`` times the CPU restatement of the reference's algorithm (oracle/, the NumPy
backend's algorithm in C, all host threads) on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

BETA_C_2D = math.log(1.0 + math.sqrt(2.0)) / 2.0
BETA_3D = 0.221654626
L2_FLUSH_BYTES = 256 << 20

WORKLOADS = {
    # name: (variant, shape, algorithm, beta, init, seed, sweeps per step, bytes/update)
    "msc16384": ("msc", (16384, 16384), "metropolis", BETA_C_2D, "hot", 7, 1000, 0.375),
    "int8_1024": ("int8", (1024, 1024), "metropolis", BETA_C_2D, "hot", 1, 1000, 3.0),
    "int8_3d_256": ("int8", (256, 256, 256), "heatbath", BETA_3D, "cold", 0, 2000, 3.0),
}
DESCRIPTION = {
    "msc16384": "msc 2D Metropolis L=16384 (16384x128 u64 words per colour), periodic, T=T_c, "
                "hot start seed 7, 1000 sweeps per step",
    "int8_1024": "int8 2D Metropolis L=1024 compressed checkerboard, beta_c, hot start seed 1, "
                 "1000 sweeps per step",
    "int8_3d_256": "int8 3D heat bath L=256, beta=0.221654626, cold start, 2000 sweeps per step "
                   "with (E, M) every 10 sweeps",
}
MEASURE_EVERY = {"int8_3d_256": 10}
KERNEL = {"msc": "msc_strip_kernel", "int8": "int8_half_kernel"}


# ------------------------------------------------------------------------- helpers -------
def dist_env() -> tuple[int, int, int]:
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profile_traffic(kernel: str, workload: str) -> float | None:
    """DRAM bytes per launch of ``kernel`` from the committed ncu summary, if there is one."""
    p = ROOT / "profiles" / f"{kernel}_{workload}.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch"):
            try:
                return float(line.split("=")[1].split()[0])
            except (IndexError, ValueError):
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int) -> None:
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self) -> None:
        for line in self.proc.stdout:  # type: ignore[union-attr]
            self.lines.append(line.strip())

    def __exit__(self, *exc) -> None:
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9], strict=False):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "power_w_max": max(power) if power else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------ B200 arm -------
def make_sim(wl: str, seed_offset: int = 0):
    from pyising_b200.backend import B200Int8, B200MultiSpin

    variant, shape, alg, beta, init, seed, _, _ = WORKLOADS[wl]
    cls = B200MultiSpin if variant == "msc" else B200Int8
    return cls(shape, beta, seed=seed + seed_offset, algorithm=alg, init=init)


def tune_workload(wl: str, device: int) -> dict:
    """The autotuner's launch knobs for a workload's shape (measured on a scratch lattice before
    any timing; not written to the user's tuning cache)."""
    from pyising_b200 import autotune

    variant, shape, alg, beta, *_ = WORKLOADS[wl]
    res = autotune.tune(variant, shape, alg, beta, device=device, save=False)
    return {"config": res["config"], "default_flips_per_ns": round(res["default_flips_per_ns"], 1),
            "tuned_flips_per_ns": round(res["flips_per_ns"], 1),
            "seconds": round(res["seconds"], 2)}


def run_device(wl: str, steps: int, warmup: int, rank: int, world: int, local: int,
               dist, tuned: dict | None = None) -> dict:
    """Device-resident timing: K steps, CUDA events on the launching stream, L2 flushed."""
    import torch

    from pyising_b200 import autotune

    variant, shape, alg, beta, init, seed, sweeps, bpu = WORKLOADS[wl]
    every = MEASURE_EVERY.get(wl, 0)
    sim = make_sim(wl, rank)
    if tuned:
        autotune.apply(sim, tuned["config"])
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    st0 = sim.state()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def step():
        if every:
            sim.sweep_measured(sweeps, every)
        else:
            sim.sweep(sweeps)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    # restart from the workload's own start so the timed steps are the job itself
    sim.load_colour_arrays(st0["c0"], st0["c1"])
    sim.t = 0
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for i in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
                events[i][0].record(stream)
            step()
            with torch.cuda.stream(stream):
                events[i][1].record(stream)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ms = [a.elapsed_time(b) for a, b in events]
    total_ms = sum(ms)
    if dist is not None:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    n = int(np.prod(shape))
    flips = n * sweeps * steps * world
    value = flips / (total_ms * 1e6)
    launches = 2 * sweeps * steps  # half-sweeps: the unit of the roofline's launch time
    avg_launch_ms = total_ms / launches
    # kernels launched in the timed region: every half-sweep, plus one counter node per
    # replayed graph chunk and one counter reset per call; a persistent run is one launch
    cfg = (tuned or {}).get("config", {})
    if cfg.get("schedule") == "persistent" and variant == "int8" and len(shape) == 2:
        per_step = 1
    elif cfg.get("schedule") == "launches":
        per_step = 2 * sweeps
    else:
        g = every if every else int(cfg.get("graph_chunk", 32))
        per_step = 2 * sweeps + (sweeps // g + 1 if sweeps >= 2 * g else 0)
    M, E = sim.observables_int()
    out = {"value": value, "ms_per_step": total_ms / steps, "step_ms": ms,
           "launches": launches, "gpu_launches": per_step * steps,
           "avg_launch_ms": avg_launch_ms, "flips_per_step": n * sweeps,
           "final_M": M, "final_E": E, "clocks": clk.summary(), "n_spins": n,
           "bytes_per_update": bpu, "sim": sim}
    del flush
    return out


def run_e2e(wl: str, steps: int, rank: int, world: int, dist, tuned: dict | None = None) -> dict:
    """The same job through the public API with host buffers: upload the start configuration,
    sweep, download the final colour arrays and read (M, E), every step."""
    import torch

    from pyising_b200 import autotune

    variant, shape, alg, beta, init, seed, sweeps, bpu = WORKLOADS[wl]
    every = MEASURE_EVERY.get(wl, 0)
    sim = make_sim(wl, rank)
    if tuned:
        autotune.apply(sim, tuned["config"])
    st0 = sim.state()

    def pinned_like(a: np.ndarray) -> np.ndarray:
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        return t.numpy().view(a.dtype).reshape(a.shape)

    # the step's input and result live in pinned host buffers (allocated once, outside the
    # timed region), as a serving caller would keep them
    c0, c1 = pinned_like(st0["c0"]), pinned_like(st0["c1"])
    c0[...] = st0["c0"]
    c1[...] = st0["c1"]
    out = (pinned_like(st0["c0"]), pinned_like(st0["c1"]))
    h2d = c0.nbytes + c1.nbytes + sim.table.nbytes
    d2h = c0.nbytes + c1.nbytes + 16 + (sweeps // every) * 16 if every else c0.nbytes + c1.nbytes + 16
    sim.sweep(2)
    sim.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    finals = []
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.load_colour_arrays(c0, c1)
        sim.t = 0
        sim._upload_table()
        if every:
            sim.sweep_measured(sweeps, every)
        else:
            sim.sweep(sweeps)
        sim.colour_arrays(out)
        finals.append(sim.observables_int())
    sim.synchronize()
    dt = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([dt], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dt = float(t.item())
    n = int(np.prod(shape))
    return {"value": n * sweeps * steps * world / (dt * 1e9), "unit": "flips/ns",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "ms_per_step": dt * 1e3 / steps, "host_buffers": "pinned",
            # every step runs the same job from the same start: identical (M, E) each time
            "steps_identical": all(f == finals[0] for f in finals)}


def rng_ceiling(sim, variant: str) -> dict:
    from pyising_b200._lib import philox_rate

    rate = philox_rate(sim.device, 512, 5)
    if variant == "msc":
        mean = sim.philox_calls_per_word(2)
        wmax = sim.philox_calls_per_word(2, warp=True)
        calls_per_update = mean / 64.0
        return {"philox_calls_per_ns": rate, "calls_per_word_mean": mean,
                "calls_per_word_warp_max": wmax, "calls_per_update": calls_per_update,
                "ceiling_flips_per_ns": rate / calls_per_update,
                "ceiling_warp_max_flips_per_ns": rate / (wmax / 64.0)}
    return {"philox_calls_per_ns": rate, "calls_per_update": 0.25,
            "ceiling_flips_per_ns": rate / 0.25}


def cpu_baseline(wl: str, budget_s: float = 10.0) -> dict:
    """The oracle (the reference's algorithm in C, all host threads) on a bounded sample."""
    import oracle

    variant, shape, alg, beta, init, seed, sweeps, bpu = WORKLOADS[wl]
    cores = oracle.cpu_count()
    oracle.set_threads(cores)
    sim = oracle.create(variant, shape=shape, beta=beta, seed=seed, algorithm=alg, init=init)
    t0 = time.perf_counter()
    sim.sweep(1)
    one = max(time.perf_counter() - t0, 1e-6)
    n = max(1, min(sweeps, int(budget_s / one)))
    t0 = time.perf_counter()
    sim.sweep(n)
    dt = time.perf_counter() - t0
    rate = int(np.prod(shape)) * n / (dt * 1e9)
    return {"value": rate, "unit": "flips/ns", "cores": cores, "kind": "port",
            "sample": f"{n} sweeps of the same lattice (shape {list(shape)}, {variant}, "
                      f"{alg}) on the C oracle, {cores} threads, {dt:.1f} s"}


TC_3D = 1.0 / BETA_3D


def c4_jobs(sweeps: int = 5000, every: int = 10):
    """The batched-ensemble config: 96 2D int8 Metropolis lattices, L = 2^k with k uniform in
    6..12, T uniform in [2.0, 2.6], seed = index, NumPy hot start; draws from default_rng(0)."""
    from pyising_b200.ensemble import Job
    from pyising_b200.lattice import random_lattice

    rng = np.random.default_rng(0)
    ks = rng.integers(6, 13, size=96)
    Ts = rng.uniform(2.0, 2.6, size=96)
    return [Job((2 ** int(k), 2 ** int(k)), 1.0 / float(T), sweeps, seed=i, measure_every=every,
                init=random_lattice((2 ** int(k), 2 ** int(k)), i))
            for i, (k, T) in enumerate(zip(ks, Ts, strict=True))]


def c5_jobs(n_jobs: int, seed: int = 2026):
    """The served-stream config: Poisson arrivals at 200 jobs/s; 70% 2D (L log-uniform in
    128..8192, int8 or msc 50/50, Metropolis, T within +-15% of T_c), 30% 3D (L log-uniform in
    32..256, int8 heat bath, T within +-15% of the 3D T_c); sweeps log-uniform in 100..10000;
    (M, E) every 10 sweeps; L rounded to the layout multiple; device seeded start (seed = index).
    Returns (arrival times in s, jobs)."""
    from pyising_b200.ensemble import Job

    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / 200.0, size=n_jobs))
    jobs = []
    for i in range(n_jobs):
        sweeps = int(np.exp(rng.uniform(np.log(100), np.log(10000))))
        if rng.random() < 0.7:
            variant = "msc" if rng.random() < 0.5 else "int8"
            m = 128 if variant == "msc" else 8
            L = int(np.exp(rng.uniform(np.log(128), np.log(8192))))
            L = max(m, int(round(L / m)) * m)
            T = (1.0 / BETA_C_2D) * rng.uniform(0.85, 1.15)
            jobs.append(Job((L, L), 1.0 / T, sweeps, seed=i, variant=variant, measure_every=10,
                            init="philox"))
        else:
            L = int(np.exp(rng.uniform(np.log(32), np.log(256))))
            L = max(8, int(round(L / 8)) * 8)
            T = TC_3D * rng.uniform(0.85, 1.15)
            jobs.append(Job((L, L, L), 1.0 / T, sweeps, seed=i, algorithm="heatbath",
                            measure_every=10, init="philox"))
    return arrivals, jobs


def sequential_plain(jobs) -> tuple[float, list]:
    """The same jobs one at a time through the single-lattice API (upload or device start,
    sweeps with the fused measurement, series back to the host); returns (seconds, series)."""
    import torch

    from pyising_b200.backend import B200Int8, B200MultiSpin

    out = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for j in jobs:
        cls = B200MultiSpin if j.variant == "msc" else B200Int8
        sim = cls(j.shape, j.beta, seed=j.seed, algorithm=j.algorithm, init=j.init)
        out.append(sim.sweep_measured(j.sweeps, j.measure_every))
        del sim
    torch.cuda.synchronize()
    return time.perf_counter() - t0, out


def class_of(job) -> str:
    if job.variant == "msc":
        return "msc 2D Metropolis"
    return f"int8 {len(job.shape)}D {job.algorithm}"


def best_kernel_rates(jobs) -> dict:
    """Per kernel class of ``jobs``: the autotuned single-lattice rate of the class's largest
    shape (device-timed; smaller shapes are launch-bound and never faster), and the class's
    Philox calls per update (0.25 for int8; the measured calls per word / 64 for msc)."""
    from pyising_b200 import autotune
    from pyising_b200.backend import B200MultiSpin

    largest: dict[str, tuple] = {}
    for j in jobs:
        k = class_of(j)
        if k not in largest or j.n_spins > int(np.prod(largest[k][0])):
            largest[k] = (tuple(j.shape), j.algorithm, j.variant, j.beta)
    rates, calls = {}, {}
    for k, (shape, alg, variant, beta) in largest.items():
        rates[k] = round(autotune.tune(variant, shape, alg, beta, save=False)["flips_per_ns"], 1)
        if variant == "msc":
            sim = B200MultiSpin(shape, beta, seed=12345, init="philox")
            calls[k] = round(sim.philox_calls_per_word(2) / 64.0, 5)
            del sim
        else:
            calls[k] = 0.25
    return {"flips_per_ns": rates, "philox_calls_per_update": calls}


def ratio_bound(jobs, t_seq: float, best: dict, t_batched: float) -> dict:
    """How far the batched/sequential ratio can go.  ``at_best_kernel``: the sequential time over
    the time the jobs' flips take at their class's best rate (the autotuned single-lattice rate,
    or the batched run's own rate when that is higher); ``at_philox_ceiling``: over the time
    the Philox blocks alone take at the measured Philox rate, which no kernel can beat."""
    from pyising_b200._lib import philox_rate

    flips = sum(j.n_spins * j.sweeps for j in jobs)
    rates = best["flips_per_ns"]
    t_kernel = sum(j.n_spins * j.sweeps / (rates[class_of(j)] * 1e9) for j in jobs)
    t_kernel = min(t_kernel, t_batched)
    rate = philox_rate(0, 512, 5)
    t_philox = sum(j.n_spins * j.sweeps * best["philox_calls_per_update"][class_of(j)]
                   for j in jobs) / (rate * 1e9)
    return {"class_best_flips_per_ns": rates,
            "philox_calls_per_update": best["philox_calls_per_update"],
            "philox_calls_per_ns": round(rate, 1),
            "best_kernel_s": round(t_kernel, 3),
            "at_best_kernel": round(t_seq / t_kernel, 3),
            "philox_s": round(t_philox, 3),
            "at_philox_ceiling": round(t_seq / t_philox, 3),
            "best_kernel_flips_per_ns": round(flips / t_kernel / 1e9, 1)}


def c4_oracle_check(jobs, results) -> dict:
    """Every member's series and final lattice against the oracle (all host threads), after
    the timed region: the checker, not a measured path."""
    import oracle

    oracle.set_threads(oracle.cpu_count())
    t0 = time.perf_counter()
    bad = []
    for i, (job, res) in enumerate(zip(jobs, results, strict=True)):
        ref = oracle.OracleInt8(job.shape, job.beta, seed=job.seed, init=job.init)
        series = ref.sweep(job.sweeps, measure_every=job.measure_every)
        if not (np.array_equal(series, res.series) and np.array_equal(ref.get_lattice(),
                                                                      res.lattice)):
            bad.append(i)
    return {"identical": not bad, "members": len(jobs), "mismatched": bad,
            "compared": "every (M, E) of the series and the final lattice",
            "oracle_seconds": round(time.perf_counter() - t0, 1),
            "oracle_threads": oracle.cpu_count()}


def run_batched_ensemble(check_oracle: bool = True) -> dict:
    """C4: batched vs one at a time, every lattice's series compared (and with the oracle)."""
    import torch

    from pyising_b200 import autotune
    from pyising_b200.ensemble import Ensemble

    import dataclasses

    jobs = [dataclasses.replace(j, keep_lattice=True) for j in c4_jobs()]
    flips = sum(j.n_spins * j.sweeps for j in jobs)
    tuned = autotune.tune_ensemble(jobs, sweeps=256)
    with Ensemble(memory_budget=120e9) as ens:
        for name, v in tuned["config"].items():
            ens.set_knob(name, v)
        ids = [ens.add(j) for j in jobs]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ens.run()
        t_batch = time.perf_counter() - t0
        results = [ens.result(i) for i in ids]
        batched = [r.series for r in results]
    t_seq, seq = sequential_plain(jobs)
    same = all(np.array_equal(a, b) for a, b in zip(batched, seq, strict=True))
    oracle_check = c4_oracle_check(jobs, results) if check_oracle else None
    return {"workload": "96 2D int8 Metropolis lattices, L=2^k k~U{6..12}, T~U[2.0,2.6], "
                        "seed=index, NumPy hot start, 5000 sweeps, (E,M) every 10; "
                        "draws from default_rng(0)",
            "flips": flips, "batched_s": round(t_batch, 3), "sequential_s": round(t_seq, 3),
            "batched_flips_per_ns": round(flips / t_batch / 1e9, 2),
            "sequential_flips_per_ns": round(flips / t_seq / 1e9, 2),
            "speedup": round(t_seq / t_batch, 3), "bit_identical": bool(same),
            "bound": ratio_bound(jobs, t_seq, best_kernel_rates(jobs), t_batch),
            "oracle_identical": oracle_check["identical"] if oracle_check else None,
            "oracle_check": oracle_check,
            "tuned_batch_knobs": tuned["config"],
            "timed": "uploads of the start lattices, all sweeps, series and final lattices "
                     "back to the host"}


def run_served_stream(n_jobs: int, baseline_jobs: int | None = None) -> dict:
    """C5: Poisson arrivals of ``n_jobs`` jobs into the server; the same jobs one at a time with
    the plain kernels (all of them, or the first ``baseline_jobs`` as a seeded subset), and the
    server's queue depth and memory use sampled every 50 ms."""
    import threading

    from pyising_b200 import autotune
    from pyising_b200.ensemble import Server

    arrivals, jobs = c5_jobs(n_jobs)
    flips = sum(j.n_spins * j.sweeps for j in jobs)
    submit_t = [0.0] * n_jobs
    ids = [0] * n_jobs
    tuned = autotune.tune_ensemble(jobs[: min(n_jobs, 100)], sweeps=256)
    budget = int(120e9)
    peaks = {"pending": 0, "active": 0, "used_bytes": 0}
    with Server(memory_budget=budget) as srv:
        for name, v in tuned["config"].items():
            srv.set_knob(name, v)
        start = time.perf_counter()
        done = threading.Event()

        def feeder():
            for i, job in enumerate(jobs):
                delay = start + arrivals[i] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                submit_t[i] = time.perf_counter()
                ids[i] = srv.submit(job)

        def monitor():
            while not done.wait(0.05):
                st = srv.status()
                for k in peaks:
                    peaks[k] = max(peaks[k], int(st[k]))

        th, mon = threading.Thread(target=feeder), threading.Thread(target=monitor)
        th.start()
        mon.start()
        th.join()
        results = []
        for i in range(n_jobs):
            srv.wait(ids[i])
            results.append(srv.result(ids[i]))
            srv.release(ids[i])
        done.set()
        mon.join()
    lat = np.array([r.latency_s for r in results])
    end = max(submit_t[i] + lat[i] for i in range(n_jobs))
    served_s = end - submit_t[0]
    nb = n_jobs if baseline_jobs is None else max(1, min(baseline_jobs, n_jobs))
    base_flips = sum(j.n_spins * j.sweeps for j in jobs[:nb])
    t_seq, seq = sequential_plain(jobs[:nb])
    same = all(np.array_equal(r.series, s) for r, s in zip(results[:nb], seq, strict=True))
    served_rate = flips / served_s / 1e9
    offered_rate = flips / (arrivals[-1] * 1e9)
    seq_rate = base_flips / t_seq / 1e9
    return {"workload": f"{n_jobs} jobs of the served-stream mix (Poisson 200 jobs/s; 70% 2D "
                        "L~logU[128,8192] int8|msc, 30% 3D L~logU[32,256] int8 heat bath; "
                        "T_c +-15%; sweeps~logU[100,10000]; (E,M) every 10; device seeded "
                        "start), seed 2026",
            "jobs": n_jobs, "flips": flips, "offered_flips_per_ns": round(offered_rate, 2),
            "arrival_window_s": round(float(arrivals[-1]), 3),
            "served_s": round(served_s, 3), "served_flips_per_ns": round(served_rate, 2),
            "keeps_up": bool(served_rate >= 0.98 * offered_rate),
            "sequential_jobs": nb,
            "sequential_subset": ("all jobs" if nb == n_jobs else
                                  f"the first {nb} jobs of the stream (seeded subset)"),
            "sequential_s": round(t_seq, 3),
            "sequential_flips_per_ns": round(seq_rate, 2),
            "speedup": round(served_rate / seq_rate, 3),
            "bound": ratio_bound(jobs[:nb], t_seq, best_kernel_rates(jobs[:nb]),
                                 served_s * base_flips / flips),
            "latency_p50_s": round(float(np.percentile(lat, 50)), 4),
            "latency_p99_s": round(float(np.percentile(lat, 99)), 4),
            "latency_max_s": round(float(lat.max()), 4),
            "peak_pending_jobs": peaks["pending"], "peak_active_jobs": peaks["active"],
            "peak_used_bytes": peaks["used_bytes"],
            "bit_identical": bool(same), "bit_identical_jobs": nb,
            "memory_budget_bytes": budget, "tuned_batch_knobs": tuned["config"]}


def run_slabs(wl: str, parts: int = 2, sweeps: int = 200) -> dict:
    """The workload's lattice cut into `parts` slabs on this GPU (neighbour rows read in place),
    timed with CUDA events on the slabs' stream after a warm-up; shows the slab path's own cost
    against the single-lattice kernels (on separate GPUs the slabs run concurrently)."""
    import torch

    from pyising_b200.slab import SlabSimulation

    variant, shape, alg, beta, init, seed, _, _ = WORKLOADS[wl]
    sim = SlabSimulation(shape, beta, seed=seed, algorithm=alg, variant=variant, init="philox",
                         parts=parts, devices=[torch.cuda.current_device()])
    st = sim.runner.streams[0]
    sim.sweep(20)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    sim.sweep(sweeps)
    b.record(st)
    b.synchronize()
    ms = a.elapsed_time(b)
    sim.close()
    n = int(np.prod(shape))
    return {"workload": f"{DESCRIPTION[wl].split(',')[0]} as {parts} slabs on one GPU",
            "parts": parts, "sweeps": sweeps, "flips_per_ns": round(n * sweeps / (ms * 1e6), 2),
            "exchange": "neighbour edge rows read in place (no copies)"}


def main_b200(args, rank: int, world: int, local: int, dist) -> dict | None:
    import torch

    wl = args.workload
    variant, shape, alg, beta, init, seed, sweeps, bpu = WORKLOADS[wl]
    tuned = tune_workload(wl, local) if args.tune else None
    dev = run_device(wl, args.steps, args.warmup, rank, world, local, dist, tuned)
    sim = dev.pop("sim")
    e2e = run_e2e(wl, args.steps, rank, world, dist, tuned)
    if rank != 0:
        return None
    peaks = measured_peaks()
    n = dev["n_spins"]
    bytes_per_launch = bpu * n / 2  # one colour = half the spins per launch
    achieved = bytes_per_launch / (dev["avg_launch_ms"] * 1e-3) / 1e9
    traffic = profile_traffic(KERNEL[variant], wl)
    rng = rng_ceiling(sim, variant)
    hbm_ceiling = peaks["hbm_gbs"] / bpu
    line = {
        "metric": "flips/ns", "value": round(dev["value"], 2), "unit": "flips/ns",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dev["ms_per_step"], 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64" if variant == "msc" else "int8",
        "data": "synthetic (seeded hot/cold start; no dataset)",
        "config": {"workload": DESCRIPTION[wl], "variant": variant, "shape": list(shape),
                   "algorithm": alg, "beta": beta, "sweeps_per_step": sweeps,
                   "l2": "flushed between steps (256 MiB write); the lattice stays "
                         "L2-resident within a step",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "launch_knobs": tuned if tuned else "library defaults"},
        "pct_hbm_roofline": round(100 * dev["value"] / hbm_ceiling, 2),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1),
                     "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": round(achieved / peaks["hbm_gbs"], 4),
                     "traffic": traffic,
                     "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs)",
                     "kernel": KERNEL[variant],
                     "bytes_per_launch": bytes_per_launch,
                     "avg_launch_ms": round(dev["avg_launch_ms"], 5)},
        "rng_roofline": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in rng.items()},
        "e2e": {k: (round(v, 2) if isinstance(v, float) else v) for k, v in e2e.items()},
        "gpu_launches": dev["gpu_launches"],
        "clocks": dev["clocks"],
        "final_M_E": [dev["final_M"], dev["final_E"]],
    }
    if world == 1:
        line["cpu_baseline"] = cpu_baseline(wl, args.cpu_budget)
        line["cpu_baseline"]["value"] = round(line["cpu_baseline"]["value"], 4)
    if args.extras and world == 1:
        extras = {}
        for other in WORKLOADS:
            if other == wl:
                continue
            t_other = tune_workload(other, local) if args.tune else None
            d = run_device(other, 3, 3, 0, 1, local, None, t_other)
            d.pop("sim")
            v, _, _, _, _, _, sw, b = WORKLOADS[other]
            # int8: one Philox block per 4 sites, so the integer-pipe ceiling is rate / 0.25
            rng_ceiling_other = rng["philox_calls_per_ns"] / 0.25 if v == "int8" else None
            extras[other] = {"flips_per_ns": round(d["value"], 2),
                             "ms_per_step": round(d["ms_per_step"], 4),
                             "pct_hbm_roofline": round(100 * d["value"] * b / peaks["hbm_gbs"], 2),
                             "pct_philox_roofline": (round(100 * d["value"] / rng_ceiling_other, 2)
                                                     if rng_ceiling_other else None),
                             "description": DESCRIPTION[other],
                             "launch_knobs": t_other if t_other else "library defaults"}
        line["other_configs"] = extras
    if args.extras and world == 1:
        line["slab_decomposition"] = run_slabs(wl)
    if args.batch and world == 1:
        line["batched_ensemble"] = run_batched_ensemble(args.c4_oracle)
    if args.serve_jobs > 0 and world == 1:
        line["served_stream"] = run_served_stream(args.serve_jobs, args.serve_baseline_jobs)
    torch.cuda.synchronize()
    return line


def main_reference(args, rank: int) -> dict | None:
    """The reference's algorithm on the host cores (the oracle port), one bounded sample per
    step; rank 0 only."""
    if rank != 0:
        return None
    import oracle

    wl = args.workload
    variant, shape, alg, beta, init, seed, sweeps, bpu = WORKLOADS[wl]
    cores = oracle.cpu_count()
    oracle.set_threads(cores)
    sim = oracle.create(variant, shape=shape, beta=beta, seed=seed, algorithm=alg, init=init)
    t0 = time.perf_counter()
    sim.sweep(1)
    one = max(time.perf_counter() - t0, 1e-6)
    per_step = max(1, min(sweeps, int(args.ref_step_s / one)))
    for _ in range(args.warmup):
        sim.sweep(per_step)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        sim.sweep(per_step)
        times.append(time.perf_counter() - t0)
    n = int(np.prod(shape))
    value = n * per_step * len(times) / (sum(times) * 1e9)
    sample = (f"{per_step} sweeps per step of the {variant} lattice {list(shape)} ({alg}) on the "
              f"C restatement of the reference algorithm, {cores} threads")
    return {"impl": "reference", "metric": "flips/ns", "value": round(value, 4),
            "unit": "flips/ns", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * sum(times) / len(times), 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "u64" if variant == "msc" else "int8", "data": "synthetic",
            "config": {"workload": DESCRIPTION[wl], "variant": variant, "shape": list(shape),
                       "sweeps_per_step": per_step},
            "cpu_baseline": {"value": round(value, 4), "unit": "flips/ns", "cores": cores,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(value, 4), "unit": "flips/ns", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def profile_case(which: str, L: int, n: int) -> int:
    """One small sweep case for profilers (ncu) and quick timing; prints the final exact (M, E)
    (batch: of the first lattice) and no JSON line.

    int8: 2D Metropolis L x L at beta_c, NumPy hot start seed 7; hb3: 3D heat bath L^3 at
    beta = 0.221654626, cold start; msc: 2D multi-spin Metropolis L x L at beta_c, hot start
    seed 7; sw: n Swendsen-Wang updates of a 2D int8 L x L lattice at beta_c from a cold start;
    batch: an ensemble of 2D int8 Metropolis lattices L x L, L/2 x L/2 (four each) and L/4 x L/4
    (sixteen) at temperatures 2.0 .. 2.6, device seeded starts, n sweeps with (M, E) every 10,
    through the batched kernel; batch1: one 2D int8 Metropolis lattice L x L at beta_c alone in a
    batch, device seeded start, no measurement; slab2 / mscslab2: a 2D int8 / msc Metropolis
    L x L lattice at beta_c cut into two slabs on device 0 (neighbour rows read in place),
    device seeded start."""
    from pyising_b200.backend import B200Int8, B200MultiSpin
    if which == "int8":
        sim = B200Int8((L, L), BETA_C_2D, seed=7, init="hot")
    elif which == "hb3":
        sim = B200Int8((L, L, L), 0.221654626, seed=0, algorithm="heatbath", init="cold")
    elif which == "msc":
        sim = B200MultiSpin((L, L), BETA_C_2D, seed=7, init="hot")
    elif which == "sw":
        sim = B200Int8((L, L), BETA_C_2D, seed=7, init="cold")
        sim.cluster_sweep(n)
        sim.synchronize()
        print(which, L, n, sim.observables_int())
        return 0
    elif which == "batch":
        from pyising_b200.ensemble import Ensemble, Job

        sizes = [L] + [L // 2] * 4 + [L // 4] * 16
        jobs = [Job((s, s), 1.0 / (2.0 + 0.6 * i / len(sizes)), n, seed=i, measure_every=10,
                    init="philox") for i, s in enumerate(sizes)]
        with Ensemble() as ens:
            ids = [ens.add(j) for j in jobs]
            ens.run()
            series = ens.result(ids[0]).series
        print(which, L, n, tuple(int(x) for x in series[-1]) if len(series) else None)
        return 0
    elif which in ("slab2", "mscslab2"):
        from pyising_b200.slab import SlabSimulation

        sim = SlabSimulation((L, L), BETA_C_2D, seed=7, variant="msc" if which == "mscslab2"
                             else "int8", init="philox", parts=2, devices=[0])
        sim.sweep(n)
        sim.synchronize()
        print(which, L, n, sim.observables_int())
        sim.close()
        return 0
    elif which == "batch1":
        from pyising_b200.ensemble import Ensemble, Job

        with Ensemble() as ens:
            i = ens.add(Job((L, L), BETA_C_2D, n, seed=7, init="philox", keep_lattice=True))
            ens.run()
            lat = ens.result(i).lattice
        print(which, L, n, int(lat.astype("int64").sum()))
        return 0
    else:
        raise SystemExit(f"unknown case {which!r}")
    sim.sweep(n)
    sim.synchronize()
    print(which, L, n, sim.observables_int())
    return 0


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="msc16384")
    ap.add_argument("--no-extras", dest="extras", action="store_false")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="time the library's default launch knobs instead of tuned ones")
    ap.add_argument("--no-batch", dest="batch", action="store_false",
                    help="skip the 96-lattice batched ensemble")
    ap.add_argument("--no-c4-oracle", dest="c4_oracle", action="store_false",
                    help="skip the oracle check of the 96 ensemble members (about 2 minutes)")
    ap.add_argument("--serve-jobs", type=int, default=300,
                    help="jobs of the served stream (0 = skip; the configuration has 20000)")
    ap.add_argument("--serve-baseline-jobs", type=int, default=None,
                    help="time the one-at-a-time baseline on the first N jobs only")
    ap.add_argument("--cpu-budget", type=float, default=10.0,
                    help="seconds of oracle work for cpu_baseline")
    ap.add_argument("--ref-step-s", type=float, default=2.0,
                    help="seconds of oracle work per step of --impl reference")
    ap.add_argument("--profile-case", nargs=3, metavar=("CASE", "L", "SWEEPS"),
                    help="run one small case for a profiler and exit (CASE: int8, hb3, msc, sw, "
                         "batch, batch1, slab2, mscslab2)")
    args = ap.parse_args()
    if args.profile_case:
        which, L, n = args.profile_case
        return profile_case(which, int(L), int(n))
    if args.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    rank, world, local = dist_env()
    if args.impl == "reference":
        line = main_reference(args, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0

    import torch

    torch.cuda.set_device(local)
    os.environ["PYISING_B200_DEVICE"] = str(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as td

        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                              device_id=torch.device("cuda", local))
        dist = td
    try:
        line = main_b200(args, rank, world, local, dist)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
