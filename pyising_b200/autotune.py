"""Autotuner of the launch knobs, per (GPU, variant, algorithm, lattice shape).

The sweep kernels have knobs that change speed but never results (the random numbers are keyed
by site, sweep and colour, and every schedule visits the same sites with the same rule):

* ``band``          int8: rows of one plane a thread walks while the opposite colour's rows
                    slide through its registers (the halo reuse depth); 0 = occupancy default;
* ``chunk_width``   int8: bytes per thread and row, 16, 8 or 4 (4, 2 or 1 words of 4 sites);
* ``blocks_per_sm`` grid size in blocks of 256 threads per SM;
* ``msc_kernel``    msc: schedule: word ranges per warp, or 32-word column strips walked down a
                    band of rows with 4 or 3 Philox blocks per word at intake and registers
                    bounded for 2, 3 or 4 resident blocks;
* ``msc_waves``     msc: warps per resident warp (ranges or strip bands of the work-stack kernels);
* ``graph_chunk``   sweeps per captured CUDA graph of an unmeasured run;
* ``schedule``      ``"auto"`` (graphs), ``"launches"``, ``"persistent"`` or ``"temporal"``
                    (2D int8: two sweeps per launch on shared-memory tiles).

:func:`tune` measures them on a scratch lattice of the given shape (device seeded start, CUDA
events on the simulation's stream) by coordinate descent from the defaults, and stores the best
configuration in a JSON cache (``$PYISING_B200_TUNE_CACHE``, else
``~/.cache/pyising_b200/tune.json``) keyed by the GPU, variant, algorithm and shape.  New
simulations pick up a cached configuration automatically (:func:`apply_cached`); with
``PYISING_B200_AUTOTUNE=1`` a shape without one is tuned on first use.

The reference has no counterpart: its CUDA kernels use one fixed launch shape
(src/pyising/backends/cupy_backend.py:68-72,129-135).
"""

from __future__ import annotations

import ctypes
import json
import math
import os
import threading
import time
from pathlib import Path

from . import _lib
from ._lib import check, lib

KNOBS = {"band": 1, "chunk_width": 2, "blocks_per_sm": 3, "msc_waves": 4, "graph_chunk": 5,
         "msc_kernel": 9}
DEFAULTS = {"band": 0, "chunk_width": 16, "blocks_per_sm": 8, "msc_waves": 1, "graph_chunk": 32,
            "msc_kernel": 0, "schedule": "auto"}

_lock = threading.Lock()
_cache_mem: dict[Path, dict] = {}  # cache file contents by path, read once per process


def cache_path() -> Path:
    env = os.environ.get("PYISING_B200_TUNE_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "pyising_b200" / "tune.json"


_names: dict[int, str] = {}


def device_name(device: int = 0) -> str:
    if device not in _names:
        buf = ctypes.create_string_buffer(256)
        check(lib().ising_device_name(int(device), buf, len(buf)), "device_name")
        _names[device] = buf.value.decode()
    return _names[device]


def key(device: str, variant: str, algorithm: str, shape) -> str:
    return f"{device}|{variant}|{algorithm}|{'x'.join(str(int(s)) for s in shape)}"


def search_space(variant: str, shape, algorithm: str = "metropolis") -> dict[str, list]:
    """Values tried per knob (the first one is the default)."""
    shape = tuple(int(s) for s in shape)
    lh = shape[-1] // 2
    space: dict[str, list] = {}
    if variant == "int8":
        space["band"] = [0, 1, 2, 4, 8, 16]
        space["chunk_width"] = [16, 4] + ([8] if lh % 8 == 0 else [])
    else:
        # 0 = automatic; 1 = word ranges; 2..7 = column strips with (intake blocks, register
        # bound) variants, where every row holds whole 32-word strips
        space["msc_kernel"] = [0, 1] + ([2, 3, 4, 5, 6, 7] if (lh // 64) % 32 == 0 else [])
        space["msc_waves"] = [1, 2, 4]
    space["blocks_per_sm"] = [8, 4, 16]
    if variant == "int8" and len(shape) == 2:
        space["schedule"] = ["auto", "launches", "persistent"]
        if lh % 16 == 0 and shape[0] % 8 == 0 and shape[0] >= 16 and 32 * lh <= 96 * 1024:
            space["schedule"].append("temporal")
    else:
        space["schedule"] = ["auto", "launches"]
    space["graph_chunk"] = [32, 8, 128]
    return space


# ------------------------------------------------------------------------------ cache -------
def _read(p: Path) -> dict:
    try:
        data = json.loads(p.read_text())
    except (OSError, ValueError):
        return {}
    return data if isinstance(data, dict) else {}


def load_cache(path: Path | None = None) -> dict[str, dict]:
    p = Path(path) if path is not None else cache_path()
    with _lock:
        if p not in _cache_mem:
            _cache_mem[p] = _read(p)
        return _cache_mem[p]


def save_entry(k: str, entry: dict, path: Path | None = None) -> None:
    """Adds one entry to the cache file (read-modify-write, replaced atomically)."""
    p = Path(path) if path is not None else cache_path()
    with _lock:
        data = _read(p)
        data[k] = entry
        p.parent.mkdir(parents=True, exist_ok=True)
        tmp = p.with_suffix(p.suffix + f".{os.getpid()}.tmp")
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        os.replace(tmp, p)
        _cache_mem[p] = data


def lookup(k: str, path: Path | None = None) -> dict | None:
    entry = load_cache(path).get(k)
    return entry.get("config") if isinstance(entry, dict) else None


# ------------------------------------------------------------------------- knobs -----------
def apply(sim, config: dict) -> None:
    """Sets the knobs of ``config`` on a simulation (unknown or inapplicable keys are skipped:
    a configuration tuned for int8 carries no msc knob and vice versa)."""
    space = search_space(sim.variant, sim.shape, sim.algorithm)
    for name, value in config.items():
        if name == "schedule":
            if value in space["schedule"]:
                sim.set_schedule(value)
        elif name in KNOBS and name in space:
            check(lib().ising_set_knob(sim._h, KNOBS[name], int(value)), f"set_knob {name}")


def current(sim) -> dict:
    out = {}
    for name in search_space(sim.variant, sim.shape, sim.algorithm):
        if name in KNOBS:
            v = ctypes.c_int()
            check(lib().ising_get_knob(sim._h, KNOBS[name], ctypes.byref(v)), "get_knob")
            out[name] = int(v.value)
    return out


def apply_cached(sim) -> bool:
    """Applies the cached configuration for the simulation's key, tuning first when
    ``PYISING_B200_AUTOTUNE=1`` and none is cached.  Returns whether one was applied."""
    if not cache_path().exists() and os.environ.get("PYISING_B200_AUTOTUNE") != "1":
        return False
    k = key(device_name(sim.device), sim.variant, sim.algorithm, sim.shape)
    cfg = lookup(k)
    if cfg is None and os.environ.get("PYISING_B200_AUTOTUNE") == "1":
        cfg = tune(sim.variant, sim.shape, sim.algorithm, sim.beta, device=sim.device)["config"]
    if cfg is None:
        return False
    apply(sim, cfg)
    return True


# ------------------------------------------------------------------------- tuning ----------
def _time(sim, sweeps: int, reps: int) -> float:
    """Best of ``reps`` device-timed runs of ``sweeps`` sweeps, in flips/ns."""
    best = math.inf
    ms = ctypes.c_float()
    for _ in range(reps):
        check(lib().ising_time_sweeps(sim._h, sim.t, int(sweeps), ctypes.byref(ms)),
              "time_sweeps")
        sim.t += int(sweeps)
        best = min(best, float(ms.value))
    return sim.n_spins * sweeps / (best * 1e6)


def tune(variant: str, shape, algorithm: str = "metropolis", beta: float | None = None,
         device: int = 0, target_ms: float = 20.0, reps: int = 3, save: bool = True,
         path: Path | None = None) -> dict:
    """Coordinate-descent search over :func:`search_space` on a scratch lattice; returns
    ``{"config": best knobs, "flips_per_ns": its rate, "default_flips_per_ns": ..., "trials":
    [(config, rate), ...]}`` and stores it in the cache when ``save``."""
    from .backend import B200Int8, B200MultiSpin
    from .lattice import BETA_C_2D

    shape = tuple(int(s) for s in shape)
    if beta is None:
        beta = BETA_C_2D if len(shape) == 2 else 0.221654626
    cls = B200MultiSpin if variant == "msc" else B200Int8
    prev = os.environ.get("PYISING_B200_AUTOTUNE")
    os.environ["PYISING_B200_AUTOTUNE"] = "0"  # the scratch lattice must not recurse
    try:
        sim = cls(shape, beta, seed=12345, algorithm=algorithm, init="philox")
    finally:
        if prev is None:
            os.environ.pop("PYISING_B200_AUTOTUNE", None)
        else:
            os.environ["PYISING_B200_AUTOTUNE"] = prev
    space = search_space(variant, shape, algorithm)
    cfg = {k: DEFAULTS[k] for k in space}
    apply(sim, cfg)
    # sweeps per timed run: about target_ms at a first estimate of the rate, and at least two
    # of the longest graph chunk tried, so that the graph schedules are what gets timed
    _time(sim, 64, 1)  # warm-up: module loading, first graph captures
    probe = _time(sim, 64, 1)
    sweeps = int(target_ms * 1e6 * probe / sim.n_spins)
    sweeps = min(max(sweeps, 2 * max(space.get("graph_chunk", [32]))), 4096)
    t_start = time.perf_counter()
    best_rate = _time(sim, sweeps, reps)
    default_rate = best_rate
    trials = [(dict(cfg), best_rate)]
    for name, values in space.items():
        for v in values:
            if v == cfg[name]:
                continue
            trial = dict(cfg, **{name: v})
            try:
                apply(sim, trial)
            except ValueError:
                continue
            rate = _time(sim, sweeps, reps)
            trials.append((trial, rate))
            if rate > best_rate:
                best_rate, cfg = rate, trial
        apply(sim, cfg)
    result = {"config": cfg, "flips_per_ns": best_rate, "default_flips_per_ns": default_rate,
              "sweeps_per_trial": sweeps, "trials": trials,
              "seconds": time.perf_counter() - t_start}
    if save:
        entry = {"config": cfg, "flips_per_ns": round(best_rate, 2),
                 "default_flips_per_ns": round(default_rate, 2), "when": time.time()}
        save_entry(key(device_name(device), variant, algorithm, shape), entry, path)
    del sim
    return result


BATCH_SPACE = {"band": [8, 4, 2, 16], "items_per_slot": [6, 3, 12], "graph_chunk": [32, 8, 0]}


def tune_ensemble(jobs, sweeps: int = 200, device: int = 0) -> dict:
    """Coordinate descent over the batch knobs (:data:`BATCH_SPACE`: band cap, items per
    resident block, sweeps per replayed graph chunk) on copies of ``jobs`` shortened to
    ``sweeps`` sweeps (same shapes, variants and temperatures, so the same kernel
    classes and work lists); returns ``{"config": ..., "flips_per_ns": ..., "trials": ...}``."""
    import dataclasses

    from .ensemble import Ensemble

    short = [dataclasses.replace(j, sweeps=min(j.sweeps, sweeps)) for j in jobs]

    def run(cfg: dict) -> float:
        with Ensemble(device=device) as ens:
            for name, v in cfg.items():
                ens.set_knob(name, v)
            ids = [ens.add(j) for j in short]
            ens.run(2)  # admission, first work list and module loading outside the timing
            # the flips still to do: the first sweep (two epochs) already ran
            flips = sum(j.n_spins * (j.sweeps - ens.status(i)[1])
                        for j, i in zip(short, ids, strict=True))
            t0 = time.perf_counter()
            ens.run()
            dt = time.perf_counter() - t0
        return flips / (dt * 1e9)

    cfg = {k: v[0] for k, v in BATCH_SPACE.items()}
    best = run(cfg)
    trials = [(dict(cfg), best)]
    for name, values in BATCH_SPACE.items():
        for v in values[1:]:
            trial = dict(cfg, **{name: v})
            rate = run(trial)
            trials.append((trial, rate))
            if rate > best:
                best, cfg = rate, trial
    return {"config": cfg, "flips_per_ns": best, "default_flips_per_ns": trials[0][1],
            "trials": trials}


def main(argv: list[str] | None = None) -> int:
    """``python -m pyising_b200.autotune int8|msc L [L [L]] [--algorithm heatbath]``"""
    import argparse

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("variant", choices=sorted(_lib.VARIANT))
    ap.add_argument("shape", type=int, nargs="+")
    ap.add_argument("--algorithm", default="metropolis", choices=sorted(_lib.ALGORITHM))
    ap.add_argument("--beta", type=float, default=None)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    res = tune(args.variant, args.shape, args.algorithm, args.beta, device=args.device)
    print(json.dumps({k: v for k, v in res.items() if k != "trials"}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
