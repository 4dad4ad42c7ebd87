"""The B200 backend classes: ``B200Int8`` (int8 checkerboard, 2D/3D, Metropolis and heat bath)
and ``B200MultiSpin`` (64 spins per uint64, 2D Metropolis).

They implement the pyising simulation interface (src/pyising/backends/base.py:19-139) on top of
the C ABI of ``libising_b200.so``; every sweep, measurement and layout conversion runs in the
sm_100a kernels, and ``sweep(n)`` issues all ``2n`` half-sweeps in one C call.  Results are
bit-identical to pyising's NumPy backend (src/pyising/backends/numpy_backend.py) for the same
seed and start.
"""

from __future__ import annotations

import ctypes
import math
import os
from typing import ClassVar

import numpy as np

from . import _lib
from ._lib import check, lib
from .base import IsingSimulation


def default_device() -> int:
    return int(os.environ.get("PYISING_B200_DEVICE", "0"))


class _B200Simulation(IsingSimulation):
    backend: ClassVar[str] = "b200"
    gpu: ClassVar[bool] = True
    _variant_code: ClassVar[int] = 0

    def _setup(self) -> None:
        self._h = ctypes.c_void_p()
        shape = (ctypes.c_int64 * 3)(*(list(self.shape) + [0] * (3 - self.ndim)))
        self.device = default_device()
        check(lib().ising_create(self.ndim, shape, self._variant_code,
                                 _lib.ALGORITHM[self.algorithm], self.seed, self.device,
                                 ctypes.byref(self._h)), "create")
        self._upload_table()
        self.cluster_t = 0
        # launch knobs picked by the autotuner for this GPU and shape, if any (speed only)
        from . import autotune

        autotune.apply_cached(self)

    def __del__(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().ising_destroy(h)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
            self._h = None

    # ---- hooks -------------------------------------------------------------------------------
    def _upload_table(self) -> None:
        tab = np.ascontiguousarray(self.table, dtype=np.uint32)
        check(lib().ising_set_table(self._h, tab.ctypes.data, len(tab)), "set_table")

    def _half_sweep(self, color: int) -> None:
        check(lib().ising_half_sweep(self._h, int(color), self.t), "half_sweep")

    def _fill_cold(self) -> None:
        check(lib().ising_fill_cold(self._h), "fill_cold")

    def _fill_philox(self) -> None:
        """``init="philox"``: the device seeded start of ``ising_fill_philox`` keyed by the
        simulation's seed (no host work; not pyising's NumPy hot start)."""
        check(lib().ising_fill_philox(self._h, self.seed), "fill_philox")

    def set_lattice(self, lat: np.ndarray) -> None:
        full = np.ascontiguousarray(np.asarray(lat, dtype=np.int8).reshape(self.shape))
        check(lib().ising_set_lattice(self._h, full.ctypes.data), "set_lattice")

    def get_lattice(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.int8)
        check(lib().ising_get_lattice(self._h, out.ctypes.data), "get_lattice")
        return out

    def synchronize(self) -> None:
        check(lib().ising_sync(self._h), "sync")

    # ---- the hot path -----------------------------------------------------------------------
    def sweep(self, n: int = 1) -> None:
        """``n`` full sweeps in one C call (asynchronous; ``self.t`` advances by ``n``)."""
        n = int(n)
        if n <= 0:
            return
        check(lib().ising_sweep(self._h, self.t, n, 0, None), "sweep")
        self.t += n

    def sweep_measured(self, n: int, every: int) -> np.ndarray:
        """``n`` sweeps with exact ``(M, E)`` after every ``every``-th one, measured inside the
        colour-1 half-sweep; returns an int64 array of shape ``(n // every, 2)``.  This is the
        device-resident form of pyising.observables.sample (src/pyising/observables.py:61-74)."""
        n, every = int(n), int(every)
        if every <= 0:
            raise ValueError("every must be positive")
        out = np.zeros((n // every, 2), dtype=np.int64)
        check(lib().ising_sweep(self._h, self.t, n, every, out.ctypes.data), "sweep")
        self.t += n
        return out

    def observables_int(self) -> tuple[int, int]:
        """Exact integers ``(M, E)``: ``M = sum s``, ``E = -sum_<ij> s_i s_j``."""
        m, e = ctypes.c_int64(), ctypes.c_int64()
        check(lib().ising_observables(self._h, ctypes.byref(m), ctypes.byref(e)), "observables")
        return int(m.value), int(e.value)

    def observables(self) -> tuple[float, float]:
        """``(m, e)`` per spin, as pyising's GPU backends return them."""
        m, e = self.observables_int()
        return m / self.n_spins, e / self.n_spins

    def magnetization(self) -> float:
        return self.observables()[0]

    def energy(self) -> float:
        return self.observables()[1]

    def device_bytes(self) -> int:
        b = ctypes.c_int64()
        check(lib().ising_device_bytes(self._h, ctypes.byref(b)), "device_bytes")
        return int(b.value)

    def set_seed(self, seed: int) -> None:
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        check(lib().ising_set_seed(self._h, self.seed), "set_seed")

    SCHEDULES = {"auto": 0, "launches": 1, "graphs": 2, "persistent": 3, "temporal": 4}

    def set_schedule(self, schedule: str = "auto", test_mute_band: int = -1) -> None:
        """How sweeps are issued: ``"auto"``, ``"launches"`` (one kernel per half-sweep),
        ``"graphs"`` (replayed CUDA graphs), ``"persistent"`` (one cooperative launch for all
        sweeps; 2D int8) or ``"temporal"`` (graphs of launches that each run two sweeps on
        shared-memory tiles; small 2D int8 lattices).  Results are identical.  ``test_mute_band`` >= 0 is a test hook that
        makes one band of a persistent run stop publishing, so the run reports a time-out."""
        check(lib().ising_set_schedule(self._h, self.SCHEDULES[schedule], int(test_mute_band)),
              "set_schedule")

    def set_stream(self, stream: int | None) -> None:
        """Issue work on an existing CUDA stream (e.g. ``torch.cuda.current_stream().cuda_stream``)."""
        check(lib().ising_set_stream(self._h, stream or None), "set_stream")

    # ---- checkpoint / resume -----------------------------------------------------------------
    def colour_arrays(self, out: tuple[np.ndarray, np.ndarray] | None = None
                      ) -> tuple[np.ndarray, np.ndarray]:
        """The two colour arrays in their device layout (compressed int8 or packed uint64).
        ``out``: two C-contiguous arrays of that shape and dtype to fill (e.g. pinned host
        buffers reused across calls); new arrays otherwise."""
        if out is None:
            a, b = self._colour_buffers()
        else:
            a, b = (self._checked_buffer(x) for x in out)
        check(lib().ising_download(self._h, a.ctypes.data, b.ctypes.data), "download")
        return a, b

    def load_colour_arrays(self, c0: np.ndarray, c1: np.ndarray) -> None:
        """Uploads two colour arrays in the device layout; C-contiguous arrays of the right
        shape and dtype are read in place (no host copy)."""
        shape, dtype = self._colour_spec()
        src = []
        for x in (c0, c1):
            x = np.asarray(x)
            if x.dtype != dtype or x.shape != shape or not x.flags.c_contiguous:
                x = np.ascontiguousarray(x, dtype=dtype).reshape(shape)
            src.append(x)
        check(lib().ising_upload(self._h, src[0].ctypes.data, src[1].ctypes.data), "upload")

    def _colour_buffers(self):
        shape, dtype = self._colour_spec()
        return np.empty(shape, dtype), np.empty(shape, dtype)

    def _checked_buffer(self, x: np.ndarray) -> np.ndarray:
        shape, dtype = self._colour_spec()
        if x.dtype != dtype or x.shape != shape or not x.flags.c_contiguous:
            raise ValueError(f"colour buffer must be C-contiguous {dtype} of shape {shape}")
        return x

    def state(self) -> dict:
        """Everything needed to resume bit-exactly: the RNG is keyed by (site, t, colour, seed)."""
        c0, c1 = self.colour_arrays()
        return {"shape": self.shape, "variant": self.variant, "algorithm": self.algorithm,
                "beta": self.beta, "seed": self.seed, "t": self.t, "c0": c0, "c1": c1}

    @classmethod
    def from_state(cls, st: dict) -> _B200Simulation:
        sim = cls(st["shape"], st["beta"], seed=st["seed"], algorithm=st["algorithm"],
                  init="cold")
        sim.load_colour_arrays(st["c0"], st["c1"])
        sim.t = int(st["t"])
        return sim


class B200Int8(_B200Simulation):
    """int8 compressed checkerboard (2D/3D, Metropolis and heat bath)."""

    variant = "int8"
    stream = "int8"
    _variant_code = 0

    def _colour_spec(self):
        return (self.rows, self.lh), np.dtype(np.int8)


    # ---- cluster updates (Swendsen-Wang on the device) ------------------------------------
    def bond_threshold(self) -> int:
        """Integer threshold of the bond probability p = 1 - exp(-2 beta)."""
        from .lattice import prob_to_threshold

        return prob_to_threshold(1.0 - math.exp(-2.0 * self.beta)) if self.beta > 0 else 0

    def cluster_sweep(self, n: int = 1, seed: int | None = None,
                      measure: bool = False) -> np.ndarray | None:
        """``n`` Swendsen-Wang updates (steps ``self.cluster_t`` ..), keyed by ``seed`` (the
        simulation's seed by default).  The Metropolis/heat-bath sweep counter ``t`` is not
        touched; the cluster step counter ``cluster_t`` advances by ``n``.  With ``measure``,
        returns the exact ``(M, E)`` after every step as an ``(n, 2)`` int64 array."""
        n = int(n)
        if n <= 0:
            return np.zeros((0, 2), np.int64) if measure else None
        key = self.seed if seed is None else int(seed) & 0xFFFFFFFFFFFFFFFF
        out = np.zeros((n, 2), np.int64) if measure else None
        check(lib().ising_cluster_sweep(self._h, self.cluster_t, n, key, self.bond_threshold(),
                                        out.ctypes.data if measure else None), "cluster_sweep")
        self.cluster_t += n
        return out

    def cluster_labels(self, step: int = 0, seed: int | None = None) -> tuple[np.ndarray,
                                                                              np.ndarray]:
        """One Swendsen-Wang labeling without flips: (labels (2, rows, Lx/2) int32 = each
        site's cluster root, bonds (rows, Lx/2) uint8 = active bonds of each colour-0 site)."""
        key = self.seed if seed is None else int(seed) & 0xFFFFFFFFFFFFFFFF
        labels = np.empty((2, self.rows, self.lh), np.int32)
        bonds = np.empty((self.rows, self.lh), np.uint8)
        check(lib().ising_cluster_labels(self._h, int(step), key, self.bond_threshold(),
                                         labels.ctypes.data, bonds.ctypes.data),
              "cluster_labels")
        return labels, bonds


class B200MultiSpin(_B200Simulation):
    """Multi-spin coding: 64 spins per uint64, bit-sliced neighbour count, lazy comparison."""

    variant = "msc"
    dims = (2,)
    algorithms = ("metropolis",)
    layout_multiple = 128
    stream = "msc"
    bytes_per_update = 3.0 / 8.0
    _variant_code = 1

    def _colour_spec(self):
        return (self.rows, self.lh // 64), np.dtype(np.uint64)

    def philox_calls_per_word(self, sweeps: int = 2, warp: bool = False) -> float:
        """Mean (or per-warp maximum) Philox calls per word; advances the lattice like
        ``sweep(sweeps)`` (src/pyising/backends/cupy_backend.py:137-144)."""
        mean, wmax = ctypes.c_double(), ctypes.c_double()
        check(lib().ising_msc_calls_per_word(self._h, self.t, int(sweeps), ctypes.byref(mean),
                                             ctypes.byref(wmax)), "calls_per_word")
        self.t += int(sweeps)
        return float(wmax.value if warp else mean.value)
