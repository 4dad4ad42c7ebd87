"""CPU oracle for the pyising sweep hot path — TEST INFRASTRUCTURE, never product code.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` import this package.
It wraps ``liboracle.so`` (``oracle/ising_oracle.c``, a plain-C restatement of pyising's NumPy
backend) and restates the host-side layout helpers of ``src/pyising/lattice.py`` in NumPy.

Parity is pinned against golden vectors produced by the reference itself
(``tests/golden/make_golden.py``; checked by ``tests/test_oracle_golden.py``).
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
UINT32_MAX = 0xFFFFFFFF

_lib = None


def build(force: bool = False) -> Path:
    """Compile ``liboracle.so`` with the Makefile beside this file."""
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < (
            HERE / "ising_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        P, I64, U64, U32, I = (ctypes.c_void_p, ctypes.c_int64, ctypes.c_uint64,
                               ctypes.c_uint32, ctypes.c_int)
        sigs = {
            "orc_philox": (None, [P, U32, U32, P]),
            "orc_philox_range": (None, [U64, I64, U32, U32, U32, U32, U32, P]),
            "orc_set_threads": (None, [I]),
            "orc_max_threads": (I, []),
            "orc_threshold_table": (None, [ctypes.c_double, I, I, P]),
            "orc_int8_half": (None, [P, P, I, P, I, U32, U64, P, I]),
            "orc_int8_observables": (None, [P, P, I, P, P, P]),
            "orc_int8_sweeps": (None, [P, P, I, P, U64, I64, U64, P, I, I64, P]),
            "orc_msc_half": (I64, [P, P, P, I, U32, U64, U32, U32]),
            "orc_msc_observables": (None, [P, P, P, P, P]),
            "orc_msc_sweeps": (I64, [P, P, P, U64, I64, U64, U32, U32, I64, P]),
            "orc_set_fast": (None, [I]),
            "orc_fast_active": (I, []),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def set_fast(on: bool) -> None:
    """int8 sweeps: the AVX-512 variant of the half-sweep where the host has it (default), or
    the plain restatement; the two are bit-identical."""
    lib().orc_set_fast(int(bool(on)))


def fast_active() -> bool:
    return bool(lib().orc_fast_active())


def max_threads() -> int:
    return int(lib().orc_max_threads())


def _p(a: np.ndarray) -> int:
    assert a.flags.c_contiguous
    return a.ctypes.data


# ---------------------------------------------------------------- Philox and streams -------
def split_seed(seed: int) -> tuple[int, int]:
    """philox.py:20-23."""
    seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    return seed & UINT32_MAX, seed >> 32


def philox4x32(ctr, key) -> tuple[int, int, int, int]:
    c = np.asarray([int(x) & UINT32_MAX for x in ctr], dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().orc_philox(_p(c), int(key[0]) & UINT32_MAX, int(key[1]) & UINT32_MAX, _p(out))
    return tuple(int(x) for x in out)  # type: ignore[return-value]


def philox_range(q0: int, n: int, c1: int, c2: int, c3: int, k0: int, k1: int) -> np.ndarray:
    out = np.zeros((n, 4), dtype=np.uint32)
    lib().orc_philox_range(q0, n, c1 & UINT32_MAX, c2 & UINT32_MAX, c3 & UINT32_MAX,
                           k0 & UINT32_MAX, k1 & UINT32_MAX, _p(out))
    return out


def site_uniforms(n_sites: int, sweep: int, color: int, seed: int) -> np.ndarray:
    """int8 stream (philox.py:54-64): site n takes word n%4 of Philox((n//4, t, c, 0))."""
    k0, k1 = split_seed(seed)
    return philox_range(0, n_sites // 4, sweep, color, 0, k0, k1).reshape(-1)


def word_randoms(n_words: int, sweep: int, color: int, seed: int, level_pair: int):
    """msc stream (philox.py:67-78)."""
    k0, k1 = split_seed(seed)
    r = philox_range(0, n_words, sweep, color, 1 + level_pair, k0, k1).astype(np.uint64)
    s = np.uint64(32)
    return r[:, 0] | (r[:, 1] << s), r[:, 2] | (r[:, 3] << s)


# ------------------------------------------------------------ thresholds and layouts -------
def threshold_table(beta: float, ndim: int, algorithm: str) -> np.ndarray:
    """lattice.py:121-142, through the C restatement."""
    alg = {"metropolis": 0, "heatbath": 1}[algorithm]
    out = np.zeros(2 * ndim + 1, dtype=np.uint32)
    lib().orc_threshold_table(float(beta), int(ndim), alg, _p(out))
    return out


def threshold_table_py(beta: float, ndim: int, algorithm: str) -> np.ndarray:
    """Same table in Python floats (lattice.py:121-142), to cross-check the C one."""
    def thr(p: float) -> int:
        return UINT32_MAX if p >= 1.0 else min(int(math.floor(p * 2.0**32)), UINT32_MAX)
    z = 2 * ndim
    xs = range(-z, z + 1, 2)
    if algorithm == "metropolis":
        vals = [UINT32_MAX if x <= 0 else thr(math.exp(-2.0 * beta * x)) for x in xs]
    else:
        vals = [thr(1.0 / (1.0 + math.exp(-2.0 * beta * x))) for x in xs]
    return np.array(vals, dtype=np.uint32)


def row_parity(shape) -> np.ndarray:
    """lattice.py:43-47."""
    return (np.indices(tuple(shape[:-1])).sum(axis=0) % 2).reshape(-1).astype(np.int64)


def to_compressed(lat: np.ndarray):
    """lattice.py:50-61."""
    shape = lat.shape
    lx = shape[-1]
    flat = lat.reshape(-1, lx)
    rp = row_parity(shape)
    out = []
    for c in (0, 1):
        p = (rp + c) % 2
        cols = 2 * np.arange(lx // 2)[None, :] + p[:, None]
        out.append(np.ascontiguousarray(np.take_along_axis(flat, cols, axis=1)))
    return out[0], out[1]


def from_compressed(c0: np.ndarray, c1: np.ndarray, shape) -> np.ndarray:
    """lattice.py:64-72."""
    lx = shape[-1]
    flat = np.empty((c0.shape[0], lx), dtype=c0.dtype)
    rp = row_parity(shape)
    for c, arr in ((0, c0), (1, c1)):
        p = (rp + c) % 2
        cols = 2 * np.arange(lx // 2)[None, :] + p[:, None]
        np.put_along_axis(flat, cols, arr, axis=1)
    return flat.reshape(shape)


def pack_bits(comp: np.ndarray) -> np.ndarray:
    """lattice.py:75-82: bit b of word w is compressed site 64w+b, 1 = spin +1."""
    rows, lh = comp.shape
    bits = (comp > 0).astype(np.uint8).reshape(rows, lh // 64, 64)
    return np.packbits(bits, axis=2, bitorder="little").view("<u8").reshape(rows, lh // 64)


def unpack_bits(words: np.ndarray) -> np.ndarray:
    """lattice.py:85-90."""
    rows, nw = words.shape
    b = np.unpackbits(np.ascontiguousarray(words).view(np.uint8).reshape(rows, nw * 8),
                      axis=1, bitorder="little")
    return (b.astype(np.int8) * 2 - 1).reshape(rows, nw * 64)


def random_lattice(shape, seed: int) -> np.ndarray:
    """lattice.py:93-96 (NumPy PCG64 default_rng)."""
    rng = np.random.default_rng(seed)
    return (rng.integers(0, 2, size=tuple(shape), dtype=np.int8) * 2 - 1).astype(np.int8)


def energy_magnetization(lat: np.ndarray) -> tuple[int, int]:
    """Exact integer (M, E) of a full lattice, from the definitions (lattice.py:108-118)."""
    lat64 = lat.astype(np.int64)
    e = 0
    for ax in range(lat.ndim):
        e -= int(np.sum(lat64 * np.roll(lat64, 1, axis=ax)))
    return int(lat64.sum()), e


def philox_start(shape, seed: int) -> np.ndarray:
    """The device seeded start of the product (``init="philox"``; not part of the reference):
    compressed site n of colour c is +1 iff bit n % 32 of word (n // 32) % 4 of
    Philox((n // 128, 0, c, 0xFFFFFFFF), seed) is set.  Returns the full lattice."""
    shape = tuple(int(s) for s in shape)
    rows = int(np.prod(shape[:-1]))
    sites = rows * shape[-1] // 2
    groups = (sites + 127) // 128
    k0, k1 = split_seed(seed)
    cols = []
    for c in (0, 1):
        r = philox_range(0, groups, 0, c, 0xFFFFFFFF, k0, k1)  # (groups, 4) uint32
        bits = np.unpackbits(r.astype("<u4").view(np.uint8).reshape(groups, 16), axis=1,
                             bitorder="little").reshape(-1)[:sites]
        cols.append((bits.astype(np.int8) * 2 - 1).reshape(rows, shape[-1] // 2))
    return from_compressed(cols[0], cols[1], shape)


# --------------------------------------------------------------- simulations -------------
def _shape_arr(shape) -> np.ndarray:
    return np.asarray(list(shape) + [0] * (3 - len(shape)), dtype=np.int64)


class OracleInt8:
    """int8 compressed checkerboard on the CPU (numpy_backend.py:14-51)."""

    stream = "int8"

    def __init__(self, shape, beta, seed=0, algorithm="metropolis", init="hot"):
        self.shape = tuple(int(s) for s in shape)
        self.ndim = len(self.shape)
        self.algorithm = algorithm
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.beta = float(beta)
        self.t = 0
        self.table = threshold_table(self.beta, self.ndim, algorithm)
        if isinstance(init, np.ndarray):
            self.set_lattice(init)
        elif init == "cold":
            self.set_lattice(np.ones(self.shape, np.int8))
        else:
            self.set_lattice(random_lattice(self.shape, self.seed))

    @property
    def n_spins(self) -> int:
        return int(np.prod(self.shape))

    def set_beta(self, beta: float) -> None:
        self.beta = float(beta)
        self.table = threshold_table(self.beta, self.ndim, self.algorithm)

    def set_lattice(self, lat: np.ndarray) -> None:
        c0, c1 = to_compressed(np.asarray(lat, dtype=np.int8).reshape(self.shape))
        self.c = [np.ascontiguousarray(c0), np.ascontiguousarray(c1)]

    def get_lattice(self) -> np.ndarray:
        return from_compressed(self.c[0], self.c[1], self.shape)

    def sweep(self, n: int = 1, measure_every: int = 0) -> np.ndarray | None:
        n = int(n)
        series = None
        if measure_every > 0:
            series = np.zeros((n // measure_every, 2), dtype=np.int64)
        sh = _shape_arr(self.shape)
        lib().orc_int8_sweeps(_p(self.c[0]), _p(self.c[1]), self.ndim, _p(sh), self.t, n,
                              self.seed, _p(self.table), int(self.algorithm == "heatbath"),
                              int(measure_every), _p(series) if series is not None else None)
        self.t += n
        return series

    def half_sweep(self, color: int) -> None:
        sh = _shape_arr(self.shape)
        lib().orc_int8_half(_p(self.c[color]), _p(self.c[1 - color]), self.ndim, _p(sh), color,
                            self.t & UINT32_MAX, self.seed, _p(self.table),
                            int(self.algorithm == "heatbath"))

    def observables_int(self) -> tuple[int, int]:
        m, e = ctypes.c_int64(), ctypes.c_int64()
        sh = _shape_arr(self.shape)
        lib().orc_int8_observables(_p(self.c[0]), _p(self.c[1]), self.ndim, _p(sh),
                                   ctypes.byref(m), ctypes.byref(e))
        return m.value, e.value

    def observables(self) -> tuple[float, float]:
        m, e = self.observables_int()
        return m / self.n_spins, e / self.n_spins


class OracleMultiSpin:
    """Packed 64-spin words, 2D Metropolis (numpy_backend.py:86-131)."""

    stream = "msc"

    def __init__(self, shape, beta, seed=0, algorithm="metropolis", init="hot"):
        self.shape = tuple(int(s) for s in shape)
        self.ndim = 2
        self.algorithm = "metropolis"
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.beta = float(beta)
        self.t = 0
        self.table = threshold_table(self.beta, 2, "metropolis")
        self.calls = 0
        if isinstance(init, np.ndarray):
            self.set_lattice(init)
        elif init == "cold":
            self.set_lattice(np.ones(self.shape, np.int8))
        else:
            self.set_lattice(random_lattice(self.shape, self.seed))

    @property
    def n_spins(self) -> int:
        return int(np.prod(self.shape))

    def set_beta(self, beta: float) -> None:
        self.beta = float(beta)
        self.table = threshold_table(self.beta, 2, "metropolis")

    def set_lattice(self, lat: np.ndarray) -> None:
        c0, c1 = to_compressed(np.asarray(lat, dtype=np.int8).reshape(self.shape))
        self.w = [np.ascontiguousarray(pack_bits(c0)), np.ascontiguousarray(pack_bits(c1))]

    def get_lattice(self) -> np.ndarray:
        return from_compressed(unpack_bits(self.w[0]), unpack_bits(self.w[1]), self.shape)

    def sweep(self, n: int = 1, measure_every: int = 0) -> np.ndarray | None:
        n = int(n)
        series = None
        if measure_every > 0:
            series = np.zeros((n // measure_every, 2), dtype=np.int64)
        sh = _shape_arr(self.shape)
        self.calls += lib().orc_msc_sweeps(
            _p(self.w[0]), _p(self.w[1]), _p(sh), self.t, n, self.seed, int(self.table[3]),
            int(self.table[4]), int(measure_every),
            _p(series) if series is not None else None)
        self.t += n
        return series

    def observables_int(self) -> tuple[int, int]:
        m, e = ctypes.c_int64(), ctypes.c_int64()
        sh = _shape_arr(self.shape)
        lib().orc_msc_observables(_p(self.w[0]), _p(self.w[1]), _p(sh), ctypes.byref(m),
                                  ctypes.byref(e))
        return m.value, e.value

    def observables(self) -> tuple[float, float]:
        m, e = self.observables_int()
        return m / self.n_spins, e / self.n_spins


def create(variant: str, **kw):
    return {"int8": OracleInt8, "msc": OracleMultiSpin}[variant](**kw)


def cpu_count() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1
