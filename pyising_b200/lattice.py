"""Host-side lattice conventions the backend shares with pyising (src/pyising/lattice.py).

Only what the product path needs on the host: shape validation, the integer acceptance table
(built in FP64 on the host, as the reference does) and the NumPy hot start.  The colour split and
bit packing run on the device (``csrc/layout_kernels.cu``).
"""

from __future__ import annotations

import math

import numpy as np

UINT32_MAX = 0xFFFFFFFF

#: Critical couplings (src/pyising/exact.py:11-15): 2D exact, 3D simple cubic.
BETA_C_2D = math.log(1.0 + math.sqrt(2.0)) / 2.0
TC_2D = 1.0 / BETA_C_2D


def check_shape(shape, multiple: int = 8) -> tuple[int, ...]:
    """2D or 3D, every extent even and >= 2, last extent a multiple of ``multiple``
    (src/pyising/lattice.py:25-34)."""
    shape = tuple(int(s) for s in shape)
    if len(shape) not in (2, 3):
        raise ValueError(f"only 2D and 3D lattices are supported, got shape {shape}")
    if any(s < 2 or s % 2 for s in shape):
        raise ValueError(f"all extents must be even and >= 2, got {shape}")
    if shape[-1] % multiple:
        raise ValueError(f"last extent must be a multiple of {multiple}, got {shape[-1]}")
    return shape


def prob_to_threshold(p: float) -> int:
    """Accept iff ``u32 < threshold`` (src/pyising/lattice.py:121-125)."""
    if p >= 1.0:
        return UINT32_MAX
    return min(int(math.floor(p * 2.0**32)), UINT32_MAX)


def threshold_table(beta: float, ndim: int, algorithm: str) -> np.ndarray:
    """uint32[2 ndim + 1] indexed by ``(X + 2 ndim) // 2`` (src/pyising/lattice.py:128-142).

    Metropolis: ``X = s h``, entry ``floor(exp(-2 beta X) 2^32)`` and UINT32_MAX for ``X <= 0``.
    Heat bath: ``X = h``, entry ``floor(2^32 / (1 + exp(-2 beta h)))``.
    """
    z = 2 * ndim
    xs = range(-z, z + 1, 2)
    if algorithm == "metropolis":
        vals = [UINT32_MAX if x <= 0 else prob_to_threshold(math.exp(-2.0 * beta * x)) for x in xs]
    elif algorithm == "heatbath":
        vals = [prob_to_threshold(1.0 / (1.0 + math.exp(-2.0 * beta * x))) for x in xs]
    else:
        raise ValueError(f"unknown algorithm {algorithm!r}")
    return np.array(vals, dtype=np.uint32)


def random_lattice(shape, seed: int) -> np.ndarray:
    """Infinite-temperature start, i.i.d. +-1 from ``numpy.random.default_rng(seed)``
    (src/pyising/lattice.py:93-96), so hot starts match pyising's NumPy backend exactly."""
    rng = np.random.default_rng(seed)
    return (rng.integers(0, 2, size=tuple(shape), dtype=np.int8) * 2 - 1).astype(np.int8)


def row_parity(shape) -> np.ndarray:
    """Parity of the sum of the non-x indices of every row, rows in C order
    (src/pyising/lattice.py:43-47)."""
    return (np.indices(tuple(shape[:-1])).sum(axis=0) & 1).reshape(-1)


def split_colours(lat: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The two compressed colour arrays (rows, Lx/2) of a full lattice on the host: colour c of
    a row of parity p sits at x = 2j + ((p + c) % 2) (src/pyising/lattice.py:50-61)."""
    flat = np.asarray(lat).reshape(-1, lat.shape[-1])
    odd = (row_parity(lat.shape) == 1)[:, None]
    even_x, odd_x = flat[:, 0::2], flat[:, 1::2]
    return (np.ascontiguousarray(np.where(odd, odd_x, even_x)),
            np.ascontiguousarray(np.where(odd, even_x, odd_x)))


def merge_colours(c0: np.ndarray, c1: np.ndarray, shape) -> np.ndarray:
    """The full lattice from its two compressed colour arrays (src/pyising/lattice.py:64-72)."""
    shape = tuple(shape)
    odd = (row_parity(shape) == 1)[:, None]
    flat = np.empty((c0.shape[0], shape[-1]), dtype=np.int8)
    flat[:, 0::2] = np.where(odd, c1, c0)
    flat[:, 1::2] = np.where(odd, c0, c1)
    return flat.reshape(shape)


def pack_colour(comp: np.ndarray) -> np.ndarray:
    """Packed words (rows, Lh/64) of a compressed colour array: bit b of word w is site 64w + b,
    set for +1 (src/pyising/lattice.py:75-82)."""
    rows, lh = comp.shape
    bits = (np.asarray(comp) > 0).reshape(rows, lh // 64, 64)
    return np.packbits(bits, axis=2, bitorder="little").view("<u8").reshape(rows, lh // 64)


def unpack_colour(words: np.ndarray) -> np.ndarray:
    """The compressed int8 colour array of packed words (src/pyising/lattice.py:85-90)."""
    rows, nw = words.shape
    bytes_ = np.ascontiguousarray(words).view(np.uint8).reshape(rows, 8 * nw)
    return np.unpackbits(bytes_, axis=1, bitorder="little").astype(np.int8) * 2 - 1
