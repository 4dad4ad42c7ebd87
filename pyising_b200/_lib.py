"""ctypes binding of ``libising_b200.so`` (the C ABI declared in ``include/ising_b200.h``).

There is no fallback: if the library is missing or cannot be loaded, :func:`lib` raises, and a
failing C call raises the Python exception matching pyising's own (``ValueError`` for bad
arguments as in src/pyising/lattice.py:25-34, ``MemoryError``, ``RuntimeError``).
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libising_b200.so"

OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_TIMEOUT, ERR_STATE = 0, 1, 2, 3, 4, 5
VARIANT = {"int8": 0, "msc": 1}
ALGORITHM = {"metropolis": 0, "heatbath": 1}

P = ctypes.c_void_p
I = ctypes.c_int  # noqa: E741
I64 = ctypes.c_int64
U64 = ctypes.c_uint64
U32 = ctypes.c_uint32
PI64 = ctypes.POINTER(ctypes.c_int64)
PD = ctypes.POINTER(ctypes.c_double)

# name -> (restype, argtypes); every entry point of include/ising_b200.h
SIGNATURES: dict[str, tuple] = {
    "ising_last_error": (ctypes.c_char_p, []),
    "ising_version": (I, []),
    "ising_device_count": (I, [ctypes.POINTER(I)]),
    "ising_device_name": (I, [I, ctypes.c_char_p, I]),
    "ising_create": (I, [I, PI64, I, I, U64, I, ctypes.POINTER(P)]),
    "ising_destroy": (I, [P]),
    "ising_set_stream": (I, [P, P]),
    "ising_set_table": (I, [P, P, I]),
    "ising_set_seed": (I, [P, U64]),
    "ising_set_lattice": (I, [P, P]),
    "ising_get_lattice": (I, [P, P]),
    "ising_upload": (I, [P, P, P]),
    "ising_download": (I, [P, P, P]),
    "ising_fill_cold": (I, [P]),
    "ising_sweep": (I, [P, U64, I64, I64, P]),
    "ising_half_sweep": (I, [P, I, U64]),
    "ising_observables": (I, [P, PI64, PI64]),
    "ising_sync": (I, [P]),
    "ising_device_bytes": (I, [P, PI64]),
    "ising_msc_calls_per_word": (I, [P, U64, I64, PD, PD]),
    "ising_sweep_static": (I, [I, PI64, I, I, U64, P, I, P, P, U64, I64, I64, P, P]),
    "ising_fill_philox": (I, [P, U64]),
    "ising_set_schedule": (I, [P, I, I]),
    "ising_cluster_sweep": (I, [P, U64, I64, U64, U32, P]),
    "ising_cluster_labels": (I, [P, U64, U64, U32, P, P]),
    "ising_set_knob": (I, [P, I, I]),
    "ising_get_knob": (I, [P, I, ctypes.POINTER(I)]),
    "ising_time_sweeps": (I, [P, U64, I64, ctypes.POINTER(ctypes.c_float)]),
    "ising_selftest_bounded_wait": (I, [I, ctypes.POINTER(I)]),
    "ising_batch_create": (I, [I, I64, ctypes.POINTER(P)]),
    "ising_batch_add": (I, [P, P, PI64]),
    "ising_batch_run": (I, [P, I64, PI64]),
    "ising_batch_status": (I, [P, I64, ctypes.POINTER(I), PI64]),
    "ising_batch_result": (I, [P, I64, P, P]),
    "ising_batch_release": (I, [P, I64]),
    "ising_batch_set_knob": (I, [P, I, I]),
    "ising_batch_get_knob": (I, [P, I, ctypes.POINTER(I)]),
    "ising_batch_destroy": (I, [P]),
    "ising_server_create": (I, [I, I64, ctypes.POINTER(P)]),
    "ising_server_set_knob": (I, [P, I, I]),
    "ising_server_submit": (I, [P, P, PI64]),
    "ising_server_wait": (I, [P, I64, ctypes.c_double, ctypes.POINTER(I)]),
    "ising_server_result": (I, [P, I64, P, P, PD]),
    "ising_server_release": (I, [P, I64]),
    "ising_server_status": (I, [P, PI64, PI64, PI64, PI64]),
    "ising_server_destroy": (I, [P]),
    "ising_slab_create": (I, [I, PI64, I, I, U64, I64, I64, I, ctypes.POINTER(P)]),
    "ising_slab_destroy": (I, [P]),
    "ising_slab_set_stream": (I, [P, P]),
    "ising_slab_set_table": (I, [P, P, I]),
    "ising_slab_upload": (I, [P, P, P]),
    "ising_slab_download": (I, [P, P, P]),
    "ising_slab_fill_cold": (I, [P]),
    "ising_slab_fill_philox": (I, [P, U64]),
    "ising_slab_halo": (I, [P, I, I, ctypes.POINTER(P), PI64]),
    "ising_slab_set_peer": (I, [P, I, P]),
    "ising_slab_series_reset": (I, [P, I64]),
    "ising_slab_half_sweep": (I, [P, I, U64, I64]),
    "ising_slab_half_sweep_rows": (I, [P, I, U64, I64, I64, I64]),
    "ising_slab_series_read": (I, [P, I64, P]),
    "ising_slab_observables": (I, [P, PI64, PI64]),
    "ising_slab_sync": (I, [P]),
    "ising_philox_rate": (I, [I, I, I, PD]),
    "ising_philox_range": (I, [I, U32, I64, U32, U32, U32, U32, U32, P]),
}

_lib: ctypes.CDLL | None = None


class IsingError(RuntimeError):
    """A CUDA-side failure reported by the library."""


class DeviceTimeout(IsingError, TimeoutError):
    """A bounded device-side wait expired; the kernel returned early with an error status."""


def lib() -> ctypes.CDLL:
    """Load the library once; raises if it has not been built or cannot be loaded."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH.name} is not built; run `python -m pyising_b200.build` "
                "(needs nvcc for sm_100a)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    msg = lib().ising_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str = "") -> None:
    """Raise the exception that matches a non-zero status code."""
    if rc == OK:
        return
    msg = last_error()
    if what:
        msg = f"{what}: {msg}"
    if rc == ERR_INVALID:
        raise ValueError(msg)
    if rc == ERR_NOMEM:
        raise MemoryError(msg)
    if rc == ERR_TIMEOUT:
        raise DeviceTimeout(msg)
    raise IsingError(msg)


def device_count() -> int:
    """Visible CUDA devices (0 when the driver or a device is missing)."""
    n = ctypes.c_int(0)
    lib().ising_device_count(ctypes.byref(n))
    return int(n.value)


def philox_rate(device: int = 0, calls: int = 512, repeats: int = 5) -> float:
    """Measured Philox4x32-10 throughput of the device, calls/ns (best of ``repeats``)."""
    out = ctypes.c_double()
    check(lib().ising_philox_rate(device, calls, repeats, ctypes.byref(out)), "philox_rate")
    return float(out.value)


def philox_range(q0: int, n: int, c1: int, c2: int, c3: int, k0: int, k1: int,
                 device: int = 0):
    """Device Philox over counters (q0+i, c1, c2, c3); returns a (n, 4) uint32 array."""
    import numpy as np

    out = np.zeros((n, 4), dtype=np.uint32)
    check(lib().ising_philox_range(device, q0 & 0xFFFFFFFF, n, c1 & 0xFFFFFFFF, c2 & 0xFFFFFFFF,
                                   c3 & 0xFFFFFFFF, k0 & 0xFFFFFFFF, k1 & 0xFFFFFFFF,
                                   out.ctypes.data), "philox_range")
    return out
