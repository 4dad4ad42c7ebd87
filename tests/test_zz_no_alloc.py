"""ising_sweep_static, the sweep entry point that allocates nothing, against ising_sweep.

Some callers cannot call cudaMalloc: their device memory belongs to a pool they do not control,
or their loop must not take the implicit device synchronisation of cudaMalloc/cudaFree.  They
hand ising_sweep_static their own device arrays, and the measured (M, E) sums go to a fixed
array compiled into the library.  Here the caller-owned arrays are torch CUDA tensors; the new
entry point is called through the C ABI twice in a row (the second call continues the first)
and each call's series and final spins must equal those of the existing handle-based entry point
(ising_sweep) exactly, as every result here is an integer.

This file is collected last on purpose (pytest orders files by name).
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    ("int8", (64, 256), "metropolis", 0.44),
    ("int8", (16, 24), "heatbath", 0.42),
    ("int8", (16, 16, 32), "heatbath", 0.22),
    ("msc", (128, 256), "metropolis", 0.44),
    ("msc", (40, 4096), "metropolis", 0.44),  # rows of 32 words: the strip kernel
]


def _shape_arg(shape):
    return (ctypes.c_int64 * 3)(*(list(shape) + [0] * (3 - len(shape))))


@pytest.mark.parametrize("variant,shape,algorithm,beta", CASES, ids=lambda x: str(x))
def test_static_sweep_matches_handle_entry_point(variant, shape, algorithm, beta):
    import torch

    from pyising_b200._lib import ALGORITHM, VARIANT, check, lib
    from pyising_b200.backend import B200Int8, B200MultiSpin
    from pyising_b200.lattice import random_lattice, threshold_table

    seed = 2**40 + 3
    lat = random_lattice(shape, 21)
    cls = B200MultiSpin if variant == "msc" else B200Int8
    sim = cls(shape, beta, seed=seed, algorithm=algorithm, init=lat)
    c0, c1 = sim.colour_arrays()
    # the caller's own device arrays (allocated by torch, not by this library)
    d0 = torch.from_numpy(c0.view(np.uint8).reshape(-1).copy()).cuda()
    d1 = torch.from_numpy(c1.view(np.uint8).reshape(-1).copy()).cuda()
    table = np.ascontiguousarray(threshold_table(beta, len(shape), algorithm))
    stream = torch.cuda.current_stream()
    t0 = 0
    for _call in range(2):
        got = np.zeros((4, 2), dtype=np.int64)
        rc = lib().ising_sweep_static(len(shape), _shape_arg(shape), VARIANT[variant],
                                      ALGORITHM[algorithm], seed, table.ctypes.data, len(table),
                                      d0.data_ptr(), d1.data_ptr(), t0, 20, 5, got.ctypes.data,
                                      stream.cuda_stream)
        check(rc, "ising_sweep_static")
        want = sim.sweep_measured(20, 5)
        t0 += 20
        np.testing.assert_array_equal(got, want)
        torch.cuda.synchronize()
        w0, w1 = sim.colour_arrays()
        np.testing.assert_array_equal(d0.cpu().numpy(), w0.view(np.uint8).reshape(-1))
        np.testing.assert_array_equal(d1.cpu().numpy(), w1.view(np.uint8).reshape(-1))


def test_static_sweep_rejects_more_measurements_than_the_scratch_holds():
    import torch

    from pyising_b200._lib import lib

    shape = (16, 32)
    d0 = torch.ones(16 * 16, dtype=torch.int8, device="cuda")
    d1 = torch.ones(16 * 16, dtype=torch.int8, device="cuda")
    table = np.full(5, 0xFFFFFFFF, dtype=np.uint32)
    series = np.zeros((4097, 2), dtype=np.int64)
    rc = lib().ising_sweep_static(2, _shape_arg(shape), 0, 0, 1, table.ctypes.data, 5,
                                  d0.data_ptr(), d1.data_ptr(), 0, 4097, 1, series.ctypes.data,
                                  None)
    assert rc == 1  # ISING_ERR_INVALID, before any device work
    assert "at most 4096 measurements" in lib().ising_last_error().decode()
    # a host pointer in place of a device array is refused, not dereferenced by a kernel
    host = np.ones(256, dtype=np.int8)
    rc = lib().ising_sweep_static(2, _shape_arg(shape), 0, 0, 1, table.ctypes.data, 5,
                                  host.ctypes.data, d1.data_ptr(), 0, 1, 0, None, None)
    assert rc == 1
    assert "c0" in lib().ising_last_error().decode()


def _cudart():
    """The CUDA runtime torch already loaded (found by its soname), for exact-size allocations:
    torch's caching allocator hands out pieces of larger segments."""
    import torch

    torch.cuda.init()
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]
    rt.cudaFree.argtypes = [ctypes.c_void_p]
    return rt


# shapes needing 4 MiB per colour, so the short arrays (2 MiB) stay short whatever granularity
# the driver rounds allocations to
@pytest.mark.parametrize("variant,shape", [("int8", (4096, 2048)), ("msc", (8192, 8192)),
                                           ("int8", (64, 64, 2048))], ids=str)
def test_static_sweep_rejects_arrays_shorter_than_the_shape(variant, shape):
    """A colour array whose allocation ends before rows x (bytes per row) is refused before any
    launch, naming the array; an allocation of exactly the needed size is accepted."""
    from pyising_b200._lib import VARIANT, lib

    rows = int(np.prod(shape[:-1]))
    need = rows * shape[-1] // 2 if variant == "int8" else rows * shape[-1] // 128 * 8
    rt = _cudart()
    ptrs = []
    try:
        for size in (need, need // 2):
            p = ctypes.c_void_p()
            assert rt.cudaMalloc(ctypes.byref(p), size) == 0
            ptrs.append(p.value)
        full, short = ptrs
        table = np.full(2 * len(shape) + 1, 0xFFFFFFFF, dtype=np.uint32)
        for c0, c1, bad in ((short, full, "c0"), (full, short, "c1")):
            rc = lib().ising_sweep_static(len(shape), _shape_arg(shape), VARIANT[variant], 0, 1,
                                          table.ctypes.data, len(table), c0, c1, 0, 1, 0, None,
                                          None)
            assert rc == 1, bad  # ISING_ERR_INVALID
            msg = lib().ising_last_error().decode()
            assert msg.startswith(bad) and "needs" in msg, msg
        # exactly the needed bytes (both arrays the same buffer: zero sweeps, nothing runs)
        rc = lib().ising_sweep_static(len(shape), _shape_arg(shape), VARIANT[variant], 0, 1,
                                      table.ctypes.data, len(table), full, full, 0, 0, 0, None,
                                      None)
        assert rc == 0, lib().ising_last_error().decode()
    finally:
        for p in ptrs:
            rt.cudaFree(ctypes.c_void_p(p))


def test_static_sweep_rejects_arrays_of_another_device():
    """Arrays on a GPU other than the current one are refused before any launch."""
    import torch

    from pyising_b200._lib import lib

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    shape = (16, 32)
    d0 = torch.ones(256, dtype=torch.int8, device="cuda:1")
    d1 = torch.ones(256, dtype=torch.int8, device="cuda:1")
    table = np.full(5, 0xFFFFFFFF, dtype=np.uint32)
    with torch.cuda.device(0):
        rc = lib().ising_sweep_static(2, _shape_arg(shape), 0, 0, 1, table.ctypes.data, 5,
                                      d0.data_ptr(), d1.data_ptr(), 0, 1, 0, None, None)
    assert rc == 1
    assert "lives on device 1" in lib().ising_last_error().decode()
