"""CPU tests of the boundary: the C-ABI library loads and exports every entry point of
include/ising_b200.h, argument validation happens before any device call, and the host-side
Python layer mirrors pyising's errors.  No compute call needs a GPU here."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "ising_b200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ising_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from pyising_b200 import build
    from pyising_b200._lib import lib as load

    build.build()
    return load()


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("ising_create", "ising_destroy", "ising_set_table", "ising_set_lattice",
                 "ising_get_lattice", "ising_upload", "ising_download", "ising_fill_cold",
                 "ising_sweep", "ising_half_sweep", "ising_observables", "ising_sync",
                 "ising_last_error", "ising_device_count"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    from pyising_b200._lib import SIGNATURES

    for name in declared_functions():
        assert hasattr(lib, name), f"{name} declared in the header but not exported"
        assert name in SIGNATURES, f"{name} has no ctypes signature"


def test_version_and_errors_without_device(lib):
    assert lib.ising_version() >= 100
    n = ctypes.c_int(-1)
    lib.ising_device_count(ctypes.byref(n))
    assert n.value >= 0


@pytest.mark.parametrize("ndim,shape,variant,alg,msg", [
    (4, (8, 8, 8), 0, 0, "2D and 3D"),
    (2, (7, 8, 0), 0, 0, "even"),
    (2, (8, 12, 0), 0, 0, "multiple of 8"),
    (2, (8, 64, 0), 1, 0, "multiple of 128"),
    (3, (8, 8, 128), 1, 0, "2D Metropolis"),
    (2, (8, 128, 0), 1, 1, "2D Metropolis"),
    (2, (8, 8, 0), 5, 0, "variant"),
    (2, (8, 8, 0), 0, 9, "algorithm"),
])
def test_create_validates_before_touching_cuda(lib, ndim, shape, variant, alg, msg):
    h = ctypes.c_void_p()
    arr = (ctypes.c_int64 * 3)(*shape)
    rc = lib.ising_create(ndim, arr, variant, alg, 0, 0, ctypes.byref(h))
    assert rc == 1  # ISING_ERR_INVALID
    assert msg in lib.ising_last_error().decode()
    assert not h.value


def test_null_handles_are_rejected(lib):
    assert lib.ising_sweep(None, 0, 1, 0, None) == 1
    assert "null" in lib.ising_last_error().decode()
    assert lib.ising_destroy(None) == 0
    assert lib.ising_observables(None, None, None) == 1


def test_check_maps_status_to_exceptions(lib):
    from pyising_b200._lib import DeviceTimeout, IsingError, check

    check(0)
    lib.ising_sweep(None, 0, 1, 0, None)
    with pytest.raises(ValueError):
        check(1)
    with pytest.raises(MemoryError):
        check(3)
    with pytest.raises(DeviceTimeout):
        check(4)
    with pytest.raises(IsingError):
        check(2)


def test_host_lattice_helpers():
    from pyising_b200.lattice import check_shape, random_lattice, threshold_table

    assert check_shape((8, 16)) == (8, 16)
    with pytest.raises(ValueError):
        check_shape((8,))
    with pytest.raises(ValueError):
        check_shape((7, 8))
    with pytest.raises(ValueError):
        check_shape((8, 64), 128)
    t = threshold_table(0.5, 2, "metropolis")
    assert t[0] == t[1] == t[2] == 0xFFFFFFFF
    assert t[3] == int(np.exp(-2.0) * 2**32) and t[4] == int(np.exp(-4.0) * 2**32)
    assert threshold_table(0.5, 3, "heatbath")[3] == 2**31
    with pytest.raises(ValueError):
        threshold_table(0.5, 2, "glauber")
    lat = random_lattice((4, 8), 1)
    assert lat.dtype == np.int8 and set(np.unique(lat)) <= {-1, 1}


def test_registry_mirrors_pyising_errors():
    import pyising_b200 as pb

    with pytest.raises(KeyError):
        pb.load("nope", "int8")
    assert set(pb.REGISTRY) == {("b200", "int8"), ("b200", "msc")}
    if not pb.available():  # no GPU in this container: the entries are unavailable
        with pytest.raises(RuntimeError, match="not available"):
            pb.create("b200", "int8", shape=(8, 8), beta=0.4)


def test_backend_class_validation_precedes_device():
    """Shape/dims/algorithm errors are raised by the host layer before any device call."""
    from pyising_b200.backend import B200Int8, B200MultiSpin

    with pytest.raises(ValueError, match="multiple of 128"):
        B200MultiSpin((8, 64), 0.4)
    with pytest.raises(ValueError, match="dims"):
        B200MultiSpin((8, 8, 128), 0.4)
    with pytest.raises(ValueError, match="supports"):
        B200MultiSpin((8, 128), 0.4, algorithm="heatbath")
    with pytest.raises(ValueError, match="even"):
        B200Int8((7, 8), 0.4)
