"""Shared fixtures.  GPU tests carry ``@pytest.mark.gpu`` and are skipped without a device."""

from __future__ import annotations

import functools
import os
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
#: The pyising source tree (its ``src`` folder), for the tests that import the reference itself;
#: set PYISING_REFERENCE_SRC to run them (skipped when unset or absent).
REFERENCE_SRC = Path(os.environ.get("PYISING_REFERENCE_SRC", "") or "/nonexistent")


@functools.cache
def has_gpu() -> bool:
    try:
        from pyising_b200._lib import device_count

        return device_count() > 0
    except Exception:  # noqa: BLE001
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="needs a CUDA GPU")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def golden(name: str) -> dict:
    with np.load(GOLDEN / name) as z:
        return {k: z[k] for k in z.files}


def unpack_lattice(bits: np.ndarray, shape) -> np.ndarray:
    n = int(np.prod(shape))
    return (np.unpackbits(bits)[:n].astype(np.int8) * 2 - 1).reshape(shape)


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle
