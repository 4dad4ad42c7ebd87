"""Registration into the pyising reference itself (runs only where the reference source is
present; the registry and class layout need no GPU)."""

from __future__ import annotations

import sys

import pytest
from conftest import REFERENCE_SRC

pytestmark = pytest.mark.skipif(not REFERENCE_SRC.exists(), reason="pyising source not present")


@pytest.fixture(scope="module")
def pb():
    sys.path.insert(0, str(REFERENCE_SRC))
    try:
        import pyising_b200

        yield pyising_b200.register_with_pyising()
    finally:
        sys.path.remove(str(REFERENCE_SRC))


def test_registry_keys_and_cli_choice(pb):
    import pyising

    assert pb.REGISTRY[("b200", "int8")] == "b200_backend:B200Int8"
    assert pb.REGISTRY[("b200", "msc")] == "b200_backend:B200MultiSpin"
    assert "b200" in pb.BACKENDS and "b200" in pyising.BACKENDS
    assert "b200" not in pb.GPU_ONLY


def test_classes_are_pyising_simulations(pb):
    mod = sys.modules["pyising.backends.b200_backend"]
    for name, variant, stream in (("B200Int8", "int8", "int8"),
                                  ("B200MultiSpin", "msc", "msc")):
        cls = getattr(mod, name)
        assert issubclass(cls, pb.IsingSimulation)
        assert cls.backend == "b200" and cls.variant == variant and cls.stream == stream
    assert mod.B200MultiSpin.layout_multiple == 128
    assert mod.B200MultiSpin.bytes_per_update == 3.0 / 8.0
    assert mod.B200Int8.dims == (2, 3)


def test_load_without_device_is_none_or_class(pb):
    from conftest import has_gpu

    cls = pb.load("b200", "int8")
    if has_gpu():
        assert cls is not None
    else:
        # class import works; construction is what needs the device
        with pytest.raises(Exception):  # noqa: B017
            cls((8, 8), 0.4)


def test_identity_harness_sees_the_backend(pb):
    """validate.check_identity iterates REGISTRY and matches on cls.stream."""
    keys = [k for k in pb.REGISTRY if k[0] == "b200"]
    assert {k[1] for k in keys} == {"int8", "msc"}
