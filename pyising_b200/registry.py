"""Backend registry in the shape of pyising's (src/pyising/backends/__init__.py:11-62), and the
shim that registers the B200 backend into pyising itself when pyising is importable.

``create("b200", "int8", shape=..., beta=..., seed=..., algorithm=..., init=...)`` behaves like
``pyising.create``: ``KeyError`` for an unknown key, ``RuntimeError`` when the backend cannot be
used here (library not built, no CUDA device), ``ValueError`` for a bad shape/dims/algorithm.
"""

from __future__ import annotations

import importlib
import sys
import types
from functools import cache

REGISTRY: dict[tuple[str, str], str] = {
    ("b200", "int8"): "pyising_b200.backend:B200Int8",
    ("b200", "msc"): "pyising_b200.backend:B200MultiSpin",
}
BACKENDS = ("b200",)


@cache
def load(backend: str, variant: str = "int8"):
    """The simulation class, or ``None`` if it cannot be used on this machine."""
    key = (backend, variant)
    if key not in REGISTRY:
        raise KeyError(f"unknown backend/variant {backend}/{variant}; known: {sorted(REGISTRY)}")
    mod_name, cls_name = REGISTRY[key].split(":")
    try:
        mod = importlib.import_module(mod_name)
        from ._lib import device_count

        if device_count() < 1:
            return None
    except Exception:  # noqa: BLE001 - like pyising: any failure disables the entry
        return None
    return getattr(mod, cls_name, None)


def available() -> list[tuple[str, str]]:
    return [k for k in REGISTRY if load(*k) is not None]


def create(backend: str = "b200", variant: str = "int8", **kwargs):
    """Instantiate a simulation; ``RuntimeError`` if the backend is unavailable here."""
    cls = load(backend, variant)
    if cls is None:
        raise RuntimeError(f"backend {backend}/{variant} is not available on this machine")
    return cls(**kwargs)


def register_with_pyising(name: str = "b200"):
    """Register the backend into an importable pyising as ``(name, "int8")`` and
    ``(name, "msc")``.

    * A module ``pyising.backends.<name>_backend`` is placed in ``sys.modules``; its classes
      subclass both this package's classes and ``pyising.backends.base.IsingSimulation``.
    * ``REGISTRY`` gains the two keys, ``BACKENDS`` gains ``name`` (for the CLI choices at
      src/pyising/cli.py:87) and the ``load`` cache is cleared.
    * The name is not added to ``GPU_ONLY`` (that gate needs torch,
      src/pyising/backends/__init__.py:39-43); ``load`` returns ``None`` when the library or a
      device is missing because the class import or construction raises.

    Returns the pyising.backends module.
    """
    import pyising
    import pyising.backends as pb

    from .backend import B200Int8, B200MultiSpin

    mod_name = f"{name}_backend"
    full = f"{pb.__name__}.{mod_name}"
    mod = types.ModuleType(full)
    mod.__doc__ = "B200 (sm_100a) backend registered by pyising_b200.register_with_pyising."
    base = pb.IsingSimulation
    for cls in (B200Int8, B200MultiSpin):
        sub = type(cls.__name__, (cls, base), {"backend": name, "__module__": full})
        setattr(mod, cls.__name__, sub)
    sys.modules[full] = mod
    setattr(pb, mod_name, mod)
    pb.REGISTRY[(name, "int8")] = f"{mod_name}:B200Int8"
    pb.REGISTRY[(name, "msc")] = f"{mod_name}:B200MultiSpin"
    if name not in pb.BACKENDS:
        pb.BACKENDS = tuple(pb.BACKENDS) + (name,)
        pyising.BACKENDS = pb.BACKENDS
    pb.load.cache_clear()
    return pb
