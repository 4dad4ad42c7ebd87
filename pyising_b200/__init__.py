"""pyising_b200 — a B200-native (sm_100a) backend for pyising's sweep hot path.

Drop-in for pyising's ``create(backend, variant, ...)`` / ``sim.sweep(n)`` /
``sim.observables()`` API (src/pyising/backends/__init__.py:57-62, base.py:19-139):

    import pyising_b200 as pb
    sim = pb.create("b200", "int8", shape=(1024, 1024), beta=pb.BETA_C_2D, seed=1, init="hot")
    sim.sweep(1000)
    M, E = sim.observables_int()

or, with pyising installed, ``pyising_b200.register_with_pyising()`` and then
``pyising.create("b200", "msc", ...)``.  Every sweep runs in hand-written CUDA kernels behind
the C ABI of ``libising_b200.so`` (``include/ising_b200.h``); there is no CPU fallback.
"""

from .lattice import BETA_C_2D, TC_2D, check_shape, random_lattice, threshold_table
from .registry import BACKENDS, REGISTRY, available, create, load, register_with_pyising

__version__ = "0.1.0"

__all__ = ["BACKENDS", "REGISTRY", "available", "create", "load", "register_with_pyising",
           "BETA_C_2D", "TC_2D", "check_shape", "random_lattice", "threshold_table",
           "__version__"]
