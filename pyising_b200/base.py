"""The simulation interface of pyising, mirrored so the backend runs without pyising installed.

Same constructor, class variables and hooks as ``pyising.backends.base.IsingSimulation``
(src/pyising/backends/base.py:19-139).  When pyising is importable,
:func:`pyising_b200.registry.register_with_pyising` also makes the backend classes subclasses of
pyising's own ``IsingSimulation``.
"""

from __future__ import annotations

from abc import ABC, abstractmethod
from typing import ClassVar

import numpy as np

from .lattice import check_shape, random_lattice, threshold_table


class IsingSimulation(ABC):
    """A checkerboard Ising Monte Carlo simulation (J = 1, h = 0, periodic).

    Parameters as in src/pyising/backends/base.py:44-51: ``shape`` ``(L, L)`` or ``(L, L, L)``,
    ``beta``, 64-bit ``seed`` (Philox key), ``algorithm`` ``"metropolis"``/``"heatbath"``,
    ``init`` ``"hot"``, ``"cold"`` or an int8 +-1 lattice.
    """

    backend: ClassVar[str] = "base"
    variant: ClassVar[str] = "base"
    dims: ClassVar[tuple[int, ...]] = (2, 3)
    algorithms: ClassVar[tuple[str, ...]] = ("metropolis", "heatbath")
    layout_multiple: ClassVar[int] = 8
    stream: ClassVar[str] = "int8"
    bytes_per_update: ClassVar[float] = 3.0
    gpu: ClassVar[bool] = True

    def __init__(self, shape, beta: float, seed: int = 0, algorithm: str = "metropolis",
                 init: str | np.ndarray = "hot") -> None:
        self.shape = check_shape(shape, self.layout_multiple)
        self.ndim = len(self.shape)
        if self.ndim not in self.dims:
            raise ValueError(f"{self.backend}/{self.variant} supports dims {self.dims}")
        if algorithm not in self.algorithms:
            raise ValueError(f"{self.backend}/{self.variant} supports {self.algorithms}")
        self.algorithm = algorithm
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.beta = float(beta)
        self.t = 0
        self.rows = int(np.prod(self.shape[:-1]))
        self.lh = self.shape[-1] // 2
        self.table = threshold_table(self.beta, self.ndim, self.algorithm)
        self._setup()
        if isinstance(init, np.ndarray):
            self.set_lattice(init)
        elif init == "cold":
            self._fill_cold()
        elif init == "hot":
            self._fill_hot()
        elif init == "philox":
            self._fill_philox()
        else:
            raise ValueError(f"unknown init {init!r}")

    @property
    def n_spins(self) -> int:
        return int(np.prod(self.shape))

    def set_beta(self, beta: float) -> None:
        """Change the temperature; keeps the configuration and the sweep counter."""
        self.beta = float(beta)
        self.table = threshold_table(self.beta, self.ndim, self.algorithm)
        self._upload_table()

    def sweep(self, n: int = 1) -> None:
        """``n`` full sweeps, colour 0 then colour 1 (src/pyising/backends/base.py:85-90)."""
        for _ in range(int(n)):
            self._half_sweep(0)
            self._half_sweep(1)
            self.t += 1

    @abstractmethod
    def _setup(self) -> None: ...

    @abstractmethod
    def _half_sweep(self, color: int) -> None: ...

    @abstractmethod
    def get_lattice(self) -> np.ndarray: ...

    @abstractmethod
    def set_lattice(self, lat: np.ndarray) -> None: ...

    def _upload_table(self) -> None:  # noqa: B027 - optional hook
        pass

    def _fill_hot(self) -> None:
        self.set_lattice(random_lattice(self.shape, self.seed))

    def _fill_cold(self) -> None:
        self.set_lattice(np.ones(self.shape, dtype=np.int8))

    def _fill_philox(self) -> None:
        raise ValueError(f"{self.backend}/{self.variant} has no device seeded start")

    def synchronize(self) -> None:  # noqa: B027 - optional hook
        pass

    def magnetization(self) -> float:
        lat = self.get_lattice()
        return float(np.sum(lat, dtype=np.int64)) / lat.size

    def energy(self) -> float:
        lat = self.get_lattice()
        e = 0
        for ax in range(lat.ndim):
            e -= int(np.sum(lat.astype(np.int64) * np.roll(lat, 1, axis=ax)))
        return e / lat.size

    def observables(self) -> tuple[float, float]:
        return self.magnetization(), self.energy()

    def device_bytes(self) -> int:
        return int(self.n_spins * self.bytes_per_update / 3.0)
