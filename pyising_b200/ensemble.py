"""Batched ensembles and continuous-batching serving on one GPU.

The reference runs one lattice per launch (``create`` → ``sweep`` in a Python loop,
bench/run.py:121-142 and observables.sample, src/pyising/observables.py:61-74).  Here many
independent lattices of uneven size, dimension, variant and temperature advance together: every
launch updates one colour of every active lattice over a (lattice, tile) work list
(``csrc/batch.cu``), measurements stay on the device, and each lattice is bit-identical to
running it alone, because its random numbers depend only on (site, sweep, colour, seed).

* :class:`Ensemble` — add jobs, ``run()`` until all are done, read results.
* :class:`Server` — a serving loop on its own host thread: ``submit`` from any thread while
  others run; jobs are admitted by a device-memory budget at sweep boundaries.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, lib
from .lattice import check_shape, random_lattice, threshold_table

INIT_COLD, INIT_PHILOX, INIT_LATTICE = 0, 1, 2
PENDING, ACTIVE, FINISHING, DONE = 0, 1, 2, 3
STATE_NAMES = {PENDING: "pending", ACTIVE: "active", FINISHING: "finishing", DONE: "done"}


class IsingJobStruct(ctypes.Structure):
    """``ising_job`` of include/ising_b200.h."""

    _fields_ = [
        ("ndim", ctypes.c_int),
        ("shape", ctypes.c_int64 * 3),
        ("variant", ctypes.c_int),
        ("algorithm", ctypes.c_int),
        ("seed", ctypes.c_uint64),
        ("table", ctypes.c_uint32 * 7),
        ("table_n", ctypes.c_int),
        ("t0", ctypes.c_uint64),
        ("n_sweeps", ctypes.c_int64),
        ("measure_every", ctypes.c_int64),
        ("init", ctypes.c_int),
        ("lattice", ctypes.c_void_p),
        ("keep_lattice", ctypes.c_int),
    ]


@dataclass
class Job:
    """One lattice run: ``sweeps`` sweeps from sweep counter ``t0`` with ``(M, E)`` after every
    ``measure_every``-th sweep.  ``init`` is ``"hot"`` (pyising's NumPy start, seeded by
    ``seed``), ``"cold"``, ``"philox"`` (the device seeded start) or an int8 lattice."""

    shape: tuple
    beta: float
    sweeps: int
    seed: int = 0
    variant: str = "int8"
    algorithm: str = "metropolis"
    measure_every: int = 0
    init: object = "hot"
    t0: int = 0
    keep_lattice: bool = False
    table: np.ndarray | None = field(default=None, repr=False)

    def __post_init__(self) -> None:
        if self.variant not in _lib.VARIANT:
            raise ValueError(f"unknown variant {self.variant!r}")
        self.shape = check_shape(self.shape, 128 if self.variant == "msc" else 8)
        if self.variant == "msc" and (len(self.shape) != 2 or self.algorithm != "metropolis"):
            raise ValueError("msc supports 2D Metropolis only")
        if self.table is None:
            self.table = threshold_table(self.beta, len(self.shape), self.algorithm)

    @property
    def n_spins(self) -> int:
        return int(np.prod(self.shape))

    @property
    def n_measurements(self) -> int:
        return self.sweeps // self.measure_every if self.measure_every > 0 else 0

    def to_struct(self) -> tuple[IsingJobStruct, np.ndarray | None]:
        s = IsingJobStruct()
        s.ndim = len(self.shape)
        for i, v in enumerate(self.shape):
            s.shape[i] = v
        s.variant = _lib.VARIANT[self.variant]
        s.algorithm = _lib.ALGORITHM[self.algorithm]
        s.seed = int(self.seed) & 0xFFFFFFFFFFFFFFFF
        tab = np.ascontiguousarray(self.table, dtype=np.uint32)
        for i, v in enumerate(tab):
            s.table[i] = int(v)
        s.table_n = len(tab)
        s.t0 = int(self.t0) & 0xFFFFFFFFFFFFFFFF
        s.n_sweeps = int(self.sweeps)
        s.measure_every = int(self.measure_every)
        s.keep_lattice = int(bool(self.keep_lattice))
        keep = None
        if isinstance(self.init, np.ndarray):
            keep = np.ascontiguousarray(np.asarray(self.init, dtype=np.int8).reshape(self.shape))
            s.init = INIT_LATTICE
        elif self.init == "hot":
            keep = random_lattice(self.shape, self.seed)
            s.init = INIT_LATTICE
        elif self.init == "cold":
            s.init = INIT_COLD
        elif self.init == "philox":
            s.init = INIT_PHILOX
        else:
            raise ValueError(f"unknown init {self.init!r}")
        s.lattice = keep.ctypes.data if keep is not None else None
        return s, keep


@dataclass
class Result:
    series: np.ndarray            # (n_measurements, 2) int64: exact (M, E)
    lattice: np.ndarray | None    # final full lattice if keep_lattice
    latency_s: float | None = None


class Ensemble:
    """Many lattices in one batch (synchronous driver)."""

    def __init__(self, device: int = 0, memory_budget: float = 120e9) -> None:
        self._b = ctypes.c_void_p()
        check(lib().ising_batch_create(int(device), int(memory_budget), ctypes.byref(self._b)),
              "batch_create")
        self._jobs: dict[int, Job] = {}

    def add(self, job: Job) -> int:
        s, _keep = job.to_struct()
        jid = ctypes.c_int64()
        check(lib().ising_batch_add(self._b, ctypes.byref(s), ctypes.byref(jid)), "batch_add")
        self._jobs[jid.value] = job
        return int(jid.value)

    BATCH_KNOBS = {"band": 1, "items_per_slot": 6, "graph_chunk": 5}

    def set_knob(self, name: str, value: int) -> None:
        """Batch launch knob (``"band"``: longest band of a kernel class, ``"items_per_slot"``:
        work items per resident block, ``"graph_chunk"``: sweeps replayed from one captured
        graph while the batch is stable, 0 = none); results are identical for every value."""
        check(lib().ising_batch_set_knob(self._b, self.BATCH_KNOBS[name], int(value)),
              "batch_set_knob")

    def get_knob(self, name: str) -> int:
        v = ctypes.c_int()
        check(lib().ising_batch_get_knob(self._b, self.BATCH_KNOBS[name], ctypes.byref(v)),
              "batch_get_knob")
        return int(v.value)

    def run(self, max_epochs: int = 0) -> int:
        """Advance until every job is done (or ``max_epochs`` half-sweeps); returns epochs run."""
        n = ctypes.c_int64()
        check(lib().ising_batch_run(self._b, int(max_epochs), ctypes.byref(n)), "batch_run")
        return int(n.value)

    def status(self, jid: int) -> tuple[str, int]:
        st, sw = ctypes.c_int(), ctypes.c_int64()
        check(lib().ising_batch_status(self._b, jid, ctypes.byref(st), ctypes.byref(sw)),
              "batch_status")
        return STATE_NAMES[st.value], int(sw.value)

    def result(self, jid: int) -> Result:
        job = self._jobs[jid]
        series = np.zeros((job.n_measurements, 2), dtype=np.int64)
        lat = np.empty(job.shape, dtype=np.int8) if job.keep_lattice else None
        check(lib().ising_batch_result(self._b, jid, series.ctypes.data if series.size else None,
                                       lat.ctypes.data if lat is not None else None),
              "batch_result")
        return Result(series, lat)

    def release(self, jid: int) -> None:
        check(lib().ising_batch_release(self._b, jid), "batch_release")
        self._jobs.pop(jid, None)

    def close(self) -> None:
        if getattr(self, "_b", None) is not None and self._b.value:
            lib().ising_batch_destroy(self._b)
            self._b = None

    def __enter__(self) -> Ensemble:
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


class Server:
    """Continuous-batching serving loop (a host thread inside the library)."""

    def __init__(self, device: int = 0, memory_budget: float = 120e9) -> None:
        self._s = ctypes.c_void_p()
        check(lib().ising_server_create(int(device), int(memory_budget), ctypes.byref(self._s)),
              "server_create")
        self._jobs: dict[int, Job] = {}

    def submit(self, job: Job) -> int:
        s, _keep = job.to_struct()
        jid = ctypes.c_int64()
        check(lib().ising_server_submit(self._s, ctypes.byref(s), ctypes.byref(jid)),
              "server_submit")
        self._jobs[jid.value] = job
        return int(jid.value)

    def set_knob(self, name: str, value: int) -> None:
        """Batch launch knob of the server's engine (see :meth:`Ensemble.set_knob`)."""
        check(lib().ising_server_set_knob(self._s, Ensemble.BATCH_KNOBS[name], int(value)),
              "server_set_knob")

    def wait(self, jid: int, timeout: float | None = None) -> str:
        st = ctypes.c_int()
        check(lib().ising_server_wait(self._s, jid, -1.0 if timeout is None else float(timeout),
                                      ctypes.byref(st)), "server_wait")
        return STATE_NAMES[st.value]

    def result(self, jid: int) -> Result:
        job = self._jobs[jid]
        series = np.zeros((job.n_measurements, 2), dtype=np.int64)
        lat = np.empty(job.shape, dtype=np.int8) if job.keep_lattice else None
        lat_s = ctypes.c_double()
        check(lib().ising_server_result(self._s, jid, series.ctypes.data if series.size else None,
                                        lat.ctypes.data if lat is not None else None,
                                        ctypes.byref(lat_s)), "server_result")
        return Result(series, lat, float(lat_s.value))

    def release(self, jid: int) -> None:
        check(lib().ising_server_release(self._s, jid), "server_release")
        self._jobs.pop(jid, None)

    def status(self) -> dict:
        p, a, u, e = (ctypes.c_int64() for _ in range(4))
        check(lib().ising_server_status(self._s, ctypes.byref(p), ctypes.byref(a),
                                        ctypes.byref(u), ctypes.byref(e)), "server_status")
        return {"pending": p.value, "active": a.value, "used_bytes": u.value, "epoch": e.value}

    def close(self) -> None:
        if getattr(self, "_s", None) is not None and self._s.value:
            lib().ising_server_destroy(self._s)
            self._s = None

    def __enter__(self) -> Server:
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass
