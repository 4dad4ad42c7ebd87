"""Slab decomposition: one lattice too large (or too slow) for one GPU, split over several.

The lattice's first axis (rows y in 2D, planes z in 3D) is cut into contiguous slabs
(:func:`partition`); each slab lives on one GPU as an ``ising_slab`` handle of the C ABI, which
holds the slab's rows plus one halo row (2D) or plane (3D) of each colour on each side.  Before
a half-sweep of colour c, the opposite colour's edge rows are copied into the neighbouring
slabs' halos (periodic along the axis); the half-sweep kernels then read the halos instead of
wrapping.  Random numbers are keyed by global site index, sweep and colour, so the slabs
together give exactly the spins and (M, E) series of one GPU running the whole lattice (and of
pyising's NumPy backend, src/pyising/backends/numpy_backend.py:26-124).

Three exchanges:

* :class:`PeerExchange` (the default within one process): every slab in this process (several
  GPUs of one process, or several slabs on one GPU); no copies: the kernels read the
  neighbouring slabs' edge rows in place, over NVLink between GPUs, ordered by CUDA events.
* :class:`LocalExchange`: the same slabs, halos filled by device copies (peer copies between
  GPUs).
* :class:`RingExchange`: one slab per rank of a ``torch.distributed`` process group, ranks in
  slab order; each exchange is one batch of two sends and two receives to the neighbouring
  ranks (NCCL over NVLink on GPUs, gloo on CPU), and (M, E) sums are one int64 all-reduce.

Per sweep that is 2 exchanges of Lx/2 bytes (int8 2D), Lx/2 * Ly bytes (int8 3D) or Lx/16 bytes
(msc) per halo, against a half-sweep over the whole slab.
"""

from __future__ import annotations

import contextlib
import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib
from .lattice import (check_shape, merge_colours, pack_colour, random_lattice, split_colours,
                      threshold_table, unpack_colour)

HALO_LOW, HALO_HIGH, EDGE_LOW, EDGE_HIGH = 0, 1, 2, 3


def partition(extent: int, parts: int) -> list[tuple[int, int]]:
    """Balanced ``(begin, count)`` ranges of a first axis of ``extent`` over ``parts`` slabs
    (the first ``extent % parts`` slabs one row or plane longer)."""
    if parts < 1 or parts > extent:
        raise ValueError(f"cannot cut an axis of {extent} into {parts} slabs")
    q, r = divmod(extent, parts)
    out, b = [], 0
    for i in range(parts):
        c = q + (1 if i < r else 0)
        out.append((b, c))
        b += c
    return out


class _DeviceBytes:
    """A region of library-owned device memory, seen by torch without a copy."""

    def __init__(self, ptr: int, nbytes: int) -> None:
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1",
                                         "data": (ptr, False), "version": 3, "strides": None,
                                         "stream": None}


class Slab:
    """Rows ``[begin, begin + count)`` of the first axis of the lattice ``shape`` on one GPU.

    Host colour arrays cover the owned rows only: ``(rows, Lx/2)`` int8 or ``(rows, Lx/128)``
    uint64, rows = count (2D) or count * Ly (3D).
    """

    def __init__(self, shape, table: np.ndarray, seed: int, algorithm: str, variant: str,
                 begin: int, count: int, device: int = 0) -> None:
        self.shape = tuple(int(s) for s in shape)
        self.ndim = len(self.shape)
        self.variant, self.algorithm = variant, algorithm
        self.begin, self.count, self.device = int(begin), int(count), int(device)
        inner = self.shape[1] if self.ndim == 3 else 1
        self.rows = self.count * inner
        self.row0 = self.begin * inner
        self.lh = self.shape[-1] // 2
        self._h = ctypes.c_void_p()
        sh = (ctypes.c_int64 * 3)(*(list(self.shape) + [0] * (3 - self.ndim)))
        check(lib().ising_slab_create(self.ndim, sh, _lib.VARIANT[variant],
                                      _lib.ALGORITHM[algorithm], int(seed) & (2**64 - 1),
                                      self.begin, self.count, self.device, ctypes.byref(self._h)),
              "slab_create")
        self._regions: dict[tuple[int, int], object] = {}
        self.set_table(table)

    def close(self) -> None:
        if self._h is not None and self._h.value:
            lib().ising_slab_destroy(self._h)
        self._h = None
        self._regions = {}

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def set_table(self, table: np.ndarray) -> None:
        tab = np.ascontiguousarray(table, dtype=np.uint32)
        check(lib().ising_slab_set_table(self._h, tab.ctypes.data, len(tab)), "slab_set_table")

    def set_stream(self, stream: int | None) -> None:
        check(lib().ising_slab_set_stream(self._h, stream or None), "slab_set_stream")

    def fill_cold(self) -> None:
        check(lib().ising_slab_fill_cold(self._h), "slab_fill_cold")

    def fill_philox(self, start_seed: int) -> None:
        check(lib().ising_slab_fill_philox(self._h, int(start_seed) & (2**64 - 1)),
              "slab_fill_philox")

    def _spec(self):
        if self.variant == "msc":
            return (self.rows, self.lh // 64), np.uint64
        return (self.rows, self.lh), np.int8

    def load(self, c0: np.ndarray, c1: np.ndarray) -> None:
        """Uploads the owned rows of both colours (device layout)."""
        shape, dtype = self._spec()
        a, b = (np.ascontiguousarray(x, dtype=dtype).reshape(shape) for x in (c0, c1))
        check(lib().ising_slab_upload(self._h, a.ctypes.data, b.ctypes.data), "slab_upload")

    def colour_arrays(self) -> tuple[np.ndarray, np.ndarray]:
        shape, dtype = self._spec()
        a, b = np.empty(shape, dtype), np.empty(shape, dtype)
        check(lib().ising_slab_download(self._h, a.ctypes.data, b.ctypes.data), "slab_download")
        return a, b

    def region(self, colour: int, which: int):
        """A halo (HALO_LOW/HIGH) or edge (EDGE_LOW/HIGH) of one colour as a uint8 torch tensor
        over the slab's device memory (no copy)."""
        key = (colour, which)
        if key not in self._regions:
            import torch

            ptr, nbytes = ctypes.c_void_p(), ctypes.c_int64()
            check(lib().ising_slab_halo(self._h, colour, which, ctypes.byref(ptr),
                                        ctypes.byref(nbytes)), "slab_halo")
            self._regions[key] = torch.as_tensor(_DeviceBytes(ptr.value, nbytes.value),
                                                 device=f"cuda:{self.device}")
        return self._regions[key]

    def set_peer(self, side: int, other: Slab | None) -> None:
        """Read ``other``'s edge rows in place of this slab's halos (side 0: the previous slab,
        1: the next one); ``None``: back to the own halos."""
        check(lib().ising_slab_set_peer(self._h, int(side), other._h if other is not None
                                        else None), "slab_set_peer")

    def half_sweep(self, colour: int, t: int, slot: int = -1, first: int = 0,
                   count: int | None = None) -> None:
        """Half-sweep of rows (2D) or planes (3D) ``first .. first + count - 1`` (all by
        default) of the slab."""
        n = self.count - first if count is None else count
        check(lib().ising_slab_half_sweep_rows(self._h, colour, int(t), int(slot), int(first),
                                               int(n)), "slab_half_sweep")

    def series_reset(self, pairs: int) -> None:
        check(lib().ising_slab_series_reset(self._h, int(pairs)), "slab_series_reset")

    def series_read(self, pairs: int) -> np.ndarray:
        out = np.zeros((pairs, 2), np.int64)
        check(lib().ising_slab_series_read(self._h, int(pairs), out.ctypes.data),
              "slab_series_read")
        return out

    def observables(self) -> tuple[int, int]:
        m, e = ctypes.c_int64(), ctypes.c_int64()
        check(lib().ising_slab_observables(self._h, ctypes.byref(m), ctypes.byref(e)),
              "slab_observables")
        return m.value, e.value

    def sync(self) -> None:
        check(lib().ising_slab_sync(self._h), "slab_sync")


class LocalExchange:
    """All slabs of the lattice in this process, in slab order: halos filled by device copies.

    ``start`` / ``finish`` split an exchange so that work can be issued in between (the slab
    runner's overlap mode); here the copies are issued by ``start``."""

    def exchange(self, slabs, colour: int) -> None:
        n = len(slabs)
        for i, s in enumerate(slabs):
            s.region(colour, HALO_LOW).copy_(slabs[i - 1].region(colour, EDGE_HIGH))
            s.region(colour, HALO_HIGH).copy_(slabs[(i + 1) % n].region(colour, EDGE_LOW))

    def start(self, slabs, colour: int):
        self.exchange(slabs, colour)

    def finish(self, pending) -> None:
        pass

    def allreduce(self, values: np.ndarray) -> np.ndarray:
        return values


class PeerExchange:
    """All slabs of the lattice in this process, in slab order, with no halo copies at all: each
    slab's kernels read its neighbours' edge rows in place (NVLink peer loads between GPUs, set
    up once by ``Slab.set_peer``).  An exchange only orders the work: every slab's next
    half-sweep waits for its neighbours' last half-sweeps (CUDA events across streams), which
    both makes their edges current (read after write) and keeps them from being rewritten while
    they are still read (write after read).  Slabs on one stream need nothing."""

    def __init__(self, slabs, streams=None) -> None:
        n = len(slabs)
        for i, s in enumerate(slabs):
            s.set_peer(0, slabs[i - 1])
            s.set_peer(1, slabs[(i + 1) % n])
        self.streams = list(streams) if streams is not None else None

    def exchange(self, slabs, colour: int) -> None:
        st = self.streams
        if st is None or all(x is st[0] for x in st):
            return
        import torch

        events = []
        for x in st:
            ev = torch.cuda.Event()
            ev.record(x)
            events.append(ev)
        n = len(slabs)
        for i, x in enumerate(st):
            for j in (i - 1, (i + 1) % n):
                if st[j % n] is not x:
                    x.wait_event(events[j % n])

    def start(self, slabs, colour: int):
        self.exchange(slabs, colour)

    def finish(self, pending) -> None:
        pass

    def allreduce(self, values: np.ndarray) -> np.ndarray:
        return values


class RingExchange:
    """One slab per rank of a ``torch.distributed`` group, rank r holding slab r of the first
    axis (periodic, so the last rank's high halo is rank 0's first row).  ``device`` is where
    the all-reduce runs: this rank's GPU for NCCL, ``"cpu"`` for gloo."""

    def __init__(self, group=None, device="cpu") -> None:
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.device = device

    def _global(self, r: int) -> int:
        return self.dist.get_global_rank(self.group, r) if self.group is not None else r

    def exchange(self, slabs, colour: int) -> None:
        self.finish(self.start(slabs, colour))

    def finish(self, pending) -> None:
        for w in pending or ():
            w.wait()

    def start(self, slabs, colour: int):
        """Issues the two sends and two receives; ``finish`` waits for them (on GPUs: makes
        the current stream wait), so that rows reading no halo can be updated in between."""
        (s,) = slabs
        if self.world == 1:
            LocalExchange().exchange(slabs, colour)
            return None
        d = self.dist
        prev = self._global((self.rank - 1) % self.world)
        nxt = self._global((self.rank + 1) % self.world)
        # Tag 2c: an edge sent down the ring lands in the receiver's high halo; tag 2c + 1: sent
        # up, lands in the low halo.  With two ranks prev == nxt and the tags (gloo) or the
        # order of the operations (NCCL matches a pair's messages in order) keep them apart.
        ops = [d.P2POp(d.isend, s.region(colour, EDGE_LOW), prev, self.group, 2 * colour),
               d.P2POp(d.isend, s.region(colour, EDGE_HIGH), nxt, self.group, 2 * colour + 1),
               d.P2POp(d.irecv, s.region(colour, HALO_HIGH), nxt, self.group, 2 * colour),
               d.P2POp(d.irecv, s.region(colour, HALO_LOW), prev, self.group, 2 * colour + 1)]
        return d.batch_isend_irecv(ops)

    def allreduce(self, values: np.ndarray) -> np.ndarray:
        import torch

        t = torch.as_tensor(np.ascontiguousarray(values, dtype=np.int64), device=self.device)
        self.dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()


class SlabRunner:
    """The sweep loop over the slabs of this process and an exchange.

    A slab needs ``half_sweep(colour, t, slot)``, ``region(colour, which)``,
    ``series_reset(pairs)``, ``series_read(pairs)`` and ``observables()``; the loop keeps track
    of which colour's halos are current and refreshes them only when a half-sweep (or a
    measurement) reads them.  ``streams``: CUDA streams the slabs run on, made current while
    the loop issues copies and collectives so that they are ordered with the kernels.
    """

    def __init__(self, slabs, exchange, t: int = 0, streams=(), overlap: bool = False) -> None:
        self.slabs = list(slabs)
        self.exchange = exchange
        self.t = int(t)
        self.streams = list(streams)
        self.overlap = bool(overlap)
        self._fresh = [False, False]

    @contextlib.contextmanager
    def _on_streams(self):
        with contextlib.ExitStack() as stack:
            if self.streams:
                import torch

                for st in self.streams:
                    stack.enter_context(torch.cuda.stream(st))
            yield

    def invalidate(self) -> None:
        """The slabs' spins were replaced: every halo is stale."""
        self._fresh = [False, False]

    def _refresh(self, colour: int) -> None:
        if not self._fresh[colour]:
            self.exchange.exchange(self.slabs, colour)
            self._fresh[colour] = True

    def sweep(self, n: int = 1, measure_every: int = 0) -> np.ndarray | None:
        """n sweeps (colour 0 then colour 1, as src/pyising/backends/base.py:85-90); with
        measure_every > 0 the exact (M, E) of the whole lattice after every measure_every-th
        sweep, an int64 array (n // measure_every, 2)."""
        if n < 0 or measure_every < 0:
            raise ValueError("sweep counts must be non-negative")
        n_meas = n // measure_every if measure_every > 0 else 0
        with self._on_streams():
            if n_meas:
                for s in self.slabs:
                    s.series_reset(n_meas)
            k = 0
            for i in range(n):
                slot = -1
                if measure_every > 0 and (i + 1) % measure_every == 0:
                    slot, k = k, k + 1
                self._half(0, -1)
                self._half(1, slot)
                self.t += 1
            if not n_meas:
                return None
            local = np.zeros((n_meas, 2), np.int64)
            for s in self.slabs:
                local += s.series_read(n_meas)
            return self.exchange.allreduce(local).reshape(n_meas, 2)

    def _half(self, colour: int, slot: int) -> None:
        """One half-sweep of every slab.  In overlap mode, with halos to refresh and slabs of at
        least three rows (planes), the rows that read no halo are issued between the start and
        the finish of the exchange, the first and last row after it."""
        other = colour ^ 1
        if (self.overlap and not self._fresh[other] and
                all(s.count >= 3 for s in self.slabs)):
            pending = self.exchange.start(self.slabs, other)
            for s in self.slabs:
                s.half_sweep(colour, self.t, slot, 1, s.count - 2)
            self.exchange.finish(pending)
            self._fresh[other] = True
            for s in self.slabs:
                s.half_sweep(colour, self.t, slot, 0, 1)
                s.half_sweep(colour, self.t, slot, s.count - 1, 1)
        else:
            self._refresh(other)
            for s in self.slabs:
                s.half_sweep(colour, self.t, slot)
        self._fresh[colour] = False

    def observables_int(self) -> tuple[int, int]:
        """Exact (M, E) of the whole lattice."""
        with self._on_streams():
            self._refresh(0)
            local = np.zeros(2, np.int64)
            for s in self.slabs:
                local += np.asarray(s.observables(), np.int64)
            tot = self.exchange.allreduce(local)
        return int(tot[0]), int(tot[1])


class SlabSimulation:
    """One lattice over a slab decomposition, with pyising's simulation calls.

    ``group``: a ``torch.distributed`` process group (or ``"default"`` for the default one),
    one slab per rank on this rank's current CUDA device, NCCL halos (:class:`RingExchange`).
    Otherwise every slab lives in this process: ``parts`` slabs (default: one per GPU) on
    ``devices`` (default: all GPUs, round robin), the kernels reading their neighbours' edge rows
    in place (``exchange="peer"``, :class:`PeerExchange`) or from halo copies
    (``exchange="copy"``, :class:`LocalExchange`).
    ``init``: ``"hot"`` (NumPy's PCG64 start of pyising, generated on every rank), ``"cold"``,
    ``"philox"`` (the device seeded start, no host work) or a full int8 lattice.  ``overlap``
    (default: with a process group) updates the rows that read no halo while the halos are in
    flight.
    """

    def __init__(self, shape, beta: float, seed: int = 0, algorithm: str = "metropolis",
                 variant: str = "int8", init="hot", *, parts: int | None = None,
                 devices=None, group=None, exchange: str = "peer",
                 overlap: bool | None = None) -> None:
        import torch

        if variant not in ("int8", "msc"):
            raise ValueError(f"unknown variant {variant!r}")
        self.variant = variant
        self.shape = check_shape(shape, 128 if variant == "msc" else 8)
        self.ndim = len(self.shape)
        if variant == "msc" and (self.ndim != 2 or algorithm != "metropolis"):
            raise ValueError("msc supports 2D Metropolis only")
        if algorithm not in ("metropolis", "heatbath"):
            raise ValueError(f"unknown algorithm {algorithm!r}")
        self.algorithm = algorithm
        self.seed = int(seed) & (2**64 - 1)
        self.beta = float(beta)
        self.table = threshold_table(self.beta, self.ndim, algorithm)
        self.n_spins = int(np.prod(self.shape))
        if group is not None:
            import torch.distributed as dist

            g = None if group == "default" else group
            rank, world = dist.get_rank(g), dist.get_world_size(g)
            ranges = partition(self.shape[0], world)
            dev = torch.cuda.current_device()
            self.slabs = [Slab(self.shape, self.table, self.seed, algorithm, variant,
                               *ranges[rank], device=dev)]
            ring = RingExchange(g, device=f"cuda:{dev}")
        else:
            ndev = torch.cuda.device_count()
            devices = list(devices) if devices is not None else list(range(ndev))
            parts = parts if parts is not None else len(devices)
            ranges = partition(self.shape[0], parts)
            self.slabs = [Slab(self.shape, self.table, self.seed, algorithm, variant, b, c,
                               device=devices[i % len(devices)])
                          for i, (b, c) in enumerate(ranges)]
            if exchange not in ("peer", "copy"):
                raise ValueError(f"unknown exchange {exchange!r}")
        streams = {}
        for s in self.slabs:
            if s.device not in streams:
                streams[s.device] = torch.cuda.Stream(device=s.device)
            s.set_stream(streams[s.device].cuda_stream)
        if group is None:
            ex = (PeerExchange(self.slabs, [streams[s.device] for s in self.slabs])
                  if exchange == "peer" else LocalExchange())
        else:
            ex = ring
        # overlap the exchange with the rows that read no halo: by default between processes,
        # where the exchange is NCCL traffic (in one process it only adds launches)
        if overlap is None:
            overlap = group is not None
        self.runner = SlabRunner(self.slabs, ex, streams=list(streams.values()), overlap=overlap)
        if isinstance(init, np.ndarray):
            self.set_lattice(init)
        elif init == "hot":
            self.set_lattice(random_lattice(self.shape, self.seed))
        elif init == "cold":
            for s in self.slabs:
                s.fill_cold()
            self.runner.invalidate()
        elif init == "philox":
            for s in self.slabs:
                s.fill_philox(self.seed)
            self.runner.invalidate()
        else:
            raise ValueError(f"unknown init {init!r}")

    @property
    def t(self) -> int:
        return self.runner.t

    @t.setter
    def t(self, value: int) -> None:
        self.runner.t = int(value)

    def set_beta(self, beta: float) -> None:
        """New temperature; keeps the spins and the sweep counter (src/pyising/backends/
        base.py:79-83)."""
        self.beta = float(beta)
        self.table = threshold_table(self.beta, self.ndim, self.algorithm)
        for s in self.slabs:
            s.set_table(self.table)

    def set_lattice(self, lat: np.ndarray) -> None:
        """A full +-1 int8 lattice; each slab takes its own rows."""
        lat = np.asarray(lat, dtype=np.int8)
        if lat.shape != self.shape:
            raise ValueError(f"lattice shape {lat.shape} != {self.shape}")
        c0, c1 = split_colours(lat)
        for s in self.slabs:
            a, b = c0[s.row0:s.row0 + s.rows], c1[s.row0:s.row0 + s.rows]
            if self.variant == "msc":
                a, b = pack_colour(a), pack_colour(b)
            s.load(a, b)
        self.runner.invalidate()

    def local_colour_arrays(self) -> list[tuple[int, np.ndarray, np.ndarray]]:
        """``(row0, c0, c1)`` of every slab in this process (compressed int8 rows)."""
        out = []
        for s in self.slabs:
            a, b = s.colour_arrays()
            if self.variant == "msc":
                a, b = unpack_colour(a), unpack_colour(b)
            out.append((s.row0, a, b))
        return out

    def get_lattice(self) -> np.ndarray:
        """The full lattice (with a process group: gathered from every rank, on every rank)."""
        parts = self.local_colour_arrays()
        if isinstance(self.runner.exchange, RingExchange) and self.runner.exchange.world > 1:
            ex = self.runner.exchange
            gathered = [None] * ex.world
            ex.dist.all_gather_object(gathered, parts, group=ex.group)
            parts = [p for ps in gathered for p in ps]
        parts.sort(key=lambda p: p[0])
        c0 = np.concatenate([p[1] for p in parts])
        c1 = np.concatenate([p[2] for p in parts])
        return merge_colours(c0, c1, self.shape)

    def sweep(self, n: int = 1) -> None:
        self.runner.sweep(n)

    def sweep_measured(self, n: int, every: int) -> np.ndarray:
        """n sweeps with the exact (M, E) after every ``every``-th: int64 (n // every, 2)."""
        if every <= 0:
            raise ValueError("every must be positive")
        return self.runner.sweep(n, every)

    def observables_int(self) -> tuple[int, int]:
        return self.runner.observables_int()

    def observables(self) -> tuple[float, float]:
        """(M / N, E / N) (src/pyising/backends/base.py:125-135)."""
        m, e = self.observables_int()
        return m / self.n_spins, e / self.n_spins

    def synchronize(self) -> None:
        for s in self.slabs:
            s.sync()

    def close(self) -> None:
        """Frees the slabs, after every stream's work is done (with peer reads a slab's memory
        may be read by its neighbours' kernels on other streams)."""
        slabs = getattr(self, "slabs", [])
        for s in slabs:
            if s._h is not None and s._h.value:
                s.sync()
        for s in slabs:
            s.close()
        self.slabs = []

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


def main(argv=None) -> int:
    """Run one lattice over slabs and print one JSON line (rank 0):

        python -m pyising_b200.slab --shape 16384 16384 --variant msc --sweeps 1000 --every 10
        torchrun --nproc-per-node 8 -m pyising_b200.slab --shape 65536 65536 --variant msc

    Under torchrun (WORLD_SIZE > 1) each rank holds one slab on its GPU (NCCL halos, exchange
    overlapped with the rows that read no halo); otherwise ``--parts`` slabs share this
    process's GPUs.  The sweeps are timed with CUDA events on every slab's stream, maximum over
    ranks; the whole-lattice (M, E) series and flips/ns are printed.
    """
    import argparse
    import json
    import os

    import torch

    ap = argparse.ArgumentParser(prog="python -m pyising_b200.slab")
    ap.add_argument("--shape", type=int, nargs="+", required=True)
    ap.add_argument("--variant", choices=["int8", "msc"], default="int8")
    ap.add_argument("--algorithm", choices=["metropolis", "heatbath"], default="metropolis")
    ap.add_argument("--beta", type=float, default=None, help="default: the critical coupling")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--init", choices=["hot", "cold", "philox"], default="philox")
    ap.add_argument("--sweeps", type=int, default=200)
    ap.add_argument("--every", type=int, default=0, help="measure (M, E) every n sweeps")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--parts", type=int, default=None, help="slabs in this process")
    args = ap.parse_args(argv)
    from .lattice import BETA_C_2D

    beta = args.beta if args.beta is not None else (BETA_C_2D if len(args.shape) == 2
                                                     else 0.221654626)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    group = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        group = "default"
    sim = SlabSimulation(args.shape, beta, seed=args.seed, algorithm=args.algorithm,
                         variant=args.variant, init=args.init, parts=args.parts, group=group)
    sim.sweep(args.warmup)
    streams = sim.runner.streams
    starts, ends = [], []
    for st in streams:
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(st)
        starts.append(ev)
    series = sim.sweep_measured(args.sweeps, args.every) if args.every else sim.sweep(args.sweeps)
    for st in streams:
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(st)
        ends.append(ev)
    for ev in ends:
        ev.synchronize()
    ms = max(a.elapsed_time(b) for a, b in zip(starts, ends))
    if group is not None:
        import torch.distributed as dist

        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    m, e = sim.observables_int()
    rank = int(os.environ.get("RANK", "0"))
    if rank == 0:
        n = int(np.prod(args.shape))
        print(json.dumps({
            "shape": args.shape, "variant": args.variant, "algorithm": args.algorithm,
            "beta": beta, "slabs": world if group else len(sim.slabs), "ranks": world,
            "sweeps": args.sweeps, "ms": round(ms, 3),
            "flips_per_ns": round(n * args.sweeps / (ms * 1e6), 2), "final_M_E": [m, e],
            "series": series.tolist() if series is not None else None}), flush=True)
    sim.close()
    if group is not None:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
