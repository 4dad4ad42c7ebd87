"""Slab decomposition of one lattice (pyising_b200.slab).

CPU: the sweep loop (SlabRunner) and both halo exchanges run on CPU slabs whose half-sweep is
a NumPy restatement of the reference update (src/pyising/backends/numpy_backend.py:26-44)
working only on the slab's rows and halos: in one process (LocalExchange) and as gloo ranks of
world size 2 and 3 (RingExchange, the code path NCCL runs on GPUs).  Spins and (M, E) series must be
bit-identical to the oracle running the whole lattice.

GPU: the C-ABI slab handles (ising_slab_*) split over several slabs on one GPU must be
bit-identical to one handle holding the whole lattice, for int8 2D/3D (Metropolis, heat bath)
and msc, uneven slabs included.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import oracle
from pyising_b200.slab import (EDGE_HIGH, EDGE_LOW, HALO_HIGH, HALO_LOW, LocalExchange,
                               RingExchange, SlabRunner, partition)


def test_partition_covers_the_axis():
    for extent in (2, 7, 16, 33):
        for parts in range(1, min(extent, 6) + 1):
            ranges = partition(extent, parts)
            assert ranges[0][0] == 0 and sum(c for _, c in ranges) == extent
            assert all(b1 == b0 + c0 for (b0, c0), (b1, _) in zip(ranges, ranges[1:]))
            assert max(c for _, c in ranges) - min(c for _, c in ranges) <= 1
    with pytest.raises(ValueError):
        partition(4, 5)
    with pytest.raises(ValueError):
        partition(4, 0)


@pytest.mark.parametrize("ndim,shape,variant,begin,count,msg", [
    (2, (16, 16, 0), 0, 0, 0, "outside the first axis"),
    (2, (16, 16, 0), 0, 10, 8, "outside the first axis"),
    (2, (16, 16, 0), 0, -1, 4, "outside the first axis"),
    (3, (8, 8, 128), 1, 0, 4, "2D Metropolis"),
    (2, (16, 12, 0), 0, 0, 4, "multiple of 8"),
    (4, (8, 8, 8), 0, 0, 4, "2D and 3D"),
])
def test_slab_create_validates_before_touching_cuda(ndim, shape, variant, begin, count, msg):
    import ctypes

    from pyising_b200._lib import lib

    h = ctypes.c_void_p()
    arr = (ctypes.c_int64 * 3)(*shape)
    rc = lib().ising_slab_create(ndim, arr, variant, 0, 0, begin, count, 0, ctypes.byref(h))
    assert rc == 1  # ISING_ERR_INVALID
    assert msg in lib().ising_last_error().decode()
    assert not h.value


def test_slab_calls_reject_null_handles():
    from pyising_b200._lib import lib

    L = lib()
    assert L.ising_slab_destroy(None) == 0
    assert L.ising_slab_half_sweep(None, 0, 0, -1) == 1
    assert "null" in L.ising_last_error().decode()
    assert L.ising_slab_halo(None, 0, 0, None, None) == 1
    assert L.ising_slab_observables(None, None, None) == 1


@pytest.mark.parametrize("shape", [(6, 16), (4, 6, 8), (10, 256)])
def test_host_colour_split_matches_the_oracle(shape):
    from pyising_b200.lattice import merge_colours, pack_colour, split_colours, unpack_colour

    lat = oracle.random_lattice(shape, 4)
    c0, c1 = split_colours(lat)
    w0, w1 = oracle.to_compressed(lat)
    np.testing.assert_array_equal(c0, w0)
    np.testing.assert_array_equal(c1, w1)
    np.testing.assert_array_equal(merge_colours(c0, c1, shape), lat)
    if shape[-1] % 128 == 0:
        np.testing.assert_array_equal(pack_colour(c0), oracle.pack_bits(w0))
        np.testing.assert_array_equal(unpack_colour(pack_colour(c1)), c1)


class CpuSlab:
    """A slab of an int8 lattice on the CPU with the C-ABI slab's interface: rows
    [begin, begin + count) of the first axis plus one halo row (2D) or plane (3D) per side,
    updated from its own rows and halos only."""

    def __init__(self, lat, begin, count, beta, seed, algorithm):
        shape = lat.shape
        self.count = count
        self.ndim = len(shape)
        self.ly = shape[1] if self.ndim == 3 else count
        inner = shape[1] if self.ndim == 3 else 1
        self.rows, self.row0 = count * inner, begin * inner
        self.halo = inner
        self.par0 = begin & 1
        self.lh = shape[-1] // 2
        self.k0, self.k1 = oracle.split_seed(seed)
        self.table = oracle.threshold_table(beta, self.ndim, algorithm)
        self.heat = algorithm == "heatbath"
        full = oracle.to_compressed(lat)
        self.a = []
        for c in (0, 1):
            arr = np.zeros((self.rows + 2 * self.halo, self.lh), np.int8)
            arr[self.halo:self.halo + self.rows] = full[c][self.row0:self.row0 + self.rows]
            self.a.append(arr)
        self.series = np.zeros((0, 2), np.int64)

    def region(self, colour, which):
        h, r, arr = self.halo, self.rows, self.a[colour]
        sl = {HALO_LOW: slice(0, h), HALO_HIGH: slice(h + r, 2 * h + r),
              EDGE_LOW: slice(h, 2 * h), EDGE_HIGH: slice(r, h + r)}[which]
        return torch.from_numpy(arr[sl].reshape(-1).view(np.uint8))

    def _rows(self, first=0, count=None):
        """Local rows of rows (2D) or planes (3D) first .. first + count - 1."""
        count = self.count - first if count is None else count
        per = self.ly if self.ndim == 3 else 1
        return np.arange(first * per, (first + count) * per)

    def _field(self, colour, r=None):
        """Sum of the opposite colour's neighbours of the owned sites of `colour` in rows r."""
        h, ly = self.halo, self.ly
        oth = self.a[1 - colour].astype(np.int64)
        r = np.arange(self.rows) if r is None else r
        z, y = (r // ly, r % ly) if self.ndim == 3 else (np.zeros_like(r), r)
        same = oth[h + r]
        par = ((self.par0 + y + z + colour) & 1)[:, None]
        field = same + np.where(par == 1, np.roll(same, -1, axis=1), np.roll(same, 1, axis=1))
        if self.ndim == 2:
            field += oth[h + r - 1] + oth[h + r + 1]
        else:
            plane = z * ly
            field += oth[h + plane + (y + 1) % ly] + oth[h + plane + (y - 1) % ly]
            field += oth[h + r + ly] + oth[h + r - ly]
        return field

    def half_sweep(self, colour, t, slot=-1, first=0, count=None):
        r = self._rows(first, count)
        if len(r) == 0:
            return
        own = self.a[colour][self.halo + r]
        field = self._field(colour, r)
        q0, n = (self.row0 + r[0]) * self.lh // 4, len(r) * self.lh // 4
        u = oracle.philox_range(q0, n, t, colour, 0, self.k0, self.k1).reshape(own.shape)
        d = 2 * self.ndim
        if self.heat:
            new = np.where(u < self.table[(field + d) // 2], 1, -1).astype(np.int8)
        else:
            x = own * field
            flip = (x <= 0) | (u < self.table[(x + d) // 2])
            new = np.where(flip, -own, own).astype(np.int8)
        self.a[colour][self.halo + r] = new
        if slot >= 0:
            self.series[slot] += self._observe(r)

    def _observe(self, r):
        s1 = self.a[1][self.halo + r].astype(np.int64)
        m = int(s1.sum() + self.a[0][self.halo + r].astype(np.int64).sum())
        return m, -int((s1 * self._field(1, r)).sum())

    def observables(self):
        return self._observe(np.arange(self.rows))

    def series_reset(self, pairs):
        self.series = np.zeros((pairs, 2), np.int64)

    def series_read(self, pairs):
        return self.series[:pairs].copy()

    def compressed(self):
        return [x[self.halo:self.halo + self.rows] for x in self.a]


CASES = [((10, 16), 0.44, "metropolis", 12345, 3),
         ((6, 4, 8), 0.22, "heatbath", 7, 2),
         ((8, 6, 16), 0.3, "metropolis", 2**40 + 1, 4),
         ((14, 24), 0.6, "heatbath", 99, 5)]


def _oracle_run(shape, beta, algorithm, seed, sweeps, every):
    lat = oracle.random_lattice(shape, seed)
    sim = oracle.OracleInt8(shape, beta, seed=seed, algorithm=algorithm, init=lat)
    series = sim.sweep(sweeps, measure_every=every)
    return lat, series, sim.get_lattice(), sim.observables_int()


def _assemble(shape, slabs):
    c0 = np.concatenate([s.compressed()[0] for s in slabs])
    c1 = np.concatenate([s.compressed()[1] for s in slabs])
    return oracle.from_compressed(c0, c1, shape)


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("shape,beta,algorithm,seed,parts", CASES)
def test_local_exchange_matches_whole_lattice(shape, beta, algorithm, seed, parts, overlap):
    lat, series, final, obs = _oracle_run(shape, beta, algorithm, seed, 6, 2)
    slabs = [CpuSlab(lat, b, c, beta, seed, algorithm) for b, c in partition(shape[0], parts)]
    runner = SlabRunner(slabs, LocalExchange(), overlap=overlap)
    got = runner.sweep(6, 2)
    np.testing.assert_array_equal(got, series)
    np.testing.assert_array_equal(_assemble(shape, slabs), final)
    assert runner.observables_int() == obs
    assert runner.t == 6


def _ring_worker(rank, world, port, queue):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = []
        for shape, beta, algorithm, seed, _ in CASES:
            lat = oracle.random_lattice(shape, seed)
            b, c = partition(shape[0], world)[rank]
            for overlap in (False, True):
                slab = CpuSlab(lat, b, c, beta, seed, algorithm)
                runner = SlabRunner([slab], RingExchange(None, device="cpu"), overlap=overlap)
                series = runner.sweep(5, 1)
                runner.sweep(2)
                obs = runner.observables_int()
                out.append((series, b, slab.compressed(), obs))
        queue.put((rank, out))
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_ring_exchange_gloo(world):
    """World 2: both ring neighbours are the same rank; world 3: they differ."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ring_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for k, (shape, beta, algorithm, seed, _) in enumerate(CASES):
        lat = oracle.random_lattice(shape, seed)
        sim = oracle.OracleInt8(shape, beta, seed=seed, algorithm=algorithm, init=lat)
        want_series = sim.sweep(5, measure_every=1)
        sim.sweep(2)
        for kk in (2 * k, 2 * k + 1):  # without and with overlap
            for rank in range(world):
                series, _, _, obs = got[rank][kk]
                np.testing.assert_array_equal(series, want_series)
                assert obs == sim.observables_int()
            parts = sorted(((got[r][kk][1], r), got[r][kk][2]) for r in range(world))
            c0 = np.concatenate([p[1][0] for p in parts])
            c1 = np.concatenate([p[1][1] for p in parts])
            np.testing.assert_array_equal(oracle.from_compressed(c0, c1, shape),
                                          sim.get_lattice())


# ------------------------------------------------------------------------------ GPU ---------
GPU_CASES = [
    ("int8", (64, 96), "metropolis", 0.44, 2),
    ("int8", (30, 48), "heatbath", 0.5, 3),   # uneven slabs, odd first rows
    ("int8", (12, 10, 40), "metropolis", 0.22, 3),
    ("int8", (10, 8, 32), "heatbath", 0.25, 4),
    ("msc", (34, 256), "metropolis", 0.44, 3),
    ("msc", (38, 4096), "metropolis", 0.44, 3),  # 32-word rows: the strip schedule, odd slabs
    ("msc", (20, 8192), "metropolis", 0.3, 2),
    ("int8", (32, 64), "heatbath", -0.3, 2),  # negative beta: the per-site lookup rule
]


@pytest.mark.gpu
@pytest.mark.parametrize("exchange,overlap", [("peer", False), ("copy", False), ("copy", True)])
@pytest.mark.parametrize("variant,shape,algorithm,beta,parts", GPU_CASES)
def test_gpu_slabs_match_one_handle(variant, shape, algorithm, beta, parts, exchange, overlap):
    from pyising_b200.backend import B200Int8, B200MultiSpin
    from pyising_b200.slab import SlabSimulation

    seed = 2024
    one_cls = B200MultiSpin if variant == "msc" else B200Int8
    one = one_cls(shape, beta, seed=seed, algorithm=algorithm, init="hot")
    split = SlabSimulation(shape, beta, seed=seed, algorithm=algorithm, variant=variant,
                           init="hot", parts=parts, devices=[0], exchange=exchange,
                           overlap=overlap)
    np.testing.assert_array_equal(split.get_lattice(), one.get_lattice())
    want = one.sweep_measured(12, 3)
    got = split.sweep_measured(12, 3)
    np.testing.assert_array_equal(got, want)
    one.sweep(5)
    split.sweep(5)
    assert split.t == one.t == 17
    np.testing.assert_array_equal(split.get_lattice(), one.get_lattice())
    assert split.observables_int() == one.observables_int()
    split.close()


@pytest.mark.gpu
@pytest.mark.parametrize("variant,shape", [("int8", (24, 40)), ("int8", (6, 8, 16)),
                                           ("msc", (20, 128))])
def test_gpu_slab_philox_start_and_oracle(variant, shape):
    from pyising_b200.slab import SlabSimulation

    split = SlabSimulation(shape, 0.4 if len(shape) == 2 else 0.2, seed=77, variant=variant,
                           init="philox", parts=3, devices=[0])
    lat = oracle.philox_start(shape, 77)
    np.testing.assert_array_equal(split.get_lattice(), lat)
    sim = oracle.create(variant, shape=shape, beta=split.beta, seed=77, init=lat)
    np.testing.assert_array_equal(split.sweep_measured(4, 2), sim.sweep(4, measure_every=2))
    np.testing.assert_array_equal(split.get_lattice(), sim.get_lattice())
    split.set_beta(0.1)
    sim.set_beta(0.1)
    split.sweep(3)
    sim.sweep(3)
    np.testing.assert_array_equal(split.get_lattice(), sim.get_lattice())
    split.close()


@pytest.mark.gpu
def test_gpu_slab_argument_errors():
    from pyising_b200.slab import Slab

    tab = oracle.threshold_table(0.4, 2, "metropolis")
    with pytest.raises(ValueError):
        Slab((16, 16), tab, 0, "metropolis", "int8", 10, 8)  # beyond the axis
    with pytest.raises(ValueError):
        Slab((16, 16), tab, 0, "metropolis", "int8", 0, 0)
    with pytest.raises(ValueError):
        Slab((16, 16, 16), tab, 0, "metropolis", "msc", 0, 4)
    s = Slab((16, 16), tab, 0, "metropolis", "int8", 4, 4)
    with pytest.raises(ValueError):
        s.half_sweep(0, 0, slot=0)  # no series reset
    with pytest.raises(ValueError):
        s.half_sweep(2, 0)
    far = Slab((16, 16), tab, 0, "metropolis", "int8", 12, 4)
    other = Slab((16, 32), tab, 0, "metropolis", "int8", 0, 4)
    with pytest.raises(ValueError):
        s.set_peer(0, far)  # [12, 16) is not the low neighbour of [4, 8)
    with pytest.raises(ValueError):
        s.set_peer(1, other)  # another lattice
    with pytest.raises(ValueError):
        s.set_peer(2, far)
    s.set_peer(1, Slab((16, 16), tab, 0, "metropolis", "int8", 8, 8))
    s.set_peer(1, None)
    for x in (s, far, other):
        x.close()


def _nccl_world1_worker(port, queue):
    import torch.distributed as dist

    from pyising_b200.backend import B200Int8
    from pyising_b200.slab import SlabSimulation

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        shape = (6, 8, 32)
        one = B200Int8(shape, 0.25, seed=5, algorithm="heatbath", init="hot")
        split = SlabSimulation(shape, 0.25, seed=5, algorithm="heatbath", init="hot",
                               group="default")
        ok = bool(np.array_equal(split.sweep_measured(6, 2), one.sweep_measured(6, 2)))
        ok = ok and bool(np.array_equal(split.get_lattice(), one.get_lattice()))
        ok = ok and split.observables_int() == one.observables_int()
        split.close()
        queue.put(ok)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_gpu_slab_process_group_world1_nccl():
    """The process-group path (one slab per rank, NCCL all-reduce) on a world of one rank."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_world1_worker, args=(_free_port(), q))
    p.start()
    ok = q.get(timeout=240)
    p.join(timeout=60)
    assert p.exitcode == 0 and ok
