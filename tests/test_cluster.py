"""Swendsen-Wang cluster updates on the device (ising_cluster_sweep / ising_cluster_labels).

There is no bit-exact reference for them (pyising's own cluster sampler is a CPU Wolff with
NumPy's generator, src/pyising/cluster.py:32-104), so the labeling is checked exactly against a
CPU union-find over the same active bonds, the bond rule against the spins, and the dynamics
statistically against the exact finite-torus energy (host FP64, pyising_b200.physics).
"""

from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def neighbours(shape, c0_row, j):
    """Colour-1 neighbours of colour-0 site (row, j) in the order of the bond bits."""
    ndim = len(shape)
    lh = shape[-1] // 2
    ly = shape[-2]
    lz = shape[0] if ndim == 3 else 1
    y, z = c0_row % ly, c0_row // ly
    par = (y + z) & 1
    plane = z * ly
    out = [c0_row * lh + j,
           c0_row * lh + ((j + 1) % lh if par else (j - 1) % lh),
           (plane + (y + 1) % ly) * lh + j,
           (plane + (y - 1) % ly) * lh + j]
    if ndim == 3:
        out += [(((z + 1) % lz) * ly + y) * lh + j, (((z - 1) % lz) * ly + y) * lh + j]
    return out


def components_min(n, edges):
    parent = list(range(n))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in edges:
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[max(ra, rb)] = min(ra, rb)
    return np.array([find(x) for x in range(n)])


KNOB_CLUSTER_TILE = 7


def set_cluster_tile(sim, tile):
    from pyising_b200._lib import check, lib

    check(lib().ising_set_knob(sim._h, KNOB_CLUSTER_TILE, int(tile)), "set_knob")


# tile 0: automatic (16 rows x 32 positions); 1: single-level; 32 and 100: tiles of 2 and 6 rows
# x 16 positions, so many bonds are united by the cross-tile kernel; 6144: tiles as tall as the
# lattice
@pytest.mark.parametrize("tile", [0, 1, 32, 100, 6144])
@pytest.mark.parametrize("shape,beta", [((16, 32), 0.3), ((16, 32), 0.7), ((24, 40), 0.44),
                                        ((8, 8, 16), 0.22), ((8, 8, 16), 0.5)])
def test_labels_are_the_components_of_the_active_bonds(oracle_mod, shape, beta, tile):
    from pyising_b200.backend import B200Int8

    sim = B200Int8(shape, beta, seed=77, init=oracle_mod.random_lattice(shape, 5))
    set_cluster_tile(sim, tile)
    sim.sweep(3)
    c0, c1 = sim.colour_arrays()
    labels, bonds = sim.cluster_labels(step=9)
    rows, lh = c0.shape
    S = rows * lh
    edges, aligned, active = [], 0, 0
    for r in range(rows):
        for j in range(lh):
            nbs = neighbours(shape, r, j)
            for k, m in enumerate(nbs):
                same = c0[r, j] == c1.reshape(-1)[m]
                aligned += int(same)
                if bonds[r, j] >> k & 1:
                    assert same, "an active bond joins anti-aligned spins"
                    active += 1
                    edges.append((r * lh + j, S + m))
            assert bonds[r, j] >> len(nbs) == 0
    want = components_min(2 * S, edges)
    np.testing.assert_array_equal(labels.reshape(-1), want)
    p = 1.0 - math.exp(-2.0 * beta)
    assert abs(active - p * aligned) < 5 * math.sqrt(aligned * p * (1 - p)) + 1


def test_cluster_updates_do_not_depend_on_the_tile_size():
    from pyising_b200.backend import B200Int8

    out = []
    for shape, tile in [((128, 96), 0), ((128, 96), 32), ((128, 96), 1000), ((128, 96), 6144),
                        ((16, 24, 32), 0), ((16, 24, 32), 77), ((16, 24, 32), 1024)]:
        sim = B200Int8(shape, 0.44 if len(shape) == 2 else 0.22, seed=9, init="hot")
        set_cluster_tile(sim, tile)
        series = sim.cluster_sweep(6, measure=True)
        out.append((shape, series, sim.get_lattice()))
    for (shape_a, sa, la), (shape_b, sb, lb) in zip(out, out[1:]):
        if shape_a == shape_b:
            np.testing.assert_array_equal(sa, sb)
            np.testing.assert_array_equal(la, lb)


def test_cluster_tile_knob_range():
    from pyising_b200.backend import B200Int8

    sim = B200Int8((16, 16), 0.4, init="cold")
    for bad in (-1, 2, 31, 6145):
        with pytest.raises(ValueError):
            set_cluster_tile(sim, bad)


@pytest.mark.parametrize("shape,tile", [((64, 64), 0), ((64, 64), 1), ((8, 16, 32), 0)], ids=str)
def test_bounded_union_find_loops_report_a_timeout(shape, tile):
    """The test hook writes a two-site cycle into the labels after the unions: every root walk
    that reaches it spends its step budget (or sees another thread's error) and returns, the
    call reports ISING_ERR_TIMEOUT within a fraction of a second, and the context still works."""
    import time

    from pyising_b200._lib import DeviceTimeout, IsingError, check, lib
    from pyising_b200.backend import B200Int8

    sim = B200Int8(shape, 2.0, seed=5, init="cold")  # every bond active: one spanning cluster
    set_cluster_tile(sim, tile)
    check(lib().ising_set_knob(sim._h, 8, 1), "set_knob")  # ISING_KNOB_TEST_LABEL_CYCLE
    t0 = time.perf_counter()
    with pytest.raises(DeviceTimeout):
        sim.cluster_sweep(2)
    assert time.perf_counter() - t0 < 5.0
    with pytest.raises(IsingError):
        sim.cluster_labels()
    # the context is usable: the same handle without the hook, and a fresh one, both work
    check(lib().ising_set_knob(sim._h, 8, 0), "set_knob")
    sim.set_lattice(np.ones(shape, np.int8))
    sim.cluster_sweep(2)
    fresh = B200Int8(shape, 2.0, seed=5, init="cold")
    fresh.cluster_sweep(2)
    np.testing.assert_array_equal(sim.get_lattice(), fresh.get_lattice())
    fresh.sweep(3)
    assert set(np.unique(fresh.get_lattice())) <= {-1, 1}


def test_cluster_sweeps_are_deterministic_and_keep_the_lattice_valid():
    from pyising_b200.backend import B200Int8

    runs = []
    for _ in range(3):  # the union order varies between runs; the clusters must not
        sim = B200Int8((256, 256), 0.44, seed=3, init="cold")
        sim.cluster_sweep(40)
        runs.append(sim.get_lattice())
    np.testing.assert_array_equal(runs[0], runs[1])
    np.testing.assert_array_equal(runs[0], runs[2])
    assert set(np.unique(runs[0])) <= {-1, 1}
    sim = B200Int8((64, 64), 0.0, seed=3, init="cold")  # beta = 0: no bonds, every spin random
    sim.cluster_sweep(1)
    assert abs(sim.get_lattice().mean()) < 0.1


@pytest.mark.parametrize("T", [2.0, 2.269185314213022, 3.0])
def test_cluster_dynamics_sample_the_exact_energy(T):
    from pyising_b200.backend import B200Int8
    from pyising_b200.physics import binning_error, energy_torus

    L = 32
    sim = B200Int8((L, L), 1.0 / T, seed=1234, init="cold")
    sim.cluster_sweep(200)
    e = []
    for _ in range(3000):
        sim.cluster_sweep(1)
        e.append(sim.observables_int()[1] / L**2)
    e = np.array(e)
    err = binning_error(e)
    assert abs(e.mean() - energy_torus(T, L)) < 4.5 * err, (e.mean(), energy_torus(T, L), err)


def test_measured_cluster_series_and_binder_scan():
    from pyising_b200.backend import B200Int8
    from pyising_b200.physics import TC_2D, cluster_binder_scan, equilibrated

    sim = B200Int8((32, 32), 0.44, seed=8, init="cold")
    series = sim.cluster_sweep(50, measure=True)
    assert series.shape == (50, 2) and sim.cluster_t == 50
    assert tuple(series[-1]) == sim.observables_int()
    lat = equilibrated((32, 32), 2.0, seed=4, steps=50)
    assert abs(abs(lat.mean()) - 0.9113) < 0.06  # ordered at T = 2.0
    out = cluster_binder_scan([8, 16], [2.15, 2.25, 2.35, 2.45], therm=100, meas=3000)
    assert abs(out["crossings"]["8-16"] - TC_2D) < 0.08, out
