"""Generate the golden fixtures in this folder by running the pyising reference itself.

Run once, with --reference pointing at the reference source; the GPU host never runs
this.  Every array comes from the reference's own functions: ``pyising.philox``,
``pyising.lattice`` and the NumPy backends (``src/pyising/backends/numpy_backend.py``).

    python tests/golden/make_golden.py --reference <pyising checkout>/src [--quick]

Files written (all ``.npz``):
  philox.npz      Philox4x32-10 known answers: the Random123 vectors listed in the reference's
                  tests/test_philox.py plus 512 seeded random (counter, key) pairs.
  streams.npz     site_uniforms / word_randoms samples, split_seed.
  tables.npz      threshold_table for several (beta, ndim, algorithm).
  int8_cases.npz  the int8 identity cases of tests/test_backends.py:22-36 and
                  validate.py:72-75, plus the set_beta/split-sweep case.
  msc_cases.npz   the msc identity cases of tests/test_backends.py:39-51 and validate.py:75.
  c1_int8_L1024.npz   1024^2 int8 Metropolis, beta_c, seed 1, hot start, 1000 sweeps.
  c2_msc.npz          msc 1024^2 x 1000 sweeps and 2048^2 x 200 sweeps, T_c, seed 7, hot.
  c3_int8_3d_L64.npz  64^3 int8 heat bath, beta 0.221654626, cold, 2000 sweeps, (M, E) every 10.
  c4_batch.npz        the first lattices (L <= 128) of the seeded 96-lattice ensemble, 500 sweeps.
  exact.npz       pyising.exact: energy_torus / specific_heat_torus on a (T, L) grid,
                  magnetization_2d and energy_2d on a T grid (``--only exact`` writes just this).
Lattices are stored as np.packbits(lat > 0) with their shape.
"""

from __future__ import annotations

import argparse
import ast
import math
import sys
import time
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def packed(lat: np.ndarray) -> np.ndarray:
    return np.packbits((lat > 0).reshape(-1))


def me(lat: np.ndarray) -> tuple[int, int]:
    """Exact integers from the reference's per-spin floats (N <= 2^28, exact in float64)."""
    from pyising.lattice import energy_per_spin, magnetization

    n = lat.size
    return int(round(magnetization(lat) * n)), int(round(energy_per_spin(lat) * n))


def _literal(node):
    """Tuples/lists of integer constants, allowing ``(x,) * n`` (no other evaluation)."""
    if isinstance(node, ast.Constant) and isinstance(node.value, int):
        return node.value
    if isinstance(node, (ast.Tuple, ast.List)):
        return tuple(_literal(e) for e in node.elts)
    if isinstance(node, ast.BinOp) and isinstance(node.op, ast.Mult):
        seq, n = _literal(node.left), _literal(node.right)
        if isinstance(seq, tuple) and isinstance(n, int):
            return seq * n
    raise ValueError(f"unsupported node {ast.dump(node)[:80]}")


def kat_vectors(ref_root: Path):
    """The Random123 known-answer list in the reference's tests/test_philox.py, read as text."""
    src = (ref_root.parent / "tests" / "test_philox.py").read_text()
    tree = ast.parse(src)
    for node in tree.body:
        if isinstance(node, ast.Assign) and getattr(node.targets[0], "id", "") == "KAT":
            return list(_literal(node.value))
    raise RuntimeError("KAT list not found")


def write_exact() -> None:
    """The reference's exact finite-torus and infinite-lattice results (src/pyising/exact.py)."""
    from pyising import exact

    Ts = np.array([1.5, 1.8, 2.0, 2.2, exact.TC_2D, 2.4, 2.6, 3.0, 4.0])
    Ls = np.array([4, 8, 16, 32, 64, 128])
    e = np.array([[exact.energy_torus(float(T), int(L)) for L in Ls] for T in Ts])
    c = np.array([[exact.specific_heat_torus(float(T), int(L)) for L in Ls] for T in Ts])
    np.savez_compressed(OUT / "exact.npz", T=Ts, L=Ls, energy_torus=e, specific_heat_torus=c,
                        magnetization_2d=exact.magnetization_2d(Ts), energy_2d=exact.energy_2d(Ts))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="the pyising source folder (the checkout's src/)")
    ap.add_argument("--quick", action="store_true", help="skip the long config runs")
    ap.add_argument("--only", choices=["exact"], default=None, help="write one fixture only")
    args = ap.parse_args()
    ref_root = Path(args.reference)
    sys.path.insert(0, str(ref_root))
    write_exact()
    if args.only == "exact":
        return 0
    from pyising import backends as B
    from pyising.exact import BETA_C_2D
    from pyising.lattice import random_lattice, threshold_table
    from pyising.philox import philox4x32, site_uniforms, split_seed, word_randoms

    t_start = time.time()
    # ---- Philox ------------------------------------------------------------------------
    kat = kat_vectors(ref_root)
    rng = np.random.default_rng(20261203)
    ctr = rng.integers(0, 2**32, size=(512, 4), dtype=np.uint64)
    key = rng.integers(0, 2**32, size=(512, 2), dtype=np.uint64)
    out = np.zeros((512, 4), dtype=np.uint32)
    for i in range(512):
        r = philox4x32(*[int(x) for x in ctr[i]], int(key[i, 0]), int(key[i, 1]))
        out[i] = [int(x) for x in r]
    np.savez_compressed(
        OUT / "philox.npz",
        kat_ctr=np.array([k[0] for k in kat], dtype=np.uint32),
        kat_key=np.array([k[1] for k in kat], dtype=np.uint32),
        kat_out=np.array([k[2] for k in kat], dtype=np.uint32),
        rnd_ctr=ctr.astype(np.uint32), rnd_key=key.astype(np.uint32), rnd_out=out)

    # ---- streams -------------------------------------------------------------------------
    su = site_uniforms(64, 5, 1, 2**40 + 3)
    wr = [word_randoms(16, 3, 0, 12345, lp) for lp in range(3)]
    np.savez_compressed(
        OUT / "streams.npz", site_uniforms=su, split_seed=np.array(split_seed(2**40 + 3)),
        word_randoms=np.array([[a, b] for a, b in wr], dtype=np.uint64))

    # ---- tables --------------------------------------------------------------------------
    cases = []
    vals = []
    for beta in (0.0, 0.22, 0.221654626, 0.3, 0.37, 0.42, 0.44, BETA_C_2D, 0.5, 1.0, 3.0,
                 -0.2):
        for ndim in (2, 3):
            for alg in ("metropolis", "heatbath"):
                cases.append((beta, ndim, 0 if alg == "metropolis" else 1))
                t = threshold_table(beta, ndim, alg)
                vals.append(np.pad(t.astype(np.uint64), (0, 7 - len(t)),
                                   constant_values=2**40))
    np.savez_compressed(OUT / "tables.npz", cases=np.array(cases, dtype=np.float64),
                        tables=np.array(vals, dtype=np.uint64))

    # ---- int8 identity cases -------------------------------------------------------------
    rec = {}
    idx = 0
    for shape in [(16, 24), (8, 8, 16), (64, 32)]:
        for alg in ("metropolis", "heatbath"):
            lat = random_lattice(shape, 5)
            beta = 0.42 if len(shape) == 2 else 0.22
            sim = B.load("numpy", "int8")(shape, beta, seed=2**40 + 7, algorithm=alg, init=lat)
            sim.sweep(6)
            rec[f"case{idx}"] = np.array([len(shape), *shape, *([0] * (3 - len(shape)))])
            rec[f"meta{idx}"] = np.array([beta, 2**40 + 7, 6, 5, 0 if alg == "metropolis" else 1],
                                         dtype=np.float64)
            rec[f"final{idx}"] = packed(sim.get_lattice())
            idx += 1
    for shape, alg in [((32, 64), "metropolis"), ((32, 64), "heatbath"),
                       ((8, 8, 16), "metropolis"), ((8, 8, 16), "heatbath")]:
        lat = random_lattice(shape, 2024)
        beta = 0.42 if len(shape) == 2 else 0.22
        sim = B.load("numpy", "int8")(shape, beta, seed=99, algorithm=alg, init=lat)
        sim.sweep(8)
        rec[f"case{idx}"] = np.array([len(shape), *shape, *([0] * (3 - len(shape)))])
        rec[f"meta{idx}"] = np.array([beta, 99, 8, 2024, 0 if alg == "metropolis" else 1],
                                     dtype=np.float64)
        rec[f"final{idx}"] = packed(sim.get_lattice())
        idx += 1
    # set_beta + split sweeps (tests/test_backends.py:54-68)
    lat = random_lattice((128, 128), 1)
    a = B.load("numpy", "int8")((128, 128), 0.3, seed=3, init=lat)
    a.sweep(2)
    a.set_beta(0.5)
    a.sweep(3)
    rec["set_beta_final"] = packed(a.get_lattice())
    rec["n_cases"] = np.array(idx)
    np.savez_compressed(OUT / "int8_cases.npz", **rec)

    # ---- msc identity cases --------------------------------------------------------------
    rec = {}
    idx = 0
    for shape, beta, seed, init_seed, n in [((128, 128), 0.44, 11, 9, 5),
                                            ((64, 384), 0.44, 11, 9, 5),
                                            ((128, 256), 0.42, 99, 2024, 8)]:
        lat = random_lattice(shape, init_seed)
        sim = B.load("numpy", "msc")(shape, beta, seed=seed, init=lat)
        sim.sweep(n)
        rec[f"case{idx}"] = np.array(shape)
        rec[f"meta{idx}"] = np.array([beta, seed, n, init_seed], dtype=np.float64)
        rec[f"final{idx}"] = packed(sim.get_lattice())
        idx += 1
    lat = random_lattice((128, 128), 1)
    a = B.load("numpy", "msc")((128, 128), 0.3, seed=3, init=lat)
    a.sweep(2)
    a.set_beta(0.5)
    a.sweep(3)
    rec["set_beta_final"] = packed(a.get_lattice())
    rec["n_cases"] = np.array(idx)
    np.savez_compressed(OUT / "msc_cases.npz", **rec)
    print(f"small fixtures done in {time.time() - t_start:.1f} s", flush=True)
    if args.quick:
        return 0

    # ---- C1: int8 2D L=1024, beta_c, seed 1, hot, 1000 sweeps ----------------------------
    shape = (1024, 1024)
    sim = B.create("numpy", "int8", shape=shape, beta=BETA_C_2D, seed=1,
                   init=random_lattice(shape, 1))
    series = []
    for _ in range(10):
        sim.sweep(100)
        series.append(me(sim.get_lattice()))
    np.savez_compressed(OUT / "c1_int8_L1024.npz", shape=np.array(shape), beta=BETA_C_2D,
                        seed=1, sweeps=1000, series_every=100, series=np.array(series),
                        final=packed(sim.get_lattice()))
    print(f"C1 done in {time.time() - t_start:.1f} s", flush=True)

    # ---- C2 parity shapes: msc, T_c, seed 7, hot --------------------------------------------
    rec = {}
    for L, n in ((1024, 1000), (2048, 200)):
        shape = (L, L)
        sim = B.create("numpy", "msc", shape=shape, beta=BETA_C_2D, seed=7,
                       init=random_lattice(shape, 7))
        sim.sweep(n)
        rec[f"final{L}"] = packed(sim.get_lattice())
        rec[f"me{L}"] = np.array(me(sim.get_lattice()))
        rec[f"sweeps{L}"] = np.array(n)
    np.savez_compressed(OUT / "c2_msc.npz", beta=BETA_C_2D, seed=7, **rec)
    print(f"C2 done in {time.time() - t_start:.1f} s", flush=True)

    # ---- C3 parity shape: 3D L=64 heat bath, cold, 2000 sweeps, (M, E) every 10 -----------
    shape = (64, 64, 64)
    beta3 = 0.221654626
    sim = B.create("numpy", "int8", shape=shape, beta=beta3, seed=0, algorithm="heatbath",
                   init="cold")
    series = []
    for _ in range(200):
        sim.sweep(10)
        series.append(me(sim.get_lattice()))
    np.savez_compressed(OUT / "c3_int8_3d_L64.npz", shape=np.array(shape), beta=beta3, seed=0,
                        sweeps=2000, series_every=10, series=np.array(series),
                        final=packed(sim.get_lattice()))
    print(f"C3 done in {time.time() - t_start:.1f} s", flush=True)

    # ---- C4: the seeded ensemble draw; the first lattices with L <= 128 ---------------------
    rng = np.random.default_rng(0)
    ks = rng.integers(6, 13, size=96)
    Ts = rng.uniform(2.0, 2.6, size=96)
    picked = [i for i in range(96) if 2 ** int(ks[i]) <= 128][:6]
    rec = {"ks": ks, "Ts": Ts, "picked": np.array(picked)}
    for i in picked:
        L = 2 ** int(ks[i])
        shape = (L, L)
        sim = B.create("numpy", "int8", shape=shape, beta=1.0 / Ts[i], seed=i,
                       init=random_lattice(shape, i))
        series = []
        for _ in range(50):
            sim.sweep(10)
            series.append(me(sim.get_lattice()))
        rec[f"final{i}"] = packed(sim.get_lattice())
        rec[f"series{i}"] = np.array(series)
    np.savez_compressed(OUT / "c4_batch.npz", sweeps=500, every=10, **rec)
    print(f"all done in {time.time() - t_start:.1f} s (beta_c = {BETA_C_2D!r}, "
          f"ln(1+sqrt2)/2 = {math.log(1 + math.sqrt(2)) / 2!r})")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
