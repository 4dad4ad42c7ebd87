"""Physics validation suite of the B200 backend -> JSON (after src/pyising/validate.py).

    python -m pyising_b200.validate [--quick] [--out validation.json]

Every scan runs as batched ensembles (pyising_b200.physics), one lattice per (size,
temperature, kind), each bit-identical to running it alone:

1. 2D energy per spin vs the exact finite-lattice value (Kaufman / Ferdinand-Fisher) at every
   temperature, for Metropolis (int8 and multi-spin coding) and heat bath; |m| vs Onsager-Yang.
2. 2D Binder-cumulant crossings of several sizes vs Onsager's T_c.
3. 3D Binder-cumulant crossings vs the simple-cubic critical coupling (Ferrenberg, Xu & Landau).
4. 3D Metropolis vs heat bath energies (two different Markov chains, one equilibrium).
5. 2D and 3D Binder crossings again from Swendsen-Wang cluster chains on the device.

The reference equilibrates its starts and runs its Binder scans and 3D comparison with a CPU
Wolff sampler (src/pyising/validate.py:45-50,127-178); here the starts come from Swendsen-Wang
updates on the device (item 1), the batched local-update chains run long enough near T_c to
outlast their autocorrelation (items 2-4), and item 5 repeats the crossings with cluster
chains.  Bitwise identity against the NumPy oracle is
the job of the test suite (tests/), which is where the oracle may be imported.
"""

from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from .physics import BETA_C_3D, TC_2D, TC_3D, binder_scan, temperature_scan

# Sizes, temperatures and run lengths: QUICK as the reference's QUICK (3D Binder sizes 8 and 16:
# int8 rows need Lx % 8 == 0), FULL with the reference's FULL sizes and temperature grids
# (src/pyising/validate.py:28-42) and local-update run lengths.
QUICK = {
    "L2": 128, "T2": [1.8, 2.1, TC_2D, 2.5, 3.0], "therm": 1000, "meas": 500, "every": 4,
    "binder2_L": [8, 16], "binder2_T": list(np.linspace(2.2, 2.34, 5)),
    "binder2_therm": 4000, "binder2_meas": 20000, "binder2_every": 2,
    "binder3_L": [8, 16], "binder3_T": list(np.linspace(4.45, 4.57, 5)),
    "binder3_therm": 4000, "binder3_meas": 20000, "binder3_every": 2,
    "L3": 16, "T3": [4.0, TC_3D, 5.0],
    "equilibrate": 100, "cluster2_L": [8, 16], "cluster3_L": [8, 16], "cluster_therm": 100,
    "cluster_meas": 2000,
}
FULL = {
    "L2": 128, "T2": sorted(list(np.round(np.linspace(1.6, 3.4, 19), 3)) + [TC_2D]),
    "therm": 2000, "meas": 2000, "every": 10,
    "binder2_L": [8, 16, 32, 64], "binder2_T": list(np.round(np.linspace(2.20, 2.34, 15), 4)),
    "binder2_therm": 40000, "binder2_meas": 100000, "binder2_every": 5,
    "binder3_L": [8, 16, 32], "binder3_T": list(np.round(np.linspace(4.47, 4.55, 9), 4)),
    "binder3_therm": 20000, "binder3_meas": 50000, "binder3_every": 5,
    "L3": 32, "T3": [3.5, 4.2, TC_3D, 5.0, 6.0],
    "equilibrate": 300, "cluster2_L": [8, 16, 32, 64], "cluster3_L": [8, 16, 32],
    "cluster_therm": 200, "cluster_meas": 10000,
}


def _near(T: float, tc: float) -> bool:
    return abs(T - tc) < 0.15 * tc / 2.27


def scan_2d(cfg: dict, log=print) -> list[dict]:
    """Item 1: four times more measurements within 0.15 of T_c (longest autocorrelations)."""
    near = [T for T in cfg["T2"] if _near(T, TC_2D)]
    far = [T for T in cfg["T2"] if not _near(T, TC_2D)]
    rows = []
    for Ts, mult in ((far, 1), (near, 4)):
        if Ts:
            rows += temperature_scan(cfg["L2"], Ts, cfg["therm"], cfg["meas"] * mult,
                                     cfg["every"], equilibrate=cfg["equilibrate"])
    rows.sort(key=lambda r: (r["variant"], r["algorithm"], r["T"]))
    for r in rows:
        log(f"  2D {r['variant']:<5} {r['algorithm']:<10} T={r['T']:.4f} |m|={r['abs_m']:.5f} "
            f"(Yang {r['m_exact_inf']:.5f}) e={r['e']:.6f}+-{r['e_err']:.6f} "
            f"(exact L={r['L']}: {r['e_exact_L']:.6f}, z={r['e_z']:+.2f})")
    return rows


def binder(cfg: dict, dim: int, log=print) -> dict:
    """Items 2 and 3: Binder cumulants of every size and temperature, crossings of
    consecutive sizes; the estimate is the crossing of the two largest sizes."""
    k = f"binder{dim}"
    out = binder_scan(cfg[f"{k}_L"], cfg[f"{k}_T"], cfg[f"{k}_therm"], cfg[f"{k}_meas"],
                      cfg[f"{k}_every"], dim=dim,
                      algorithm="metropolis" if dim == 2 else "heatbath")
    ref = TC_2D if dim == 2 else TC_3D
    Ls = cfg[f"{k}_L"]
    est = out["crossings"][f"{Ls[-2]}-{Ls[-1]}"]
    out.update({"dim": dim, "L": Ls, "Tc_reference": ref, "Tc_estimate": est,
                "Tc_rel_error": abs(est - ref) / ref})
    out["U4"] = {str(L): v for L, v in out["U4"].items()}
    out["U4_err"] = {str(L): v for L, v in out["U4_err"].items()}
    for pair, tc in out["crossings"].items():
        log(f"  Binder crossing {dim}D L={pair}: T = {tc:.5f} (reference {ref:.5f})")
    return out


def cluster_binder(cfg: dict, dim: int, log=print) -> dict:
    """Items 2 and 3 again with Swendsen-Wang chains on the device, at the reference's sizes
    (its Wolff scans, src/pyising/validate.py:127-150)."""
    from .physics import cluster_binder_scan

    Ls = cfg[f"cluster{dim}_L"]
    out = cluster_binder_scan(Ls, cfg[f"binder{dim}_T"], cfg["cluster_therm"],
                              cfg["cluster_meas"], dim=dim)
    ref = TC_2D if dim == 2 else TC_3D
    est = out["crossings"][f"{Ls[-2]}-{Ls[-1]}"]
    out.update({"dim": dim, "L": Ls, "Tc_reference": ref, "Tc_estimate": est,
                "Tc_rel_error": abs(est - ref) / ref, "updates": "Swendsen-Wang"})
    out["U4"] = {str(L): v for L, v in out["U4"].items()}
    out["U4_err"] = {str(L): v for L, v in out["U4_err"].items()}
    for pair, tc in out["crossings"].items():
        log(f"  Swendsen-Wang Binder crossing {dim}D L={pair}: T = {tc:.5f} (reference {ref:.5f})")
    return out


def scan_3d(cfg: dict, log=print) -> list[dict]:
    """Item 4: Metropolis and heat bath at the same L and T (independent seeds); their energy
    difference in units of its combined standard error."""
    L = cfg["L3"]
    near = [T for T in cfg["T3"] if _near(T, TC_3D)]
    far = [T for T in cfg["T3"] if not _near(T, TC_3D)]
    rows = []
    for Ts, mult in ((far, 1), (near, 4)):
        if Ts:
            rows += temperature_scan(L, Ts, cfg["therm"], cfg["meas"] * mult, cfg["every"],
                                     kinds=(("int8", "metropolis"), ("int8", "heatbath")), dim=3,
                                     seed=11)
    out = []
    for T in sorted(cfg["T3"]):
        m = next(r for r in rows if r["T"] == T and r["algorithm"] == "metropolis")
        h = next(r for r in rows if r["T"] == T and r["algorithm"] == "heatbath")
        err = float(np.hypot(m["e_err"], h["e_err"]))
        out.append({"L": L, "T": float(T), "metropolis": m, "heatbath": h,
                    "e_z": (m["e"] - h["e"]) / err if err > 0 else float("nan")})
        log(f"  3D T={T:.4f} Metropolis e={m['e']:.5f}+-{m['e_err']:.5f}  heat bath "
            f"e={h['e']:.5f}+-{h['e_err']:.5f}  z={out[-1]['e_z']:+.2f}")
    return out


def summarize(res: dict) -> dict:
    s2 = res["scan2d"]
    away = [r for r in s2 if abs(r["T"] - TC_2D) > 0.2 and r["T"] < TC_2D]
    return {
        "e_max_abs_err_vs_exact_L": max(abs(r["e"] - r["e_exact_L"]) for r in s2),
        "e_max_abs_z": max(abs(r["e_z"]) for r in s2),
        "m_max_abs_err_vs_yang_away_from_Tc": max(
            (abs(r["abs_m"] - r["m_exact_inf"]) for r in away), default=float("nan")),
        "Tc2d_estimate": res["binder2d"]["Tc_estimate"],
        "Tc2d_rel_error": res["binder2d"]["Tc_rel_error"],
        "Tc3d_estimate": res["binder3d"]["Tc_estimate"],
        "Tc3d_rel_error": res["binder3d"]["Tc_rel_error"],
        "e3d_max_abs_z_metropolis_vs_heatbath": max(abs(r["e_z"]) for r in res["scan3d"]),
        "Tc2d_cluster_estimate": res["binder2d_cluster"]["Tc_estimate"],
        "Tc2d_cluster_rel_error": res["binder2d_cluster"]["Tc_rel_error"],
        "Tc3d_cluster_estimate": res["binder3d_cluster"]["Tc_estimate"],
        "Tc3d_cluster_rel_error": res["binder3d_cluster"]["Tc_rel_error"],
    }


def run(quick: bool = False, out: str | Path | None = None, log=print) -> dict:
    """The whole suite; returns the result dict (and writes it as JSON when ``out``)."""
    cfg = QUICK if quick else FULL
    t0 = time.time()
    res: dict = {"quick": quick, "config": cfg, "beta_c_3d": BETA_C_3D}
    log("[1/5] 2D energy and magnetisation vs exact results (Swendsen-Wang equilibrated starts)")
    res["scan2d"] = scan_2d(cfg, log)
    log("[2/5] 2D Binder crossing")
    res["binder2d"] = binder(cfg, 2, log)
    log("[3/5] 3D Binder crossing")
    res["binder3d"] = binder(cfg, 3, log)
    log("[4/5] 3D Metropolis vs heat bath")
    res["scan3d"] = scan_3d(cfg, log)
    log("[5/5] 2D and 3D Binder crossings from Swendsen-Wang chains")
    res["binder2d_cluster"] = cluster_binder(cfg, 2, log)
    res["binder3d_cluster"] = cluster_binder(cfg, 3, log)
    res["summary"] = summarize(res)
    res["seconds"] = time.time() - t0
    log(json.dumps(res["summary"]))
    if out is not None:
        Path(out).parent.mkdir(parents=True, exist_ok=True)
        Path(out).write_text(json.dumps(res, indent=1, default=float))
        log(f"wrote {out} ({res['seconds']:.0f} s)")
    return res


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--out", default="validation.json")
    args = ap.parse_args(argv)
    run(quick=args.quick, out=args.out)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
