"""Run one small sweep case, for profilers (ncu) and quick timing.

    python -m pyising_b200.profile_case {int8|hb3|msc|sw|batch|batch1|slab2|mscslab2} L SWEEPS

int8: 2D Metropolis L x L at beta_c, NumPy hot start seed 7; hb3: 3D heat bath L^3 at
beta = 0.221654626, cold start; msc: 2D multi-spin Metropolis L x L at beta_c, hot start seed 7;
sw: SWEEPS Swendsen-Wang updates of a 2D int8 L x L lattice at beta_c from a cold start;
batch: an ensemble of 2D int8 Metropolis lattices L x L, L/2 x L/2 (four each) and L/4 x L/4
(sixteen) at temperatures 2.0 .. 2.6, device seeded starts, SWEEPS sweeps with (M, E) every 10,
through the batched kernel; batch1: one 2D int8 Metropolis lattice L x L at beta_c alone in a
batch, device seeded start, no measurement; slab2 / mscslab2: a 2D int8 / msc Metropolis L x L
lattice at beta_c cut into two slabs on device 0 (neighbour rows read in place), device seeded
start.  Prints the final exact (M, E) (batch: of the first lattice).
"""

from __future__ import annotations

import sys

from .backend import B200Int8, B200MultiSpin
from .lattice import BETA_C_2D


def main(argv: list[str]) -> int:
    which, L, n = argv[0], int(argv[1]), int(argv[2])
    if which == "int8":
        sim = B200Int8((L, L), BETA_C_2D, seed=7, init="hot")
    elif which == "hb3":
        sim = B200Int8((L, L, L), 0.221654626, seed=0, algorithm="heatbath", init="cold")
    elif which == "msc":
        sim = B200MultiSpin((L, L), BETA_C_2D, seed=7, init="hot")
    elif which == "sw":
        sim = B200Int8((L, L), BETA_C_2D, seed=7, init="cold")
        sim.cluster_sweep(n)
        sim.synchronize()
        print(which, L, n, sim.observables_int())
        return 0
    elif which == "batch":
        from .ensemble import Ensemble, Job

        sizes = [L] + [L // 2] * 4 + [L // 4] * 16
        jobs = [Job((s, s), 1.0 / (2.0 + 0.6 * i / len(sizes)), n, seed=i, measure_every=10,
                    init="philox") for i, s in enumerate(sizes)]
        with Ensemble() as ens:
            ids = [ens.add(j) for j in jobs]
            ens.run()
            series = ens.result(ids[0]).series
        print(which, L, n, tuple(int(x) for x in series[-1]) if len(series) else None)
        return 0
    elif which in ("slab2", "mscslab2"):
        from .slab import SlabSimulation

        sim = SlabSimulation((L, L), BETA_C_2D, seed=7, variant="msc" if which == "mscslab2"
                             else "int8", init="philox", parts=2, devices=[0])
        sim.sweep(n)
        sim.synchronize()
        print(which, L, n, sim.observables_int())
        sim.close()
        return 0
    elif which == "batch1":
        from .ensemble import Ensemble, Job

        with Ensemble() as ens:
            i = ens.add(Job((L, L), BETA_C_2D, n, seed=7, init="philox", keep_lattice=True))
            ens.run()
            lat = ens.result(i).lattice
        print(which, L, n, int(lat.astype("int64").sum()))
        return 0
    else:
        raise SystemExit(f"unknown case {which!r}")
    sim.sweep(n)
    sim.synchronize()
    print(which, L, n, sim.observables_int())
    return 0


if __name__ == "__main__":
    raise SystemExit(main(sys.argv[1:]))
