"""Physics checks of the sweep path, in FP64 on the host, driven through the batched kernel.

The exact results follow pyising's src/pyising/exact.py and the estimators its
src/pyising/observables.py, restated from the published formulas:

* :func:`magnetization_2d` — Onsager/Yang spontaneous magnetisation (exact.py:19-25);
* :func:`energy_2d` — Onsager's energy per spin of the infinite square lattice (exact.py:28-38);
* :func:`log_partition_torus`, :func:`energy_torus`, :func:`specific_heat_torus` — the exact
  partition function of the finite periodic m x n lattice (Kaufman 1949; Ferdinand & Fisher
  1969; exact.py:51-94);
* :func:`binning_error`, :func:`binder`, :func:`jackknife_binder_error`, :func:`crossing`
  (observables.py:31-85).

:func:`temperature_scan` runs a whole scan (every temperature, algorithm and variant) as ONE
batched ensemble — each lattice bit-identical to running it alone — and summarises the exact
integer (M, E) series on the host; :func:`binder_scan` does the same for Binder cumulants of
several sizes.  The reference's own scan (src/pyising/validate.py:95-125) runs one lattice at
a time from a CPU Wolff start; this one starts ordered below T_c and from the device seeded
start above it, and thermalises with local sweeps.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

#: Onsager: sinh(2 / T_c) = 1 (src/pyising/exact.py:11-12).
TC_2D = 2.0 / math.log(1.0 + math.sqrt(2.0))
BETA_C_2D = 1.0 / TC_2D
#: Simple-cubic critical coupling (Ferrenberg, Xu & Landau 2018; src/pyising/exact.py:13-15).
BETA_C_3D = 0.221654626
TC_3D = 1.0 / BETA_C_3D


# ------------------------------------------------------------------ exact results --------
def magnetization_2d(T):
    """(1 - sinh(2/T)^-4)^(1/8) below T_c, 0 above."""
    T = np.asarray(T, dtype=float)
    s = np.sinh(2.0 / T)
    with np.errstate(invalid="ignore", divide="ignore"):
        inner = np.clip(1.0 - s ** -4.0, 0.0, None)
    return np.where(T < TC_2D, inner ** 0.125, 0.0)


def energy_2d(T):
    """u(K) = -coth 2K [1 + (2/pi)(2 tanh^2 2K - 1) K_1(k^2)], k = 2 sinh 2K / cosh^2 2K
    (K_1 the complete elliptic integral of the first kind, parameter m = k^2)."""
    from scipy.special import ellipk

    K = 1.0 / np.asarray(T, dtype=float)
    k = 2.0 * np.sinh(2.0 * K) / np.cosh(2.0 * K) ** 2
    m = np.minimum(k * k, 1.0 - 1e-16)  # the logarithmic singularity sits at T_c
    t2 = np.tanh(2.0 * K) ** 2
    return -(1.0 / np.tanh(2.0 * K)) * (1.0 + (2.0 / np.pi) * (2.0 * t2 - 1.0) * ellipk(m))


def _log_2cosh(x):
    a = np.abs(x)
    return a + np.log1p(np.exp(-2.0 * a))


def _log_abs_2sinh(x):
    a = np.abs(x)
    with np.errstate(divide="ignore"):
        return a + np.log1p(-np.exp(-2.0 * a)), np.sign(x)


def log_partition_torus(K: float, m: int, n: int) -> float:
    """ln Z of the m x n periodic square lattice at coupling K.

    Z = (1/2) (2 sinh 2K)^(mn/2) (Z_1 + Z_2 + Z_3 + Z_4), with Z_1 = prod_r 2 cosh(m g_{2r+1}/2),
    Z_2 = prod_r 2 sinh(m g_{2r+1}/2), Z_3, Z_4 the same over g_{2r} (r = 0 .. n-1), where
    cosh g_l = cosh 2K coth 2K - cos(pi l / n) and g_0 = 2K + ln tanh K (negative above T_c, so
    Z_4 changes sign there).  Summed in log space with signs.
    """
    r = np.arange(n)
    c = math.cosh(2.0 * K) / math.tanh(2.0 * K)

    def gam(l):
        g = np.arccosh(np.maximum(c - np.cos(np.pi * l / n), 1.0))
        return np.where(l == 0, 2.0 * K + math.log(math.tanh(K)), g)

    parts = []
    for g in (gam(2 * r + 1), gam(2 * r)):
        parts.append((float(np.sum(_log_2cosh(m * g / 2.0))), 1.0))
        ls, sg = _log_abs_2sinh(m * g / 2.0)
        parts.append((float(np.sum(ls)), float(np.prod(sg))))
    top = max(v for v, _ in parts)
    s = sum(sg * math.exp(v - top) for v, sg in parts if np.isfinite(v))
    return (-math.log(2.0) + 0.5 * m * n * math.log(2.0 * math.sinh(2.0 * K)) + top
            + math.log(s))


def energy_torus(T: float, L: int, h: float = 1e-5) -> float:
    """Exact energy per spin of the L x L torus: -(d ln Z / dK) / L^2 (central difference)."""
    K = 1.0 / T
    return -(log_partition_torus(K + h, L, L) - log_partition_torus(K - h, L, L)) / (2 * h) / L**2


def specific_heat_torus(T: float, L: int, h: float = 1e-4) -> float:
    """Exact specific heat per spin of the L x L torus: K^2 (d^2 ln Z / dK^2) / L^2."""
    K = 1.0 / T
    f = [log_partition_torus(K + s * h, L, L) for s in (-1, 0, 1)]
    return K * K * (f[0] - 2.0 * f[1] + f[2]) / (h * h) / L**2


# ------------------------------------------------------------------ estimators -----------
def binning_error(x, n_bins: int = 32) -> float:
    """Standard error of the mean from n_bins equal blocks."""
    x = np.asarray(x, dtype=float)
    nb = min(n_bins, x.size)
    if nb < 2:
        return float("nan")
    blocks = x[: x.size // nb * nb].reshape(nb, -1).mean(axis=1)
    return float(blocks.std(ddof=1) / math.sqrt(nb))


def binder(m) -> float:
    """U_4 = 1 - <m^4> / (3 <m^2>^2)."""
    m = np.asarray(m, dtype=float)
    return float(1.0 - np.mean(m ** 4) / (3.0 * np.mean(m ** 2) ** 2))


def jackknife_binder_error(m, n_bins: int = 32) -> float:
    """Blocked jackknife error of :func:`binder`."""
    m = np.asarray(m, dtype=float)
    nb = min(n_bins, m.size)
    if nb < 2:
        return float("nan")
    blocks = m[: m.size // nb * nb].reshape(nb, -1)
    m2, m4 = (blocks ** 2).mean(axis=1), (blocks ** 4).mean(axis=1)
    s2, s4 = m2.sum(), m4.sum()
    jk = 1.0 - ((s4 - m4) / (nb - 1)) / (3.0 * ((s2 - m2) / (nb - 1)) ** 2)
    return float(math.sqrt((nb - 1) * np.mean((jk - jk.mean()) ** 2)))


def crossing(Ts, u_a, u_b) -> float:
    """Temperature where two Binder curves cross (linear interpolation of their difference)."""
    d = np.asarray(u_a, dtype=float) - np.asarray(u_b, dtype=float)
    for i in range(len(d) - 1):
        if d[i] == 0:
            return float(Ts[i])
        if d[i] * d[i + 1] < 0:
            return float(Ts[i] - d[i] * (Ts[i + 1] - Ts[i]) / (d[i + 1] - d[i]))
    return float("nan")


@dataclass
class Summary:
    """Per-spin estimates from an exact (M, E) series after thermalisation."""

    abs_m: float
    abs_m_err: float
    e: float
    e_err: float
    binder: float
    binder_err: float
    n: int

    @classmethod
    def from_series(cls, series: np.ndarray, n_spins: int, skip: int = 0) -> Summary:
        s = np.asarray(series, dtype=np.int64)[skip:]
        m = s[:, 0].astype(float) / n_spins
        e = s[:, 1].astype(float) / n_spins
        am = np.abs(m)
        return cls(float(am.mean()), binning_error(am), float(e.mean()), binning_error(e),
                   binder(m), jackknife_binder_error(m), int(len(s)))


# ------------------------------------------------------------------ cluster updates ------
def equilibrated(shape, T: float, seed: int, steps: int = 300) -> np.ndarray:
    """An equilibrium start: ``steps`` Swendsen-Wang updates on the device from a cold start
    (pyising equilibrates with CPU Wolff updates, src/pyising/validate.py:45-50)."""
    from .backend import B200Int8

    sim = B200Int8(tuple(shape), 1.0 / T, seed=seed, init="cold")
    sim.cluster_sweep(steps)
    return sim.get_lattice()


def cluster_binder_scan(Ls, Ts, therm: int, meas: int, dim: int = 2, seed: int = 21) -> dict:
    """Binder cumulants from Swendsen-Wang chains (one lattice per (L, T), (M, E) after every
    update measured on the device) and the crossings of consecutive sizes; the cluster dynamics
    decorrelate near T_c in a few updates, as pyising's Wolff scans do
    (src/pyising/validate.py:127-150)."""
    from .backend import B200Int8

    Ts = [float(t) for t in Ts]
    u = {L: [0.0] * len(Ts) for L in Ls}
    err = {L: [0.0] * len(Ts) for L in Ls}
    for a, L in enumerate(Ls):
        for i, T in enumerate(Ts):
            sim = B200Int8((L,) * dim, 1.0 / T, seed=seed + 1000 * a + i, init="cold")
            sim.cluster_sweep(therm)
            s = Summary.from_series(sim.cluster_sweep(meas, measure=True), L ** dim)
            u[L][i], err[L][i] = s.binder, s.binder_err
    crossings = {f"{a}-{b}": crossing(Ts, u[a], u[b]) for a, b in zip(Ls, Ls[1:])}
    return {"T": Ts, "U4": u, "U4_err": err, "crossings": crossings}


# ------------------------------------------------------------------ batched scans --------
def temperature_scan(L: int, Ts, therm: int, meas: int, every: int,
                     kinds=(("int8", "metropolis"), ("msc", "metropolis"),
                            ("int8", "heatbath")), seed: int = 7, dim: int = 2,
                     equilibrate: int = 0) -> list[dict]:
    """Every (kind, T) of a scan as one batched ensemble; returns a row per lattice with the
    estimates and, in 2D, the exact finite-torus energy and the Onsager-Yang magnetisation.

    Each lattice gets its own seed (seed + 1000 k + i): with one shared seed the counter-based
    uniforms would be identical at every temperature and the errors would correlate.  With
    ``equilibrate`` > 0 every lattice starts from that many Swendsen-Wang updates
    (:func:`equilibrated`), else ordered below T_c and disordered above."""
    from .ensemble import Ensemble, Job

    shape = (L,) * dim
    tc = TC_2D if dim == 2 else TC_3D
    jobs, keys = [], []
    for k, (variant, alg) in enumerate(kinds):
        for i, T in enumerate(Ts):
            if equilibrate > 0:
                init = equilibrated(shape, T, seed=int(1000 * T) + k, steps=equilibrate)
            else:
                # ordered start below T_c (a hot start can freeze into a long-lived striped
                # state there), device seeded disordered start above
                init = "cold" if T < tc else "philox"
            jobs.append(Job(shape, 1.0 / T, therm + meas * every, seed=seed + 1000 * k + i,
                            variant=variant, algorithm=alg, measure_every=every, init=init))
            keys.append((variant, alg, float(T)))
    rows = []
    with Ensemble() as ens:
        ids = [ens.add(j) for j in jobs]
        ens.run()
        for (variant, alg, T), jid in zip(keys, ids, strict=True):
            s = Summary.from_series(ens.result(jid).series, L ** dim, skip=therm // every)
            row = {"variant": variant, "algorithm": alg, "L": L, "T": T, **s.__dict__}
            if dim == 2:
                row["e_exact_L"] = energy_torus(T, L)
                row["m_exact_inf"] = float(magnetization_2d(T))
                row["e_z"] = (s.e - row["e_exact_L"]) / s.e_err if s.e_err > 0 else float("nan")
            rows.append(row)
    return rows


def binder_scan(Ls, Ts, therm: int, meas: int, every: int, dim: int = 2,
                algorithm: str = "metropolis", seed: int = 11) -> dict:
    """Binder cumulants U_4(L, T) of every size and temperature in one batched ensemble, and
    the crossing temperatures of consecutive sizes."""
    from .ensemble import Ensemble, Job

    Ts = [float(t) for t in Ts]
    jobs, keys = [], []
    for a, L in enumerate(Ls):
        for i, T in enumerate(Ts):
            jobs.append(Job((L,) * dim, 1.0 / T, therm + meas * every, seed=seed + 1000 * a + i,
                            algorithm=algorithm, measure_every=every, init="philox"))
            keys.append((L, i))
    u = {L: [0.0] * len(Ts) for L in Ls}
    err = {L: [0.0] * len(Ts) for L in Ls}
    with Ensemble() as ens:
        ids = [ens.add(j) for j in jobs]
        ens.run()
        for (L, i), jid in zip(keys, ids, strict=True):
            s = Summary.from_series(ens.result(jid).series, L ** dim, skip=therm // every)
            u[L][i], err[L][i] = s.binder, s.binder_err
    crossings = {f"{a}-{b}": crossing(Ts, u[a], u[b]) for a, b in zip(Ls, Ls[1:])}
    return {"T": Ts, "U4": u, "U4_err": err, "crossings": crossings}
