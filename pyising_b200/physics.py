"""Physics checks of the sweep path, in FP64 on the host, driven through the batched kernel.

The exact results and estimators are written from the published physics; they provide the
quantities pyising checks with (values, not code, of src/pyising/exact.py:19-94 and
src/pyising/observables.py:28-85):

* :func:`magnetization_2d` — Onsager/Yang spontaneous magnetisation;
* :func:`energy_2d` — Onsager's energy per spin of the infinite square lattice;
* :func:`log_partition_torus`, :func:`energy_torus`, :func:`specific_heat_torus` — Kaufman's
  exact partition function of the finite periodic m x n lattice with its first and second
  derivatives in K taken analytically (pyising differentiates ln Z numerically; the two agree
  to the truncation error of its differences, and this one agrees with a full enumeration of
  small tori to rounding);
* :func:`binning_error`, :func:`binder`, :func:`jackknife_binder_error`, :func:`crossing` —
  block-mean error, Binder cumulant, its blocked jackknife error, crossing of two curves.

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
    """Spontaneous magnetisation per spin of the infinite square lattice (Onsager 1949, proved
    by Yang 1952): m = [1 - sinh(2K)^-4]^(1/8) for T < T_c, 0 above (K = 1/T, J = 1)."""
    K = 1.0 / np.asarray(T, dtype=float)
    ordered = K > BETA_C_2D
    s4 = np.sinh(2.0 * np.where(ordered, K, BETA_C_2D)) ** 4
    return np.where(ordered, np.maximum(1.0 - 1.0 / s4, 0.0) ** 0.125, 0.0)


def energy_2d(T):
    """Energy per spin of the infinite square lattice (Onsager 1944):

        u = -coth(2K) [1 + (2/pi) (2 tanh^2(2K) - 1) K(q)],   q = 2 sinh(2K) / cosh^2(2K),

    with K(q) the complete elliptic integral of the first kind of modulus q (scipy's ``ellipk``
    takes the parameter q^2).  At T_c, q = 1 and the prefactor 2 tanh^2 - 1 vanishes faster than
    K(q) diverges, so the bracket is exactly 1 there (u = -sqrt 2)."""
    from scipy.special import ellipk

    K = 1.0 / np.asarray(T, dtype=float)
    c2, s2 = np.cosh(2.0 * K), np.sinh(2.0 * K)
    q2 = (2.0 * s2 / (c2 * c2)) ** 2
    regular = q2 < 1.0
    elliptic = np.where(regular, ellipk(np.where(regular, q2, 0.0)), 0.0)
    bracket = 1.0 + (2.0 / np.pi) * (2.0 * (s2 / c2) ** 2 - 1.0) * elliptic
    return -(c2 / s2) * bracket


def _lncosh2(x):
    """ln(2 cosh x) without overflow."""
    return np.logaddexp(x, -x)


def _lnsinh2(x):
    """ln|2 sinh x| without overflow (x != 0)."""
    a = np.abs(x)
    with np.errstate(divide="ignore"):
        return a + np.log(-np.expm1(-2.0 * a))


class _KaufmanTorus:
    """ln Z of the m x n periodic square lattice and its first two derivatives in K, analytic.

    Kaufman (1949), in the form of Ferdinand & Fisher (1969):

        Z = 1/2 (2 sinh 2K)^(mn/2) (Z_1 + Z_2 + Z_3 + Z_4),
        Z_1 = prod_{l odd} 2 cosh(m g_l / 2),   Z_2 = prod_{l odd} 2 sinh(m g_l / 2),
        Z_3 = prod_{l even} 2 cosh(m g_l / 2),  Z_4 = prod_{l even} 2 sinh(m g_l / 2),

    l = 0 .. 2n-1, with cosh g_l = c(K) - cos(pi l / n), c(K) = sinh 2K + 1/sinh 2K, for l >= 1
    and g_0 = 2K + ln tanh K, which changes sign at T_c (so Z_4 < 0 above T_c and Z_4 = 0 at
    it).  Every factor but the one of g_0 is strictly positive (c >= 2), so each product is
    kept as a log-magnitude plus its log-derivatives, and the g_0 factor of Z_4 is carried
    separately: that keeps dZ_4/dK right at T_c, where Z_4 vanishes but its derivative does not.
    The derivatives of g follow from cosh g = c(K): g' = c' / sinh g, g'' = (c'' - cosh g g'^2)
    / sinh g.
    """

    def __init__(self, K: float, m: int, n: int):
        self.K, self.m, self.n = float(K), int(m), int(n)
        s = math.sinh(2.0 * K)
        ch = math.cosh(2.0 * K)
        l_odd = np.arange(1, 2 * n, 2, dtype=float)
        l_even = np.arange(2, 2 * n, 2, dtype=float)  # l = 0 is handled on its own
        c = s + 1.0 / s
        dc = 2.0 * ch * (1.0 - 1.0 / (s * s))
        ddc = 4.0 * s - 4.0 / s + 8.0 * ch * ch / s ** 3
        half = 0.5 * self.m
        self.x_odd = self._angles(l_odd, c, dc, ddc, half)
        self.x_even = self._angles(l_even, c, dc, ddc, half)
        g0 = 2.0 * K + math.log(math.tanh(K))
        self.x0 = (half * g0, half * (2.0 + 2.0 / s), half * (-4.0 * ch / (s * s)))
        self.lnpre = (0.5 * m * n) * math.log(2.0 * s)
        self.dlnpre = m * n * ch / s
        self.ddlnpre = -2.0 * m * n / (s * s)

    def _angles(self, l, c, dc, ddc, half):
        cg = c - np.cos(np.pi * l / self.n)
        g = np.arccosh(cg)
        sg = np.sqrt((cg - 1.0) * (cg + 1.0))
        dg = dc / sg
        ddg = (ddc - cg * dg * dg) / sg
        return half * g, half * dg, half * ddg

    @staticmethod
    def _cosh_product(x, dx, ddx):
        """(ln prod 2cosh x, its K-derivative, its second K-derivative)."""
        t = np.tanh(x)
        return (float(np.sum(_lncosh2(x))), float(np.sum(t * dx)),
                float(np.sum((1.0 - t * t) * dx * dx + t * ddx)))

    @staticmethod
    def _sinh_product(x, dx, ddx):
        """(ln prod 2sinh x, its K-derivative, its second K-derivative), every x > 0."""
        ct = 1.0 / np.tanh(x)
        return (float(np.sum(_lnsinh2(x))), float(np.sum(ct * dx)),
                float(np.sum((1.0 - ct * ct) * dx * dx + ct * ddx)))

    def derivatives(self) -> tuple[float, float, float]:
        """(ln Z, d ln Z / dK, d^2 ln Z / dK^2)."""
        x0, dx0, ddx0 = self.x0
        # each term: (log-magnitude, value, first, second derivative) / exp(log-magnitude)
        terms = []
        for lnz, d1, d2 in (self._cosh_product(*self.x_odd), self._sinh_product(*self.x_odd)):
            terms.append((lnz, 1.0, d1, d2 + d1 * d1))
        # Z_3: the g_0 factor 2 cosh x0 is regular, fold it in
        lnz, d1, d2 = self._cosh_product(*self.x_even)
        t0 = math.tanh(x0)
        d1 += t0 * dx0
        d2 += (1.0 - t0 * t0) * dx0 * dx0 + t0 * ddx0
        terms.append((lnz + float(_lncosh2(x0)), 1.0, d1, d2 + d1 * d1))
        # Z_4 = f0 * R, f0 = 2 sinh x0 (may vanish), R = the remaining product
        lnr, r1, r2 = self._sinh_product(*self.x_even)
        f0 = 2.0 * math.sinh(x0)
        f1 = 2.0 * math.cosh(x0) * dx0
        f2 = f0 * dx0 * dx0 + 2.0 * math.cosh(x0) * ddx0
        terms.append((lnr, f0, f1 + f0 * r1, f2 + 2.0 * f1 * r1 + f0 * (r2 + r1 * r1)))
        top = max(t[0] for t in terms)
        w = [math.exp(t[0] - top) for t in terms]
        s0 = sum(wi * t[1] for wi, t in zip(w, terms))
        s1 = sum(wi * t[2] for wi, t in zip(w, terms))
        s2 = sum(wi * t[3] for wi, t in zip(w, terms))
        lnz = -math.log(2.0) + self.lnpre + top + math.log(s0)
        d1 = self.dlnpre + s1 / s0
        d2 = self.ddlnpre + s2 / s0 - (s1 / s0) ** 2
        return lnz, d1, d2


def log_partition_torus(K: float, m: int, n: int) -> float:
    """ln Z of the m x n periodic square lattice at coupling K (J = 1, h = 0)."""
    return _KaufmanTorus(K, m, n).derivatives()[0]


def energy_torus(T: float, L: int) -> float:
    """Exact energy per spin of the L x L torus, u = -(1/L^2) d ln Z / dK."""
    return -_KaufmanTorus(1.0 / T, L, L).derivatives()[1] / (L * L)


def specific_heat_torus(T: float, L: int) -> float:
    """Exact specific heat per spin of the L x L torus, c = (K^2 / L^2) d^2 ln Z / dK^2."""
    K = 1.0 / T
    return K * K * _KaufmanTorus(K, L, L).derivatives()[2] / (L * L)


# ------------------------------------------------------------------ estimators -----------
def _blocks(x, n_bins: int) -> np.ndarray | None:
    """The series cut into ``min(n_bins, len)`` equal consecutive blocks (the tail that does not
    fill a block is dropped), one row per block; None when fewer than two blocks exist."""
    x = np.asarray(x, dtype=float)
    nb = min(int(n_bins), x.size)
    if nb < 2:
        return None
    size = x.size // nb
    return x[: nb * size].reshape(nb, size)


def binning_error(x, n_bins: int = 32) -> float:
    """Standard error of the mean of a correlated series, from the scatter of block means
    (Flyvbjerg & Petersen 1989): blocks longer than the autocorrelation time are independent."""
    b = _blocks(x, n_bins)
    if b is None:
        return float("nan")
    means = b.mean(axis=1)
    nb = means.size
    var = float(np.sum((means - means.mean()) ** 2)) / (nb - 1)
    return math.sqrt(var / nb)


def _binder_from_moments(m2: float, m4: float) -> float:
    return 1.0 - m4 / (3.0 * m2 * m2)


def binder(m) -> float:
    """Binder's fourth-order cumulant U_4 = 1 - <m^4> / (3 <m^2>^2) (Binder 1981): 2/3 in the
    ordered phase, 0 for a Gaussian order parameter."""
    m2 = np.asarray(m, dtype=float) ** 2
    return _binder_from_moments(float(m2.mean()), float((m2 * m2).mean()))


def jackknife_binder_error(m, n_bins: int = 32) -> float:
    """Jackknife error of :func:`binder` over blocks: U_4 is recomputed with each block left
    out, and sigma^2 = (n - 1)/n sum_j (U_j - mean U)^2 (Efron 1982)."""
    b = _blocks(m, n_bins)
    if b is None:
        return float("nan")
    sq = b * b
    block_m2, block_m4 = sq.mean(axis=1), (sq * sq).mean(axis=1)
    nb = block_m2.size
    tot2, tot4 = float(block_m2.sum()), float(block_m4.sum())
    u = np.array([_binder_from_moments((tot2 - a) / (nb - 1), (tot4 - c) / (nb - 1))
                  for a, c in zip(block_m2, block_m4)])
    return math.sqrt((nb - 1) / nb * float(np.sum((u - u.mean()) ** 2)))


def crossing(Ts, u_a, u_b) -> float:
    """First temperature at which two Binder curves meet: the first grid point where their
    difference is zero, or the zero of the straight line through the first pair of neighbours
    with opposite signs; NaN when they do not cross on the grid."""
    T = np.asarray(Ts, dtype=float)
    d = np.asarray(u_a, dtype=float) - np.asarray(u_b, dtype=float)
    sign = np.sign(d)
    hits = np.flatnonzero((sign[:-1] == 0) | (sign[:-1] * sign[1:] < 0))
    if hits.size == 0:
        return float("nan")
    i = int(hits[0])
    if d[i] == 0:
        return float(T[i])
    frac = d[i] / (d[i] - d[i + 1])
    return float(T[i] + frac * (T[i + 1] - T[i]))


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
