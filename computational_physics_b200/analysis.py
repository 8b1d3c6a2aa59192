"""Error analysis of Monte Carlo time series and the exact finite-lattice reference values.

* :func:`binning_error` -- blocking analysis (Flyvbjerg & Petersen, J. Chem. Phys. 91, 461
  (1989)): the series is pair-averaged repeatedly; the standard error of the mean at each
  level rises while samples are correlated and plateaus once blocks are independent.  The
  estimate is the largest error among levels that still hold at least ``min_blocks``
  blocks, which is conservative under autocorrelation.  The reference prints plain means
  without errors (ising/src/ising_2d.cpp:127-162).
* :func:`exact_energy_heat` -- E/N and C/N of the periodic M x N Ising model (J = 1) from
  the Kaufman / Ferdinand-Fisher partition function
      Z = 1/2 (2 sinh 2K)^(MN/2) (Z1 + Z2 + Z3 + Z4)
  (the quantities of ising/verification/FF_internalEnergy_specificHeat*.c), here by
  differentiating ln Z numerically in 60-digit arithmetic: E/N = -(1/MN) d lnZ/dK,
  C/N = K^2/(MN) d^2 lnZ/dK^2.
"""
from __future__ import annotations

import math
from functools import lru_cache

import mpmath as mp
import numpy as np

KC = 0.5 * math.log(1.0 + math.sqrt(2.0))

__all__ = ["binning_error", "BinningResult", "exact_energy_heat", "exact_energy", "KC", "energy_series",
           "gate_energy"]


class BinningResult(tuple):
    """(mean, error, tau_int, levels): tau_int = (error / naive error)^2 / 2 in sample units."""

    __slots__ = ()

    def __new__(cls, mean, error, tau, levels):
        return super().__new__(cls, (mean, error, tau, levels))

    mean = property(lambda s: s[0])
    error = property(lambda s: s[1])
    tau_int = property(lambda s: s[2])
    levels = property(lambda s: s[3])


def binning_error(x, min_blocks: int = 32) -> BinningResult:
    x = np.asarray(x, np.float64)
    n = len(x)
    if n < 2:
        return BinningResult(float(x.mean()) if n else float("nan"), float("inf"), float("nan"), [])
    mean = float(x.mean())
    levels = []
    y = x.copy()
    while len(y) >= min_blocks:
        m = len(y)
        err = float(np.sqrt(y.var(ddof=1) / m)) if m > 1 else float("inf")
        levels.append((m, err))
        if m < 2 * min_blocks:
            break
        y = 0.5 * (y[0:m - m % 2:2] + y[1:m - m % 2:2])
    if not levels:
        levels = [(n, float(np.sqrt(x.var(ddof=1) / n)))]
    error = max(e for _, e in levels)
    naive = levels[0][1]
    tau = 0.5 * (error / naive) ** 2 if naive > 0 else float("nan")
    return BinningResult(mean, error, tau, levels)


def _ln_partition(K, M: int, N: int):
    """ln Z of the periodic M x N lattice at coupling K (mpmath number)."""
    c2 = mp.cosh(2 * K) / mp.tanh(2 * K)
    half = mp.mpf(M) / 2
    lnZ = []
    signs = []
    for odd in (True, False):
        gam = []
        for i in range(N):
            r = 2 * i + 1 if odd else 2 * i
            if r == 0:
                gam.append(2 * K + mp.log(mp.tanh(K)))
            else:
                cl = c2 - mp.cos(r * mp.pi / N)
                gam.append(mp.log(cl + mp.sqrt(cl * cl - 1)))
        for hyper in (mp.cosh, mp.sinh):
            s = mp.mpf(0)
            sign = 1
            for gm in gam:
                v = 2 * hyper(half * gm)
                if v == 0:
                    sign = 0
                    break
                if v < 0:
                    sign = -sign
                s += mp.log(abs(v))
            lnZ.append(s)
            signs.append(sign)
    top = max(lnZ)
    total = mp.fsum(sg * mp.exp(l - top) for sg, l in zip(signs, lnZ))
    return (mp.mpf(M) * N / 2) * mp.log(2 * mp.sinh(2 * K)) + top + mp.log(total) - mp.log(2)


@lru_cache(maxsize=4096)
def exact_energy_heat_precise(K: float, M: int, N: int | None = None, dps: int = 60) -> tuple[float, float]:
    """(E/N, C/N) of the M x N periodic lattice at K = J/T, by differentiating ln Z in
    `dps`-digit arithmetic (slow: about a second per call at L = 256)."""
    N = M if N is None else N
    with mp.workdps(dps):
        f = lambda k: _ln_partition(k, M, N)
        K = mp.mpf(K)
        d1 = mp.diff(f, K, 1)
        d2 = mp.diff(f, K, 2)
        return float(-d1 / (M * N)), float(K * K * d2 / (M * N))


def _log2hyper(a: np.ndarray, cosh: bool):
    """ln|2 cosh a| or ln|2 sinh a| and the sign, without overflow."""
    x = np.abs(a)
    if cosh:
        return x + np.log1p(np.exp(-2 * x)), np.ones_like(a)
    with np.errstate(divide="ignore"):
        return x + np.log(-np.expm1(-2 * x)), np.sign(a)


@lru_cache(maxsize=65536)
def exact_energy_heat(K: float, M: int, N: int | None = None) -> tuple[float, float]:
    """(E/N, C/N) of the M x N periodic lattice at K = J/T: the closed-form derivatives of
    Z1..Z4 evaluated in float64 log space (microseconds; E/N agrees with the 60-digit route
    to ~1e-13)."""
    N = M if N is None else N
    K = float(K)
    s2, c2 = math.sinh(2 * K), math.cosh(2 * K)
    r = np.arange(2 * N, dtype=np.float64)
    cl = c2 / math.tanh(2 * K) - np.cos(r * math.pi / N)
    root = np.sqrt(np.maximum(cl * cl - 1.0, 0.0))
    cp = 2 * c2 * (1 - 1 / (s2 * s2))
    cpp = 8 / s2 ** 3 * c2 * c2 + 4 * (s2 - 1 / s2)
    with np.errstate(divide="ignore", invalid="ignore"):
        g = np.log(cl + root)
        gp = cp / root
        gpp = cpp / root - cp * cp * cl / root ** 3
    g[0] = 2 * K + math.log(math.tanh(K))
    gp[0] = 2 * (1 + 1 / s2)
    gpp[0] = -4 / (s2 * math.tanh(2 * K))
    half = M / 2.0
    lnZ, sgn, D1, D2 = [], [], [], []
    for odd, cosh in ((True, True), (True, False), (False, True), (False, False)):
        idx = slice(1, None, 2) if odd else slice(0, None, 2)
        a = half * g[idx]
        lz, sg = _log2hyper(a, cosh)
        with np.errstate(divide="ignore", invalid="ignore"):
            t = np.tanh(a) if cosh else 1 / np.tanh(a)
        # Z''/Z = (sum u)^2 + sum v with u = M/2 g' t, v = M/2 g'' t + (M/2 g')^2 q, where
        # t^2 + q = 1 for both (tanh, sech^2) and (coth, -csch^2); so
        # Z''/Z = (sum u)^2 - sum u^2 + sum ((M/2 g')^2 + M/2 g'' t).  The one term that can be
        # huge (coth of gamma_0 near 0) is split off so nothing cancels catastrophically.
        u = half * gp[idx] * t
        d1 = float(np.sum(u))
        k = int(np.argmax(np.abs(u)))
        rest = d1 - u[k]
        cross = 2 * u[k] * rest + rest * rest - (float(np.sum(u * u)) - u[k] * u[k])
        d2 = cross + float(np.sum((half * gp[idx]) ** 2 + half * gpp[idx] * t))
        lnZ.append(float(np.sum(lz)))
        sgn.append(float(np.prod(sg)))
        D1.append(d1)
        D2.append(d2)
    top = max(lnZ)
    w = np.array([s * math.exp(l - top) for s, l in zip(sgn, lnZ)])
    w /= w.sum()
    # A vanishing Z_x (sinh of gamma_0 = 0 at K_c) has weight 0 and a finite product w * D.
    d1w = sum(x * y for x, y in zip(w, D1) if x != 0)
    d2w = sum(x * y for x, y in zip(w, D2) if x != 0)
    e = -(d1w / (M * N) + 1 / math.tanh(2 * K))
    c = (d2w - d1w * d1w) * K * K / (M * N) - 2 * K * K / s2 ** 2
    return float(e), float(c)


def exact_energy(T: float, L0: int, L1: int | None = None) -> float:
    """E/N of the periodic L0 x L1 lattice at temperature T."""
    L1 = L0 if L1 is None else L1
    return exact_energy_heat(1.0 / float(T), int(L0), int(L1))[0]


def energy_series(samples: np.ndarray, num_sites: int) -> np.ndarray:
    """E/N per measurement from the exact integer sums (e, m) the engine records."""
    return -np.asarray(samples, np.float64)[:, 0] / num_sites


def gate_energy(samples: np.ndarray, L0: int, L1: int, T: float, nsigma: float = 2.0) -> dict:
    """E/N of a run against the exact value: mean, binned error, z-score and pass flag."""
    E = energy_series(samples, L0 * L1)
    b = binning_error(E)
    exact = exact_energy(T, L0, L1)
    z = (b.mean - exact) / b.error if b.error > 0 else float("inf")
    return {"mean": b.mean, "error": b.error, "tau_int": b.tau_int, "exact": exact, "z": z,
            "pass": abs(z) <= nsigma, "samples": len(E)}
