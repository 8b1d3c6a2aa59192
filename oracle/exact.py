"""Test infrastructure: exact internal energy and specific heat per spin of the finite
periodic 2D Ising model (J = 1), the physics oracle for the Swendsen-Wang sweep.

Restates the Ferdinand-Fisher / Kaufman partial partition functions Z1..Z4 that the
reference evaluates in ising/verification/FF_internalEnergy_specificHeat.c:10-272
(long double) and FF_internalEnergy_specificHeat_mpfr.c:67-593 (512-bit MPFR):

  gamma_0   = 2K + ln tanh K
  gamma_r   = arccosh(cosh(2K) coth(2K) - cos(r pi / N)),  r > 0
  Z1 = prod_{i<N} 2 cosh(M/2 gamma_{2i+1}),  Z2 = prod 2 sinh(M/2 gamma_{2i+1})
  Z3 = prod_{i<N} 2 cosh(M/2 gamma_{2i}),    Z4 = prod 2 sinh(M/2 gamma_{2i})
  E/N = -( sum_x (Z_x'/Z_x) w_x / (M N) + coth 2K ),         w_x = Z_x / sum_y Z_y
  C/N = K^2/(MN) (sum_x (Z_x''/Z_x) w_x - (sum_x (Z_x'/Z_x) w_x)^2) - 2K^2 / sinh^2 2K

with the derivative sums of FF_..._specificHeat.c:95-191.  The long-double program
overflows (NaN) for L >= 256; here every quantity is an mpmath number at 60 significant
digits, so any lattice size works.  Pinned against the reference program's printed
values in tests/golden/exact_ff.json.
"""
from __future__ import annotations

import math

import mpmath as mp

KC = 0.5 * math.log(1.0 + math.sqrt(2.0))


def _gammas(K, M: int, N: int):
    c2, s2 = mp.cosh(2 * K), mp.sinh(2 * K)
    t2 = mp.tanh(2 * K)
    cp = 2 * c2 * (1 - 1 / (s2 * s2))                       # c_l'
    cpp = 8 / (s2 ** 3) * c2 * c2 + 4 * (s2 - 1 / s2)         # c_l''
    g, gp, gpp = {}, {}, {}
    for r in range(0, 2 * N):
        if r == 0:
            g[r] = 2 * K + mp.log(mp.tanh(K))
            gp[r] = 2 * (1 + 1 / s2)
            gpp[r] = -4 / (s2 * t2)
        else:
            cl = c2 / t2 - mp.cos(r * mp.pi / N)
            root = mp.sqrt(cl * cl - 1)
            g[r] = mp.log(cl + root)
            gp[r] = cp / root
            gpp[r] = cpp / root - cp * cp * cl / root ** 3
    return g, gp, gpp


def exact_energy_heat(K: float, M: int, N: int | None = None, dps: int = 60) -> tuple[float, float]:
    """(E/N, C/N) of the M x N periodic lattice at coupling K = J / T."""
    N = M if N is None else N
    with mp.workdps(dps):
        K = mp.mpf(K)
        g, gp, gpp = _gammas(K, M, N)
        half = mp.mpf(M) / 2
        Z, D1, D2 = [], [], []
        for x in (1, 2, 3, 4):
            rs = [2 * i + 1 for i in range(N)] if x in (1, 2) else [2 * i for i in range(N)]
            hyper = mp.cosh if x in (1, 3) else mp.sinh
            z = mp.mpf(1)
            for r in rs:
                z *= 2 * hyper(half * g[r])
            # Z'/Z and Z''/Z: tanh for cosh products (x = 1, 3), coth for sinh products (x = 2, 4).
            s1 = mp.mpf(0)
            s2 = mp.mpf(0)
            for r in rs:
                a = half * g[r]
                if x in (1, 3):
                    th = mp.tanh(a)
                    s1 += gp[r] * th
                    s2 += gpp[r] * th + half * gp[r] ** 2 / mp.cosh(a) ** 2
                else:
                    ct = 1 / mp.tanh(a)
                    s1 += gp[r] * ct
                    s2 += gpp[r] * ct - half * gp[r] ** 2 / mp.sinh(a) ** 2
            d1 = half * s1
            d2 = d1 * d1 + half * s2
            Z.append(z)
            D1.append(d1)
            D2.append(d2)
        total = Z[0] + Z[1] + Z[2] + Z[3]
        w = [z / total for z in Z]
        temp = sum(d * wx for d, wx in zip(D1, w))
        e = -(temp / (M * N) + 1 / mp.tanh(2 * K))
        c = sum(d * wx for d, wx in zip(D2, w))
        c = (c - temp * temp) * K * K / (M * N) - 2 * K * K / mp.sinh(2 * K) ** 2
        return float(e), float(c)


def exact_energy(T: float, L: int) -> float:
    """E/N of the periodic L x L lattice at temperature T (K = 1/T)."""
    return exact_energy_heat(1.0 / float(T), L, L)[0]
