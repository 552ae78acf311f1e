"""Resistive-wall wake functions: CPU restatement for the parity tests.

Test infrastructure only (the library never imports it).  Restates
WakeFunction::GetyokoyaFactor and its L functions (WakeFunction.cpp:723-941),
the sector reader's factor bookkeeping (WakeFunction.cpp:332-361) and
GetRWLRWakeFun (WakeFunction.cpp:499-552).  The special functions the
reference takes from GSL (>= 2.7: gsl_sf_gamma, gsl_sf_fact, gsl_sf_hyperg_2F1,
gsl_sf_ellint_Kcomp) come from mpmath at 30 digits here, independently of the
library's series and AGM.
"""
from __future__ import annotations

import math

import mpmath as mp

PI = 4 * math.atan(1.0)
C_LIGHT = 299792458.0
FACTOR_GAUSS_SI = 120 * PI * C_LIGHT / (4 * PI)  # Global.h:37-39


def yokoya_factors(a, b):
    """(longitudinal, dipole x, dipole y, quadrupole x, quadrupole y) of an
    elliptical pipe with half apertures a > b."""
    with mp.workdps(30):
        a, b = mp.mpf(a), mp.mpf(b)
        f = mp.sqrt(abs(a * a - b * b))
        mu = mp.acosh(a / f)
        x = mp.exp(-4 * mu)
        cache = {}

        def term(n, s):  # sqrt2 pi e^{-(2n+1+2s) mu} G(n+1/2+s)/G(1/2)/(n+s)! 2F1(...)
            if (n, s) not in cache:
                cache[n, s] = (mp.sqrt(2) * mp.pi * mp.exp(-(2 * n + 1 + 2 * s) * mu)
                               * mp.gamma(n + s + mp.mpf(1) / 2) / mp.gamma(mp.mpf(1) / 2)
                               / mp.factorial(n + s)
                               * mp.hyp2f1(mp.mpf(1) / 2, n + s + mp.mpf(1) / 2, n + s + 1, x))
            return cache[n, s]

        kcomp = 2 * mp.sqrt(2) * mp.exp(-mu) * mp.ellipk(x)  # modulus sqrt(x): parameter x
        coef = [2 * mp.sqrt(2) / mp.pi * b / f] + [mp.sqrt(2) / mp.pi * (b / f) ** 3] * 4
        coef[3] = -coef[3]
        t = [mp.mpf(0)] * 5
        for L in range(50):
            kl = 2 if L == 0 else 1
            for P in range(50):
                kp = 2 if P == 0 else 1
                l1 = term(abs(P - L), 0) if P != L else kcomp
                l0 = l1 + term(P + L, 0)
                ld1, ld2 = term(abs(P - L), 0), term(P + L, 1)
                sg = -1 if (P + L) % 2 else 1
                c2 = mp.cosh(2 * P * mu) * mp.cosh(2 * L * mu)
                t[0] += l0 * sg / c2 / kp / kl
                t[1] += ((ld1 + ld2) * sg / mp.cosh((2 * P + 1) * mu) / mp.cosh((2 * L + 1) * mu)
                         * (2 * P + 1) * (2 * L + 1))
                t[2] += ((ld1 - ld2) * sg / mp.sinh((2 * P + 1) * mu) / mp.sinh((2 * L + 1) * mu)
                         * (2 * P + 1) * (2 * L + 1))
                t[3] += l0 * sg / c2 * (2 * P) ** 2 / kl
                t[4] += l0 * sg / c2 * (2 * P) ** 2 / kl
        return [float(coef[i] * t[i]) for i in range(5)]


def sector_factors(rx, ry):
    """Per sector, the factors RWWakeParaReadIn leaves: computed for x > y,
    swapped (x <-> y) for x < y, and those of the previous sector (1 for the
    first) for a round one."""
    out, cur = [], [1.0] * 5
    for a, b in zip(rx, ry):
        if a > b:
            cur = yokoya_factors(a, b)
        elif a < b:
            y = yokoya_factors(b, a)
            cur = [y[0], y[2], y[1], y[4], y[3]]
        out.append(list(cur))
    return out


def rw_lr_wake(sec, yok, beta_ip_x, beta_ip_y, tau):
    """GetRWLRWakeFun at tau <= 0: sec = dict of per-sector lists radius_x,
    radius_y, length, beta_x, beta_y, num, sigma."""
    if tau == 0:
        return [0.0, 0.0, 0.0]
    w = [0.0, 0.0, 0.0]
    for i in range(len(sec["radius_x"])):
        r = min(sec["radius_x"][i], sec["radius_y"][i])
        sig = sec["sigma"][i] * FACTOR_GAUSS_SI
        g = math.sqrt(1.0 / sig) * sec["length"][i] * sec["num"][i]
        w[0] += g / r ** 3 * yok[i][1] * sec["beta_x"][i]
        w[1] += g / r ** 3 * yok[i][2] * sec["beta_y"][i]
        w[2] += g / r * yok[i][0]
    w[0] *= -2.0 / PI / abs(tau) ** 0.5 * FACTOR_GAUSS_SI / beta_ip_x
    w[1] *= -2.0 / PI / abs(tau) ** 0.5 * FACTOR_GAUSS_SI / beta_ip_y
    w[2] *= 1.0 / 2.0 / PI / C_LIGHT / abs(tau) ** 1.5 * FACTOR_GAUSS_SI
    return w
