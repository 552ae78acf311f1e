"""The library's resistive-wall wake functions (cg_yokoya_factors, series 2F1
and AGM K) against the mpmath restatement (oracle/rw.py), the flat-pipe limit
of the Yokoya factors, and the sector bookkeeping of the reference's reader."""
import ctypes as C
import math

import numpy as np
import pytest

from cetasim_b200 import _abi
from oracle import rw


@pytest.mark.parametrize("a,b", [(2.0, 1.0), (1.5, 1.0), (1.05, 1.0), (10.0, 1.0)])
def test_yokoya_factors_match_mpmath(lib, a, b):
    out = np.zeros(5)
    assert lib.cg_yokoya_factors(a, b, _abi.ptr(out)) == 0
    ref = rw.yokoya_factors(a, b)
    assert np.allclose(out, ref, rtol=1e-11, atol=1e-13)


def test_flat_pipe_limit():
    """b/a -> 0: 1, pi^2/24, pi^2/12, -pi^2/24, pi^2/24 (Yokoya 1993).  The
    reference truncates the double series at 50 x 50 terms, which holds to
    a/b ~ 20 (flatter pipes are beyond its truncation)."""
    y = rw.yokoya_factors(20.0, 1.0)
    p = math.pi ** 2
    assert np.allclose(y, [1.0, p / 24, p / 12, -p / 24, p / 24], rtol=1e-2)


def test_rw_lr_wake_matches_the_oracle(lib):
    sec = {"radius_x": [0.02, 0.03, 0.01, 0.015], "radius_y": [0.02, 0.01, 0.02, 0.015],
           "length": [10.0, 5.0, 2.0, 1.0], "beta_x": [8.0, 10.0, 4.0, 6.0],
           "beta_y": [9.0, 7.0, 5.0, 3.0], "num": [12, 4, 2, 1],
           "sigma": [5.8e7, 1.4e6, 3.7e7, 5.8e7]}
    s = _abi.RwSectors()
    s.n = 4
    for f, v in sec.items():
        getattr(s, f)[:4] = v
    yok = rw.sector_factors(sec["radius_x"], sec["radius_y"])
    assert yok[3] == yok[2]  # the round sector keeps the previous factors
    for tau in (0.0, -2e-9, -1e-6, -3e-4):
        out = np.zeros(3)
        assert lib.cg_rw_lr_wake(C.byref(s), 7.0, 6.0, tau, _abi.ptr(out)) == 0
        ref = rw.rw_lr_wake(sec, yok, 7.0, 6.0, tau)
        assert np.allclose(out, ref, rtol=1e-11, atol=0)


def test_rw_pseudo_wake_matches_scipy():
    """The oracle's fu_z of GetRWPusdoWakeFun (Bessel I by its series) against
    scipy's exponentially scaled Bessel I of the four orders directly."""
    from scipy.special import ive
    import oracle
    lib = oracle.load()
    for u in (0.05, -0.05, 0.5, -0.5, 3.0, -3.0, 10.0, -10.0, 30.0, -39.0):
        x = u * u / 4
        ref = abs(u) ** 1.5 * (np.sign(u) * (ive(-0.25, x) - ive(0.75, x))
                               + (-ive(0.25, x) + ive(-0.75, x)))
        scale = abs(u) ** 1.5 * (ive(-0.25, x) + ive(0.75, x) + ive(0.25, x) + ive(-0.75, x))
        assert abs(lib.or_rw_fz(u) - ref) <= 1e-12 * scale  # the terms cancel for u > 0
    assert lib.or_rw_fz(0.005) == 0.0 and lib.or_rw_fz(41.0) == 0.0
