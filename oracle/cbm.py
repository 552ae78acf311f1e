"""Coupled-bunch mode analysis: CPU restatement for the parity tests.

Test infrastructure only (the library never imports it).  It restates the
"ideal" method of MPBeam::GetCBMGR (MPBeam.cpp:1496-1575: per plane the
normalised complex amplitude of each bunch, turned by its betatron phase
-2 pi Q h_j / H, then GSL's forward complex FFT over the bunches, whose
convention is X_k = sum_j z_j exp(-2 pi i j k / M)) and the growth-rate fit of
MPBeam.cpp:1781-1830 (FittingGSL::FitALinear, FittingGSL.cpp:231-243, which
calls gsl_fit_wlinear of GSL >= 2.7: weighted means accumulated as running
means, then the running weighted second moments; slope = cov / var).
"""
from __future__ import annotations

import numpy as np


def cbm_record(mean, harm, H, beta, alpha, tunes, beta_z):
    """mean: (M, 6) bunch centroids (x, x', y, y', z, dp); harm: (M,) bunch
    harmonic numbers; beta, alpha: Twiss (x, y) at section 0; tunes (Qx, Qy,
    Qz).  Returns amp, arg, aver, iq_amp, iq_arg, each (3, M): |X_k|,
    atan2(Re X_k, Im X_k) (the reference's argument order, MPBeam.cpp:1567-1569),
    the centroids, and the IQ average at the scan frequency (k + Q) f0
    (MPBeam.cpp:1586-1625 with the frequencies of MPBeam.cpp:153-158 and
    f0 t0 = 1): |IQ_k| and arg IQ_k."""
    mean = np.asarray(mean, dtype=np.float64)
    harm = np.asarray(harm, dtype=np.float64)
    M = len(harm)
    amp = np.zeros((3, M))
    arg = np.zeros((3, M))
    aver = np.zeros((3, M))
    iq_amp = np.zeros((3, M))
    iq_arg = np.zeros((3, M))
    for pl in range(3):
        u, up = mean[:, 2 * pl], mean[:, 2 * pl + 1]
        if pl < 2:  # MPBeam.cpp:1536-1537
            sb = np.sqrt(beta[pl])
            z = u / sb - 1j * (sb * up + alpha[pl] / sb * u)
        else:       # MPBeam.cpp:1538 (alpha_z = 0)
            sb = np.sqrt(beta_z)
            z = u / sb + 1j * (sb * up)
        z = z * np.exp(1j * (-2.0 * np.pi * tunes[pl] * harm / H))
        X = np.fft.fft(z)
        amp[pl] = np.sqrt(X.real ** 2 + X.imag ** 2)
        arg[pl] = np.arctan2(X.real, X.imag)
        aver[pl] = u
        f = np.arange(M)[:, None] + tunes[pl]
        iq = (u[None, :] * np.exp(-2j * np.pi * f * harm[None, :] / H)).sum(axis=1) / M
        iq_amp[pl] = np.abs(iq)
        iq_arg[pl] = np.angle(iq)
    return amp, arg, aver, iq_amp, iq_arg


def wlinear_slope(x, y, w=None):
    """gsl_fit_wlinear's slope (running weighted means, GSL 2.7 fit/linear.c)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    w = np.ones_like(x) if w is None else np.asarray(w, dtype=np.float64)
    W = wm_x = wm_y = 0.0
    for xi, yi, wi in zip(x, y, w):
        if wi > 0:
            W += wi
            wm_x += (xi - wm_x) * (wi / W)
            wm_y += (yi - wm_y) * (wi / W)
    W = wm_dx2 = wm_dxdy = 0.0
    for xi, yi, wi in zip(x, y, w):
        if wi > 0:
            dx, dy = xi - wm_x, yi - wm_y
            W += wi
            wm_dx2 += (dx * dx - wm_dx2) * (wi / W)
            wm_dxdy += (dx * dy - wm_dxdy) * (wi / W)
    return wm_dxdy / wm_dx2


def cbm_growth(amp_hist, first, last, interval, t0):
    """Growth rates (3, M) in 1/s: the fit of log |X_k| over records
    [first, last) against n x interval turns, slope / t0 (MPBeam.cpp:1781-1830)."""
    amp_hist = np.asarray(amp_hist, dtype=np.float64)
    x = np.arange(last - first) * float(interval)
    _, P, M = amp_hist.shape
    rate = np.zeros((P, M))
    for pl in range(P):
        for k in range(M):
            rate[pl, k] = wlinear_slope(x, np.log(amp_hist[first:last, pl, k])) / t0
    return rate


def analytic(u):
    """GetHilbertAnalytical (MPBeam.cpp:1937-1989) without the Gaussian filter,
    which the reference builds but does not apply: forward FFT, terms
    1 .. N/2 doubled (the N/2 term of an even N kept single), terms above N/2
    zeroed, inverse FFT with 1/N."""
    u = np.asarray(u, dtype=np.float64)
    N = len(u)
    w = np.zeros(N)
    w[0] = 1.0
    w[1:N // 2 + 1] = 2.0
    if N % 2 == 0:
        w[N // 2] = 1.0
    return np.fft.ifft(np.fft.fft(u) * w)


def cbm_hilbert(aver_hist, harm, H, beta, alpha, tunes, beta_z, first, last, interval, t0):
    """The Hilbert method of GetCBMGR (MPBeam.cpp:1680-1725, 1781-1830):
    aver_hist (N, 3, M) centroid records.  Returns mode rates (3, M), bunch
    rates (3, M), mode amplitudes (N, 3, M), analytic signals (N, 3, M)."""
    aver_hist = np.asarray(aver_hist, dtype=np.float64)
    N, _, M = aver_hist.shape
    ana = np.zeros((N, 3, M), dtype=np.complex128)
    for pl in range(3):
        for j in range(M):
            ana[:, pl, j] = analytic(aver_hist[:, pl, j])
    hamp = np.zeros((N, 3, M))
    for n in range(N):
        mean = np.zeros((M, 6))
        for pl in range(3):
            mean[:, 2 * pl] = ana[n, pl].real
            mean[:, 2 * pl + 1] = -ana[n, pl].imag
        hamp[n] = cbm_record(mean, harm, H, beta, alpha, tunes, beta_z)[0]
    return (cbm_growth(hamp, first, last, interval, t0),
            cbm_growth(np.abs(ana), first, last, interval, t0), hamp, ana)
