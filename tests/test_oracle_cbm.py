"""The coupled-bunch mode oracle (oracle/cbm.py) against closed forms: a pure
mode lands in its DFT bin, and the GSL-form fit is the least-squares slope."""
import numpy as np

from oracle import cbm


def test_pure_mode_lands_in_its_bin():
    M, H, mu = 16, 16, 5
    harm = np.arange(M)
    beta, alpha, tunes = (4.0, 2.5), (0.0, 0.0), (0.0, 0.0, 0.0)
    j = np.arange(M)
    mean = np.zeros((M, 6))
    # alpha = 0, x / sqrt(b) = cos and sqrt(b) x' = sin: z_j = cos - i sin
    mean[:, 0] = np.sqrt(beta[0]) * np.cos(2 * np.pi * mu * j / M)
    mean[:, 1] = np.sin(2 * np.pi * mu * j / M) / np.sqrt(beta[0])
    amp, arg, aver, iq_amp, _ = cbm.cbm_record(mean, harm, H, beta, alpha, tunes, 1.0)
    # z_j = cos - i sin = exp(-2 pi i mu j / M): all weight in bin M - mu
    assert abs(amp[0, M - mu] - M) < 1e-12
    assert np.max(np.delete(amp[0], M - mu)) < 1e-12
    assert np.array_equal(aver[0], mean[:, 0])
    # the IQ scan at (k + 0) f0 over uniform bunches sees the cos pattern in bins mu, M - mu
    half = np.sqrt(beta[0]) / 2
    assert abs(iq_amp[0, mu] - half) < 1e-12 and abs(iq_amp[0, M - mu] - half) < 1e-12


def test_fit_is_the_least_squares_slope():
    rng = np.random.default_rng(3)
    x = np.arange(40) * 25.0
    y = 1e-4 * x + 0.3 + rng.normal(0, 1e-3, len(x))
    assert abs(cbm.wlinear_slope(x, y) - np.polyfit(x, y, 1)[0]) < 1e-15 * 1e3


def test_growth_recovers_an_exponential():
    t0, interval, g = 2.5e-6, 10, 120.0  # 1/s
    n = np.arange(30)
    amp = np.exp(g * t0 * interval * n)[:, None, None] * np.ones((1, 3, 4))
    rate = cbm.cbm_growth(amp, 5, 30, interval, t0)
    assert np.allclose(rate, g, rtol=1e-9)


def test_analytic_signal_of_a_sinusoid():
    n = np.arange(64)
    a = cbm.analytic(np.cos(2 * np.pi * 5 * n / 64 + 0.3))
    assert np.allclose(a, np.exp(1j * (2 * np.pi * 5 * n / 64 + 0.3)), atol=1e-12)


def test_analytic_signal_of_an_odd_length_record():
    n = np.arange(63)
    a = cbm.analytic(np.sin(2 * np.pi * 4 * n / 63))
    assert np.allclose(a, -1j * np.exp(1j * 2 * np.pi * 4 * n / 63), atol=1e-12)


def test_iq_scan_phase_form_equals_the_reference_form():
    """The IQ average with the phase (k + Q) h / H (f0 t0 = 1) against the
    reference's form exp(-i 2 pi f t) with f = (k + Q) f0 and t = h t0 / H
    evaluated in floating point (MPBeam.cpp:153-158, 1597-1611): amplitude
    and argument (arg of the average, MPBeam.cpp:1617-1619) in all three
    planes."""
    rng = np.random.default_rng(4)
    M, H = 80, 3840
    tunes = (18.213, 10.137, 0.0049)
    harm = np.sort(rng.choice(H, M, replace=False))
    t0 = 2.3057e-6
    f0 = 1.0 / t0
    mean = np.zeros((M, 6))
    for pl in range(3):
        mean[:, 2 * pl] = rng.normal(0, 1e-5, M) * (1 + pl)
    _, _, _, iq_amp, iq_arg = cbm.cbm_record(mean, harm, H, (10.0, 5.0), (0.0, 0.0), tunes, 1.0)
    t = harm * (t0 / H)
    for pl in range(3):
        u = mean[:, 2 * pl]
        for k in range(M):
            ref = np.mean(u * np.exp(-1j * 2.0 * np.pi * ((k + tunes[pl]) * f0) * t))
            assert abs(iq_amp[pl, k] - abs(ref)) <= 1e-11 * np.abs(u).max()
            if abs(ref) > 1e-3 * np.abs(u).max():
                d = np.angle(np.exp(1j * (iq_arg[pl, k] - np.angle(ref))))
                assert abs(d) <= 1e-8, (pl, k, d)
