"""Coupled-bunch mode history and growth rates on the GPU (cg_cbm_*) against
the oracle (oracle/cbm.py) on the same bunch moments."""
import numpy as np
import pytest

from helpers import pair, particles, small
from oracle import cbm

pytestmark = pytest.mark.gpu


def _oracle_record(wl, g):
    s0 = wl.sections[0]
    r = wl.cfg.ring
    mean = np.array([list(m.mean) for m in g.moments()])
    return cbm.cbm_record(mean, wl.harm, r.harmonics, (s0.beta_x, s0.beta_y),
                          (s0.alpha_x, s0.alpha_y), (r.work_qx, r.work_qy, r.work_qz), r.beta_z)


def _with_mode(parts, mu, amp, n_bunch):
    """Bunch centroids displaced by a travelling x and y pattern of mode mu."""
    out = []
    for j, c in enumerate(parts):
        c = c.copy()
        ph = 2 * np.pi * mu * j / n_bunch
        c[0] += amp * np.cos(ph)
        c[1] += 1e-2 * amp * np.sin(ph)
        c[2] += 0.5 * amp * np.sin(ph)
        c[4] += 1e-3 * np.cos(ph)
        out.append(c)
    return out


def test_record_matches_the_oracle():
    wl = small("fast_ion", 0.05)
    parts = _with_mode(particles(wl, seed=31), 7, 2e-5, wl.n_bunches)
    g, _ = pair(wl, parts)
    g.cbm_init(4)
    g.cbm_record()
    amp, arg, aver, iqa, iqg = g.cbm_history()
    assert amp.shape == (1, 3, wl.n_bunches)
    oa, og, ov, oqa, oqg = _oracle_record(wl, g)
    for dev_a, dev_g, ora_a, ora_g in ((amp[0], arg[0], oa, og), (iqa[0], iqg[0], oqa, oqg)):
        scale = ora_a.max(axis=1, keepdims=True)
        assert np.max(np.abs(dev_a - ora_a) / scale) < 1e-11
        big = ora_a > 1e-6 * scale  # phases of the modes that carry the signal
        dphi = np.angle(np.exp(1j * (dev_g - ora_g)))
        assert np.max(np.abs(dphi[big])) < 1e-9
    assert np.array_equal(aver[0], ov)


def test_growth_of_a_synthetic_mode():
    """Records of a mode whose amplitude grows as exp(g t): the device fit
    returns g for that mode, and the oracle's fit of the device history."""
    wl = small("fast_ion", 0.02)
    # centred bunches: the centroids are the mode pattern alone
    base = [c - c.mean(axis=1, keepdims=True) for c in particles(wl, seed=32)]
    g, _ = pair(wl, base)
    t0, interval, rate = wl.cfg.ring.t0, 50, 400.0
    n_rec = 12
    g.cbm_init(n_rec)
    for n in range(n_rec):
        a = 1e-6 * np.exp(rate * t0 * interval * n)
        g.upload_beam(_with_mode(base, 3, a, wl.n_bunches))
        g.cbm_record()
    amp, _, _, iqa, _ = g.cbm_history()
    for method, hist in ((0, amp), (1, iqa)):
        dev = g.cbm_growth(2, n_rec, interval, method)
        ora = cbm.cbm_growth(hist, 2, n_rec, interval, t0)
        assert np.allclose(dev, ora, rtol=1e-9, atol=1e-6, equal_nan=True)
        # the x mode the centroids carry grows at the set rate
        k = int(np.argmax(hist[-1, 0]))
        assert abs(dev[0, k] / rate - 1) < 1e-3


def test_hilbert_method_matches_the_oracle():
    """Records of betatron-like turn-by-turn centroids: the device's analytic
    signals, mode amplitudes and both fits against the oracle on the same
    centroid history."""
    wl = small("fast_ion", 0.02)
    base = [c - c.mean(axis=1, keepdims=True) for c in particles(wl, seed=33)]
    g, _ = pair(wl, base)
    r = wl.cfg.ring
    t0, interval, n_rec = r.t0, 1, 40
    g.cbm_init(n_rec)
    M = wl.n_bunches
    for n in range(n_rec):
        parts = []
        for j, c in enumerate(base):
            c = c.copy()
            ph = 2 * np.pi * (r.work_qx * n + 3 * j / M)
            c[0] += 1e-6 * np.exp(2e-2 * n) * np.cos(ph)
            c[2] += 5e-7 * np.sin(ph + 0.2 * j)
            c[4] += 1e-4 * np.cos(2 * np.pi * r.work_qz * n + j)
            parts.append(c)
        g.upload_beam(parts)
        g.cbm_record()
    _, _, aver, _, _ = g.cbm_history()
    mr, br, hamp, harg, ana = g.cbm_hilbert(5, n_rec - 5, interval)
    s0 = wl.sections[0]
    omr, obr, ohamp, oana = cbm.cbm_hilbert(
        aver, wl.harm, r.harmonics, (s0.beta_x, s0.beta_y), (s0.alpha_x, s0.alpha_y),
        (r.work_qx, r.work_qy, r.work_qz), r.beta_z, 5, n_rec - 5, interval, t0)
    scale = np.abs(oana).max(axis=0, keepdims=True)
    assert np.max(np.abs(ana - oana) / scale) < 1e-10
    assert np.max(np.abs(hamp - ohamp) / ohamp.max(axis=(0, 2), keepdims=True)) < 1e-10
    # rates of the modes that carry signal through the fit window (the others
    # fit the logarithm of rounding noise)
    live = ohamp[5:n_rec - 5].min(axis=0) > 1e-6 * ohamp.max(axis=(0, 2))[:, None]
    assert live.sum() > 10
    assert np.allclose(mr[live], omr[live], rtol=1e-7, atol=1e-3)
    assert np.allclose(br, obr, rtol=1e-7, atol=1e-3)
