"""The field surrogate (no reference counterpart) on the GPU through the C ABI:
the tensor-core forward pass and the training gradients against the FP64
network oracle (oracle/mlp.py), the exact-field training data against the
oracle's field, training to the hold-out target, and the surrogate ion kick
against the exact kick.  Tolerances are stated per test."""
import numpy as np
import pytest

import oracle
from cetasim_b200 import surrogate as S
from cetasim_b200.beam import MPBeam
from helpers import TRAPPED, particles, small
from oracle import mlp

pytestmark = pytest.mark.gpu


# The field error target of the learned path: the largest error of G over
# the domain, relative to the peak |G|.
TARGET = 1e-3


@pytest.fixture(scope="module")
def trained():
    # 2^20 exact-field samples, the training schedule of S.train (300 epochs,
    # on a B200 about 24 s)
    return S.train(seed=2024)


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(0, 1, n), rng.uniform(0, 1, n), rng.uniform(0.05, 1, n)],
                    1).astype(np.float32)


def test_forward_matches_fp64_oracle():
    # BF16 weights are the model; activations enter the tensor cores as two
    # BF16 terms and accumulate in FP32: <= 1e-5 of the output scale
    w = mlp.init(7)
    x = _inputs(1000, 1)
    out = S.evaluate(w, x)
    ref, _ = mlp.forward(w, x)
    assert np.abs(out - ref).max() <= 1e-5 * np.abs(ref).max()


def test_training_gradients_match_fp64_oracle():
    w = mlp.init(9)
    x, t = S.dataset(11, 512)
    loss, g = S.gradient(w, x, t)
    lref, gref = mlp.loss_and_grad(w, x, t)
    assert abs(loss - lref) <= 1e-6 * lref
    for o, n in ((mlp.W1, 192), (mlp.B1, 64), (mlp.W2, 4096), (mlp.B2, 64), (mlp.W3, 4096),
                 (mlp.B3, 64), (mlp.W4, 128), (mlp.B4, 2)):
        assert np.linalg.norm(g[o:o + n] - gref[o:o + n]) <= 1e-4 * np.linalg.norm(gref[o:o + n])


def test_training_data_is_the_exact_field():
    x, t = S.dataset(13, 4096)
    ref = mlp.field_target(x, oracle.gaussian_field)
    assert np.abs(t - ref).max() <= 1e-6 * np.abs(ref).max()   # float32 rounding


def test_trained_network_meets_holdout_rms_target(trained):
    w, stats = trained
    loss, rms, worst, seconds = stats
    # hold-out (2^16 samples of another seed): RMS error of G <= 1e-3 of the
    # peak |G|
    assert rms <= TARGET, stats
    # independent check of the hold-out claim with the oracle's field
    x, _ = S.dataset(99, 1 << 14)
    ref = mlp.field_target(x, oracle.gaussian_field)
    err = S.evaluate(w, x) - ref
    assert np.sqrt(np.mean(err ** 2)) <= TARGET * np.abs(ref).max()


def test_trained_network_meets_holdout_max_target(trained):
    _, stats = trained
    assert stats[2] <= TARGET, stats


def test_network_field_vanishes_on_the_axes(trained):
    """The outputs are a N_x and b N_y: exactly zero field across x = 0
    (G_x) and y = 0 (G_y), as the Gaussian's field is odd in x and in y."""
    w, _ = trained
    rng = np.random.default_rng(5)
    x = np.stack([np.zeros(256), rng.uniform(0, 1, 256), rng.uniform(0.05, 1, 256)], 1)
    assert np.all(S.evaluate(w, x)[:, 0] == 0)
    x = np.stack([rng.uniform(0, 1, 256), np.zeros(256), rng.uniform(0.05, 1, 256)], 1)
    assert np.all(S.evaluate(w, x)[:, 1] == 0)


def test_trained_network_gains_over_untrained_and_round_beam(trained):
    """What training buys: the same network at its initial weights, and the
    cheap closed-form alternative that needs no network (the round-beam field
    with sigma = sqrt(sigma_x sigma_y)), are both orders of magnitude worse."""
    w, _ = trained
    x, _ = S.dataset(101, 1 << 14)
    ref = mlp.field_target(x, oracle.gaussian_field)
    peak = np.abs(ref).max()
    rms = lambda e: np.sqrt(np.mean(e ** 2)) / peak
    trained_err = rms(S.evaluate(w, x) - ref)
    untrained_err = rms(S.evaluate(mlp.init(2024), x) - ref)
    a, b, r = x[:, 0].astype(float), x[:, 1].astype(float), x[:, 2].astype(float)
    px, py, s = 8 * a, 8 * b * r, np.sqrt(r)
    r2 = px * px + py * py
    g = (1 - np.exp(-r2 / (2 * s * s))) / r2
    round_err = rms(np.stack([px * g, py * g], 1) - ref)
    assert trained_err * 100 < untrained_err
    assert trained_err * 100 < round_err


def _kick_pair(weights, parts):
    wl = small("fast_ion", 0.02, bunch_current=TRAPPED)
    out = []
    for w in (None, weights):
        g = MPBeam(wl)
        for j, c in enumerate(parts):
            g.upload(j, c)
        if w is not None:
            g.set_surrogate(w)
        g.MPBeamRMSCal(0)
        g.SSBeamIonEffectOneInteractionPoint(0, 0)
        out.append((g, [g.download(j)[0] for j in range(wl.n_bunches)]))
    return wl, out


def test_surrogate_kick_against_exact_kick(trained):
    w, _ = trained
    wl = small("fast_ion", 0.02, bunch_current=TRAPPED)
    parts = particles(wl, seed=4, spread=3.0)
    wl, ((ge, ce), (gs, cs)) = _kick_pair(w, parts)
    dex = np.concatenate([c[1] - p[1] for c, p in zip(ce, parts)])
    dsx = np.concatenate([c[1] - p[1] for c, p in zip(cs, parts)])
    dey = np.concatenate([c[3] - p[3] for c, p in zip(ce, parts)])
    dsy = np.concatenate([c[3] - p[3] for c, p in zip(cs, parts)])
    scale = max(np.abs(dex).max(), np.abs(dey).max())
    err = np.concatenate([dsx - dex, dsy - dey])
    # kick error relative to the largest kick: RMS within the target
    assert np.sqrt(np.mean(err ** 2)) <= TARGET * scale
    # positions are untouched by the kick
    for a, b in zip(ce, cs):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])
    # the exact path's audit of the surrogate at the same IP reports the
    # largest field error it sees (a positive, finite ratio)
    d, f = gs.surrogate_audit(0)
    assert 0 < f and 0 < d < f


def test_surrogate_kick_max_error_meets_target(trained):
    w, _ = trained
    wl = small("fast_ion", 0.02, bunch_current=TRAPPED)
    parts = particles(wl, seed=4, spread=3.0)
    wl, ((ge, ce), (gs, cs)) = _kick_pair(w, parts)
    err = np.concatenate([np.concatenate([c[q] - e[q] for c, e in zip(cs, ce)]) for q in (1, 3)])
    dex = np.concatenate([np.concatenate([e[q] - p[q] for e, p in zip(ce, parts)]) for q in (1, 3)])
    assert np.abs(err).max() <= TARGET * np.abs(dex).max()
    d, f = gs.surrogate_audit(0)
    assert d <= TARGET * f


def test_points_outside_the_domain_take_the_exact_path(trained):
    w, _ = trained
    wl = small("fast_ion", 0.02, bunch_current=TRAPPED)
    parts = particles(wl, seed=4, spread=3.0)
    # the first particle of every bunch 40 sigma away horizontally: outside
    # |x| <= 8 sigma of the cloud even with the bunch size it inflates
    far = [c.copy() for c in parts]
    for c in far:
        c[0, 0] += 40 * np.sqrt(wl.gen[0] * 10.0)
    wl, ((ge, ce), (gs, cs)) = _kick_pair(w, far)
    for a, b in zip(ce, cs):
        assert a[1][0] == b[1][0] and a[3][0] == b[3][0]
        assert not np.array_equal(a[1][1:], b[1][1:])   # the others took the network


def test_turns_with_surrogate_and_periodic_audit(trained):
    w, _ = trained
    wl = small("fast_ion", 0.01, bunch_current=TRAPPED)
    g = MPBeam(wl)
    for j, c in enumerate(particles(wl, seed=5)):
        g.upload(j, c)
    g.set_surrogate(w, audit_interval=4)
    g.Run(0, 8)
    n, last, worst = g.surrogate_audit_stats()
    # two audits made, each a positive error ratio, the worst one kept
    assert n == 2 and 0 < last <= worst < 1


def test_coupled_bunch_growth_rate_with_the_surrogate(trained):
    """The fast-ion instability of the 80-bunch train at 1e-8 Pa (ten times
    the benchmark pressure, so that the vertical coupled-bunch mode grows by
    about e^2 within 400 turns; radiation damping off): the growth rate of
    the dominant vertical mode from the GetCBMGR-form estimator
    (cg_cbm_growth, the DFT modes) with the surrogate in the electron-ion
    kicks is within 5 % of the exact path's."""
    from cetasim_b200 import configs
    w, _ = trained
    turns, rates = 400, {}
    for arm in ("exact", "surrogate"):
        wl = configs.make("fast_ion", n_scale=0.05)
        for k in range(wl.cfg.n_sections):
            wl.sections[k].pressure = 1e-8
        wl.cfg.flag_synrad = 0
        g = MPBeam(wl)
        for j, c in enumerate(particles(wl, seed=5, spread=0.2)):
            g.upload(j, c)
        if arm == "surrogate":
            g.set_surrogate(w)
        g.cbm_init(turns + 1)
        for n in range(turns):
            g.Run(n, 1)
            g.MPBeamRMSCal(0)
            g.cbm_record()
        amp = g.cbm_history()[0]
        mode = int(np.argmax(amp[-1, 1, :]))
        rates[arm] = (mode, g.cbm_growth(100, turns, 1.0, 0)[1, mode])
        g.close()
    (me, re), (ms, rs) = rates["exact"], rates["surrogate"]
    assert me == ms and re > 100.0            # the same mode, growing (1/s)
    assert abs(rs - re) <= 0.05 * re, rates
