"""Broadband impedance (runBBIFlag 1) on the GPU through the C ABI: one kick
and whole turns (the turn graph) against the reference's own runs
(tests/golden/ref_bbi.npz),
the profile and potentials against the oracle restatement, run-to-run and
checkpoint determinism, and the out-of-range error.

The frequency-domain kick is the reference's FFT product applied as the
equivalent circular convolution, so it agrees with the reference to
rounding: 1e-11 of the largest kick per coordinate for one kick, 1e-10 of the
coordinates' rms after the turns.  The time-domain kick follows the
reference's loops; its profile sums are in fixed point (order-independent),
so it too agrees to rounding."""
import tempfile

import numpy as np
import pytest

import bbicases
import oracle
from cetasim_b200 import _abi
from cetasim_b200.beam import MPBeam
from refcases import parts_digest

pytestmark = pytest.mark.gpu

KICK_TOL = 1e-11
TURN_TOL = 1e-10


def _kick_err(got, want, start):
    e = np.zeros(6)
    for q in range(6):
        k = np.max(np.abs(want[q] - start[q]))
        d = np.max(np.abs(got[q] - want[q]))
        e[q] = d / k if k > 0 else d
    return e


@pytest.mark.parametrize("case", list(bbicases.CASES))
def test_kick_matches_the_reference(case):
    g = bbicases.golden()
    td = bbicases.CASES[case][3]
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = bbicases.build(case, d)
    assert parts_digest(parts) == bytes(g[f"{case}/digest"]).decode()
    b = MPBeam(wl)
    bbicases.start(b, parts)
    b.BBImpBeamInteraction()
    for j in bbicases.KEEP[case]:
        c, _ = b.download(j)
        err = _kick_err(c, g[f"{case}/kick{j}"], parts[j])
        assert err.max() <= KICK_TOL, (j, err)
    if not td:
        # the five potentials at the bins that hold particles (the GPU
        # evaluates them there only) against the reference's arrays
        lo = int(g[f"{case}/pot_lo"][0])
        want = g[f"{case}/pot"]
        a, got = b.bbi_profile(0)
        for q in range(5):
            if not wl.cfg.bbi.sim[q]:
                continue
            mask = got[1 + q] != 0
            idx = np.nonzero(mask)[0] + a
            assert idx.size and np.all((idx >= lo) & (idx < lo + want.shape[1]))
            sc = np.max(np.abs(want[q]))
            assert np.max(np.abs(got[1 + q][mask] - want[q][idx - lo])) <= KICK_TOL * sc, q


@pytest.mark.parametrize("case", list(bbicases.CASES))
def test_profile_matches_the_oracle(case):
    """The smoothed charge profile (the reference's profileForBunchBBImp of
    the charge, or densityProfile in the time domain) of every kept bunch."""
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = bbicases.build(case, d)
    b = MPBeam(wl)
    o = oracle.OracleBeam(wl)
    bbicases.start(b, parts)
    bbicases.start(o, parts)
    b.BBImpBeamInteraction()
    o.BBImpBeamInteraction()
    for j in bbicases.KEEP[case]:
        a, got = b.bbi_profile(j)
        want = o.bbi_profile(j)[0]
        assert got.shape[1] > 0
        sc = np.max(np.abs(want))
        assert np.max(np.abs(got[0] - want[a:a + got.shape[1]])) <= 1e-12 * sc
        # nothing of the profile outside the bins the GPU keeps
        outside = np.concatenate([want[:a], want[a + got.shape[1]:]])
        assert np.all(outside == 0)


@pytest.mark.parametrize("case", list(bbicases.CASES))
def test_turns_match_the_reference(case):
    g = bbicases.golden()
    turns = bbicases.CASES[case][2]
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = bbicases.build(case, d)
    b = MPBeam(wl)
    bbicases.start(b, parts)
    b.Run(0, turns)  # the turn graph: the kick between the damping and the LR wake
    for j in bbicases.KEEP[case]:
        c, s = b.download(j)
        assert np.array_equal(s, g[f"{case}/surv{j}"])
        err = bbicases.coord_rel_err(c, g[f"{case}/coords{j}"])
        assert err.max() <= TURN_TOL, (j, err)


def test_runs_repeat_bit_for_bit_and_resume():
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = bbicases.build("fd_train_lr", d)
    runs = []
    for _ in range(2):
        b = MPBeam(wl)
        bbicases.start(b, parts)
        b.Run(0, 2)
        runs.append([b.download(j)[0] for j in range(wl.n_bunches)])
    for x, y in zip(*runs):
        assert np.array_equal(x, y)
    b = MPBeam(wl)
    bbicases.start(b, parts)
    b.Run(0, 1)
    blob = b.checkpoint()
    b2 = MPBeam(wl)
    b2.restore(blob)
    b2.Run(1, 1)
    for j in range(wl.n_bunches):
        assert np.array_equal(b2.download(j)[0], runs[0][j])


def test_particle_outside_the_profile_is_an_error():
    """A particle beyond zMax: the reference indexes outside its profile; the
    library skips it and reports CG_ERR_INVALID."""
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = bbicases.build("fd_single", d)
    p = parts[0].copy()
    p[4, 3] = 5.0  # zMax = dz (n - 1) = 0.32 m
    b = MPBeam(wl)
    b.upload(0, p)
    with pytest.raises(_abi.CgError) as e:
        b.BBImpBeamInteraction()
    assert e.value.code == 1  # CG_ERR_INVALID
