"""Broadband impedance (runBBIFlag 1) in the oracle restatement against the
reference's own build: the committed fixtures of its runs
(tests/golden/ref_bbi.npz, made by tests/golden/make_bbi_golden.py) and the
input parser's reading of the BBI keys and tables.

The frequency-domain path of the reference uses FFTW (here its r2c / c2r as
direct sums in oracle/ref_shim) and the oracle its own direct sums, so those
results agree to rounding (1e-12 of the kick); the time-domain path is
plain loops in both and agrees bit for bit."""
import tempfile

import numpy as np
import pytest

import bbicases
import oracle
from refcases import parts_digest

FD_TOL = 1e-12


def _kick_err(got, want, start):
    """Largest difference per coordinate over the largest kick."""
    e = np.zeros(6)
    for q in range(6):
        k = np.max(np.abs(want[q] - start[q]))
        d = np.max(np.abs(got[q] - want[q]))
        e[q] = d / k if k > 0 else d
    return e


@pytest.mark.parametrize("case", list(bbicases.CASES))
def test_oracle_kick_matches_the_reference(case):
    g = bbicases.golden()
    td = bbicases.CASES[case][3]
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = bbicases.build(case, d)
    assert parts_digest(parts) == bytes(g[f"{case}/digest"]).decode()
    o = oracle.OracleBeam(wl)
    bbicases.start(o, parts)
    o.BBImpBeamInteraction()
    for j in bbicases.KEEP[case]:
        c, _ = o.download(j)
        want = g[f"{case}/kick{j}"]
        if td:
            assert np.array_equal(c, want), (j, np.max(np.abs(c - want)))
        else:
            assert np.all(_kick_err(c, want, parts[j]) <= FD_TOL), _kick_err(c, want, parts[j])
    if not td:
        lo = int(g[f"{case}/pot_lo"][0])
        want = g[f"{case}/pot"]
        got = o.bbi_profile(0)[1:, lo:lo + want.shape[1]]
        for q in range(5):
            sc = np.max(np.abs(want[q]))
            assert np.max(np.abs(got[q] - want[q])) <= FD_TOL * max(sc, 1e-300), q


@pytest.mark.parametrize("case", list(bbicases.CASES))
def test_oracle_turns_match_the_reference(case):
    g = bbicases.golden()
    turns, td = bbicases.CASES[case][2], bbicases.CASES[case][3]
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = bbicases.build(case, d)
    o = oracle.OracleBeam(wl)
    bbicases.start(o, parts)
    o.Run(0, turns)
    for j in bbicases.KEEP[case]:
        c, s = o.download(j)
        assert np.array_equal(s, g[f"{case}/surv{j}"])
        want = g[f"{case}/coords{j}"]
        if td:
            assert np.array_equal(c, want), (j, np.max(np.abs(c - want)))
        else:
            assert np.all(bbicases.coord_rel_err(c, want) <= 1e-11), bbicases.coord_rel_err(c, want)


def test_input_parser_reads_the_bbi_settings():
    with tempfile.TemporaryDirectory() as d:
        wl, _, _ = bbicases.build("fd_single_zq", d)
        b = wl.cfg.bbi
        assert b.flag == 1 and b.time_domain == 0
        assert [b.sim[i] for i in range(5)] == [1, 0, 0, 1, 0]
        want = bbicases.resonator_table(640, 300e9)
        assert b.n_rows == 640
        assert np.array_equal(wl.bbi_table, want)
        wl, _, _ = bbicases.build("td_train", d + "/td")
        b = wl.cfg.bbi
        assert b.flag == 1 and b.time_domain == 1 and b.n_rows == 300
        assert np.array_equal(wl.bbi_table, bbicases.wake_table(300, 0.4e-3, 60))


def test_oracle_rejects_a_table_narrower_than_the_bucket():
    """The filtered bins must lie inside the profile (MPBunch.cpp:2360-2368
    reads outside it otherwise): a 20-sample table at 300 GHz spans 9.5 mm."""
    with tempfile.TemporaryDirectory() as d:
        wl, _, _ = bbicases.build("fd_single", d)
    wl.set_bbi(bbicases.resonator_table(20, 300e9), 0)
    with pytest.raises(Exception):
        oracle.OracleBeam(wl)
