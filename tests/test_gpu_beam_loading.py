"""Cavities with beam loading (rfMode 1) on the GPU through the C ABI: the
resonators' set-up and whole turns against the reference's own runs
(tests/golden/ref_beam_loading.npz), single RF steps against the oracle
restatement (which reproduces the reference bit for bit), and checkpoint /
resume of the cavity state.  Tolerances: 1e-10 relative (the recurrence
follows the reference's operations with CUDA's sin, cos and exp)."""
import tempfile

import numpy as np
import pytest

import blcases
import oracle
from cetasim_b200.beam import MPBeam
from refcases import parts_digest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _pairs(states):
    return np.array([[v for z in s[:3] for v in (z.real, z.imag)] for s in states])


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-300))


@pytest.mark.parametrize("case", list(blcases.CASES))
def test_turns_reproduce_the_reference_runs(case):
    g = blcases.golden()
    turns = blcases.CASES[case][2]
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = blcases.build(case, d)
    assert parts_digest(parts) == bytes(g[f"{case}/digest"]).decode()
    b = MPBeam(wl)
    blcases.start(b, parts)
    cav = blcases.loaded_cavities(wl)
    # the set-up (host restatement of InitialcavityResonator)
    assert _rel(_pairs([b.resonator(c) for c in cav]), g[f"{case}/res_init"]) <= 1e-13
    b.Run(0, turns)  # the turn graph
    for j in blcases.KEEP[case]:
        c, s = b.download(j)
        want = g[f"{case}/coords{j}"]
        assert np.array_equal(s, g[f"{case}/surv{j}"])
        alive = s == 0
        err = blcases.coord_rel_err(c, want, alive)
        assert err.max() <= TOL, (j, err)
    for i, c in enumerate(cav):
        got = _pairs([b.resonator(c)])[0]
        want = g[f"{case}/res_final"][i]
        # each complex value against its own size
        for q in range(0, 6, 2):
            assert abs(complex(*got[q:q + 2]) - complex(*want[q:q + 2])) <= TOL * (
                abs(complex(*want[q:q + 2])) + 1e-300), (c, q)
    info = np.array([[[v for z in b.rf_info(j, c) for v in (z.real, z.imag)] for c in cav]
                     for j in range(wl.n_bunches)])
    want = g[f"{case}/info"]
    for q in range(0, 8, 2):
        num = np.abs((info[..., q] - want[..., q]) + 1j * (info[..., q + 1] - want[..., q + 1]))
        den = np.abs(want[..., q] + 1j * want[..., q + 1]) + 1e-300
        assert np.max(num / den) <= TOL, q


@pytest.mark.parametrize("case", ["single_binned", "train_binned_fb", "ragged_harmonic"])
def test_staged_rf_steps_match_the_oracle(case):
    """cg_rf_kick and cg_longi_drift three times: momenta, resonator state
    and bunch averages against the oracle after each step."""
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = blcases.build(case, d)
    b = MPBeam(wl)
    o = oracle.OracleBeam(wl)
    blcases.start(b, parts)
    blcases.start(o, parts)
    cav = blcases.loaded_cavities(wl)
    for _ in range(3):
        b.BeamMomtumUpdateDueToRFTest()
        o.BeamMomtumUpdateDueToRFTest()
        b.BeamLongiPosTransferOneTurn()
        o.BeamLongiPosTransferOneTurn()
        for j in range(wl.n_bunches):
            got, s = b.download(j)
            want, _ = o.download(j)
            alive = s == 0
            assert blcases.coord_rel_err(got, want, alive).max() <= 1e-12
        for c in cav:
            for x, y in zip(b.resonator(c), o.resonator(c)):
                assert abs(x - y) <= 1e-12 * (abs(y) + 1e-300)


def test_checkpoint_resumes_the_cavity_state():
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = blcases.build("train_binned_fb", d)
    b = MPBeam(wl)
    blcases.start(b, parts)
    b.Run(0, 1)
    blob = b.checkpoint()
    b.Run(1, 2)
    end = [b.download(j) for j in range(wl.n_bunches)], b.resonator(0)
    b.restore(blob)
    b.Run(1, 2)
    again = [b.download(j) for j in range(wl.n_bunches)], b.resonator(0)
    for (x, s), (y, t) in zip(end[0], again[0]):
        assert np.array_equal(x, y) and np.array_equal(s, t)
    assert end[1] == again[1]
