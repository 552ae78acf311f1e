"""Cavities with beam loading (rfMode 1) in the oracle restatement against
the reference's own build: the committed fixtures of its runs
(tests/golden/ref_beam_loading.npz, made by tests/golden/make_bl_golden.py)
and, where the build is present, step-by-step live comparisons of the RF
step (MPBeam::BeamMomtumUpdateDueToRFTest, MPBeam.cpp:2621-2704)."""
import tempfile

import numpy as np
import pytest

import blcases
import oracle
from oracle import ref
from refcases import parts_digest

live = pytest.mark.skipif(not ref.available(), reason="oracle/_ref/libcetasim_ref.so not built")


def _pairs(states):
    return np.array([[v for z in s[:3] for v in (z.real, z.imag)] for s in states])


@pytest.mark.parametrize("case", list(blcases.CASES))
def test_oracle_reproduces_the_reference_runs(case):
    g = blcases.golden()
    turns = blcases.CASES[case][2]
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = blcases.build(case, d)
    assert parts_digest(parts) == bytes(g[f"{case}/digest"]).decode()
    o = oracle.OracleBeam(wl)
    blcases.start(o, parts)
    cav = blcases.loaded_cavities(wl)
    # the set-up's resonator state (steady-state induced voltage, generator
    # voltage and current): bit for bit
    assert np.array_equal(_pairs([o.resonator(c) for c in cav]), g[f"{case}/res_init"])
    o.Run(0, turns)
    # after the run: coordinates, survival, resonator state and every bunch's
    # BunchRFModeInfo bit for bit
    for j in blcases.KEEP[case]:
        c, s = o.download(j)
        assert np.array_equal(s, g[f"{case}/surv{j}"])
        assert np.array_equal(c, g[f"{case}/coords{j}"]), (j, np.max(np.abs(c - g[f"{case}/coords{j}"])))
    assert np.array_equal(_pairs([o.resonator(c) for c in cav]), g[f"{case}/res_final"])
    info = np.array([[[v for z in o.rf_info(j, c) for v in (z.real, z.imag)] for c in cav]
                     for j in range(wl.n_bunches)])
    assert np.array_equal(info, g[f"{case}/info"])


@live
@pytest.mark.parametrize("case", ["single_binned", "train_binned_fb", "ragged_harmonic"])
def test_rf_step_against_the_live_reference(case):
    """Three RF steps alone, with a drift between them so that the bins move:
    the momenta, the resonator state and the bunch averages after each."""
    with tempfile.TemporaryDirectory() as d:
        wl, path, parts = blcases.build(case, d)
        r = ref.RefBeam(path, seed=wl.cfg.seed)
        r.set_emit_nat([0.0, 0.0, 0.0])
        o = oracle.OracleBeam(wl)
        blcases.start(r, parts)
        blcases.start(o, parts)
        cav = blcases.loaded_cavities(wl)
        for _ in range(3):
            r.BeamMomtumUpdateDueToRFTest()
            o.BeamMomtumUpdateDueToRFTest()
            r.BeamLongiPosTransferOneTurn()
            o.BeamLongiPosTransferOneTurn()
            for j in range(wl.n_bunches):
                assert np.array_equal(r.download(j)[0], o.download(j)[0])
            for c in cav:
                assert r.resonator(c)[:3] == o.resonator(c)
                for j in range(wl.n_bunches):
                    assert r.rf_info(j, c) == o.rf_info(j, c)
        r.close()


def test_input_reads_the_cavity_settings():
    """The library's input reader takes every beam-loading key the reference
    reads (ReadInputSettings.cpp:192-362) and derives the resonators'
    loaded Q, frequency, detuning angle and filling time as
    CavityResonator::Initial (CavityResonator.cpp:89-104)."""
    with tempfile.TemporaryDirectory() as d:
        wl, _, _ = blcases.build("train_binned_fb", d)
    r = wl.cfg.ring
    assert r.rf_mode[0] == 1 and r.res_type[0] == 1 and r.res_excite[0] == 1
    assert r.res_dir_fb[0] == 1 and r.res_dir_fb_gain[0] == 0.3 and r.rf_bunch_bins == blcases.BINS
    assert r.res_ql[0] == r.res_q0[0] / (1 + r.res_coupling[0])
    fh = float(r.cav_harm[0] * r.harmonics) * r.f0
    assert r.res_fre[0] == fh + r.res_detune[0]
    assert r.res_tf[0] == 2 * r.res_ql[0] / (2 * (4 * np.arctan(1.0)) * r.res_fre[0])


@live
def test_ideal_cavity_bunch_info_against_the_live_reference():
    """BunchRFModeInfo of the ideal main cavity beside the loaded harmonic
    one: the voltage at each bunch's last particle (Bunch.cpp:466-478)."""
    with tempfile.TemporaryDirectory() as d:
        wl, path, parts = blcases.build("ragged_harmonic", d)
        r = ref.RefBeam(path, seed=wl.cfg.seed)
        r.set_emit_nat([0.0, 0.0, 0.0])
        o = oracle.OracleBeam(wl)
        blcases.start(r, parts)
        blcases.start(o, parts)
        for b in (r, o):
            b.MPBeamRMSCal(0)
            b.BeamMomtumUpdateDueToRFTest()
        for j in range(0, wl.n_bunches, 37):
            assert o.rf_info(j, 0) == r.rf_info(j, 0)
        r.close()
