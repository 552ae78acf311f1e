"""Whole turns (MPBeam::Run order) on the GPU through cg_run_turns against the
oracle's turn loop, and the fused graph path against the staged calls."""
import numpy as np
import pytest

from helpers import TRAPPED, coord_err, moments_close, pair, particles, small

pytestmark = pytest.mark.gpu


def test_1000_turns_quantum_excitation_off_1e10():
    # the parity gate: same initial particles, QE off, coordinates agree to
    # <= 1e-10 relative after 1000 turns (map + RF + drift + loss + damping)
    wl = small("plain_single", 0.02, qe=False, flag_sr_wake=0)
    g, o = pair(wl, particles(wl))
    g.Run(0, 1000)
    o.Run(0, 1000)
    assert coord_err(g, o, wl).max() <= 1e-10


def test_turns_with_sr_wake_and_quantum_excitation():
    wl = small("plain_single", 0.05, sr_bins=40)
    g, o = pair(wl, particles(wl))
    g.Run(0, 60)
    o.Run(0, 60)
    assert coord_err(g, o, wl).max() <= 1e-9
    g.MPBeamRMSCal(0)
    o.MPBeamRMSCal(0)
    assert not moments_close(g.moments(), o.moments(), 1e-9)


def test_fast_ion_turns():
    wl = small("fast_ion", 0.01, bunch_current=TRAPPED)  # 80 bunches x 200, 20 IPs
    g, o = pair(wl, particles(wl, seed=21, spread=2.0))
    g.Run(0, 5)
    o.Run(0, 5)
    assert coord_err(g, o, wl).max() <= 1e-9
    for k in (0, 19):
        ig, io = g.ions(k), o.ions(k)
        assert len(ig[0]) == len(io[0])
        if len(io[0]):
            assert np.allclose(ig[0], io[0], rtol=1e-9, atol=1e-9 * np.max(np.abs(io[0])))


def test_batched_train_turns_without_ions():
    # ragged 900-bunch train, 50 sections, LR wake + FIR + synchrotron radiation
    wl = small("batched_uneven", 0.002, flag_beam_ion=0)
    g, o = pair(wl, particles(wl, seed=8, spread=3.0))
    g.Run(0, 3)
    o.Run(0, 3)
    assert coord_err(g, o, wl).max() <= 1e-9


def test_batched_train_turns_with_ions_statistics():
    # with the ion chain on, a 1e-15 change of one coordinate grows to 1e-5
    # in two turns in the oracle itself (the ion motion over 900 passages is
    # chaotic), so the comparison is on bunch moments
    wl = small("batched_uneven", 0.002, bunch_current=TRAPPED)
    g, o = pair(wl, particles(wl, seed=8, spread=3.0))
    g.Run(0, 2)
    o.Run(0, 2)
    g.MPBeamRMSCal(0)
    o.MPBeamRMSCal(0)
    mg, mo = g.moments(), o.moments()
    for f in ("rms_x", "rms_y", "bunch_length", "energy_spread"):
        a = np.array([getattr(m, f) for m in mg])
        b = np.array([getattr(m, f) for m in mo])
        assert np.max(np.abs(a / b - 1)) < 1e-3, f
    ex = np.array([m.emit[0] for m in mg]) / np.array([m.emit[0] for m in mo])
    assert np.max(np.abs(ex - 1)) < 1e-3


def test_graph_equals_staged_calls():
    wl = small("fast_ion", 0.01)
    parts = particles(wl, seed=2)
    g1, _ = pair(wl, parts)
    g2, _ = pair(wl, parts)
    g1.Run(0, 2)
    K = wl.cfg.n_sections
    for n in range(2):
        for k in range(K):
            g2.MPBeamRMSCal(k)
            g2.SSBeamIonEffectOneInteractionPoint(n, k)
            g2.BeamTransferPerInteractionPointDueToLatticeT(k)
        g2.BeamMomtumUpdateDueToRFTest()
        g2.BeamLongiPosTransferOneTurn()
        g2.BeamEnergyLossOneTurn()
        g2.BeamSynRadDamping(n)
        g2.MarkParticleLostInBunch()
    for j in range(wl.n_bunches):
        a, sa = g1.download(j)
        b, sb = g2.download(j)
        assert np.array_equal(a, b) and np.array_equal(sa, sb)
