"""The oracle restatement pinned to the reference's own compiled code.

Fixture tests (always): the oracle tracks each case of tests/refcases.py
from the same input files and particles as the reference did when it wrote
tests/golden/ref_tracking.npz, and must reproduce its coordinates, survival
flags and moments.  Live tests (when oracle/_ref is built): the reference
build itself beside the oracle, stage by stage.
"""
import numpy as np
import pytest

import oracle
import refcases
from oracle import ref

# oracle vs reference: identical arithmetic except w(z) (the oracle's own
# evaluation, within ~1e-16 of Faddeeva::w), so bit-equal without ions
TOL = {"plain_sr": 0.0, "plain_1000": 0.0, "batched_lr_fir": 0.0, "fast_ion": 1e-13,
       "trapping_slice": 1e-12}

live = pytest.mark.skipif(not ref.available(), reason="oracle/_ref/libcetasim_ref.so not built")


# plain_sr_1000's 1000 short-range-wake turns take the oracle minutes; the
# CUDA path is checked against that fixture (test_gpu_ref.py)
@pytest.mark.parametrize("case", [c for c in refcases.CASES if c != "plain_sr_1000"])
def test_oracle_reproduces_reference_fixture(case, tmp_path):
    g = refcases.golden()
    wl, _, parts = refcases.build(case, str(tmp_path))
    assert refcases.parts_digest(parts) == bytes(g[f"{case}/digest"]).hex(), \
        "the seeded initial particles changed"
    o = oracle.OracleBeam(wl)
    refcases.start(case, o, wl, parts)
    o.Run(0, refcases.CASES[case][2])
    o.MPBeamRMSCal(0)
    worst = 0.0
    for j in g[f"{case}/bunches"]:
        c, s = o.download(int(j))
        want, ws = g[f"{case}/coords/{j}"], g[f"{case}/surv/{j}"]
        assert np.array_equal(s, ws), f"bunch {j}: survival flags differ"
        worst = max(worst, refcases.coord_rel_err(c, want, s == 0).max())
    assert worst <= TOL[case], worst
    got = refcases.moments_array(o.moments())
    want = g[f"{case}/moments"]
    assert np.array_equal(got[:, 0], want[:, 0])  # survivors
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
    assert np.max(rel[:, 1:]) <= max(TOL[case], 1e-13) * 10 or np.max(np.abs(got - want)) == 0


@live
def test_derived_ring_constants_match_the_reference(tmp_path):
    wl, path, _ = refcases.build("fast_ion", str(tmp_path))
    r = ref.RefBeam(path, seed=wl.cfg.seed)
    rr = r.ring()
    c = wl.cfg.ring
    assert rr["r_gamma"] == c.r_gamma and rr["r_beta"] == c.r_beta
    assert rr["t0"] == c.t0 and rr["f0"] == c.f0 and rr["work_qz"] == c.work_qz
    assert [rr["damp_x"], rr["damp_y"], rr["damp_z"]] == list(c.synch_rad_damp_time)[:3]
    for j in (0, 41, 79):
        bi = r.bunch_info(j)
        assert bi["harm"] == wl.harm[j] and bi["ne"] == wl.ne[j]


@live
def test_stage_by_stage_moments_and_sr_bins(tmp_path):
    """Moments at every IP of one turn and the SR bin geometry and counts
    (MPBunch.cpp:1899-1918), bit for bit."""
    wl, path, parts = refcases.build("plain_sr", str(tmp_path))
    r = ref.RefBeam(path, seed=wl.cfg.seed)
    r.set_emit_nat([0.0, 0.0, 0.0])
    o = oracle.OracleBeam(wl)
    for j, c in enumerate(parts):
        r.upload(j, c)
        o.upload(j, c)
    for b in (r, o):
        b.MPBeamRMSCal(0)
        b.BeamTransferPerInteractionPointDueToLatticeT(0)
        b.MPBeamRMSCal(0)
        b.BeamMomtumUpdateDueToRFTest()
        b.BeamLongiPosTransferOneTurn()
        b.BeamEnergyLossOneTurn()
        b.BeamSynRadDamping(0)
    # transmission is set by the mark-lost stage only (the reference's member
    # keeps its initial 1.0 until then): compared in the fixture tests
    assert np.array_equal(refcases.moments_array(r.moments())[:, :-1],
                          refcases.moments_array(o.moments())[:, :-1])
    # the reference's geometry from the state the SR step will bin; the
    # oracle reports the geometry its SR step used
    zlo, dz, counts = r.sr_bins(0, wl.cfg.sr_bins)
    r.SRWakeBeamIntaction(0)
    o.SRWakeBeamIntaction(0)
    ozlo, odz, ocounts = o.sr_bins(0)
    assert (zlo, dz) == (ozlo, odz)
    assert np.array_equal(counts, ocounts)
    for j in range(wl.n_bunches):
        assert np.array_equal(r.download(j)[0], o.download(j)[0])


@live
def test_ion_clouds_mid_train_match(tmp_path):
    """Cloud contents after the train passed IP 0 of the first turn (births
    from the shared counter-based stream, kicks, drift, losses)."""
    wl, path, parts = refcases.build("fast_ion", str(tmp_path))
    r = ref.RefBeam(path, seed=wl.cfg.seed)
    r.set_emit_nat([0.0, 0.0, 0.0])
    o = oracle.OracleBeam(wl)
    for j, c in enumerate(parts):
        r.upload(j, c)
        o.upload(j, c)
    for b in (r, o):
        b.MPBeamRMSCal(0)
        b.MPBeamRMSCal(0)
        b.SSBeamIonEffectOneInteractionPoint(0, 0)
    # the clouds were cleared by the 3760-bucket gap only at the next IP call;
    # compare the electrons the clouds kicked
    worst = 0.0
    for j in range(wl.n_bunches):
        cr, sr = r.download(j)
        co, so = o.download(j)
        assert np.array_equal(sr, so)
        worst = max(worst, refcases.coord_rel_err(co, cr, so == 0).max())
    assert worst <= 1e-13, worst
    xr = r.ions(0)
    xo = o.ions(0)
    assert len(xr[0]) == len(xo[0])
    for a, b in zip(xr, xo):
        np.testing.assert_allclose(b, a, rtol=1e-12, atol=1e-300)


@live
def test_reference_exit_becomes_a_status(tmp_path):
    """Bunch::MarkLostParticle exits below 50 % transmission
    (Bunch.cpp:194-197); the harness returns a status instead."""
    wl, path, parts = refcases.build("plain_1000", str(tmp_path))
    r = ref.RefBeam(path, seed=wl.cfg.seed)
    c = parts[0].copy()
    c[4][: len(c[4]) * 2 // 3] = 10.0  # |z| beyond C / 2h: longitudinally lost
    r.upload(0, c)
    with pytest.raises(RuntimeError, match="exit"):
        r.MarkParticleLostInBunch()


@live
def test_refuses_a_directory_with_sdds_files(tmp_path):
    wl, path, _ = refcases.build("plain_1000", str(tmp_path))
    (tmp_path / "keep.sdds").write_text("x")
    with pytest.raises(RuntimeError, match="refusing"):
        ref.RefBeam(path, seed=1)
