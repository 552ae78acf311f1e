"""The CUDA path against the reference's own compiled code.

Each case of tests/refcases.py is written as the reference's input files,
read by the library's parser, and tracked on the GPU from the same seeded
particles the reference tracked when it wrote tests/golden/ref_tracking.npz
(quantum excitation off; ion births from the shared counter-based stream).
Where oracle/_ref is present (it ships with the build), further cases run
the reference beside the GPU in the same test.
"""
import os
import shutil

import numpy as np
import pytest

import refcases
from cetasim_b200.beam import MPBeam
from oracle import ref

pytestmark = pytest.mark.gpu

# GPU vs reference, max |delta| / rms of each coordinate over alive particles.
# The GPU's transcendentals, fused multiply-adds and w(z) differ from the
# host's by ulps; 1000 turns of the linear map grow that to ~1e-12.
TOL = {"plain_sr": 1e-10, "plain_1000": 1e-10, "plain_sr_1000": 1e-10, "fast_ion": 1e-10, "batched_lr_fir": 1e-10,
       "trapping_slice": 1e-10}


def run_gpu(case, d):
    wl, path, parts = refcases.build(case, d)
    g = MPBeam(wl)
    refcases.start(case, g, wl, parts)
    g.Run(0, refcases.CASES[case][2])
    g.MPBeamRMSCal(0)
    return wl, parts, g


@pytest.mark.parametrize("case", list(refcases.CASES))
def test_gpu_reproduces_reference_fixture(case, tmp_path):
    gold = refcases.golden()
    wl, parts, g = run_gpu(case, str(tmp_path))
    assert refcases.parts_digest(parts) == bytes(gold[f"{case}/digest"]).hex()
    worst = 0.0
    for j in gold[f"{case}/bunches"]:
        c, s = g.download(int(j))
        want, ws = gold[f"{case}/coords/{j}"], gold[f"{case}/surv/{j}"]
        assert np.array_equal(s, ws), f"bunch {j}: survival flags differ"
        worst = max(worst, refcases.coord_rel_err(c, want, s == 0).max())
    assert worst <= TOL[case], f"{case}: {worst:.3e}"
    got = refcases.moments_array(g.moments())
    want = gold[f"{case}/moments"]
    assert np.array_equal(got[:, 0], want[:, 0])  # survivors per bunch
    # centroids and z extremes against the bunch sizes, the rest relatively
    # (columns of refcases.moments_array)
    bx, by = wl.sections[0].beta_x, wl.sections[0].beta_y
    scale = np.abs(want).copy()
    scale[:, 1] = want[:, 13]
    scale[:, 2] = np.sqrt(want[:, 7] / bx)
    scale[:, 3] = want[:, 14]
    scale[:, 4] = np.sqrt(want[:, 8] / by)
    scale[:, 5] = scale[:, 19] = scale[:, 20] = want[:, 17]
    scale[:, 6] = want[:, 18]
    rel = np.abs(got[:, 1:] - want[:, 1:]) / np.maximum(scale[:, 1:], 1e-300)
    assert np.max(rel) <= 1e-8, f"{case}: moments {np.max(rel):.3e}"


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_gpu_and_reference_side_by_side_fast_ion_ip_records(tmp_path):
    """One turn of the trapped fast-ion train: the electrons after every IP
    against the reference run stage by stage."""
    wl, path, parts = refcases.build("fast_ion", str(tmp_path))
    r = ref.RefBeam(path, seed=wl.cfg.seed)
    r.set_emit_nat([0.0, 0.0, 0.0])
    g = MPBeam(wl)
    for j, c in enumerate(parts):
        r.upload(j, c)
        g.upload(j, c)
    for b in (r, g):
        b.MPBeamRMSCal(0)
    for k in range(wl.cfg.n_sections):
        for b in (r, g):
            b.MPBeamRMSCal(k)
            b.SSBeamIonEffectOneInteractionPoint(0, k)
            b.BeamTransferPerInteractionPointDueToLatticeT(k)
        worst = 0.0
        for j in range(0, wl.n_bunches, 7):
            cr, sr = r.download(j)
            cg, sg = g.download(j)
            assert np.array_equal(sr, sg)
            worst = max(worst, refcases.coord_rel_err(cg, cr, sr == 0).max())
        assert worst <= 1e-11, f"IP {k}: {worst:.3e}"
        if k % 5 == 0:
            # the last bunch's kick on every ion of the cloud (ionAccumuFx/Fy)
            fxr, fyr = r.ion_forces(k)
            fxg, fyg, _ = g.ion_forces(k)
            assert len(fxg) == len(fxr)
            for a, b in ((fxg, fxr), (fyg, fyr)) if len(fxr) else ():
                assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b)), k
    # after the last IP: every bunch's totIonCharge (MPBunch.cpp:1208-1209)
    import ctypes as C
    q = np.empty(wl.n_bunches)
    g._check(g.lib.cg_bunch_ion_charge(g.h, q.ctypes.data_as(C.POINTER(C.c_double))))
    want = np.array([r.bunch_ion_charge(j) for j in range(wl.n_bunches)])
    assert np.max(np.abs(q - want)) <= 1e-12 * np.max(np.abs(want))
    # the ideal cavity's voltage at each bunch's last particle after an RF step
    for b in (r, g):
        b.BeamMomtumUpdateDueToRFTest()
    for j in range(0, wl.n_bunches, 7):
        want = r.rf_info(j, 0)
        got = g.rf_info(j, 0)
        for a, b_ in zip(got, want):
            assert abs(a - b_) <= 1e-12 * abs(want[0])


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_initial_distribution_statistics_match_the_reference_generator(tmp_path):
    """k_gaussian against the reference's own MPBunch::DistriGenerator
    (type 3, MPBunch.cpp:98-298), which the reference build ran when it set
    the beam up: 1e5 macroparticles each.  Both keep every draw inside the
    3-sigma cuts; second moments agree within 5 sampling sigmas (2.5 %), and
    the normalised transverse amplitude and longitudinal radius have the same
    law (two-sample Kolmogorov-Smirnov)."""
    from scipy import stats
    from cetasim_b200 import configs, input_dat
    wl = configs.make("plain_single", n_scale=1.0)
    path = input_dat.write_case(str(tmp_path), wl, n_turns=1)
    wl = input_dat.load_case(path)
    r = ref.RefBeam(path, seed=11)
    cr, _ = r.download(0)
    g = MPBeam(wl)
    g.generate(seed=11)
    cg, sg = g.download(0)
    assert (sg == 0).all()
    s0 = wl.sections[0]
    ex, ey, sz, sdp = wl.gen
    rb2 = wl.cfg.ring.r_beta ** 2
    for c in (cr, cg):
        # the cuts of MPBunch.cpp:145 and :256
        assert np.all((c[4] / sz) ** 2 + (c[5] * rb2 / sdp) ** 2 < 9.0)
        assert np.all(c[0] ** 2 / (ex * s0.beta_x) + c[2] ** 2 / (ey * s0.beta_y) <= 9.0)
    n = cr.shape[1]
    for d in range(6):
        vr, vg = np.var(cr[d]), np.var(cg[d])
        assert abs(vg / vr - 1) <= 5 * np.sqrt(2 / n), (d, vg / vr)
    ax = lambda c: c[0] ** 2 / (ex * s0.beta_x) + c[1] ** 2 * s0.beta_x / ex
    lz = lambda c: (c[4] / sz) ** 2 + (c[5] * rb2 / sdp) ** 2
    for f in (ax, lz):
        assert stats.ks_2samp(f(cr), f(cg)).pvalue > 1e-4


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_quantum_excitation_statistics_over_seeds(tmp_path):
    """Radiation damping with quantum excitation ON: the reference draws its
    noise from mt19937 (Bunch.cpp:989-1023, seeded here per run through the
    hooks), the CUDA path from Philox, so single runs differ.  From the same
    initial beam (1.5x the matched size in all planes) 8 seeded runs on each
    side over 400 turns: the seed-averaged emittances, bunch length and
    energy spread agree within 4 standard errors of their difference, and
    both sit between the initial and the equilibrium values."""
    from cetasim_b200 import configs, input_dat
    wl = configs.make("plain_single", n_scale=0.02)
    wl.cfg.flag_sr_wake = 0
    path = input_dat.write_case(str(tmp_path / "case"), wl, n_turns=400)
    wl = input_dat.load_case(path)
    turns, seeds = 400, 8
    parts = [1.5 * c for c in refcases.particles(wl, seed=3)]

    def fields(m):
        return [m.emit[0], m.emit[1], m.bunch_length, m.energy_spread]

    got = {"ref": [], "gpu": []}
    for s in range(seeds):
        # the reference writes .sdds files where it runs: a fresh copy per run
        d = tmp_path / f"seed{s}"
        shutil.copytree(os.path.dirname(path), d, ignore=shutil.ignore_patterns("*.sdds"))
        r = ref.RefBeam(str(d / "input.dat"), seed=1000 + s)
        r.upload(0, parts[0])
        r.Run(0, turns)
        r.MPBeamRMSCal(0)
        got["ref"].append(fields(r.moments()[0]))
        r.close()
        wl.cfg.seed = 1000 + s
        g = MPBeam(wl)
        g.upload(0, parts[0])
        g.Run(0, turns)
        g.MPBeamRMSCal(0)
        got["gpu"].append(fields(g.moments()[0]))
        g.close()
    a, b = np.array(got["ref"]), np.array(got["gpu"])
    se = np.sqrt(a.var(0, ddof=1) / seeds + b.var(0, ddof=1) / seeds)
    diff = np.abs(a.mean(0) - b.mean(0))
    assert np.all(diff <= 4 * se + 1e-3 * np.abs(a.mean(0))), (a.mean(0), b.mean(0), se)
    # the beam is damping towards equilibrium in both
    init = [1.5 ** 2 * wl.gen[0], 1.5 ** 2 * wl.gen[1], 1.5 * wl.gen[2], 1.5 * wl.gen[3]]
    for m in (a.mean(0), b.mean(0)):
        assert m[0] < 0.95 * init[0] and m[2] < 0.99 * init[2]


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("case, bunches", [("batched_lr_fir", [0, 450]), ("fast_ion", [0, 79])])
def test_particle_phase_advance_matches_the_reference(tmp_path, case, bunches):
    """The accumulated phase advance of every particle of two bunches over
    the case's turns (Bunch.cpp:715-731; the turn graph, with the segmented
    maps of the ion train) against the reference."""
    wl, path, parts = refcases.build(case, str(tmp_path))
    r = ref.RefBeam(path, seed=wl.cfg.seed)
    r.set_emit_nat([0.0, 0.0, 0.0])
    g = MPBeam(wl)
    refcases.start(case, r, wl, parts)
    refcases.start(case, g, wl, parts)
    g.set_phase_track(bunches)
    turns = refcases.CASES[case][2]
    r.Run(0, turns)
    g.Run(0, turns)
    for j in bunches:
        a, b = g.phase_adv(j), r.phase_adv(j)
        # a particle whose turn-to-turn phase change lies within rounding of
        # zero can take the other branch of the reference's rule (tmp >= 0 ?
        # tmp : tmp + 2 pi, Bunch.cpp:725-727): then its sum differs by 2 pi
        d = a - b
        wraps = np.round(d / (2 * np.pi))
        assert np.max(np.abs(d - 2 * np.pi * wraps)) <= 1e-9 * np.max(np.abs(b)), j
        assert np.count_nonzero(wraps) <= max(1, 0.01 * wraps.size), (j, np.count_nonzero(wraps))
