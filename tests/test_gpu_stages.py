"""Each MPBeam stage on the GPU (through the C ABI) against the oracle on the
same seeded particles.  Tolerances are relative to the rms of each
coordinate (or to the kick's own scale) and are stated per test."""
import numpy as np
import pytest

from helpers import TRAPPED, coord_err, moments_close, pair, particles, small

pytestmark = pytest.mark.gpu


def test_moments_all_fields():
    wl = small("fast_ion", 0.02)  # 80 bunches x 400
    g, o = pair(wl, particles(wl))
    for k in (0, 7):
        g.MPBeamRMSCal(k)
        o.MPBeamRMSCal(k)
        assert not moments_close(g.moments(), o.moments(), 1e-13)


def test_moments_ragged_bunches_with_losses():
    wl = small("batched_uneven", 0.01)  # 900 bunches of 50..500
    wl_parts = particles(wl, seed=3)
    rng = np.random.default_rng(5)
    surv = [(rng.random(len(c[0])) < 0.1).astype(np.uint8) for c in wl_parts]
    g, o = pair(wl, wl_parts, surv)
    g.MPBeamRMSCal(3)
    o.MPBeamRMSCal(3)
    assert not moments_close(g.moments(), o.moments(), 1e-13)


def test_section_maps_one_turn():
    wl = small("fast_ion", 0.05)
    g, o = pair(wl, particles(wl))
    for k in range(wl.cfg.n_sections):
        g.BeamTransferPerInteractionPointDueToLatticeT(k)
        o.BeamTransferPerInteractionPointDueToLatticeT(k)
    assert coord_err(g, o, wl).max() <= 1e-13


def test_lost_particles_are_not_mapped():
    wl = small("plain_single", 0.01)
    parts = particles(wl)
    surv = [np.zeros(len(parts[0][0]), dtype=np.uint8)]
    surv[0][::7] = 1
    g, o = pair(wl, parts, surv)
    g.BeamTransferPerInteractionPointDueToLatticeT(0)
    cg_, _ = g.download(0)
    assert np.array_equal(cg_[:, ::7], parts[0][:, ::7])


def test_longitudinal_stages():
    wl = small("plain_single", 0.02)
    parts = particles(wl)
    surv = [np.zeros(len(parts[0][0]), dtype=np.uint8)]
    surv[0][::11] = 2  # lost particles still get RF, drift and energy loss
    g, o = pair(wl, parts, surv)
    for st in ("BeamMomtumUpdateDueToRFTest", "BeamLongiPosTransferOneTurn", "BeamEnergyLossOneTurn"):
        getattr(g, st)()
        getattr(o, st)()
        assert coord_err(g, o, wl, alive_only=False).max() <= 1e-14, st


@pytest.mark.parametrize("qe", [False, True])
def test_synrad_same_philox_draws(qe):
    wl = small("plain_single", 0.02, qe=qe)
    g, o = pair(wl, particles(wl))
    for turn in (0, 1, 12345):
        g.BeamSynRadDamping(turn)
        o.BeamSynRadDamping(turn)
    assert coord_err(g, o, wl).max() <= 1e-13


def test_mark_lost_flags_and_transmission():
    wl = small("fast_ion", 0.01)
    parts = particles(wl)
    rng = np.random.default_rng(2)
    for c in parts:
        idx = rng.choice(len(c[0]), 20, replace=False)
        c[0][idx[:8]] = 0.2   # beyond the 0.1 m aperture
        c[4][idx[5:14]] = 0.5  # beyond C/(2h)
    g, o = pair(wl, parts)
    tg = g.MarkParticleLostInBunch()
    to = o.MarkParticleLostInBunch()
    assert np.array_equal(tg, to)
    for j in range(wl.n_bunches):
        assert np.array_equal(g.download(j)[1], o.download(j)[1])


def test_sr_wake_bins_bit_exact_and_kick():
    wl = small("plain_single", 0.05)  # 5000 particles, 100 bins
    g, o = pair(wl, particles(wl))
    g.MPBeamRMSCal(0)
    o.MPBeamRMSCal(0)
    dp0 = g.download(0)[0][5].copy()
    z = g.download(0)[0][4]
    for turn in range(3):
        g.SRWakeBeamIntaction(turn)
        o.SRWakeBeamIntaction(turn)
        zlo_g, dz_g, cnt_g = g.sr_bins(0)
        zlo_o, dz_o, cnt_o = o.sr_bins(0)
        assert abs(zlo_g - zlo_o) <= 1e-14 * abs(zlo_o) and abs(dz_g - dz_o) <= 1e-14 * dz_o
        # counts are integers: bit-exact given the geometry
        idx = ((z - zlo_g) / dz_g).astype(np.int64)
        idx = idx[(idx >= 0) & (idx < wl.cfg.sr_bins)]
        assert np.array_equal(cnt_g, np.bincount(idx, minlength=wl.cfg.sr_bins))
        if zlo_g == zlo_o and dz_g == dz_o:
            assert np.array_equal(cnt_g, cnt_o)
    kick_g = g.download(0)[0][5] - dp0
    kick_o = o.download(0)[0][5] - dp0
    assert np.max(np.abs(kick_g - kick_o)) <= 1e-11 * np.max(np.abs(kick_o))


def test_sr_wake_transverse_potentials_accumulate_as_the_oracle():
    """The x, y potentials the reference accumulates for its potentials file
    (MPBunch.cpp:1981-1993, both from the horizontal centroids), over turns
    with the beam moving, against the oracle; the z row is the kick's."""
    wl = small("plain_single", 0.05)
    g, o = pair(wl, particles(wl))
    g.set_sr_potentials(True)
    for turn in range(3):
        for b in (g, o):
            b.MPBeamRMSCal(0)
            b.SRWakeBeamIntaction(turn)
            b.BeamTransferPerInteractionPointDueToLatticeT(0)
        pg, po = g.sr_potentials(0), o.sr_potentials(0)
        for q in range(3):
            sc = np.max(np.abs(po[q]))
            assert sc > 0 and np.max(np.abs(pg[q] - po[q])) <= 1e-11 * sc, (turn, q)


def test_lr_wake_and_fir_over_turns():
    wl = small("batched_uneven", 0.004)  # 900 bunches x 20..200
    g, o = pair(wl, particles(wl, seed=9, spread=5.0))
    for turn in range(4):
        g.MPBeamRMSCal(wl.cfg.n_sections - 1)
        o.MPBeamRMSCal(wl.cfg.n_sections - 1)
        g.LRWakeBeamIntaction()
        o.LRWakeBeamIntaction()
        g.MPBeamRMSCal(0)
        o.MPBeamRMSCal(0)
        g.FIRBunchByBunchFeedback(turn + 1)
        o.FIRBunchByBunchFeedback(turn + 1)
    assert coord_err(g, o, wl, alive_only=False).max() <= 1e-11


def test_ion_chain_one_interaction_point():
    wl = small("fast_ion", 0.02, bunch_current=TRAPPED)  # 80 bunches x 400
    g, o = pair(wl, particles(wl, seed=4, spread=3.0))
    for turn in range(2):
        for k in (0, 1):
            g.MPBeamRMSCal(k)
            o.MPBeamRMSCal(k)
            g.SSBeamIonEffectOneInteractionPoint(turn, k)
            o.SSBeamIonEffectOneInteractionPoint(turn, k)
            rg, ro = g.cloud_record(k), o.cloud_record(k)
            assert np.array_equal(rg[..., 5], ro[..., 5])  # ion counts
            # coefficient and rms: relative; centroids: against the rms size
            assert np.allclose(rg[..., :3], ro[..., :3], rtol=1e-11, atol=0)
            scale = np.maximum(ro[..., 1:3], 1e-300)
            assert np.all(np.abs(rg[..., 3:5] - ro[..., 3:5]) <= 1e-11 * scale)
            ig, io = g.ions(k), o.ions(k)
            assert len(ig[0]) == len(io[0])
            for a, b in zip(ig, io):
                if len(b):
                    assert np.allclose(a, b, rtol=1e-11, atol=1e-11 * np.max(np.abs(b)))
    assert coord_err(g, o, wl).max() <= 1e-12


def test_ion_chain_near_threshold_statistics():
    """At the benchmark current (ions near their trapping threshold) the ion
    motion is chaotic: counts agree exactly and the cloud Gaussians seen by
    the electrons agree statistically."""
    wl = small("fast_ion", 0.02)
    g, o = pair(wl, particles(wl, seed=4, spread=3.0))
    g.MPBeamRMSCal(0)
    o.MPBeamRMSCal(0)
    g.SSBeamIonEffectOneInteractionPoint(0, 0)
    o.SSBeamIonEffectOneInteractionPoint(0, 0)
    rg, ro = g.cloud_record(0), o.cloud_record(0)
    assert np.array_equal(rg[..., 5], ro[..., 5])
    # the first bunches see clouds of a few ions, identical to rounding
    assert np.allclose(rg[:5, :, :5], ro[:5, :, :5], rtol=1e-9)
    # over the train, rms sizes agree on average within 1 %
    for q in (1, 2):
        assert abs(rg[:, 0, q].mean() / ro[:, 0, q].mean() - 1) < 1e-2


def test_ion_chain_two_species():
    """CO and CO2 clouds at the same IP (one trajectory set per species): the
    records of both species and the clouds against the oracle, both species
    trapped (H2 would sit below the critical mass at this current, where the
    ion motion is chaotic)."""
    wl = small("fast_ion", 0.02, bunch_current=TRAPPED)
    ion = wl.cfg.ion
    ion.n_species = 2
    ion.mass_number[1] = 44.0
    ion.cross_section[1] = 2.5e-22
    ion.gas_percent[0], ion.gas_percent[1] = 0.8, 0.2
    g, o = pair(wl, particles(wl, seed=8, spread=3.0))
    for k in (0, 1):
        g.MPBeamRMSCal(k)
        o.MPBeamRMSCal(k)
        g.SSBeamIonEffectOneInteractionPoint(0, k)
        o.SSBeamIonEffectOneInteractionPoint(0, k)
        rg, ro = g.cloud_record(k), o.cloud_record(k)
        assert rg.shape == ro.shape == (wl.n_bunches, 2, 6)
        assert np.array_equal(rg[..., 5], ro[..., 5])
        assert np.allclose(rg[..., :3], ro[..., :3], rtol=1e-11, atol=0)
        for p in (0, 1):
            ig, io = g.ions(k, p), o.ions(k, p)
            assert len(ig[0]) == len(io[0])
    assert coord_err(g, o, wl).max() <= 1e-12


def test_kick_autotuner_keeps_the_beam_and_shapes_agree():
    """The autotuner times the kick shapes on the live beam and puts px, py
    back; every shape computes the same kicks bit for bit."""
    import ctypes as C
    wl = small("fast_ion", 0.02, bunch_current=TRAPPED)
    parts = particles(wl, seed=6, spread=3.0)
    g, _ = pair(wl, parts)
    g.MPBeamRMSCal(0)
    g.SSBeamIonEffectOneInteractionPoint(0, 0)
    before = [g.download(j) for j in range(wl.n_bunches)]
    choice, ms = g.autotune(0, reps=3)
    n = len(ms) - 4
    assert 0 <= choice < 2 * n and np.all(ms > 0) and ms[choice % n] == ms[:n].min()
    after = [g.download(j) for j in range(wl.n_bunches)]
    for (a, s), (b, t) in zip(before, after):
        assert np.array_equal(a, b) and np.array_equal(s, t)
    kicked = []
    for v in range(n):
        for j, (c, s) in enumerate(before):
            g.upload(j, c, s)
        g.set_kick_variant(v)
        t = C.c_double()
        g._check(g.lib.cg_time_stage(g.h, 1, 0, 1, C.byref(t)))
        kicked.append([g.download(j)[0] for j in range(wl.n_bunches)])
    for other in kicked[1:]:
        for a, b in zip(kicked[0], other):
            assert np.array_equal(a, b)


def test_kick_inside_the_map_pass_repeats_the_separate_kernels():
    wl = small("fast_ion", 0.01, bunch_current=TRAPPED)
    parts = particles(wl, seed=7)
    import ctypes as C
    from cetasim_b200 import _abi
    nv = C.c_int()
    _abi.load().cg_kick_variants(C.byref(nv))
    runs = []
    for v in (0, nv.value):  # nv = the first kick shape inside the map pass
        g, _ = pair(wl, parts)
        g.set_kick_variant(v)
        g.Run(0, 4)
        runs.append([g.download(j)[0] for j in range(wl.n_bunches)])
    worst = max(np.max(np.abs(a - b) / (np.abs(b).max(axis=1, keepdims=True) + 1e-300))
                for a, b in zip(*runs))
    assert worst <= 1e-14


@pytest.mark.parametrize("name,scale,groups", [("fast_ion", 0.01, 3), ("batched_uneven", 0.01, 6)])
def test_turns_with_the_asynchronous_map_pass_repeat_the_register_pass(name, scale, groups):
    """Whole turns (pipelined, with ions, wakes and feedback) with the map pass
    that keeps each CTA's next chunk in flight give the coordinates, survival
    flags and clouds of the register pass bit for bit."""
    wl = small(name, scale, bunch_current=TRAPPED)
    parts = particles(wl, seed=10)
    runs = []
    from cetasim_b200.beam import MPBeam
    for on in (False, True):
        g = MPBeam(wl)
        for j, c in enumerate(parts):
            g.upload(j, c)
        g.set_pipeline(groups, 64, True)
        g.set_map_async(on)
        assert g.map_async() == on
        g.Run(0, 3)
        runs.append(([g.download(j) for j in range(wl.n_bunches)],
                     [g.ions(k) for k in (0, wl.cfg.n_sections - 1)]))
    (ca, ia), (cb, ib) = runs
    for (x, s), (y, t) in zip(ca, cb):
        assert np.array_equal(x, y) and np.array_equal(s, t)
    for u, v in zip(ia, ib):
        for p, q in zip(u, v):
            assert np.array_equal(p, q)


def test_turns_with_reserved_walk_sms_repeat_the_shared_ones():
    """Walk CTAs that reserve their SM's shared memory (no kick or map CTA
    beside them) give the same turns bit for bit."""
    from cetasim_b200.beam import MPBeam
    wl = small("batched_uneven", 0.01, bunch_current=TRAPPED)
    parts = particles(wl, seed=13)
    runs = []
    for on in (False, True):
        g = MPBeam(wl)
        for j, c in enumerate(parts):
            g.upload(j, c)
        g.set_pipeline(8, 64, True)
        g.set_walk_reserve(on)
        g.Run(0, 3)
        runs.append(([g.download(j) for j in range(wl.n_bunches)],
                     [g.ions(k) for k in (0, wl.cfg.n_sections - 1)]))
    (ca, ia), (cb, ib) = runs
    for (x, s), (y, t) in zip(ca, cb):
        assert np.array_equal(x, y) and np.array_equal(s, t)
    for u, v in zip(ia, ib):
        for p, q in zip(u, v):
            assert np.array_equal(p, q)


@pytest.mark.parametrize("groups,ramp", [(3, False), (4, True), (16, False), (2, True)])
def test_pipelined_turn_repeats_the_unpipelined_turn(groups, ramp):
    """The ion walk in segments with records, kicks and maps overlapping the
    next segment gives the same turn bit for bit."""
    wl = small("fast_ion", 0.01, bunch_current=TRAPPED)
    parts = particles(wl, seed=9)
    runs = []
    for gcount in (1, groups):
        g, _ = pair(wl, parts)
        g.set_pipeline(gcount, 0, ramp)
        g.Run(0, 4)
        runs.append(([g.download(j) for j in range(wl.n_bunches)],
                     [g.ions(k) for k in (0, wl.cfg.n_sections - 1)],
                     g.cloud_record(wl.cfg.n_sections - 1)))
    (ca, ia, ra), (cb, ib, rb) = runs
    for (x, s), (y, t) in zip(ca, cb):
        assert np.array_equal(x, y) and np.array_equal(s, t)
    for u, v in zip(ia, ib):
        for p, q in zip(u, v):
            assert np.array_equal(p, q)
    assert np.array_equal(ra, rb)


def _stage(g, stage, k, reps=1):
    import ctypes as C
    t = C.c_double()
    g._check(g.lib.cg_time_stage(g.h, stage, k, reps, C.byref(t)))


@pytest.mark.parametrize("name,scale,kick", [("batched_uneven", 0.05, False),
                                             ("fast_ion", 0.15, False),
                                             ("fast_ion", 0.15, True)])
def test_streamed_map_pass_repeats_the_register_pass(name, scale, kick):
    """The map pass with each CTA's next chunk staged in shared memory by
    cp.async (stages 8, 9) gives the coordinates and moments of the register
    pass (stages 5, 7) bit for bit, on ragged bunches (partial chunks and
    tiles) with lost particles."""
    wl = small(name, scale, bunch_current=TRAPPED if kick else None)
    parts = particles(wl, seed=11, spread=3.0 if kick else 1.0)
    rng = np.random.default_rng(12)
    surv = [(rng.random(len(c[0])) < 0.1).astype(np.uint8) for c in parts]
    runs = []
    for stage in ((7, 9) if kick else (5, 8)):
        g, _ = pair(wl, parts, surv)
        g.MPBeamRMSCal(0)
        if kick:
            g.SSBeamIonEffectOneInteractionPoint(0, 0)
        _stage(g, stage, 0, reps=3)  # three passes: the per-bunch counters rearm
        runs.append(([g.download(j) for j in range(wl.n_bunches)], g.moments()))
    (ca, ma), (cb, mb) = runs
    for (x, s), (y, t) in zip(ca, cb):
        assert np.array_equal(x, y) and np.array_equal(s, t)
    assert bytes(ma) == bytes(mb)


def test_pipeline_autotuner_restores_the_beam_and_shapes_agree():
    """The pipeline autotuner runs whole turns with every shape and puts the
    beam and the clouds back; the walk CTA size changes only the summation
    order of the cloud moments."""
    wl = small("fast_ion", 0.01, bunch_current=TRAPPED)
    parts = particles(wl, seed=13)
    g, _ = pair(wl, parts)
    g.Run(0, 2)
    before = ([g.download(j) for j in range(wl.n_bunches)], g.ions(0))
    from cetasim_b200 import _abi
    shape, ms = g.autotune_pipeline(2, reps=1)
    assert shape in _abi.PIPE_SHAPES
    assert np.all(ms > 0)
    after = ([g.download(j) for j in range(wl.n_bunches)], g.ions(0))
    for (a, s), (b, t) in zip(before[0], after[0]):
        assert np.array_equal(a, b) and np.array_equal(s, t)
    for p, q in zip(before[1], after[1]):
        assert np.array_equal(p, q)
    runs = []
    for ions in (64, 16, 8):
        h, _ = pair(wl, parts)
        h.set_pipeline(3, ions)
        h.Run(0, 4)
        runs.append([h.download(j)[0] for j in range(wl.n_bunches)])
    for other in runs[1:]:
        worst = max(np.max(np.abs(a - b) / (np.abs(b).max(axis=1, keepdims=True) + 1e-300))
                    for a, b in zip(other, runs[0]))
        assert worst <= 1e-12


@pytest.mark.parametrize("groups", [1, 3])
def test_traced_turn_equals_the_graph_turn(groups):
    """cg_trace_turn runs the turn's launches directly with timing events: the
    same beam as the turn graph, and a timeline that grows on every stream."""
    wl = small("fast_ion", 0.01, bunch_current=TRAPPED)
    parts = particles(wl, seed=17)
    a, _ = pair(wl, parts)
    b, _ = pair(wl, parts)
    for g in (a, b):
        g.set_pipeline(groups, 64)
    a.Run(0, 2)
    b.Run(0, 1)
    tr = b.trace_turn(1)
    for j in range(wl.n_bunches):
        (x, s), (y, t) = a.download(j), b.download(j)
        assert np.array_equal(x, y) and np.array_equal(s, t)
    assert tr[0][0] == "start" and tr[-1][0] == "mark_lost"
    kinds = {r[0] for r in tr}
    assert {"ion_kick", "map_pass", "long"} <= kinds
    assert ("ion_walk" in kinds) == (groups > 1) and ("ion_chain" in kinds) == (groups == 1)
    for st in (0, 1, 2):
        ts = [r[4] for r in tr if r[1] == st]
        assert all(u <= v for u, v in zip(ts, ts[1:]))
    assert tr[-1][4] >= max(r[4] for r in tr) - 1e-9


def test_upload_beam_matches_per_bunch_uploads():
    """cg_upload_beam: (6, n) rows in one 2D copy, padded rows (pitch > n) and
    scattered rows (six separate arrays) give the bunches cg_upload_bunch
    gives, survival bytes included."""
    import ctypes as C
    wl = small("batched_uneven", 0.01)
    parts = particles(wl, seed=21)
    rng = np.random.default_rng(22)
    surv = [(rng.random(len(c[0])) < 0.2).astype(np.uint8) for c in parts]
    g, _ = pair(wl, parts, surv)
    want = [g.download(j) for j in range(wl.n_bunches)]
    h, _ = pair(wl, [np.zeros_like(c) for c in parts])
    keep = []
    table = (C.c_void_p * (6 * wl.n_bunches))()
    for j, c in enumerate(parts):
        n = c.shape[1]
        if j % 3 == 0:      # contiguous (6, n)
            a = np.ascontiguousarray(c)
            rows = [a[d] for d in range(6)]
        elif j % 3 == 1:    # padded rows: pitch n + 7
            big = np.zeros((6, n + 7))
            big[:, :n] = c
            a = big
            rows = [big[d, :n] for d in range(6)]
        else:               # six separate arrays
            rows = [np.array(c[d]) for d in range(6)]
            a = rows
        keep.append(a)
        for d in range(6):
            table[6 * j + d] = rows[d].ctypes.data
    sv = [np.ascontiguousarray(x) for x in surv]
    st = (C.c_void_p * wl.n_bunches)(*[x.ctypes.data for x in sv])
    h._check(h.lib.cg_upload_beam(h.h, table, st))
    for j in range(wl.n_bunches):
        (x, s), (y, t) = want[j], h.download(j)
        assert np.array_equal(x, y) and np.array_equal(s, t)


def test_lr_wake_with_resistive_wall_over_turns():
    """Long-range wake of resonators plus resistive-wall sectors (round,
    elliptical both ways, and a round one after an elliptical one)."""
    wl = small("batched_uneven", 0.004)
    rws = wl.cfg.lr_rw
    sec = [(0.02, 0.02, 100.0, 8.0, 9.0, 2, 5.8e7), (0.03, 0.01, 20.0, 10.0, 7.0, 3, 1.4e6),
           (0.01, 0.02, 10.0, 4.0, 5.0, 1, 3.7e7), (0.015, 0.015, 5.0, 6.0, 3.0, 4, 5.8e7)]
    rws.n = len(sec)
    for i, (rx, ry, ln, bx, by, num, sig) in enumerate(sec):
        rws.radius_x[i], rws.radius_y[i], rws.length[i] = rx, ry, ln
        rws.beta_x[i], rws.beta_y[i], rws.num[i], rws.sigma[i] = bx, by, num, sig
    parts = particles(wl, seed=19, spread=5.0)
    g, o = pair(wl, parts)
    for turn in range(4):
        g.MPBeamRMSCal(wl.cfg.n_sections - 1)
        o.MPBeamRMSCal(wl.cfg.n_sections - 1)
        g.LRWakeBeamIntaction()
        o.LRWakeBeamIntaction()
    assert coord_err(g, o, wl, alive_only=False).max() <= 1e-11
    # the sectors matter: without them the kicks differ
    rws.n = 0
    g0, _ = pair(wl, parts)
    for turn in range(4):
        g0.MPBeamRMSCal(wl.cfg.n_sections - 1)
        g0.LRWakeBeamIntaction()
    assert coord_err(g0, o, wl, alive_only=False).max() > 1e-9


def test_sr_wake_with_resistive_wall():
    """Short-range wake of resistive-wall sectors (and no resonators): the
    longitudinal kicks against the oracle."""
    wl = small("plain_single", 0.05)
    wl.cfg.sr_bbr.n = 0
    rws = wl.cfg.sr_rw
    sec = [(0.012, 0.012, 200.0, 8.0, 9.0, 1, 5.8e7), (0.03, 0.01, 50.0, 10.0, 7.0, 2, 1.4e6)]
    rws.n = len(sec)
    for i, (rx, ry, ln, bx, by, num, sig) in enumerate(sec):
        rws.radius_x[i], rws.radius_y[i], rws.length[i] = rx, ry, ln
        rws.beta_x[i], rws.beta_y[i], rws.num[i], rws.sigma[i] = bx, by, num, sig
    g, o = pair(wl, particles(wl))
    g.MPBeamRMSCal(0)
    o.MPBeamRMSCal(0)
    dp0 = g.download(0)[0][5].copy()
    for turn in range(2):
        g.SRWakeBeamIntaction(turn)
        o.SRWakeBeamIntaction(turn)
    kick_g = g.download(0)[0][5] - dp0
    kick_o = o.download(0)[0][5] - dp0
    assert np.max(np.abs(kick_o)) > 0
    assert np.max(np.abs(kick_g - kick_o)) <= 1e-10 * np.max(np.abs(kick_o))
