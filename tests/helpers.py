"""Shared helpers of the GPU parity tests: small seeded workloads with the
benchmark shapes, identical initial particles for the GPU and the oracle, and
error metrics."""
import ctypes as C

import numpy as np

import oracle
from cetasim_b200 import configs


# Bunch current of the ion parity tests: with 0.125 mA per bunch CO ions sit
# near their trapping threshold (critical mass number ~23 vs 28), where each
# passage moves an ion by ~1 sigma and rounding differences grow chaotically
# along the train; at 0.02 mA the ions are deeply trapped and the comparison
# is deterministic to rounding.
TRAPPED = 0.02e-3


def small(name, n_scale, qe=True, seed=1234, bunch_current=None, **over):
    wl = configs.make(name, n_scale=n_scale, seed=seed, bunch_current=bunch_current)
    if not qe:
        for i in range(3):
            wl.cfg.ring.emit_nat[i] = 0.0
    for k, v in over.items():
        if k == "sections":
            continue
        setattr(wl.cfg, k, v)
    return wl


def particles(wl, seed=7, spread=1.0, sigma_scale=1.0):
    """Seeded 6-D Gaussian particles per bunch (host side)."""
    rng = np.random.default_rng(seed)
    ex, ey, sz, sdp = wl.gen
    out = []
    for j in range(wl.n_bunches):
        n = int(wl.n_macro[j])
        s = wl.sections[0]
        c = np.empty((6, n))
        c[0] = rng.normal(0, np.sqrt(ex * s.beta_x), n) * sigma_scale + 2e-6 * spread * rng.normal()
        c[1] = rng.normal(0, np.sqrt(ex / s.beta_x), n) * sigma_scale
        c[2] = rng.normal(0, np.sqrt(ey * s.beta_y), n) * sigma_scale + 1e-6 * spread * rng.normal()
        c[3] = rng.normal(0, np.sqrt(ey / s.beta_y), n) * sigma_scale
        c[4] = rng.normal(0, sz, n) * sigma_scale
        c[5] = rng.normal(0, sdp, n) * sigma_scale
        out.append(c)
    return out


def pair(wl, parts, surv=None):
    from cetasim_b200.beam import MPBeam
    g = MPBeam(wl)
    o = oracle.OracleBeam(wl)
    for j, c in enumerate(parts):
        s = None if surv is None else surv[j]
        g.upload(j, c, s)
        o.upload(j, c, s)
    return g, o


def coord_err(g, o, wl, alive_only=True):
    """max |gpu - oracle| / rms(oracle) per coordinate, over all bunches."""
    worst = np.zeros(6)
    for j in range(wl.n_bunches):
        cg_, sg = g.download(j)
        co, so = o.download(j)
        assert np.array_equal(sg, so), "survival flags differ"
        m = (so == 0) if alive_only else np.ones_like(so, dtype=bool)
        for d in range(6):
            scale = np.sqrt(np.mean(co[d][m] ** 2)) + 1e-300
            worst[d] = max(worst[d], np.max(np.abs(cg_[d][m] - co[d][m])) / scale)
    return worst


def moments_close(mg, mo, rtol):
    fields = ["mean", "emit", "eff_emit", "rms_x", "rms_y", "eff_rms_x", "eff_rms_y",
              "bunch_length", "energy_spread", "z_min", "z_max"]
    bad = []
    for j in range(len(mg)):
        a, b = mg[j], mo[j]
        assert a.n_alive == b.n_alive
        for f in fields:
            va, vb = np.array(getattr(a, f), ndmin=1), np.array(getattr(b, f), ndmin=1)
            scale = np.maximum(np.abs(vb), 1e-300)
            if f == "mean":
                # centroids can be ~0: compare against the bunch size scale
                scale = np.array([np.sqrt(b.emit[0] * 10), np.sqrt(b.emit[0] / 10),
                                  np.sqrt(b.emit[1] * 10), np.sqrt(b.emit[1] / 10),
                                  b.bunch_length, b.energy_spread])
            e = np.max(np.abs(va - vb) / scale)
            if not e <= rtol:
                bad.append((j, f, e))
    return bad


def write_input(d, n_turns=60, interval=5, cbmgr="cbmgr", fit=(10, 50), bunches=40,
                macro=200, extra=()):
    """A small MP-model input.dat (the reference's key = value format) and its
    twiss file in directory d: one train of `bunches` bunches every second
    bucket of a 480-bucket ring, two sections, no ions or wakes."""
    import os
    harm = 480
    gap = harm - 2 * bunches
    lines = [
        "runCalSetting = 2", f"runNTurns = {n_turns}", f"runBunchInfoPrintInterval = {interval}",
        "runSynRadDampingFlag = 1", "runBeamIonFlag = 0", "runLongRangeWake = 0",
        "runShortRangeWake = 0", "runFIRBunchByBunchFeedbackFlag = 0", "runRandomSeed = 7",
        f"runGrowthRateFittingStart = {fit[0]}", f"runGrowthRateFittingEnd = {fit[1]}",
        "ringCircRing = 288.0", "ringWorkQ = 18.21 10.17", "ringChrom = 1.0 1.0",
        "ringSynchRadDampTime = 0.02 0.02 0.01", "ringPipeAperatureX = 0.02",
        "ringPipeAperatureY = 0.01", "ringElectronBeamEnergy = 3.0e9",
        "ringAlphac = 3.0e-4 0 0", "ringU0 = 1.0e6", "ringSdelta0 = 1.0e-3",
        "ringNaturalEmit = 2.0e-9", "ringCoupling = 0.01", "ringCurrent = 0.1",
        "ringSectNum = 2", "ringTwiss = twiss.dat",
        f"rfRingHarm = {harm}", "rfResNum = 1", f"rfResHarm = 1", "rfResVol = 2.0e6",
        "bunchKappa = 0.01", "bunchEmittance = 2.0e-9", "bunchRmsBunchLength = 3.0e-3",
        "bunchRmsEnergySpread = 1.0e-3", f"bunchMacroEleNumPerBunch = {macro}",
        f"fpTotBunchNumber = {bunches}", "fpTrainNumber = 1",
        f"fpBunchNumberPerTrain = {bunches}", f"fpTrainGaps = {gap}", "fpBunchGaps = 1",
    ]
    if cbmgr:
        lines.append(f"runCBMGR = {cbmgr}")
    lines += list(extra)
    with open(os.path.join(d, "input.dat"), "w") as f:
        f.write("\n".join(lines) + "\n")
    rows = ["0.0 10.0 0.5 0.0 0.1 0.0 0.02 5.0 -0.3 0.0 0.0 0.0 0.01 144.0 1.0 300",
            "144.0 8.0 -0.4 3.1 0.2 0.01 0.02 6.0 0.2 2.9 0.0 0.0 0.01 144.0 1.0 300"]
    with open(os.path.join(d, "twiss.dat"), "w") as f:
        f.write("header\n" * 5 + "\n".join(rows) + "\n")
    return os.path.join(d, "input.dat")
