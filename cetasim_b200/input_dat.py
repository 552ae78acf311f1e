"""Writes a workload as the reference's own input files, and reads one back.

`write_case(d, wl, ...)` produces in directory d the files CETASim's
`main` reads for an MP run (ReadInputSettings::ParamRead,
ReadInputSettings.cpp:46-1085): `input.dat` with the reference's keys, the
twiss file of LatticeInterActionPoint::InitialLattice (5 header lines, 16
columns per section, LatticeInterActionPoint.cpp:181-240: s, beta_x,
alpha_x, psi_x [rad], eta_x, eta'_x, aperture_x, the same for y, length,
pressure [nTorr], temperature [K]) and the resonator files of
WakeFunction::BBRWakeParaReadIn (12 header lines, then
lRs lQ lfr txRs txQ txfr tyRs tyQ tyfr with frequencies in Hz,
WakeFunction.cpp:251-290).  `load_case(path)` builds the workload from such
an input through the library's parser (cg_config_from_input), so the CUDA
path and the reference read the same file.

Per-bunch macroparticle counts (a train of uneven bunches) are written as
the key `bunchMacroEleNumPerBunchList`, which the library reads and the
reference ignores (its bunches are all `bunchMacroEleNumPerBunch` long).
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import _abi
from .configs import Workload

PA_PER_NTORR = 1.0e-9 * 133.3224  # LatticeInterActionPoint.cpp:239


def _fmt(v) -> str:
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return repr(float(v))


def _bbr_file(path: str, b) -> None:
    rows = []
    for i in range(b.n):
        rows.append(" ".join(_fmt(v) for v in (
            b.l_rs[i], b.l_q[i], b.l_omega[i] / (2 * math.pi),
            b.tx_rs[i], b.tx_q[i], b.tx_omega[i] / (2 * math.pi),
            b.ty_rs[i], b.ty_q[i], b.ty_omega[i] / (2 * math.pi))))
    with open(path, "w") as f:
        f.write("resonator parameters\n" * 12 + "\n".join(rows) + "\n")


def fill_pattern(harm, h: int):
    """Trains of the reference's fill-pattern keys (Train.cpp:38-104) that
    place bunches at the bucket numbers `harm`: one train per run of equal
    spacing.  Returns (numbers per train, train gaps, bunch gaps)."""
    harm = [int(x) for x in harm]
    trains = []
    i = 0
    while i < len(harm):
        if i + 1 < len(harm):
            sp = harm[i + 1] - harm[i]
            j = i + 1
            while j + 1 < len(harm) and harm[j + 1] - harm[j] == sp:
                j += 1
            trains.append((i, j, sp - 1))
            i = j + 1
        else:
            trains.append((i, i, 0))
            i += 1
    npt, tgap, bgap = [], [], []
    for t, (a, b, g) in enumerate(trains):
        n = b - a + 1
        nxt = harm[trains[t + 1][0]] if t + 1 < len(trains) else harm[0] + h
        npt.append(n)
        bgap.append(g)
        tgap.append(nxt - (harm[a] + n * (g + 1)))
    return npt, tgap, bgap


def write_case(d: str, wl: Workload, n_turns: int = 1, print_interval: int | None = None, qe: bool = True,
               seed: int | None = None, extra=()) -> str:
    """The reference's input files for workload `wl` in directory d; returns
    the path of input.dat.  The print interval (default n_turns + 1) must
    not be 0, since the reference's short-range wake step takes the turn
    modulo it (MPBunch.cpp:1962), nor large, since every bunch keeps a
    history of that length (Bunch.cpp:111-115).  qe=False writes a natural emittance of 0, which
    keeps the damping and removes the quantum excitation (the excitation
    coefficients of Bunch.cpp:975-980 vanish)."""
    os.makedirs(d, exist_ok=True)
    if print_interval is None:
        print_interval = n_turns + 1
    cfg, r = wl.cfg, wl.cfg.ring
    M, K = wl.n_bunches, cfg.n_sections
    f0 = r.f0 if r.f0 else None
    if f0 is None:
        raise ValueError("the workload's ring has no derived constants")
    e_charge = 1.602017733e-19
    currents = np.asarray(wl.ne) * f0 * e_charge
    ring_current = float(currents.sum())
    npt, tgap, bgap = fill_pattern(wl.harm, int(r.harmonics))
    nm = [int(x) for x in wl.n_macro]
    kappa = r.coupling
    # The reference reads into default-initialised structs and sizes its
    # arrays at the count keys, so every group is written, in the order of
    # its example input: counts (rfResNum, ionCalGasSpec, fbDelay / fbTaps,
    # fbNumberofSections, runTBTBunchPrintNum) before their lists.
    fir, ion = cfg.fir, cfg.ion
    n_cav = int(r.n_cav)
    cav = lambda vals: " ".join(_fmt(v) for v in vals)  # noqa: E731
    lines = [
        f"ringCircRing = {_fmt(r.circ_ring)}",
        # three values: the third (nu_s) is a placeholder the reader replaces
        # by its own value from V_RF (ReadInputSettings.cpp:85-90, 1027)
        f"ringWorkQ = {_fmt(r.work_qx)} {_fmt(r.work_qy)} {_fmt(r.work_qz)}",
        "ringSynchRadDampTime = " + " ".join(_fmt(v) for v in r.synch_rad_damp_time[:3]),
        f"ringPipeAperatureX = {_fmt(r.pipe_aperture_x)}",
        f"ringPipeAperatureY = {_fmt(r.pipe_aperture_y)}",
        f"ringPipeAperatureR = {_fmt(max(r.pipe_aperture_x, r.pipe_aperture_y))}",
        f"ringElectronBeamEnergy = {_fmt(r.electron_energy)}",
        f"ringSdelta0 = {_fmt(r.sdelta0)}",
        f"ringNaturalEmit = {_fmt(r.natural_emit if qe else 0.0)}",
        f"ringCoupling = {_fmt(r.coupling)}",
        f"ringSkewQuadK = {_fmt(r.skew_quad_k)}",
        f"ringU0 = {_fmt(r.u0)}",
        f"ringCurrent = {_fmt(ring_current)}",
        f"ringChrom = {_fmt(r.chrom[0])} {_fmt(r.chrom[1])}",
        "ringAlphac = " + " ".join(_fmt(v) for v in r.alphac[:3]),
        "ringADTX = " + " ".join(_fmt(v) for v in r.adtx[:5]),
        "ringADTY = " + " ".join(_fmt(v) for v in r.adty[:5]),
        "ringTwiss = twiss.dat",
        f"ringSectNum = {K}",
        f"rfRingHarm = {int(r.harmonics)}", f"rfResNum = {n_cav}",
        "rfResHarm = " + " ".join(str(int(r.cav_harm[i])) for i in range(n_cav)),
        "rfResVol = " + cav(r.cav_vol[i] for i in range(n_cav)),
        "rfResPhase = " + cav(r.cav_phase[i] for i in range(n_cav)),
    ]
    if any(int(r.rf_mode[i]) == 1 for i in range(n_cav)):
        # cavities with beam loading: their resonator parameters as given
        ints = lambda f: " ".join(str(int(getattr(r, f)[i])) for i in range(n_cav))
        reals = lambda f: cav(getattr(r, f)[i] for i in range(n_cav))
        lines += [
            "rfMode = " + ints("rf_mode"), "rfResType = " + ints("res_type"),
            "rfResShuntImpRs = " + reals("res_rs"), "rfResQualityQ0 = " + reals("res_q0"),
            "rfResCouplingBeta = " + reals("res_coupling"), "rfResDetuneFre = " + reals("res_detune"),
            "rfResCold = " + ints("res_cold"), "rfResExciteIntability = " + ints("res_excite"),
            "rfResDirFB = " + ints("res_dir_fb"), "rfResDirFBGain = " + reals("res_dir_fb_gain"),
            "rfResDirFBPhaseShift = " + reals("res_dir_fb_phase"),
            "rfResDirFBDelay = " + reals("res_dir_fb_delay"),
            f"rfBunchBinNum = {int(r.rf_bunch_bins)}",
        ]
    else:
        # ideal cavities: the resonator parameters are not read by the
        # tracking; placeholders that keep the reference's set-up finite
        lines += [
            "rfMode = " + cav([0] * n_cav), "rfResType = " + cav([1] * n_cav),
            "rfResShuntImpRs = " + cav([0.0] * n_cav), "rfResQualityQ0 = " + cav([1.0] * n_cav),
            "rfResCouplingBeta = " + cav([0.0] * n_cav), "rfResDetuneFre = " + cav([0.0] * n_cav),
            "rfResCold = " + cav([0] * n_cav), "rfResExciteIntability = " + cav([0] * n_cav),
            "rfResDirFB = " + cav([0] * n_cav), "rfResDirFBGain = " + cav([0.0] * n_cav),
            "rfResDirFBPhaseShift = " + cav([0.0] * n_cav), "rfResDirFBDelay = " + cav([0.0] * n_cav),
            "rfBunchBinNum = 32",
        ]
    if cfg.flag_lr_wake:
        lines.append(f"lrwNTurnsWakeTrunction = {int(cfg.lr_turns) - 1}")
        if cfg.lr_bbr.n:
            _bbr_file(os.path.join(d, "lrw_bbr.dat"), cfg.lr_bbr)
            lines.append("lrwBBRInput = lrw_bbr.dat")
        if cfg.lr_rw.n:
            raise ValueError("resistive-wall sectors are not written")
    lines += [f"srwBunchBinNum = {int(cfg.sr_bins) if cfg.sr_bins else 100}",
              "srwWakePotenWriteTo = srw_poten"]
    if cfg.flag_sr_wake:
        if cfg.sr_bbr.n:
            _bbr_file(os.path.join(d, "srw_bbr.dat"), cfg.sr_bbr)
            lines.append("srwBBRInput = srw_bbr.dat")
        if cfg.sr_rw.n:
            raise ValueError("resistive-wall sectors are not written")
    lines += [
        f"fpTrainNumber = {len(npt)}", f"fpTotBunchNumber = {M}",
        "fpBunchNumberPerTrain = " + " ".join(map(str, npt)),
        "fpTrainGaps = " + " ".join(map(str, tgap)),
        "fpBunchGaps = " + " ".join(map(str, bgap)),
        "fpSetBunchChargeNum = 1", "fpSetBunchChargeIndex = 0", "fpSetBunchCharge = 1",
        f"bunchEmittance = {_fmt(wl.gen[0] * (1 + kappa))}",
        f"bunchKappa = {_fmt(kappa)}",
        f"bunchRmsBunchLength = {_fmt(wl.gen[2])}",
        f"bunchRmsEnergySpread = {_fmt(wl.gen[3])}",
        "bunchInitialStaticOffSet = 0 0 0 0 0 0",
        "bunchInitialDynamicOffSet = 0 0 0 0 0 0",
        "bunchDistributionType = 3",
        f"bunchMacroEleNumPerBunch = {nm[0]}",
    ]
    if any(n != nm[0] for n in nm):
        lines.append("bunchMacroEleNumPerBunchList = " + " ".join(map(str, nm)))
    if len(set(np.round(currents / currents.max(), 12))) > 1:
        raise ValueError("uneven bunch charges are not written (fpSetBunchCharge* keys)")
    P = ion.n_species if cfg.flag_beam_ion else 1
    lines += [
        f"ionCalGasSpec = {P}",
        "ionCalIonMassNumber = " + (" ".join(_fmt(ion.mass_number[p]) for p in range(P))
                                    if cfg.flag_beam_ion else "28"),
        "ionCalIonGasPercent = " + (" ".join(_fmt(ion.gas_percent[p]) for p in range(P))
                                    if cfg.flag_beam_ion else "1"),
        "ionCalCorsssectionEI = " + (" ".join(_fmt(ion.cross_section[p] / 1e-22) for p in range(P))
                                     if cfg.flag_beam_ion else "2.0"),
        f"ionCalIonLossBoundary = {_fmt(ion.loss_boundary if cfg.flag_beam_ion else 10.0)}",
        f"ionCalIonMaxNumber = {int(ion.max_ions) if cfg.flag_beam_ion else 100000}",
        f"ionCalMacroIonNumberGeneratedPerIP = {int(ion.macro_ions_per_ip) if cfg.flag_beam_ion else 1}",
        "ionCalIonInfoPrintInterval = 0", "ionCalIonDisWriteTo = ion_dis", "ionCalSCMethod = 1",
    ]
    if cfg.flag_fir:
        order = fir.delay + fir.taps
        nsec = max(1, int(fir.n_sections))
        lines += [
            f"fbMode = {int(fir.mode)}", f"fbNumberofSections = {nsec}",
            "fbStart = " + " ".join(str(int(fir.start[i])) for i in range(nsec)),
            "fbEnd = " + " ".join(str(min(int(fir.end[i]), 2 ** 31 - 1)) for i in range(nsec)),
            f"fbKickStrengthKx = {_fmt(fir.kick_strength[0])}",
            f"fbKickStrengthKy = {_fmt(fir.kick_strength[1])}",
            f"fbKickStrengthF = {_fmt(fir.kick_strength[2])}",
            f"fbGain = {_fmt(fir.gain)}", f"fbDelay = {int(fir.delay)}", f"fbTaps = {int(fir.taps)}",
            "fbKickerDispP = 0", "fbKickerDisp = 0",
            f"fbFIRBunchByBunchFeedbackPowerLimit = {_fmt(fir.power_limit)}",
            f"fbFIRBunchByBunchFeedbackKickerImped = {_fmt(fir.kicker_imped)}",
            # taps after the delay (ReadInputSettings.cpp:630-672)
            "fbFIRCoeffX = " + " ".join(_fmt(fir.coeff_x[i]) for i in range(fir.delay, order)),
            "fbFIRCoeffY = " + " ".join(_fmt(fir.coeff_y[i]) for i in range(fir.delay, order)),
            "fbFIRCoeffZ = " + " ".join(_fmt(fir.coeff_z[i]) for i in range(fir.delay, order)),
            "fbFIRCoeffXY = " + " ".join("0" for _ in range(fir.delay, order)),
        ]
    else:
        # the reader's post-checks walk the feedback sections (one is needed)
        lines += ["fbMode = 0", "fbNumberofSections = 1", "fbStart = 0", f"fbEnd = {max(1, n_turns)}",
                  "fbKickStrengthKx = 0", "fbKickStrengthKy = 0", "fbKickStrengthF = 0",
                  "fbGain = 0", "fbDelay = 0", "fbTaps = 1", "fbKickerDispP = 0", "fbKickerDisp = 0",
                  "fbFIRBunchByBunchFeedbackPowerLimit = 0",
                  "fbFIRBunchByBunchFeedbackKickerImped = 0",
                  "fbFIRCoeffX = 0", "fbFIRCoeffY = 0", "fbFIRCoeffZ = 0", "fbFIRCoeffXY = 0"]
    lines += [
        "driveModeOn = 0",
        "runCalSetting = 2", f"runNTurns = {n_turns}",
        "runGrowthRateFittingStart = 0", f"runGrowthRateFittingEnd = {max(1, n_turns)}",
        f"runBunchInfoPrintInterval = {print_interval}",
        "runTBTBunchPrintNum = 1", "runTBTBunchDisDataBunchIndex = 0",
        f"runSynRadDampingFlag = {int(cfg.flag_synrad)}",
        f"runBeamIonFlag = {int(cfg.flag_beam_ion)}",
        f"runFIRBunchByBunchFeedbackFlag = {int(cfg.flag_fir)}",
        f"runLongRangeWake = {int(cfg.flag_lr_wake)}",
        f"runShortRangeWake = {int(cfg.flag_sr_wake)}",
        f"runBBIFlag = {int(cfg.bbi.flag)}", "runRamping = 0",
        "runSpaceCharge = " + " ".join(str(int(v)) for v in (
            cfg.flag_sc, *(cfg.sc_mesh[i] if cfg.flag_sc else (32, 32, 33)[i] for i in range(3)))),
        f"runRandomSeed = {int(cfg.seed if seed is None else seed)}",
    ]
    if cfg.bbi.flag:
        # the broadband-impedance table as the file the reference reads
        # (5 header lines, BoardBandImp.cpp:53-58, MPBeam.cpp:762-767)
        td = int(cfg.bbi.time_domain)
        fname = "bbi_wake.dat" if td else "bbi_imped.dat"
        with open(os.path.join(d, fname), "w") as fh:
            fh.write("table\n" * 5)
            for row in np.asarray(wl.bbi_table):
                fh.write(" ".join(_fmt(v) for v in row) + "\n")
        lines += [
            f"bbiImpedSimTimeOrFreFlag = {td}",
            "bbiImpedSimLandTFlag = " + " ".join(str(int(cfg.bbi.sim[i])) for i in range(5)),
            "bbiBunchBinNumberZ = 100",
            ("bbiWakeInput = " if td else "bbiImpedInput = ") + fname,
        ]
    lines += list(extra)
    with open(os.path.join(d, "input.dat"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    rows = []
    for k in range(K):
        s = wl.sections[k]
        rows.append(" ".join(_fmt(v) for v in (
            s.s, s.beta_x, s.alpha_x, s.psi_x, s.eta_x, s.etap_x, s.aperture_x,
            s.beta_y, s.alpha_y, s.psi_y, s.eta_y, s.etap_y, s.aperture_y,
            s.length if s.length else r.circ_ring / K, s.pressure / PA_PER_NTORR, s.temperature)))
    with open(os.path.join(d, "twiss.dat"), "w") as fh:
        fh.write("twiss\n" * 5 + "\n".join(rows) + "\n")
    return os.path.join(d, "input.dat")


def load_case(path: str, name: str = "input", gen=None, lib=None) -> Workload:
    """A Workload from an input.dat through the library's own parser."""
    L = lib or _abi.load()
    cfg = _abi.Config()
    M = C.c_int()
    nm, hm, ne = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
    rc = L.cg_config_from_input(path.encode(), C.byref(cfg), C.byref(M), C.byref(nm), C.byref(hm),
                                C.byref(ne))
    if rc:
        raise _abi.CgError(rc, L.cg_parse_error().decode())
    m = M.value
    n_macro = [nm[j] for j in range(m)]
    harm = [hm[j] for j in range(m)]
    nev = [ne[j] for j in range(m)]
    K = cfg.n_sections
    secs = (_abi.Section * K)()
    C.memmove(secs, cfg.sections, C.sizeof(_abi.Section) * K)
    bbi = None
    if cfg.bbi.flag:
        cols = 6 if cfg.bbi.time_domain else 11
        bbi = np.ctypeslib.as_array(cfg.bbi.table, shape=(cfg.bbi.n_rows * cols,)).copy()
        sim = [cfg.bbi.sim[i] for i in range(5)]
    L.cg_config_free(C.byref(cfg), nm, hm, ne)  # the parser's arrays (sections copied above)
    cfg.sections = C.cast(secs, C.POINTER(_abi.Section))
    if gen is None:
        gen = (cfg.bunch_emit_x, cfg.bunch_emit_y, cfg.bunch_sigma_z, cfg.bunch_sigma_dp)
    wl = Workload(name, cfg, secs, n_macro, harm, nev, gen)
    if bbi is not None:
        wl.set_bbi(bbi, cfg.bbi.time_domain, sim)
    return wl
