"""Broadband-impedance cases (runBBIFlag 1), written as the reference's input
files so that the reference build, the oracle restatement and the CUDA path
read the same settings and tables (MPBeam::BBImpBeamInteraction,
MPBeam.cpp:1321-1346; BoardBandImp::ReadInImp, BoardBandImp.cpp:42-115;
MPBeam::GetQuasiWakePoten, MPBeam.cpp:748-801).

The tables are synthetic: broadband resonator impedances sampled from 0 to
f_max (frequency domain) and a smooth pseudo-Green wake on a z grid through
z = 0 (time domain).  Quantum excitation is off, ions and feedback off, so a
run is deterministic.
"""
import os

import numpy as np

from cetasim_b200 import configs, input_dat
from helpers import particles


def resonator_table(n, fmax, rs=(2e4, 4e5, 4e5, 1e5, 1e5), fr=(40e9, 30e9, 30e9, 30e9, 30e9), q=1.0):
    """n rows f_k = k f_max / (n - 1) of the 11 impedance columns (f, the
    real parts of Z, Dx, Dy, Qx, Qy, then their imaginary parts): a broadband
    resonator per plane, transverse ones with the (fr / f) factor."""
    f = np.arange(n) * (fmax / (n - 1))
    t = np.zeros((n, 11))
    t[:, 0] = f
    with np.errstate(divide="ignore", invalid="ignore"):
        for p in range(5):
            z = rs[p] / (1 + 1j * q * (fr[p] / f - f / fr[p]))
            if p:
                z = z * fr[p] / f
            z[0] = 0
            t[:, 1 + p] = z.real
            t[:, 6 + p] = z.imag
    return t


def wake_table(nw, dzw, cen, amp=(3e13, 2e15, 2e15, 5e14, 5e14), sigma=1.5e-3, lam=6e-3, decay=20e-3):
    """nw rows z_i = (i - cen) dzw of the 6 wake columns (z, Wz, WDx, WDy,
    WQx, WQy): a Gaussian-smoothed damped oscillation."""
    z = (np.arange(nw) - cen) * dzw
    t = np.zeros((nw, 6))
    t[:, 0] = z
    env = np.exp(-0.5 * (z / sigma) ** 2) + np.where(z > 0, np.exp(-z / decay), 0.0)
    for p in range(5):
        t[:, 1 + p] = amp[p] * env * np.cos(2 * np.pi * z / lam + 0.3 * p)
    t[cen, 0] = 0.0
    return t


# name -> (config, n_scale, turns, time domain, table, planes, long-range wake)
CASES = {
    # one bunch, frequency domain, all five planes
    "fd_single": ("plain_single", 0.005, 3, 0, lambda: resonator_table(640, 300e9), (1, 1, 1, 1, 1), False),
    # one bunch, frequency domain, longitudinal and quadrupolar x only
    "fd_single_zq": ("plain_single", 0.005, 3, 0, lambda: resonator_table(640, 300e9), (1, 0, 0, 1, 0), False),
    # one bunch, time domain, all five planes
    "td_single": ("plain_single", 0.005, 3, 1, lambda: wake_table(400, 0.5e-3, 40), (1, 1, 1, 1, 1), False),
    # the 80-bunch train, frequency domain, with the long-range wake after it
    "fd_train_lr": ("fast_ion", 0.002, 2, 0, lambda: resonator_table(256, 100e9), (1, 1, 1, 1, 1), True),
    # the 80-bunch train, time domain
    "td_train": ("fast_ion", 0.002, 2, 1, lambda: wake_table(300, 0.4e-3, 60), (1, 1, 1, 0, 1), False),
}


def build(case, d):
    """(workload read back from the written input, input path, initial particles)."""
    name, scale, turns, td, table, sim, lr = CASES[case]
    wl = configs.make(name, n_scale=scale)
    c = wl.cfg
    c.flag_beam_ion = 0
    c.flag_lr_wake = 0
    c.flag_fir = 0
    c.flag_sr_wake = 0
    if lr:
        c.flag_lr_wake = 1
        c.lr_turns = 4
        c.lr_bbr = configs.bbr([(0.0, 1.0, 1.2e9, 1e6, 1e4, 1.2e9, 1e6, 1e4, 1.2e9)])
    wl.set_bbi(table(), td, sim)
    path = input_dat.write_case(d, wl, n_turns=turns, qe=False)
    wl2 = input_dat.load_case(path, name=case)
    for i in range(3):
        wl2.cfg.ring.emit_nat[i] = 0.0
    return wl2, path, particles(wl2, seed=11, spread=1.0)


def start(beam, parts):
    for j, p in enumerate(parts):
        beam.upload(j, p)


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_bbi.npz")

# bunches whose coordinates the fixtures keep
KEEP = {"fd_single": [0], "fd_single_zq": [0], "td_single": [0],
        "fd_train_lr": list(range(0, 80, 8)), "td_train": list(range(0, 80, 8))}


def golden():
    return np.load(GOLDEN, allow_pickle=False)


def coord_rel_err(got, want):
    e = np.zeros(6)
    for q in range(6):
        sc = np.sqrt(np.mean(want[q] ** 2)) + 1e-300
        e[q] = np.max(np.abs(got[q] - want[q])) / sc
    return e
