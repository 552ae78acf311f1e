"""Cases of cavities with beam loading (rfMode 1), written as the reference's
input files so that the reference build, the oracle restatement and the CUDA
path read the same settings (MPBeam::BeamMomtumUpdateDueToRFTest,
MPBeam.cpp:2621-2704; MPBeam::InitialcavityResonator, MPBeam.cpp:236-465).

Quantum excitation is off (natural emittances 0, damping kept), ions, wakes
and feedback off, so a run is deterministic and the RF step is what moves
the bunches apart.
"""
import os

import numpy as np

from cetasim_b200 import configs, input_dat
from helpers import particles

# name -> (config, n_scale, turns, cavity settings)
# cavity settings: per cavity index, the beam-loading fields of cg_ring
MAIN = {"rf_mode": 1, "res_type": 1, "res_rs": 5e6, "res_q0": 2e4, "res_coupling": 2.0,
        "res_detune": -20e3}
CASES = {
    # one bunch, the main cavity loaded, rigid-bunch voltage
    "single_rigid": ("plain_single", 0.01, 4, {0: dict(MAIN, res_excite=0)}),
    # one bunch, bin-by-bin induced voltage (the instability setting)
    "single_binned": ("plain_single", 0.01, 4, {0: dict(MAIN, res_excite=1)}),
    # the 80-bunch train, rigid bunches
    "train_rigid": ("fast_ion", 0.002, 3, {0: dict(MAIN, res_excite=0)}),
    # the 80-bunch train, bin by bin, with the direct cavity feedback
    "train_binned_fb": ("fast_ion", 0.002, 3,
                        {0: dict(MAIN, res_excite=1, res_dir_fb=1, res_dir_fb_gain=0.3,
                                 res_dir_fb_phase=0.1, res_dir_fb_delay=1e-9)}),
    # the ragged 900-bunch train: an ideal main cavity (rfMode 0) and a passive
    # third-harmonic cavity with beam loading, bin by bin, started cold
    "ragged_harmonic": ("batched_uneven", 0.0005, 2,
                        {1: {"rf_mode": 1, "res_type": 0, "res_rs": 2e6, "res_q0": 1e4,
                             "res_coupling": 0.0, "res_detune": 150e3, "res_excite": 1,
                             "res_cold": 1}}),
}
BINS = 40


def build(case, d):
    """(workload read back from the written input, input path, initial particles)."""
    name, scale, turns, cavs = CASES[case]
    wl = configs.make(name, n_scale=scale)
    c = wl.cfg
    c.flag_beam_ion = 0
    c.flag_lr_wake = 0
    c.flag_fir = 0
    c.flag_sr_wake = 0
    r = c.ring
    if max(cavs) >= r.n_cav:
        # a second cavity: the third harmonic, no voltage asked of it; the
        # main cavity keeps the synchronous phase the reference sets for a
        # single cavity (CavityResonator.cpp:117-121)
        r.n_cav = max(cavs) + 1
        r.cav_phase[0] = np.pi - np.arcsin(r.u0 / r.cav_vol[0]) - np.pi / 2.0
        r.cav_harm[1] = 3
        r.cav_vol[1] = 0.0
        r.cav_phase[1] = 0.0
    for i, fields in cavs.items():
        for k, v in fields.items():
            getattr(r, k)[i] = v
    r.rf_bunch_bins = BINS
    path = input_dat.write_case(d, wl, n_turns=turns, qe=False)
    wl2 = input_dat.load_case(path, name=case)
    for i in range(3):
        wl2.cfg.ring.emit_nat[i] = 0.0
    return wl2, path, particles(wl2, seed=5, spread=1.0)


def loaded_cavities(wl):
    return [i for i in range(wl.cfg.ring.n_cav) if wl.cfg.ring.rf_mode[i] == 1]


def start(beam, parts):
    for j, c in enumerate(parts):
        beam.upload(j, c)


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_beam_loading.npz")

# bunches whose final coordinates the fixtures keep
KEEP = {"single_rigid": [0], "single_binned": [0], "train_rigid": list(range(0, 80, 8)),
        "train_binned_fb": list(range(0, 80, 8)), "ragged_harmonic": list(range(0, 900, 90))}


def golden():
    return np.load(GOLDEN, allow_pickle=False)


def coord_rel_err(got, want, alive):
    e = np.zeros(6)
    for q in range(6):
        sc = np.sqrt(np.mean(want[q][alive] ** 2)) + 1e-300
        e[q] = np.max(np.abs(got[q][alive] - want[q][alive])) / sc
    return e
