"""Space-charge cases (runSpaceCharge 1, 2, 3), written as the reference's
input files so that the reference build, the oracle restatement and the CUDA
path read the same settings (MPBeam::BeamTransferDueToSpaceChargePIC /
...Analytical, MPBeam.cpp:2565-2583; MPBunch.cpp:660-931; PIC2D.cpp).

Quantum excitation is off, ions, wakes and feedback off, so a run is
deterministic; the space-charge kick is the only collective effect.
"""
import os

import numpy as np

from cetasim_b200 import configs, input_dat
from helpers import particles

# name -> (config, n_scale, bunches kept, turns, flag, mesh nx ny nz)
CASES = {
    # one bunch, 2.5-D PIC on a 32 x 32 mesh, 11 slices
    "pic_single": ("plain_single", 0.008, 1, 2, 2, (32, 32, 11)),
    # 8 bunches of the fast-ion ring (20 sections), PIC on 16 x 24, 9 slices
    "pic_train": ("fast_ion", 0.01, 8, 2, 2, (16, 24, 9)),
    # one bunch, Bassetti-Erskine slices
    "be_single": ("plain_single", 0.008, 1, 2, 1, (32, 32, 11)),
    # 8 bunches, the linear (uniform-beam) field
    "linear_train": ("fast_ion", 0.01, 8, 2, 3, (32, 32, 7)),
}


def build(case, d):
    """(workload read back from the written input, input path, initial particles)."""
    name, scale, nb, turns, flag, mesh = CASES[case]
    wl = configs.make(name, n_scale=scale)
    wl.n_macro, wl.harm, wl.ne = wl.n_macro[:nb].copy(), wl.harm[:nb].copy(), wl.ne[:nb].copy()
    c = wl.cfg
    c.flag_beam_ion = 0
    c.flag_lr_wake = 0
    c.flag_fir = 0
    c.flag_sr_wake = 0
    c.flag_sc = flag
    for i in range(3):
        c.sc_mesh[i] = mesh[i]
    path = input_dat.write_case(d, wl, n_turns=turns, qe=False)
    wl2 = input_dat.load_case(path, name=case)
    for i in range(3):
        wl2.cfg.ring.emit_nat[i] = 0.0
    return wl2, path, particles(wl2, seed=13, spread=1.0)


def start(beam, parts):
    for j, p in enumerate(parts):
        beam.upload(j, p)


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_space_charge.npz")

KEEP = {"pic_single": [0], "pic_train": [0, 3, 7], "be_single": [0], "linear_train": [0, 3, 7]}


def golden():
    return np.load(GOLDEN, allow_pickle=False)


def kick_err(got, want, start):
    """Largest difference per coordinate over the largest change."""
    e = np.zeros(6)
    for q in range(6):
        k = np.max(np.abs(want[q] - start[q]))
        d = np.max(np.abs(got[q] - want[q]))
        e[q] = d / k if k > 0 else d
    return e


def coord_rel_err(got, want):
    e = np.zeros(6)
    for q in range(6):
        sc = np.sqrt(np.mean(want[q] ** 2)) + 1e-300
        e[q] = np.max(np.abs(got[q] - want[q])) / sc
    return e
