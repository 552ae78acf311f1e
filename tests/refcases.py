"""Parity cases run by the reference's own compiled sources (oracle/_ref):
the benchmark shapes at sizes the reference finishes in seconds, each
written as the reference's input files (cetasim_b200.input_dat) so that the
reference, the oracle restatement and the CUDA path read the same file.

Quantum excitation is off in every case (natural emittances 0 on all sides,
damping kept), so runs are deterministic; ion births come from the
counter-based stream shared by the harness and the device.
"""
import hashlib
import os

import numpy as np

from cetasim_b200 import configs, input_dat
from helpers import TRAPPED, particles

# name -> (config, n_scale, turns, bunch current, cfg overrides[, layout])
# layout: {"bunches": first bunches kept, "clouds": macro-ions pre-loaded per IP}
CASES = {
    # config 0's ring with the short-range wake (BBR, 100 bins)
    "plain_sr": ("plain_single", 0.005, 5, None, {}),
    # config 0's ring over 1000 turns (map, RF, drift, energy loss, damping)
    "plain_1000": ("plain_single", 0.01, 1000, None, {"flag_sr_wake": 0}),
    # config 0 itself over 1000 turns: the short-range wake on, its 100 bins
    "plain_sr_1000": ("plain_single", 0.005, 1000, None, {}),
    # config 1: 80 bunches x 25, 20 IPs, ions in the trapped regime
    "fast_ion": ("fast_ion", 0.00125, 4, TRAPPED, {}),
    # config 3's ragged 900-bunch train, 50 IPs, LR HOM wake and 9-tap FIR (no ions)
    "batched_lr_fir": ("batched_uneven", 0.001, 5, None, {"flag_beam_ion": 0}),
    # config 4's ring (every 4th bucket of h = 4000, 50 IPs, SR + HOM + FIR,
    # pre-loaded clouds): the first 150 bunches, 2000 macro-ions per IP, at a
    # current low enough that the ions' motion stays regular over the slice
    # (along the full 1000-bunch train rounding differences grow chaotically)
    "trapping_slice": ("large_trapping", 0.0002, 1, 0.005e-3, {"sr_bins": 10},
                       {"bunches": 150, "clouds": 2000}),
}

# bunches whose final coordinates the fixtures keep (all bunches' moments are kept)
KEEP_BUNCHES = {"plain_sr": None, "plain_1000": None, "plain_sr_1000": None, "fast_ion": None,
                "batched_lr_fir": list(range(0, 900, 30)), "trapping_slice": list(range(0, 150, 5))}


def build(case, d):
    """(workload read back from the written input, input path, initial particles)."""
    name, scale, turns, cur, over = CASES[case][:5]
    lay = CASES[case][5] if len(CASES[case]) > 5 else {}
    wl = configs.make(name, n_scale=scale, bunch_current=cur)
    for k, v in over.items():
        setattr(wl.cfg, k, v)
    if "bunches" in lay:
        m = lay["bunches"]
        wl.n_macro, wl.harm, wl.ne = wl.n_macro[:m].copy(), wl.harm[:m].copy(), wl.ne[:m].copy()
    path = input_dat.write_case(d, wl, n_turns=turns, qe=False)
    wl2 = input_dat.load_case(path, name=case)
    for i in range(3):
        wl2.cfg.ring.emit_nat[i] = 0.0
    return wl2, path, particles(wl2, seed=5, spread=2.0)


def clouds(case, wl):
    """The pre-loaded clouds of a case ((x, y, vx, vy) per IP) or None."""
    lay = CASES[case][5] if len(CASES[case]) > 5 else {}
    return configs.preload_clouds(wl, lay["clouds"]) if "clouds" in lay else None


def start(case, beam, wl, parts):
    """Uploads a case's particles and pre-loaded clouds into any of the three
    beams (reference, oracle, CUDA path)."""
    for j, c in enumerate(parts):
        beam.upload(j, c)
    cl = clouds(case, wl)
    if cl is not None:
        for k, (x, y, vx, vy) in enumerate(cl):
            beam.upload_ions(k, 0, x, y, vx, vy)


def parts_digest(parts):
    h = hashlib.sha256()
    for c in parts:
        h.update(np.ascontiguousarray(c, dtype=np.float64).tobytes())
    return h.hexdigest()


def run_ref(case, d):
    """The reference's own run of a case: (workload, initial particles, beam)."""
    from oracle import ref
    wl, path, parts = build(case, d)
    r = ref.RefBeam(path, seed=wl.cfg.seed)
    r.set_emit_nat([0.0, 0.0, 0.0])
    start(case, r, wl, parts)
    r.Run(0, CASES[case][2])
    return wl, parts, r


def moments_array(ms):
    """(M, 22) array of the compared moment fields."""
    rows = []
    for m in ms:
        rows.append([m.n_alive, *list(m.mean), *list(m.emit), *list(m.eff_emit), m.rms_x, m.rms_y,
                     m.eff_rms_x, m.eff_rms_y, m.bunch_length, m.energy_spread, m.z_min, m.z_max,
                     m.transmission])
    return np.array(rows, dtype=np.float64)


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_tracking.npz")


def golden():
    return np.load(GOLDEN, allow_pickle=False)


def coord_rel_err(got, want, alive):
    """max |got - want| / rms(want) per coordinate over alive particles."""
    e = np.zeros(6)
    for d in range(6):
        sc = np.sqrt(np.mean(want[d][alive] ** 2)) + 1e-300
        e[d] = np.max(np.abs(got[d][alive] - want[d][alive])) / sc
    return e
