"""Writes tests/golden/ref_bbi.npz: the reference's own runs (oracle/_ref, its
src/*.cpp) of the broadband-impedance cases of tests/bbicases.py.

Per case: the coordinates of the kept bunches after one
MPBeam::BBImpBeamInteraction from the initial particles and after the
case's turns of MPBeam::Run's loop body; for the frequency-domain cases the
five wakePotenFromBBI arrays of bunch 0 after that single kick, over the
bins from 30 below to 30 above those that hold its particles; and a digest of
the initial particles (the tests regenerate them from the same seed and check
the digest).

Run from the repository root with the reference build present:
    python tests/golden/make_bbi_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import bbicases  # noqa: E402
from oracle import ref  # noqa: E402
from refcases import parts_digest  # noqa: E402


def window(wl, parts):
    """First and last profile bin (frequency domain) of bunch 0's particles, +-30."""
    r = wl.cfg.ring
    freq_max = wl.bbi_table[-1, 0]
    n = wl.bbi_table.shape[0]
    dz = 1.0 / (2 * freq_max) * 299792458.0 * r.r_beta
    zmin = -dz * (n - 1)
    idx = ((parts[0][4] - zmin + dz / 2) / dz).astype(int)
    return max(int(idx.min()) - 30, 0), min(int(idx.max()) + 30, 2 * n - 2)


def main():
    out = {}
    for case, (_, _, turns, td, _, _, _) in bbicases.CASES.items():
        with tempfile.TemporaryDirectory() as d:
            wl, path, parts = bbicases.build(case, d)
            out[f"{case}/digest"] = np.frombuffer(parts_digest(parts).encode(), dtype=np.uint8)
            r = ref.RefBeam(path, seed=wl.cfg.seed)
            r.set_emit_nat([0.0, 0.0, 0.0])
            bbicases.start(r, parts)
            r.BBImpBeamInteraction()
            for j in bbicases.KEEP[case]:
                out[f"{case}/kick{j}"] = r.download(j)[0]
            if not td:
                a, b = window(wl, parts)
                out[f"{case}/pot_lo"] = np.array([a])
                out[f"{case}/pot"] = r.bbi_profile(0)[1:, a:b + 1]
            r.close()
        with tempfile.TemporaryDirectory() as d:
            wl, path, parts = bbicases.build(case, d)
            r = ref.RefBeam(path, seed=wl.cfg.seed)
            r.set_emit_nat([0.0, 0.0, 0.0])
            bbicases.start(r, parts)
            r.Run(0, turns)
            for j in bbicases.KEEP[case]:
                c, s = r.download(j)
                out[f"{case}/coords{j}"] = c
                out[f"{case}/surv{j}"] = s
            r.close()
        print(case, "done", flush=True)
    np.savez_compressed(bbicases.GOLDEN, **out)
    print(bbicases.GOLDEN, os.path.getsize(bbicases.GOLDEN), "bytes")


if __name__ == "__main__":
    main()
