"""Writes tests/golden/ref_beam_loading.npz: the reference's own runs
(oracle/_ref, its src/*.cpp) of the beam-loading cases of tests/blcases.py.

Per case: the resonators' state after the reference's set-up
(MPBeam::InitialcavityResonator) and after the run, every bunch's
BunchRFModeInfo after the last RF step, the final coordinates and survival
flags of the kept bunches, and a digest of the initial particles (the tests
regenerate them from the same seed and check the digest).

Run from the repository root with the reference build present:
    python tests/golden/make_bl_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import blcases  # noqa: E402
from oracle import ref  # noqa: E402
from refcases import parts_digest  # noqa: E402


def main():
    out = {}
    for case, (_, _, turns, _) in blcases.CASES.items():
        with tempfile.TemporaryDirectory() as d:
            wl, path, parts = blcases.build(case, d)
            r = ref.RefBeam(path, seed=wl.cfg.seed)
            r.set_emit_nat([0.0, 0.0, 0.0])
            blcases.start(r, parts)
            cav = blcases.loaded_cavities(wl)
            init = np.array([[v for z in r.resonator(c)[:3] for v in (z.real, z.imag)] for c in cav])
            r.Run(0, turns)
            fin = np.array([[v for z in r.resonator(c)[:3] for v in (z.real, z.imag)] for c in cav])
            info = np.array([[[v for z in r.rf_info(j, c) for v in (z.real, z.imag)] for c in cav]
                             for j in range(wl.n_bunches)])
            out[f"{case}/digest"] = np.frombuffer(parts_digest(parts).encode(), dtype=np.uint8)
            out[f"{case}/res_init"] = init
            out[f"{case}/res_final"] = fin
            out[f"{case}/info"] = info
            for j in blcases.KEEP[case]:
                c, s = r.download(j)
                out[f"{case}/coords{j}"] = c
                out[f"{case}/surv{j}"] = s
            r.close()
            print(case, "done", flush=True)
    np.savez_compressed(blcases.GOLDEN, **out)
    print(blcases.GOLDEN, os.path.getsize(blcases.GOLDEN), "bytes")


if __name__ == "__main__":
    main()
