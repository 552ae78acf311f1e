"""Writes tests/golden/ref_space_charge.npz: the reference's own runs
(oracle/_ref, its src/*.cpp) of the space-charge cases of tests/sccases.py.

Per case: px and py of the kept bunches (the only coordinates it changes)
after one space-charge step at section 0 (MPBeamRMSCal(0), then BeamTransferDueToSpaceChargePIC /
...Analytical(0)) from the initial particles and after the case's turns of
MPBeam::Run's loop body, and a digest of the initial particles.

Run from the repository root with the reference build present:
    python tests/golden/make_sc_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import sccases  # noqa: E402
from oracle import ref  # noqa: E402
from refcases import parts_digest  # noqa: E402


def main():
    out = {}
    for case, (_, _, _, turns, _, _) in sccases.CASES.items():
        with tempfile.TemporaryDirectory() as d:
            wl, path, parts = sccases.build(case, d)
            out[f"{case}/digest"] = np.frombuffer(parts_digest(parts).encode(), dtype=np.uint8)
            r = ref.RefBeam(path, seed=wl.cfg.seed)
            r.set_emit_nat([0.0, 0.0, 0.0])
            sccases.start(r, parts)
            r.MPBeamRMSCal(0)
            r.BeamTransferDueToSpaceCharge(0)
            for j in sccases.KEEP[case]:
                c = r.download(j)[0]
                # the step changes px and py only
                assert np.array_equal(c[[0, 2, 4, 5]], parts[j][[0, 2, 4, 5]])
                out[f"{case}/kick{j}"] = c[[1, 3]]
            r.close()
        with tempfile.TemporaryDirectory() as d:
            wl, path, parts = sccases.build(case, d)
            r = ref.RefBeam(path, seed=wl.cfg.seed)
            r.set_emit_nat([0.0, 0.0, 0.0])
            sccases.start(r, parts)
            r.Run(0, turns)
            for j in sccases.KEEP[case]:
                c, s = r.download(j)
                out[f"{case}/coords{j}"] = c
                out[f"{case}/surv{j}"] = s
            r.close()
        print(case, "done", flush=True)
    np.savez_compressed(sccases.GOLDEN, **out)
    print(sccases.GOLDEN, os.path.getsize(sccases.GOLDEN), "bytes")


if __name__ == "__main__":
    main()
