"""Generates tests/golden/ref_tracking.npz from the reference itself.

For every case of tests/refcases.py: the case is written as the reference's
input files, the reference's own compiled sources (oracle/_ref/
libcetasim_ref.so, built by `make -C oracle ref REF=<CETASim tree>`) track
the seeded initial particles with quantum excitation off, and the fixture
keeps the digest of the initial particles, the final coordinates and
survival flags (all bunches, or the listed ones), and every bunch's moments.

Run from the repository root after building oracle/_ref:
    python tests/golden/make_ref_golden.py [case ...]
With case names, only those cases are run and the other cases' entries of
the existing fixture are kept.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import refcases  # noqa: E402
from oracle import ref  # noqa: E402


def main():
    if not ref.available():
        sys.exit("oracle/_ref/libcetasim_ref.so is not built")
    only = sys.argv[1:]
    out = {}
    if only and os.path.exists(refcases.GOLDEN):
        old = np.load(refcases.GOLDEN)
        out = {k: old[k] for k in old.files if k.split("/")[0] not in only}
    for case in only or refcases.CASES:
        with tempfile.TemporaryDirectory() as d:
            wl, parts, r = refcases.run_ref(case, d)
            out[f"{case}/digest"] = np.frombuffer(bytes.fromhex(refcases.parts_digest(parts)),
                                                  dtype=np.uint8)
            keep = refcases.KEEP_BUNCHES[case] or list(range(wl.n_bunches))
            out[f"{case}/bunches"] = np.array(keep, dtype=np.int32)
            for j in keep:
                c, s = r.download(j)
                out[f"{case}/coords/{j}"] = c
                out[f"{case}/surv/{j}"] = s
            out[f"{case}/moments"] = refcases.moments_array(r.moments())
            r.close()
        print(case, "done", flush=True)
    np.savez_compressed(refcases.GOLDEN, **out)
    print(refcases.GOLDEN, os.path.getsize(refcases.GOLDEN), "bytes")


if __name__ == "__main__":
    main()
