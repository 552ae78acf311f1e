"""Generates tests/golden/faddeeva_golden.npz from the reference itself.

Inputs: the w(z) known-answer test of the reference's vendored Faddeeva
package (src/Faddeeva.cpp:1922-2110: 57 points and their known values), read
from the reference source, plus seeded dense grids.  Outputs: the reference's
own Faddeeva::w at every point, computed by oracle/_ref/libfaddeeva_ref.so,
which oracle/Makefile compiles from the reference's src/Faddeeva.cpp.

Run with the CETASim source tree named by CETASIM_REFERENCE:
    make -C oracle ref REF=$CETASIM_REFERENCE && python tests/golden/make_faddeeva_golden.py
"""
import ctypes
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("CETASIM_REFERENCE")
if not REF:
    sys.exit("set CETASIM_REFERENCE to the CETASim source tree (src/, include/)")


def kat_points():
    src = open(os.path.join(REF, "src", "Faddeeva.cpp")).read()
    special = {"Inf": np.inf, "-Inf": -np.inf, "NaN": np.nan}

    def val(s):
        s = s.strip()
        return special[s] if s in special else float(s)

    def block(marker):
        b = src[src.index(marker):]
        b = b[: b.index("};")]
        b = re.sub(r"/\*.*?\*/", "", b, flags=re.S)
        return [(val(a), val(c)) for a, c in re.findall(r"C\(([^,]+),([^)]+)\)", b)]

    z = block("cmplx z[NTST] = {")
    w = block("cmplx w[NTST] = {")
    assert len(z) == len(w) == 57, (len(z), len(w))
    return cplx(z), cplx(w)


def cplx(pairs):
    # set real and imaginary parts separately: a + 1j * b would turn
    # 0 + 1j * inf into nan + inf j
    out = np.empty(len(pairs), dtype=np.complex128)
    out.real = [a for a, _ in pairs]
    out.imag = [b for _, b in pairs]
    return out


def ref_w(z):
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libfaddeeva_ref.so"))
    P = ctypes.POINTER(ctypes.c_double)
    zr = np.ascontiguousarray(z.real)
    zi = np.ascontiguousarray(z.imag)
    wr, wi = np.empty_like(zr), np.empty_like(zr)
    lib.ref_faddeeva_w(zr.ctypes.data_as(P), zi.ctypes.data_as(P), wr.ctypes.data_as(P),
                       wi.ctypes.data_as(P), ctypes.c_int64(len(zr)))
    return cplx(list(zip(wr, wi)))


def main():
    kz, kw = kat_points()
    rng = np.random.default_rng(20240517)
    # first quadrant as the field kicks use it, plus near-axis and general points
    q1 = rng.uniform(0, 12, 4000) + 1j * rng.uniform(0, 12, 4000)
    axis = 10 ** rng.uniform(-10, 1.1, 2000) + 1j * 10 ** rng.uniform(-10, 1.1, 2000)
    plane = rng.uniform(-30, 30, 2000) + 1j * rng.uniform(-6, 30, 2000)
    grid = np.concatenate([q1, axis, plane])
    np.savez_compressed(os.path.join(HERE, "faddeeva_golden.npz"), kat_z=kz, kat_w=kw,
                        kat_ref=ref_w(kz), grid_z=grid, grid_ref=ref_w(grid))
    print("wrote", os.path.join(HERE, "faddeeva_golden.npz"))


if __name__ == "__main__":
    sys.exit(main())
