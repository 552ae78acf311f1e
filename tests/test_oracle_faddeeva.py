"""The oracle's w(z) pinned against the reference (CPU, no GPU needed).

Golden vectors: tests/golden/faddeeva_golden.npz, generated from the
reference's own compiled Faddeeva::w (src/Faddeeva.cpp, via oracle/_ref) and
its w(z) known-answer test (src/Faddeeva.cpp:1922-2110, 57 points, each
checked at 1e-13 relative per component by the reference's self-test).
"""
import os

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def relerr(a, b):
    with np.errstate(all="ignore"):
        e = np.abs(b - a) / np.abs(a)
    e = np.where(a == b, 0.0, e)
    e = np.where(np.isnan(a) & np.isnan(b), 0.0, e)
    return e


def test_oracle_matches_kat_known_answers(golden):
    z, w = golden["kat_z"], golden["kat_w"]
    finite = np.isfinite(z.real) & np.isfinite(z.imag)
    got = oracle.faddeeva_w(z[finite])
    e = np.maximum(relerr(w[finite].real, got.real), relerr(w[finite].imag, got.imag))
    # the reference's own tolerance for this test is 1e-13 per component
    assert e.max() <= 1e-13, (e.max(), z[finite][e.argmax()])


def test_oracle_matches_reference_outputs(golden):
    z, ref = golden["grid_z"], golden["grid_ref"]
    got = oracle.faddeeva_w(z)
    e = np.abs(got - ref) / np.abs(ref)
    assert e.max() <= 5e-14, e.max()


def test_reference_kat_binary_passes_when_built():
    kat = os.path.join(ROOT, "oracle", "_ref", "faddeeva_kat")
    if not os.path.exists(kat):
        pytest.skip("reference sources not present: oracle/_ref not built")
    import subprocess
    out = subprocess.run([kat], capture_output=True, text=True, check=True).stdout
    assert out.count("SUCCESS") == 7 and "FAIL" not in out


def test_live_reference_agrees_with_golden(golden):
    ref = oracle.ref_faddeeva_w(golden["grid_z"][:500])
    if ref is None:
        pytest.skip("oracle/_ref not built")
    assert np.array_equal(ref.view(np.float64), golden["grid_ref"][:500].view(np.float64))


def test_oracle_fast_path_matches_binary128():
    """The long-double evaluation the oracle's field kicks use."""
    import ctypes as C
    lib = oracle.load()
    rng = np.random.default_rng(0)
    z = np.concatenate([rng.uniform(0, 15, 20000) + 1j * rng.uniform(0, 15, 20000),
                        10 ** rng.uniform(-10, 1.2, 5000) + 1j * 10 ** rng.uniform(-10, 1.2, 5000)])
    zr, zi = np.ascontiguousarray(z.real), np.ascontiguousarray(z.imag)
    wr, wi = np.empty_like(zr), np.empty_like(zr)
    P = C.POINTER(C.c_double)
    lib.or_w_fast_arr(zr.ctypes.data_as(P), zi.ctypes.data_as(P), wr.ctypes.data_as(P),
                      wi.ctypes.data_as(P), C.c_int64(len(zr)))
    ref = oracle.faddeeva_w(z)
    e = np.abs(wr + 1j * wi - ref) / np.abs(ref)
    assert e.max() <= 5e-16, e.max()
