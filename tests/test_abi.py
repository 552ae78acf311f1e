"""C-ABI surface of libcetagpu.so on CPU: the library loads, exports every
symbol include/cetasim_gpu.h declares, its structs have the C layout, the
host-side derivations match the oracle bit for bit, and calls that need a
device fail with a status (no CPU fallback)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
from cetasim_b200 import _abi, configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "cetasim_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cg_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    exported = {n for n, _, _ in _abi.EXPORTS}
    assert set(names) <= exported | {"cg_config_from_input", "cg_config_free"}


def test_abi_version(lib):
    assert lib.cg_abi_version() == 3


def test_struct_layouts_match_c(built):
    sizes = (C.c_int64 * 7)()
    oracle.load().or_struct_sizes(sizes)
    py = [C.sizeof(_abi.Config), C.sizeof(_abi.Ring), C.sizeof(_abi.Section),
          C.sizeof(_abi.BunchMoments), C.sizeof(_abi.IonParams), C.sizeof(_abi.Bbr),
          C.sizeof(_abi.FirParams)]
    assert list(sizes) == py


@pytest.mark.parametrize("name", ["plain_single", "fast_ion", "batched_uneven", "large_trapping"])
def test_derivations_match_oracle_bitwise(lib, name):
    a = configs.make(name, n_scale=0.001)
    b = configs.make(name, n_scale=0.001, derive=oracle.config_derive,
                     lattice_init=oracle.lattice_init)
    ra, rb = a.cfg.ring, b.cfg.ring
    for f, _ in _abi.Ring._fields_:
        va, vb = getattr(ra, f), getattr(rb, f)
        if hasattr(va, "__len__"):
            assert list(va) == list(vb), f
        else:
            assert va == vb, f
    for k in range(a.cfg.n_sections):
        sa, sb = a.sections[k], b.sections[k]
        for f, _ in _abi.Section._fields_:
            va, vb = getattr(sa, f), getattr(sb, f)
            if hasattr(va, "__len__"):
                assert list(va) == list(vb), (k, f)
            else:
                assert va == vb, (k, f)


def test_ring_derivation_values(lib):
    wl = configs.make("fast_ion", n_scale=0.001)
    r = wl.cfg.ring
    # nu_s = 0.0049 through the reference's formula (ReadInputSettings.cpp:1027)
    assert abs(r.work_qz - 0.0049) < 2e-6
    assert abs(r.t0 - 2304.0 / 299792458.0 / r.r_beta) < 1e-20
    assert r.emit_nat[0] == pytest.approx(20e-12)
    assert r.emit_nat[1] == pytest.approx(4e-12)
    # single cavity: phase pi - asin(U0/V) - pi/2 (CavityResonator.cpp:121-124)
    phi = np.pi - np.arcsin(r.u0 / r.cav_vol[0]) - np.pi / 2
    assert r.cav_vreq_re[0] == pytest.approx(r.cav_vol[0] * np.cos(phi))


def test_lattice_maps_are_symplectic_inverses(lib):
    wl = configs.make("fast_ion", n_scale=0.001)
    for k in range(wl.cfg.n_sections):
        s = wl.sections[k]
        b1h1 = np.array(s.map_b1h1).reshape(6, 6)
        h1b1 = np.array(s.map_h1b1).reshape(6, 6)
        assert np.allclose(h1b1 @ b1h1, np.eye(6), atol=1e-13)
        # phase advances add up to 2 pi nu
    tot = sum(wl.sections[k].phase_adv_x for k in range(wl.cfg.n_sections))
    assert tot == pytest.approx(2 * np.pi * wl.cfg.ring.work_qx)


def test_create_reports_missing_device_or_succeeds(lib):
    wl = configs.make("plain_single", n_scale=0.001)
    h = C.c_void_p()
    rc = lib.cg_create(C.byref(wl.cfg), 0, C.byref(h))
    if rc == 0:
        lib.cg_destroy(h)
    else:
        assert rc == 3  # CG_ERR_CUDA: no device, and no CPU path
        assert b"no CUDA device" in lib.cg_last_error(None)


def test_invalid_configs_rejected_without_device(lib):
    wl = configs.make("plain_single", n_scale=0.001)
    wl.cfg.ring.skew_quad_k = 1e-3
    h = C.c_void_p()
    assert lib.cg_create(C.byref(wl.cfg), 0, C.byref(h)) == 8
    wl.cfg.ring.skew_quad_k = 0.0
    wl.cfg.sr_bins = 0
    assert lib.cg_create(C.byref(wl.cfg), 0, C.byref(h)) == 1
