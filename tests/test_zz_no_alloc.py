"""cg_bunch_moments_noalloc (moments of one bunch in caller-owned device
buffers, partials in a fixed static device array) against the handle-based
moments (cg_beam_rms + cg_get_moments) on the same particles.

Two calls are enqueued back to back on one stream, on bunches of different
sizes, so the second call depends on the first leaving the completion counter
at zero.  The file name keeps it last in a session, so it also runs after
every other test has used the library.  Tolerance: 1e-14 relative per field
(both paths run the same tiling and merge order)."""
import ctypes as C

import numpy as np
import pytest

from cetasim_b200 import _abi
from cetasim_b200.beam import MPBeam
from helpers import particles, small

FIELDS = ["mean", "emit", "eff_emit", "rms_x", "rms_y", "eff_rms_x", "eff_rms_y",
          "bunch_length", "energy_spread", "z_min", "z_max"]
MAX_N = 1048576  # CG_NOALLOC_MAX_PARTICLES


def _handle_moments(wl, parts, surv, j):
    g = MPBeam(wl)
    for b, c in enumerate(parts):
        g.upload(b, c, surv[b])
    g.MPBeamRMSCal(0)
    m = g.moments()[j]
    g.close()
    return m


def _device_bunch(torch, coords, surv, pad):
    n = coords.shape[1]
    d = torch.full((6, n + pad), float("nan"), dtype=torch.float64, device="cuda")
    d[:, :n] = torch.from_numpy(coords).cuda()
    s = torch.from_numpy(surv).cuda()
    return d, s


def _close(a, b, rtol):
    bad = []
    assert a.n_alive == b.n_alive
    for f in FIELDS:
        va, vb = np.array(getattr(a, f), ndmin=1), np.array(getattr(b, f), ndmin=1)
        scale = np.maximum(np.abs(vb), 1e-300)
        if f == "mean":
            scale = np.maximum(scale, [b.rms_x, b.rms_x / 10, b.rms_y, b.rms_y / 10,
                                       b.bunch_length, b.energy_spread])
        e = np.max(np.abs(va - vb) / scale)
        if not e <= rtol:
            bad.append((f, e))
    return bad


def test_rejects_sizes_beyond_the_static_scratch(lib):
    buf = (C.c_double * 8)()
    flags = (C.c_uint8 * 8)()
    out = _abi.BunchMoments()
    rc = lib.cg_bunch_moments_noalloc(C.addressof(buf), MAX_N + 1, C.addressof(flags), MAX_N + 1,
                                      10.0, 10.0, C.addressof(out), None)
    assert rc == 1  # CG_ERR_INVALID, before any device access
    msg = lib.cg_last_error(None).decode()
    assert "exceeds the static scratch" in msg and str(MAX_N) in msg
    rc = lib.cg_bunch_moments_noalloc(C.addressof(buf), 8, C.addressof(flags), 0,
                                      10.0, 10.0, C.addressof(out), None)
    assert rc == 1


@pytest.mark.gpu
def test_two_calls_match_handle_moments(lib):
    import torch

    # bunch A: one bunch of 1e5 (391 tiles, ragged last tile), 5% lost
    wa = small("plain_single", 1.0)
    pa = particles(wa, seed=21)
    rng = np.random.default_rng(4)
    sa = [(rng.random(pa[0].shape[1]) < 0.05).astype(np.uint8)]
    ref_a = _handle_moments(wa, pa, sa, 0)
    # bunch B: bunch 17 of a train of 80 x 1000 (4 tiles), 1 in 7 lost
    wb = small("fast_ion", 0.05)
    pb = particles(wb, seed=22)
    sb = [np.zeros(c.shape[1], dtype=np.uint8) for c in pb]
    sb[17][::7] = 2
    ref_b = _handle_moments(wb, pb, sb, 17)

    ca, fa = _device_bunch(torch, pa[0], sa[0], pad=37)
    cb, fb = _device_bunch(torch, pb[17], sb[17], pad=0)
    nbytes = C.sizeof(_abi.BunchMoments)
    out = torch.zeros((2, nbytes), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    secs = (wa.sections[0], wb.sections[0])

    def call(c, f, slot, sec):
        rc = lib.cg_bunch_moments_noalloc(c.data_ptr(), c.shape[1], f.data_ptr(), f.shape[0],
                                          sec.beta_x, sec.beta_y, out[slot].data_ptr(), stream)
        assert rc == 0, lib.cg_last_error(None).decode()

    call(ca, fa, 0, secs[0])  # first call on this device: resolves the scratch address
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    out.zero_()
    call(ca, fa, 0, secs[0])
    call(cb, fb, 1, secs[1])
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0  # nothing allocated by the two calls
    host = out.cpu().numpy()
    got_a = _abi.BunchMoments.from_buffer_copy(host[0].tobytes())
    got_b = _abi.BunchMoments.from_buffer_copy(host[1].tobytes())
    for got, ref, n, s in ((got_a, ref_a, pa[0].shape[1], sa[0]), (got_b, ref_b, pb[17].shape[1], sb[17])):
        assert got.n_macro == n
        assert got.n_alive == int((s == 0).sum())
        assert got.transmission == pytest.approx(got.n_alive / n, rel=1e-15)
        assert not _close(got, ref, 1e-14)
