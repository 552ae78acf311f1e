"""ORACLE (test infrastructure only): ctypes wrapper of oracle/liboracle.so,
the CPU restatement of the reference's MP tracking path (see oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this
module, and only as the checker.  The restatement is pinned against the
reference's own sources built in oracle/_ref (oracle/ref.py) and against the
fixtures they generated (tests/golden).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libfaddeeva_ref.so")

_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError("oracle/liboracle.so missing: run `make -C oracle`")
        _lib = C.CDLL(LIB)
        _lib.or_create.restype = C.c_void_p
        _lib.or_last_error.restype = C.c_char_p
        _lib.or_rw_fz.restype = C.c_double
        _lib.or_rw_fz.argtypes = [C.c_double]
        for n in ("or_destroy",):
            getattr(_lib, n).restype = None
    return _lib


def _p(a):
    if a is None:
        return None
    if a.dtype == np.float64:
        return a.ctypes.data_as(C.POINTER(C.c_double))
    if a.dtype == np.uint8:
        return a.ctypes.data_as(C.POINTER(C.c_uint8))
    if a.dtype == np.int32:
        return a.ctypes.data_as(C.POINTER(C.c_int))
    raise TypeError(a.dtype)


def faddeeva_w(z: np.ndarray) -> np.ndarray:
    lib = load()
    zr = np.ascontiguousarray(z.real, dtype=np.float64)
    zi = np.ascontiguousarray(z.imag, dtype=np.float64)
    wr, wi = np.empty_like(zr), np.empty_like(zr)
    lib.or_faddeeva_w(_p(zr), _p(zi), _p(wr), _p(wi), C.c_int64(len(zr)))
    return wr + 1j * wi


def ref_faddeeva_w(z: np.ndarray) -> np.ndarray | None:
    """The reference's own Faddeeva::w (compiled from its sources), or None."""
    if not os.path.exists(REF_LIB):
        return None
    lib = C.CDLL(REF_LIB)
    zr = np.ascontiguousarray(z.real, dtype=np.float64)
    zi = np.ascontiguousarray(z.imag, dtype=np.float64)
    wr, wi = np.empty_like(zr), np.empty_like(zr)
    lib.ref_faddeeva_w(_p(zr), _p(zi), _p(wr), _p(wi), C.c_int64(len(zr)))
    return wr + 1j * wi


def gaussian_field(x, y, sx, sy):
    lib = load()
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, sx, sy)]
    fx, fy = np.empty_like(a[0]), np.empty_like(a[0])
    lib.or_gaussian_field(*[_p(v) for v in a], _p(fx), _p(fy), C.c_int64(len(a[0])))
    return fx, fy


def config_derive(cfg_ref) -> int:
    return load().or_config_derive(cfg_ref)


def lattice_init(ring_ref, secs, n) -> int:
    return load().or_lattice_init(ring_ref, secs, n)


class OracleBeam:
    """The oracle state with the same stage-method names as cetasim_b200.MPBeam."""

    def __init__(self, wl):
        self.lib = load()
        self.wl = wl
        self.s = self.lib.or_create(C.byref(wl.cfg), wl.n_bunches, _p(wl.n_macro), _p(wl.harm),
                                    _p(wl.ne))
        if not self.s:
            raise RuntimeError("or_create failed")
        self.s = C.c_void_p(self.s)
        rws = wl.cfg.lr_rw
        if wl.cfg.flag_lr_wake and rws.n > 0:
            # the resistive-wall term of the long-range table, with Yokoya
            # factors from the mpmath restatement (oracle/rw.py)
            from . import rw
            yok = rw.sector_factors(list(rws.radius_x[:rws.n]), list(rws.radius_y[:rws.n]))
            flat = (C.c_double * (5 * rws.n))(*[v for f in yok for v in f])
            if self.lib.or_lr_add_rw(self.s, flat):
                raise RuntimeError("or_lr_add_rw failed")
        srw = wl.cfg.sr_rw
        if wl.cfg.flag_sr_wake and srw.n > 0:
            from . import rw
            yok = rw.sector_factors(list(srw.radius_x[:srw.n]), list(srw.radius_y[:srw.n]))
            flat = (C.c_double * (5 * srw.n))(*[v for f in yok for v in f])
            if self.lib.or_sr_set_rw(self.s, flat):
                raise RuntimeError("or_sr_set_rw failed")

    def close(self):
        if self.s:
            self.lib.or_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise RuntimeError(f"oracle status {rc}: {self.lib.or_last_error(self.s).decode()}")

    def upload(self, j, coords, surv=None):
        c = [np.ascontiguousarray(coords[d], dtype=np.float64) for d in range(6)]
        s = None if surv is None else np.ascontiguousarray(surv, dtype=np.uint8)
        self._check(self.lib.or_set_bunch(self.s, j, *[_p(a) for a in c], _p(s)))

    def download(self, j):
        n = int(self.wl.n_macro[j])
        c = np.empty((6, n))
        s = np.empty(n, dtype=np.uint8)
        self._check(self.lib.or_get_bunch(self.s, j, *[_p(c[d]) for d in range(6)], _p(s)))
        return c, s

    def moments(self):
        from cetasim_b200 import _abi
        out = (_abi.BunchMoments * self.wl.n_bunches)()
        self._check(self.lib.or_get_moments(self.s, out))
        return out

    def MPBeamRMSCal(self, k):
        self._check(self.lib.or_beam_rms(self.s, k))

    def SSBeamIonEffectOneInteractionPoint(self, turn, k):
        self._check(self.lib.or_beam_ion_ip(self.s, turn, k))

    def BeamTransferPerInteractionPointDueToLatticeT(self, k):
        self._check(self.lib.or_section_map(self.s, k))

    def BeamMomtumUpdateDueToRFTest(self):
        self._check(self.lib.or_rf_kick(self.s))

    def BeamLongiPosTransferOneTurn(self):
        self._check(self.lib.or_longi_drift(self.s))

    def BeamEnergyLossOneTurn(self):
        self._check(self.lib.or_energy_loss(self.s))

    def BeamSynRadDamping(self, turn):
        self._check(self.lib.or_synrad(self.s, turn))

    def LRWakeBeamIntaction(self):
        self._check(self.lib.or_lr_wake(self.s))

    def SRWakeBeamIntaction(self, turn):
        self._check(self.lib.or_sr_wake(self.s, turn))

    def BBImpBeamInteraction(self):
        self._check(self.lib.or_bbi(self.s))

    def BeamTransferDueToSpaceCharge(self, k):
        self._check(self.lib.or_space_charge(self.s, k))

    def bbi_profile(self, j):
        """6 x nbins: bunch j's smoothed charge profile and the potentials of
        the planes Z, Dx, Dy, Qx, Qy over all profile bins, from the last
        BBImpBeamInteraction."""
        nb = C.c_int()
        self._check(self.lib.or_bbi_profile(self.s, j, C.byref(nb), None))
        out = np.empty((6, nb.value))
        self._check(self.lib.or_bbi_profile(self.s, j, C.byref(nb), _p(out)))
        return out

    def FIRBunchByBunchFeedback(self, turn):
        self._check(self.lib.or_fir(self.s, turn))

    def MarkParticleLostInBunch(self):
        tr = np.empty(self.wl.n_bunches)
        rc = self.lib.or_mark_lost(self.s, _p(tr))
        self._check(rc)
        return tr

    def Run(self, turn0, n_turns):
        self._check(self.lib.or_run_turns(self.s, turn0, n_turns))

    def ions(self, k, p=0):
        cap = int(self.wl.cfg.ion.max_ions) + 8
        a = [np.empty(cap) for _ in range(4)]
        n = C.c_int()
        self._check(self.lib.or_ion_download(self.s, k, p, *[_p(x) for x in a], cap, C.byref(n)))
        return [x[: n.value] for x in a]

    def upload_ions(self, k, p, x, y, vx, vy):
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, vx, vy)]
        self._check(self.lib.or_ion_upload(self.s, k, p, *[_p(v) for v in a], len(a[0])))

    def cloud_record(self, k):
        out = np.empty((self.wl.n_bunches, max(1, self.wl.cfg.ion.n_species), 6))
        self._check(self.lib.or_ion_cloud_record(self.s, k, _p(out)))
        return out

    def resonator(self, c):
        """(vbAccum, resGenVol, resGenIg) of cavity c as complex numbers."""
        out = np.empty(6)
        self._check(self.lib.or_resonator_state(self.s, c, _p(out)))
        return complex(out[0], out[1]), complex(out[2], out[3]), complex(out[4], out[5])

    def set_resonator(self, c, vb, gen, ig):
        a = np.array([vb.real, vb.imag, gen.real, gen.imag, ig.real, ig.imag])
        self._check(self.lib.or_resonator_set(self.s, c, _p(a)))

    def rf_info(self, j, c):
        """BunchRFModeInfo of bunch j, cavity c: (cavity, generator, induced,
        self-loss) voltages as complex numbers."""
        out = np.empty(8)
        self._check(self.lib.or_rf_info(self.s, j, c, _p(out)))
        return tuple(complex(out[2 * i], out[2 * i + 1]) for i in range(4))

    def sr_potentials(self, j):
        """srWakePoten of bunch j: x, y, z rows (3 x B)."""
        out = np.empty(3 * int(self.wl.cfg.sr_bins))
        self._check(self.lib.or_sr_potentials(self.s, j, _p(out)))
        return out.reshape(3, -1)

    def sr_bins(self, j):
        zlo, dz = C.c_double(), C.c_double()
        cnt = np.empty(int(self.wl.cfg.sr_bins), dtype=np.int32)
        self._check(self.lib.or_sr_bins(self.s, j, C.byref(zlo), C.byref(dz), _p(cnt)))
        return zlo.value, dz.value, cnt
