"""ORACLE (test infrastructure only): ctypes wrapper of oracle/_ref/
libcetasim_ref.so, the reference's own multi-particle sources compiled with
the harness in oracle/ref_harness.cpp (see oracle/Makefile).  `RefBeam`
exposes the same stage-method names as cetasim_b200.MPBeam and
oracle.OracleBeam, so parity tests read alike on all three.

Only tests/, __graft_entry__.smoke() and bench.py's reference arm use this,
and only as the checker or the timed reference.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libcetasim_ref.so")
EXE = os.path.join(HERE, "_ref", "cetasim_ref")

# stage numbers of ref_stage (ref_harness.cpp)
ST_RMS, ST_ION, ST_MAP, ST_SKEW, ST_RF, ST_DRIFT, ST_ELOSS, ST_SYNRAD = range(8)
ST_LR, ST_SR, ST_FIR, ST_LOST, ST_RMS_ONLY, ST_BBI, ST_SC = range(8, 15)

MOMENT_FIELDS = ["n_alive", "n_macro", "mean", "emit", "eff_emit", "rms_x", "rms_y",
                 "eff_rms_x", "eff_rms_y", "bunch_length", "energy_spread", "z_min", "z_max",
                 "transmission"]

_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref/libcetasim_ref.so is not built "
                               "(make -C oracle ref REF=<CETASim source tree>)")
        L = C.CDLL(LIB)
        L.ref_open.restype = C.c_void_p
        L.ref_open.argtypes = [C.c_char_p, C.c_ulonglong]
        L.ref_last_error.restype = C.c_char_p
        L.ref_close.argtypes = [C.c_void_p]
        L.ref_close.restype = None
        for n in ("ref_info", "ref_bunch_info", "ref_set_emit_nat", "ref_bunch_size", "ref_set_bunch",
                  "ref_get_bunch", "ref_moments", "ref_beam_info", "ref_stage", "ref_run_turns",
                  "ref_ion_count", "ref_ion_get", "ref_ion_set", "ref_sr_bins", "ref_ring",
                  "ref_resonator", "ref_rf_info", "ref_bbi_profile", "ref_bunch_ion_charge", "ref_phase_adv"):
            getattr(L, n).restype = C.c_int
        L.cg_ref_seed.argtypes = [C.c_ulonglong, C.c_longlong]
        L.cg_ref_seed.restype = None
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class RefMoments:
    """One bunch's moments from the reference (the field names of
    cetasim_b200's BunchMoments)."""

    def __init__(self, v):
        self.n_alive = int(v[0])
        self.n_macro = int(v[1])
        self.mean = np.array(v[2:8])
        self.emit = np.array(v[8:11])
        self.eff_emit = np.array(v[11:14])
        self.rms_x, self.rms_y, self.eff_rms_x, self.eff_rms_y = (float(x) for x in v[14:18])
        self.bunch_length, self.energy_spread, self.z_min, self.z_max = (float(x) for x in v[18:22])
        self.transmission = float(v[22])


class RefBeam:
    """The reference's MPBeam on an input.dat (set-up as its main.cpp does),
    with injected particles and the Run loop body driven stage by stage."""

    def __init__(self, input_path: str, seed: int = 0):
        self.lib = load()
        h = self.lib.ref_open(os.path.abspath(input_path).encode(), C.c_ulonglong(seed))
        if not h:
            raise RuntimeError("ref_open: " + self.lib.ref_last_error().decode())
        self.h = C.c_void_p(h)
        info = (C.c_int * 4)()
        self.lib.ref_info(self.h, info)
        self.n_bunches, self.n_sections, self.n_species, self.n_macro0 = list(info)

    def close(self):
        if getattr(self, "h", None):
            self.lib.ref_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise RuntimeError(f"reference status {rc}: {self.lib.ref_last_error().decode()}")

    # -- state in / out --------------------------------------------------------
    def set_emit_nat(self, e3):
        a = np.ascontiguousarray(e3, dtype=np.float64)
        self._check(self.lib.ref_set_emit_nat(self.h, _dp(a)))

    def upload(self, j, coords, surv=None):
        c = [np.ascontiguousarray(coords[d], dtype=np.float64) for d in range(6)]
        n = len(c[0])
        s = None if surv is None else np.ascontiguousarray(surv, dtype=np.int32)
        self._check(self.lib.ref_set_bunch(self.h, j, n, *[_dp(a) for a in c],
                                           None if s is None else _ip(s)))

    def download(self, j):
        n = self.lib.ref_bunch_size(self.h, j)
        c = np.empty((6, n))
        s = np.empty(n, dtype=np.int32)
        self._check(self.lib.ref_get_bunch(self.h, j, *[_dp(c[d]) for d in range(6)], _ip(s)))
        return c, s.astype(np.uint8)

    def bunch_info(self, j):
        out = (C.c_double * 4)()
        self._check(self.lib.ref_bunch_info(self.h, j, out))
        return {"ne": out[0], "macro_charge": out[1], "harm": int(out[2]), "gap": int(out[3])}

    def ion_forces(self, k, p=0):
        cap = 1 << 20
        fx, fy = np.empty(cap), np.empty(cap)
        n = self.lib.ref_ion_forces(self.h, k, p, _dp(fx), _dp(fy), cap)
        if n < 0:
            raise RuntimeError("bad IP or species")
        return fx[:n], fy[:n]

    def phase_adv(self, j):
        n = self.lib.ref_bunch_size(self.h, j)
        out = np.empty(3 * n)
        self._check(self.lib.ref_phase_adv(self.h, j, _dp(out)))
        return out.reshape(3, n)

    def bunch_ion_charge(self, j):
        out = C.c_double()
        self._check(self.lib.ref_bunch_ion_charge(self.h, j, C.byref(out)))
        return out.value

    def ring(self):
        out = np.empty(16)
        self.lib.ref_ring(self.h, _dp(out))
        keys = ["r_gamma", "r_beta", "t0", "f0", "work_qz", "emit_nat_x", "emit_nat_y",
                "emit_nat_z", "damp_x", "damp_y", "damp_z", "u0", "sdelta0", "harmonics"]
        return dict(zip(keys, out[:14]))

    def moments(self):
        out = np.empty(26 * self.n_bunches)
        self._check(self.lib.ref_moments(self.h, _dp(out)))
        return [RefMoments(out[26 * j:26 * j + 26]) for j in range(self.n_bunches)]

    def beam_info(self):
        out = np.empty(2)
        self.lib.ref_beam_info(self.h, _dp(out))
        return out

    def ions(self, k, p=0):
        n = self.lib.ref_ion_count(self.h, k, p)
        if n < 0:
            raise RuntimeError("no such cloud")
        a = [np.empty(max(n, 1)) for _ in range(4)]
        self._check(self.lib.ref_ion_get(self.h, k, p, *[_dp(x) for x in a], max(n, 1)))
        return [x[:n] for x in a]

    def upload_ions(self, k, p, x, y, vx, vy):
        self.set_ions(k, p, x, y, vx, vy)

    def set_ions(self, k, p, x, y, vx, vy):
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, vx, vy)]
        self._check(self.lib.ref_ion_set(self.h, k, p, *[_dp(v) for v in a], len(a[0])))

    def resonator(self, c):
        """(vbAccum, resGenVol, resGenIg) as complex numbers and the derived
        (resFre, resQualityQL, resDeTunePsi, tF) of cavity c."""
        out = np.empty(10)
        self._check(self.lib.ref_resonator(self.h, c, _dp(out)))
        return (complex(out[0], out[1]), complex(out[2], out[3]), complex(out[4], out[5]),
                tuple(out[6:10]))

    def rf_info(self, j, c):
        """BunchRFModeInfo of bunch j, cavity c: (cavity, generator, induced,
        self-loss) voltages as complex numbers."""
        out = np.empty(8)
        self._check(self.lib.ref_rf_info(self.h, j, c, _dp(out)))
        return tuple(complex(out[2 * i], out[2 * i + 1]) for i in range(4))

    def sr_bins(self, j, n_bins):
        zlo, dz = C.c_double(), C.c_double()
        counts = np.empty(n_bins, dtype=np.int32)
        self._check(self.lib.ref_sr_bins(self.h, j, C.byref(zlo), C.byref(dz), _ip(counts)))
        return zlo.value, dz.value, counts

    # -- MPBeam stage methods ----------------------------------------------------
    def stage(self, s, turn=0, k=0):
        self._check(self.lib.ref_stage(self.h, s, turn, k))

    def MPBeamRMSCal(self, k):
        self.stage(ST_RMS, 0, k)

    def SSBeamIonEffectOneInteractionPoint(self, turn, k):
        self.stage(ST_ION, turn, k)

    def BeamTransferPerInteractionPointDueToLatticeT(self, k):
        self.stage(ST_MAP, 0, k)

    def BeamMomtumUpdateDueToRFTest(self):
        self.stage(ST_RF)

    def BeamLongiPosTransferOneTurn(self):
        self.stage(ST_DRIFT)

    def BeamEnergyLossOneTurn(self):
        self.stage(ST_ELOSS)

    def BeamSynRadDamping(self, turn):
        self.stage(ST_SYNRAD, turn)

    def LRWakeBeamIntaction(self):
        self.stage(ST_LR)

    def SRWakeBeamIntaction(self, turn):
        self.stage(ST_SR, turn)

    def BBImpBeamInteraction(self):
        self.stage(ST_BBI)

    def BeamTransferDueToSpaceCharge(self, k):
        self.stage(ST_SC, 0, k)

    def bbi_profile(self, j):
        """6 x (2n - 1): profileForBunchBBImp and the five wakePotenFromBBI
        arrays of bunch j (frequency domain)."""
        n = C.c_int()
        self._check(self.lib.ref_bbi_profile(self.h, j, C.byref(n), None))
        out = np.zeros((6, n.value))
        self._check(self.lib.ref_bbi_profile(self.h, j, C.byref(n), _dp(out)))
        return out

    def FIRBunchByBunchFeedback(self, turn):
        self.stage(ST_FIR, turn)

    def MarkParticleLostInBunch(self):
        self.stage(ST_LOST)

    def Run(self, turn0, n_turns):
        self._check(self.lib.ref_run_turns(self.h, turn0, n_turns))
