"""Python host API over libcetagpu.so, mirroring the reference's MPBeam stage
methods (include/MPBeam.h:131-177).  Each method forwards to one C-ABI call;
all work runs in the sm_100a kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .configs import Workload


def _load_torch_nccl():
    """The library opens whichever NCCL the process already holds, else the
    system's; PyTorch needs its own (newer) one, and two cannot share the
    soname, so PyTorch is imported first."""
    import torch  # noqa: F401


class MPBeam:
    """One device handle tracking a bunch train (MPBeam + its bunches + the
    LatticeInterActionPoint ion clouds)."""

    def __init__(self, wl: Workload, device: int = 0, shard=None):
        """shard = (rank, world, nccl_id bytes): bunch-sharded run over
        `world` processes (see cg_set_shard)."""
        self.lib = _abi.load()
        self.wl = wl
        h = C.c_void_p()
        rc = self.lib.cg_create(C.byref(wl.cfg), device, C.byref(h))
        if rc:
            raise _abi.CgError(rc, self.lib.cg_last_error(None).decode())
        self.h = h
        if shard is not None:
            _load_torch_nccl()
            rank, world, nid = shard
            idbuf = None if nid is None else C.create_string_buffer(bytes(nid), 128)
            self._check(self.lib.cg_set_shard(h, rank, world, idbuf))
        self._check(self.lib.cg_set_beam(h, wl.n_bunches, _abi.ptr(wl.n_macro), _abi.ptr(wl.harm),
                                         _abi.ptr(wl.ne)))
        j0, j1 = C.c_int(), C.c_int()
        self._check(self.lib.cg_shard_range(h, C.byref(j0), C.byref(j1)))
        self.local = range(j0.value, j1.value)

    @staticmethod
    def nccl_unique_id() -> bytes:
        _load_torch_nccl()
        lib = _abi.load()
        buf = C.create_string_buffer(128)
        rc = lib.cg_nccl_unique_id(buf)
        if rc:
            raise _abi.CgError(rc, lib.cg_last_error(None).decode())
        return buf.raw

    # -- plumbing ------------------------------------------------------------
    def _check(self, rc: int):
        if rc:
            raise _abi.CgError(rc, self.lib.cg_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.cg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state in / out --------------------------------------------------------
    def generate(self, seed: int = 99):
        ex, ey, sz, sdp = self.wl.gen
        self._check(self.lib.cg_generate_gaussian(self.h, ex, ey, sz, sdp, seed))

    def upload(self, j: int, coords: np.ndarray, surv: np.ndarray | None = None):
        c = [np.ascontiguousarray(coords[d], dtype=np.float64) for d in range(6)]
        s = None if surv is None else np.ascontiguousarray(surv, dtype=np.uint8)
        self._check(self.lib.cg_upload_bunch(self.h, j, *[_abi.ptr(a) for a in c], _abi.ptr(s)))

    def upload_beam(self, parts, surv=None):
        """Every local bunch at once (cg_upload_beam): parts[j] = (6, n_j)
        coordinates, surv[j] survival bytes or None."""
        keep = [np.ascontiguousarray(parts[j], dtype=np.float64) for j in range(self.wl.n_bunches)]
        table = (C.c_void_p * (6 * self.wl.n_bunches))()
        for j, a in enumerate(keep):
            for d in range(6):
                table[6 * j + d] = a[d].ctypes.data
        st = None
        if surv is not None:
            sk = [np.ascontiguousarray(x, dtype=np.uint8) for x in surv]
            st = (C.c_void_p * self.wl.n_bunches)(*[x.ctypes.data for x in sk])
        self._check(self.lib.cg_upload_beam(self.h, table, st))

    def download(self, j: int):
        n = int(self.wl.n_macro[j])
        c = np.empty((6, n))
        s = np.empty(n, dtype=np.uint8)
        self._check(self.lib.cg_download_bunch(self.h, j, *[_abi.ptr(c[d]) for d in range(6)],
                                               _abi.ptr(s)))
        return c, s

    def moments(self):
        out = (_abi.BunchMoments * self.wl.n_bunches)()
        self._check(self.lib.cg_get_moments(self.h, out))
        return out

    # -- MPBeam stage methods ----------------------------------------------------
    def MPBeamRMSCal(self, k: int):
        self._check(self.lib.cg_beam_rms(self.h, k))

    def SSBeamIonEffectOneInteractionPoint(self, turn: int, k: int):
        self._check(self.lib.cg_beam_ion_ip(self.h, turn, k))

    def BeamTransferPerInteractionPointDueToLatticeT(self, k: int):
        self._check(self.lib.cg_section_map(self.h, k))

    def BeamMomtumUpdateDueToRFTest(self):
        self._check(self.lib.cg_rf_kick(self.h))

    def BeamLongiPosTransferOneTurn(self):
        self._check(self.lib.cg_longi_drift(self.h))

    def BeamEnergyLossOneTurn(self):
        self._check(self.lib.cg_energy_loss(self.h))

    def BeamSynRadDamping(self, turn: int):
        self._check(self.lib.cg_synrad(self.h, turn))

    def BeamTransferDueToSpaceCharge(self, k: int):
        """BeamTransferDueToSpaceChargePIC (runSpaceCharge 2) or
        ...Analytical (1, 3) at section k."""
        self._check(self.lib.cg_space_charge(self.h, k))

    def BBImpBeamInteraction(self):
        self._check(self.lib.cg_bbi_kick(self.h))

    def bbi_profile(self, j: int):
        """(first bin, 6 x n array) of bunch j after the last
        BBImpBeamInteraction: the smoothed profile and the potentials of the
        planes Z, Dx, Dy, Qx, Qy (zero at bins without particles)."""
        lo, n = C.c_int(), C.c_int()
        self._check(self.lib.cg_bbi_profile(self.h, j, C.byref(lo), C.byref(n), None, 0))
        cap = max(1, n.value)
        out = np.zeros((6, cap))
        self._check(self.lib.cg_bbi_profile(self.h, j, C.byref(lo), C.byref(n),
                                            out.ctypes.data_as(C.POINTER(C.c_double)), cap))
        return lo.value, out[:, :n.value]

    def LRWakeBeamIntaction(self):
        self._check(self.lib.cg_lr_wake(self.h))

    def SRWakeBeamIntaction(self, turn: int):
        self._check(self.lib.cg_sr_wake(self.h, turn))

    def FIRBunchByBunchFeedback(self, turn: int):
        self._check(self.lib.cg_fir(self.h, turn))

    def MarkParticleLostInBunch(self):
        tr = np.empty(self.wl.n_bunches)
        self._check(self.lib.cg_mark_lost(self.h, _abi.ptr(tr)))
        return tr

    def Run(self, turn0: int, n_turns: int):
        self._check(self.lib.cg_run_turns(self.h, turn0, n_turns))

    # -- autotuning ---------------------------------------------------------------
    def autotune(self, k: int = 0, reps: int = 10):
        """Times the kick shapes and the map-pass forms on this beam at IP k;
        returns (choice, ms) as cg_autotune fills them (n kick shapes, then
        the map pass, with the kick, and both with the next chunk in flight)."""
        n = C.c_int()
        self._check(self.lib.cg_kick_variants(C.byref(n)))
        ms = np.zeros(n.value + 4)
        choice = C.c_int()
        self._check(self.lib.cg_autotune(self.h, k, reps, C.byref(choice), _abi.ptr(ms)))
        return choice.value, ms

    def set_kick_variant(self, v: int):
        self._check(self.lib.cg_set_kick_variant(self.h, v))

    # -- cavities with beam loading (rfMode 1) -------------------------------------
    def resonator(self, c: int):
        """(vbAccum, resGenVol, resGenIg) of cavity c as complex numbers."""
        out = np.empty(6)
        self._check(self.lib.cg_resonator_state(self.h, c, _abi.ptr(out)))
        return complex(out[0], out[1]), complex(out[2], out[3]), complex(out[4], out[5])

    def set_resonator(self, c: int, vb: complex, gen: complex, ig: complex):
        a = np.array([vb.real, vb.imag, gen.real, gen.imag, ig.real, ig.imag])
        self._check(self.lib.cg_set_resonator_state(self.h, c, _abi.ptr(a)))

    def rf_info(self, j: int, c: int):
        """BunchRFModeInfo of bunch j, cavity c after the last RF step:
        (cavity, generator, induced, self-loss) voltages as complex numbers."""
        out = np.empty(8)
        self._check(self.lib.cg_rf_info(self.h, j, c, _abi.ptr(out)))
        return tuple(complex(out[2 * i], out[2 * i + 1]) for i in range(4))

    def set_walk_reserve(self, on: bool):
        self._check(self.lib.cg_set_walk_reserve(self.h, int(bool(on))))

    def set_map_async(self, on: bool):
        self._check(self.lib.cg_set_map_async(self.h, int(bool(on))))

    def map_async(self) -> bool:
        v = C.c_int()
        self._check(self.lib.cg_map_async(self.h, C.byref(v)))
        return bool(v.value)

    def set_pipeline(self, groups: int, walk_ions: int = 0, ramp: bool = False):
        self._check(self.lib.cg_set_pipeline(self.h, groups, walk_ions, int(ramp)))

    def trace_turn(self, turn0: int, cap: int = 4096):
        """One turn as direct launches with a timing event after each: a list
        of (kind, stream, ip, segment, t_end_us) in launch order."""
        recs = (_abi.TraceRecord * cap)()
        n = C.c_int()
        self._check(self.lib.cg_trace_turn(self.h, turn0, recs, cap, C.byref(n)))
        return [(_abi.TRACE_KINDS[r.kind], r.stream, r.ip, r.segment, r.t_end_us)
                for r in recs[:n.value]]

    # -- coupled-bunch mode history (MPBeam::GetCBMGR) -----------------------------
    def cbm_init(self, capacity: int):
        self._check(self.lib.cg_cbm_init(self.h, capacity))

    def cbm_record(self):
        self._check(self.lib.cg_cbm_record(self.h))

    def cbm_history(self):
        """(amp, arg, aver, iq_amp, iq_arg), each records x 3 planes x M."""
        n = C.c_int()
        self._check(self.lib.cg_cbm_count(self.h, C.byref(n)))
        M = self.wl.n_bunches
        out = [np.zeros((n.value, 3, M)) for _ in range(5)]
        if n.value:
            self._check(self.lib.cg_cbm_history(self.h, 0, n.value, *[_abi.ptr(a) for a in out]))
        return tuple(out)

    def cbm_growth(self, first: int, last: int, interval: float, method: int = 0):
        """Growth rates (3, M) in 1/s: method 0 the DFT modes, 1 the IQ scan."""
        rate = np.zeros((3, self.wl.n_bunches))
        self._check(self.lib.cg_cbm_growth(self.h, method, first, last, float(interval),
                                           _abi.ptr(rate)))
        return rate

    def cbm_hilbert(self, first: int, last: int, interval: float):
        """The Hilbert method over all records: (mode rates (3, M), bunch
        rates (3, M), mode amplitudes and phases (N, 3, M), analytic signals
        (N, 3, M))."""
        n = C.c_int()
        self._check(self.lib.cg_cbm_count(self.h, C.byref(n)))
        M = self.wl.n_bunches
        mr, br = np.zeros((3, M)), np.zeros((3, M))
        hamp, harg = np.zeros((n.value, 3, M)), np.zeros((n.value, 3, M))
        ana = np.zeros((n.value, 3, M), dtype=np.complex128)
        self._check(self.lib.cg_cbm_hilbert(self.h, first, last, float(interval), _abi.ptr(mr),
                                            _abi.ptr(br), _abi.ptr(hamp), _abi.ptr(harg),
                                            ana.ctypes.data_as(C.c_void_p)))
        return mr, br, hamp, harg, ana

    def autotune_pipeline(self, turn0: int, reps: int = 5):
        """Times whole turns with each pipeline shape, restores the beam and
        keeps the fastest; returns ((groups, walk_ions, ramp), ms per shape
        in the order of _abi.PIPE_SHAPES)."""
        ms = np.zeros(len(_abi.PIPE_SHAPES))
        shape = (C.c_int * 3)()
        self._check(self.lib.cg_autotune_pipeline(self.h, turn0, reps, shape, _abi.ptr(ms)))
        return tuple(shape), ms

    # -- checkpoint / resume ------------------------------------------------------
    def checkpoint(self) -> bytes:
        n = C.c_size_t()
        self._check(self.lib.cg_checkpoint_size(self.h, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        self._check(self.lib.cg_checkpoint_save(self.h, buf, n.value))
        return buf.raw

    def restore(self, blob: bytes):
        buf = C.create_string_buffer(blob, len(blob))
        self._check(self.lib.cg_checkpoint_load(self.h, buf, len(blob)))

    # -- field surrogate (no reference counterpart) -------------------------------
    def set_surrogate(self, weights, audit_interval: int = 0):
        """Electron-side ion kicks from the trained surrogate (None: exact)."""
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        self._check(self.lib.cg_set_surrogate(self.h, _abi.ptr(w), audit_interval))
        self._sur_w = w

    def surrogate_audit(self, k: int):
        """(max |F_sur - F_exact|, max |F_exact|) at IP k on the current beam."""
        out = np.zeros(2)
        self._check(self.lib.cg_surrogate_audit(self.h, k, _abi.ptr(out)))
        return out

    def surrogate_audit_stats(self):
        n = C.c_int()
        last, worst = C.c_double(), C.c_double()
        self._check(self.lib.cg_surrogate_audit_stats(self.h, C.byref(n), C.byref(last),
                                                      C.byref(worst)))
        return n.value, last.value, worst.value

    # -- ion clouds --------------------------------------------------------------
    def ions(self, k: int, p: int = 0):
        cap = int(self.wl.cfg.ion.max_ions) + 8
        a = [np.empty(cap) for _ in range(4)]
        n = C.c_int()
        self._check(self.lib.cg_ion_download(self.h, k, p, *[_abi.ptr(x) for x in a], cap, C.byref(n)))
        return [x[: n.value] for x in a]

    def set_phase_track(self, bunches):
        """Tracks the accumulated phase advance of every particle of these
        bunches from now on (cg_set_phase_track)."""
        b = np.ascontiguousarray(list(bunches), dtype=np.int32)
        self._check(self.lib.cg_set_phase_track(self.h, len(b), _abi.ptr(b) if len(b) else None))

    def phase_adv(self, j: int):
        """Accumulated x, y, z phase advance of bunch j's particles (3 x n)."""
        n = int(self.wl.n_macro[j])
        out = np.empty(3 * n)
        self._check(self.lib.cg_phase_adv(self.h, j, _abi.ptr(out)))
        return out.reshape(3, n)

    def ion_forces(self, k: int, p: int = 0):
        """(fx, fy, macro-ion charge) of cloud (k, p): the last bunch's
        velocity kick on each ion."""
        cap = int(self.wl.cfg.ion.max_ions) + 8
        fx, fy = np.empty(cap), np.empty(cap)
        n, q = C.c_int(), C.c_double()
        self._check(self.lib.cg_ion_forces(self.h, k, p, _abi.ptr(fx), _abi.ptr(fy), cap, C.byref(n),
                                           C.byref(q)))
        return fx[: n.value], fy[: n.value], q.value

    def upload_ions(self, k: int, p: int, x, y, vx, vy):
        """Replaces the accumulated cloud of section k, species p."""
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, vx, vy)]
        self._check(self.lib.cg_ion_upload(self.h, k, p, *[_abi.ptr(v) for v in a], len(a[0])))

    def cloud_record(self, k: int):
        out = np.empty((self.wl.n_bunches, max(1, self.wl.cfg.ion.n_species), 6))
        self._check(self.lib.cg_ion_cloud_record(self.h, k, _abi.ptr(out)))
        return out

    def set_sr_potentials(self, on: bool):
        self._check(self.lib.cg_set_sr_potentials(self.h, int(bool(on))))

    def sr_potentials(self, j: int):
        """Bunch j's short-range potentials x, y, z (3 x B) of the last SR step."""
        B = int(self.wl.cfg.sr_bins)
        out = np.empty(3 * B)
        self._check(self.lib.cg_sr_potentials(self.h, j, _abi.ptr(out)))
        return out.reshape(3, B)

    def sr_bins(self, j: int):
        zlo, dz = C.c_double(), C.c_double()
        cnt = np.empty(int(self.wl.cfg.sr_bins), dtype=np.int32)
        self._check(self.lib.cg_sr_bins(self.h, j, C.byref(zlo), C.byref(dz), _abi.ptr(cnt)))
        return zlo.value, dz.value, cnt
