"""ctypes mirror of include/cetasim_gpu.h and the loader of libcetagpu.so.

The shared library is the product; this module only declares its C types.
Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcetagpu.so")

MAX_SPECIES = 8
MAX_CAVITIES = 4
MAX_RESONATORS = 16
MAX_FIR = 64
MAX_FB_SECTIONS = 8

D = C.c_double
I = C.c_int

STATUS = {
    0: "CG_OK", 1: "CG_ERR_INVALID", 2: "CG_ERR_OOM", 3: "CG_ERR_CUDA",
    4: "CG_ERR_ION_OVERFLOW", 5: "CG_ERR_TRANSMISSION", 6: "CG_ERR_TIMEOUT",
    7: "CG_ERR_NOT_READY", 8: "CG_ERR_UNSUPPORTED",
}


class Ring(C.Structure):
    _fields_ = [
        ("circ_ring", D), ("work_qx", D), ("work_qy", D), ("chrom", D * 2), ("alphac", D * 3),
        ("adtx", D * 5), ("adty", D * 5), ("synch_rad_damp_time", D * 3),
        ("pipe_aperture_x", D), ("pipe_aperture_y", D), ("electron_energy", D), ("sdelta0", D),
        ("natural_emit", D), ("coupling", D), ("u0", D), ("skew_quad_k", D),
        ("harmonics", I), ("n_cav", I), ("cav_harm", I * MAX_CAVITIES),
        ("cav_vol", D * MAX_CAVITIES), ("cav_phase", D * MAX_CAVITIES),
        ("r_gamma", D), ("r_beta", D), ("t0", D), ("f0", D), ("eta", D), ("work_qz", D),
        ("natural_bunch_length", D), ("beta_z", D), ("emit_nat", D * 3),
        ("cav_vreq_re", D * MAX_CAVITIES), ("cav_vreq_im", D * MAX_CAVITIES),
        ("rf_mode", I * MAX_CAVITIES), ("res_type", I * MAX_CAVITIES),
        ("res_cold", I * MAX_CAVITIES), ("res_excite", I * MAX_CAVITIES),
        ("res_dir_fb", I * MAX_CAVITIES), ("rf_bunch_bins", I),
        ("res_rs", D * MAX_CAVITIES), ("res_q0", D * MAX_CAVITIES),
        ("res_coupling", D * MAX_CAVITIES), ("res_detune", D * MAX_CAVITIES),
        ("res_dir_fb_gain", D * MAX_CAVITIES), ("res_dir_fb_phase", D * MAX_CAVITIES),
        ("res_dir_fb_delay", D * MAX_CAVITIES),
        ("res_ql", D * MAX_CAVITIES), ("res_fre", D * MAX_CAVITIES),
        ("res_psi", D * MAX_CAVITIES), ("res_tf", D * MAX_CAVITIES),
    ]


class Section(C.Structure):
    _fields_ = [
        ("s", D),
        ("beta_x", D), ("alpha_x", D), ("psi_x", D), ("eta_x", D), ("etap_x", D), ("aperture_x", D),
        ("beta_y", D), ("alpha_y", D), ("psi_y", D), ("eta_y", D), ("etap_y", D), ("aperture_y", D),
        ("length", D), ("pressure", D), ("temperature", D),
        ("phase_adv_x", D), ("phase_adv_y", D),
        ("map_b1h1", D * 36), ("map_h1b1", D * 36), ("map_h2b2", D * 36),
    ]


class IonParams(C.Structure):
    _fields_ = [
        ("n_species", I), ("mass_number", D * MAX_SPECIES), ("cross_section", D * MAX_SPECIES),
        ("gas_percent", D * MAX_SPECIES), ("loss_boundary", D), ("max_ions", I),
        ("macro_ions_per_ip", I),
    ]


class Bbr(C.Structure):
    _fields_ = [("n", I)] + [(nm, D * MAX_RESONATORS) for nm in (
        "l_rs", "l_q", "l_omega", "tx_rs", "tx_q", "tx_omega", "ty_rs", "ty_q", "ty_omega")]


class FirParams(C.Structure):
    _fields_ = [
        ("mode", I), ("delay", I), ("taps", I), ("gain", D), ("kick_strength", D * 3),
        ("power_limit", D), ("kicker_imped", D), ("coeff_x", D * MAX_FIR), ("coeff_y", D * MAX_FIR),
        ("coeff_z", D * MAX_FIR), ("n_sections", I), ("start", I * MAX_FB_SECTIONS),
        ("end", I * MAX_FB_SECTIONS),
    ]


MAX_RW = 32


class RwSectors(C.Structure):
    _fields_ = [("n", I)] + [(f, D * MAX_RW) for f in ("radius_x", "radius_y", "length",
                                                        "beta_x", "beta_y", "num", "sigma")]


class Bbi(C.Structure):
    _fields_ = [("flag", I), ("time_domain", I), ("sim", I * 5), ("n_rows", I),
                ("table", C.POINTER(D))]


BBI_MAX_BINS = 4096


class Config(C.Structure):
    _fields_ = [
        ("ring", Ring), ("n_sections", I), ("sections", C.POINTER(Section)), ("ion", IonParams),
        ("sr_bbr", Bbr), ("sr_bins", I), ("lr_bbr", Bbr), ("lr_turns", I), ("fir", FirParams),
        ("flag_synrad", I), ("flag_beam_ion", I), ("flag_lr_wake", I), ("flag_sr_wake", I),
        ("flag_fir", I), ("seed", C.c_uint64),
        ("n_turns", I), ("bunch_info_print_interval", I), ("bunch_emit_x", D), ("bunch_emit_y", D),
        ("bunch_sigma_z", D), ("bunch_sigma_dp", D),
        ("growth_fit_start", I), ("growth_fit_end", I), ("run_cbmgr", C.c_char * 256),
        ("lr_rw", RwSectors), ("sr_rw", RwSectors), ("bbi", Bbi),
        ("flag_sc", I), ("sc_mesh", I * 3),
    ]


class BunchMoments(C.Structure):
    _fields_ = [
        ("n_alive", I), ("n_macro", I), ("mean", D * 6), ("emit", D * 3), ("eff_emit", D * 3),
        ("rms_x", D), ("rms_y", D), ("eff_rms_x", D), ("eff_rms_y", D), ("bunch_length", D),
        ("energy_spread", D), ("z_min", D), ("z_max", D), ("transmission", D),
    ]


PD = C.POINTER(C.c_double)
PF = C.POINTER(C.c_float)
PU8 = C.POINTER(C.c_uint8)
PI = C.POINTER(C.c_int)

class TraceRecord(C.Structure):
    _fields_ = [("kind", C.c_int), ("stream", C.c_int), ("ip", C.c_int), ("segment", C.c_int),
                ("t_end_us", C.c_double)]


PIPE_SHAPES = [(1, 64, 0), (1, 16, 0), (2, 64, 0), (2, 64, 1), (3, 64, 0), (3, 64, 1),
               (4, 64, 0), (4, 64, 1), (3, 16, 1), (6, 64, 1), (8, 64, 1), (12, 64, 1),
               (16, 64, 1), (8, 32, 1), (12, 32, 1), (16, 32, 1)]

TRACE_KINDS = ["start", "moments", "ion_prep", "ion_walk", "ion_records", "ion_compact",
               "ion_chain", "ion_kick", "map_pass", "exchange", "lr_wake", "long", "sr_wake",
               "fir", "mark_lost"]


class SurTrainParams(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("n_train", C.c_int64), ("n_holdout", C.c_int64),
                ("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_double),
                ("l4_from", C.c_double), ("l4_weight", C.c_double)]


# (name, restype, argtypes) of every export declared in include/cetasim_gpu.h
EXPORTS = [
    ("cg_abi_version", I, []),
    ("cg_config_derive", I, [C.POINTER(Config)]),
    ("cg_lattice_init", I, [C.POINTER(Ring), C.POINTER(Section), I]),
    ("cg_config_from_input", I, [C.c_char_p, C.POINTER(Config), PI, C.POINTER(PI), C.POINTER(PI),
                                 C.POINTER(PD)]),
    ("cg_config_free", None, [C.POINTER(Config), PI, PI, PD]),
    ("cg_parse_error", C.c_char_p, []),
    ("cg_create", I, [C.POINTER(Config), I, C.POINTER(C.c_void_p)]),
    ("cg_destroy", I, [C.c_void_p]),
    ("cg_last_error", C.c_char_p, [C.c_void_p]),
    ("cg_set_beam", I, [C.c_void_p, I, PI, PI, PD]),
    ("cg_upload_bunch", I, [C.c_void_p, I, PD, PD, PD, PD, PD, PD, PU8]),
    ("cg_upload_beam", I, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("cg_download_bunch", I, [C.c_void_p, I, PD, PD, PD, PD, PD, PD, PU8]),
    ("cg_generate_gaussian", I, [C.c_void_p, D, D, D, D, C.c_uint64]),
    ("cg_beam_rms", I, [C.c_void_p, I]),
    ("cg_get_moments", I, [C.c_void_p, C.POINTER(BunchMoments)]),
    ("cg_beam_ion_ip", I, [C.c_void_p, I, I]),
    ("cg_section_map", I, [C.c_void_p, I]),
    ("cg_rf_kick", I, [C.c_void_p]),
    ("cg_longi_drift", I, [C.c_void_p]),
    ("cg_energy_loss", I, [C.c_void_p]),
    ("cg_synrad", I, [C.c_void_p, I]),
    ("cg_lr_wake", I, [C.c_void_p]),
    ("cg_sr_wake", I, [C.c_void_p, I]),
    ("cg_bbi_kick", I, [C.c_void_p]),
    ("cg_space_charge", I, [C.c_void_p, I]),
    ("cg_bunch_ion_charge", I, [C.c_void_p, PD]),
    ("cg_rf_profile", I, [C.c_void_p, I, PD, PD, PI]),
    ("cg_ion_forces", I, [C.c_void_p, I, I, PD, PD, I, PI, PD]),
    ("cg_set_phase_track", I, [C.c_void_p, I, PI]),
    ("cg_phase_adv", I, [C.c_void_p, I, PD]),
    ("cg_bbi_profile", I, [C.c_void_p, I, PI, PI, PD, I]),
    ("cg_sr_bins", I, [C.c_void_p, I, PD, PD, PI]),
    ("cg_set_sr_potentials", I, [C.c_void_p, I]),
    ("cg_sr_potentials", I, [C.c_void_p, I, PD]),
    ("cg_fir", I, [C.c_void_p, I]),
    ("cg_mark_lost", I, [C.c_void_p, PD]),
    ("cg_run_turns", I, [C.c_void_p, I, I]),
    ("cg_host_alloc", C.c_void_p, [C.c_size_t]),
    ("cg_host_free", None, [C.c_void_p]),
    ("cg_stream", C.c_void_p, [C.c_void_p]),
    ("cg_turn_launches", I, [C.c_void_p, PI]),
    ("cg_time_stage", I, [C.c_void_p, I, I, I, PD]),
    ("cg_fp64_peak", I, [PD]),
    ("cg_field_chain_latency", I, [PD]),
    ("cg_eigen_emit", I, [C.c_void_p, I, PD]),
    ("cg_ion_count", I, [C.c_void_p, I, I, PI]),
    ("cg_ion_download", I, [C.c_void_p, I, I, PD, PD, PD, PD, I, PI]),
    ("cg_ion_upload", I, [C.c_void_p, I, I, PD, PD, PD, PD, I]),
    ("cg_ion_cloud_record", I, [C.c_void_p, I, PD]),
    ("cg_ion_totals", I, [C.c_void_p, PD, PI]),
    ("cg_faddeeva_w", I, [PD, PD, PD, PD, C.c_int64]),
    ("cg_faddeeva_w_q1", I, [PD, PD, PD, PD, C.c_int64]),
    ("cg_gaussian_field", I, [PD, PD, PD, PD, PD, PD, C.c_int64]),
    ("cg_kick_variants", I, [PI]),
    ("cg_set_pipeline", I, [C.c_void_p, I, I, I]),
    ("cg_trace_turn", I, [C.c_void_p, I, C.c_void_p, I, C.POINTER(C.c_int)]),
    ("cg_yokoya_factors", I, [C.c_double, C.c_double, PD]),
    ("cg_rw_lr_wake", I, [C.c_void_p, C.c_double, C.c_double, C.c_double, PD]),
    ("cg_cbm_init", I, [C.c_void_p, I]),
    ("cg_cbm_record", I, [C.c_void_p]),
    ("cg_cbm_count", I, [C.c_void_p, C.POINTER(C.c_int)]),
    ("cg_cbm_history", I, [C.c_void_p, I, I] + [C.c_void_p] * 5),
    ("cg_cbm_growth", I, [C.c_void_p, I, I, I, C.c_double, C.c_void_p]),
    ("cg_cbm_hilbert", I, [C.c_void_p, I, I, C.c_double] + [C.c_void_p] * 5),
    ("cg_autotune_pipeline", I, [C.c_void_p, I, I, C.c_void_p, C.c_void_p]),
    ("cg_set_kick_variant", I, [C.c_void_p, I]),
    ("cg_autotune", I, [C.c_void_p, I, I, PI, PD]),
    ("cg_set_map_async", I, [C.c_void_p, I]),
    ("cg_resonator_state", I, [C.c_void_p, I, PD]),
    ("cg_set_resonator_state", I, [C.c_void_p, I, PD]),
    ("cg_rf_info", I, [C.c_void_p, I, I, PD]),
    ("cg_set_walk_reserve", I, [C.c_void_p, I]),
    ("cg_map_async", I, [C.c_void_p, PI]),
    ("cg_shard_plan", I, [PI, I, I, PI, PI]),
    ("cg_shard_exchange_size", I, [PI, I, I, PI]),
    ("cg_shard_pack", I, [PI, I, I, I, C.c_void_p, C.c_size_t, C.c_void_p]),
    ("cg_shard_unpack", I, [PI, I, I, C.c_void_p, C.c_size_t, C.c_void_p]),
    ("cg_nccl_unique_id", I, [C.c_void_p]),
    ("cg_set_shard", I, [C.c_void_p, I, I, C.c_void_p]),
    ("cg_shard_range", I, [C.c_void_p, PI, PI]),
    ("cg_checkpoint_size", I, [C.c_void_p, C.POINTER(C.c_size_t)]),
    ("cg_checkpoint_save", I, [C.c_void_p, C.c_void_p, C.c_size_t]),
    ("cg_checkpoint_load", I, [C.c_void_p, C.c_void_p, C.c_size_t]),
    ("cg_surrogate_dataset", I, [C.c_uint64, C.c_int64, PF, PF]),
    ("cg_surrogate_eval", I, [PF, PF, C.c_int64, PF]),
    ("cg_surrogate_grad", I, [PF, PF, PF, I, PF, PD]),
    ("cg_surrogate_train", I, [C.POINTER(SurTrainParams), PF, PD]),
    ("cg_set_surrogate", I, [C.c_void_p, PF, I]),
    ("cg_surrogate_audit", I, [C.c_void_p, I, PD]),
    ("cg_surrogate_audit_stats", I, [C.c_void_p, PI, PD, PD]),
    ("cg_bunch_moments_noalloc", I, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, D, D,
                                     C.c_void_p, C.c_void_p]),
]

_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Loads libcetagpu.so and declares its exports (raises if absent)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"libcetagpu.so not found at {p}: build it with `python -m cetasim_b200.build` "
            "(this package has no CPU fallback)")
    lib = C.CDLL(p)
    for name, res, args in EXPORTS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class CgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def ptr(a):
    """Pointer to a contiguous numpy array (float64 / int32 / uint8)."""
    import numpy as np
    if a is None:
        return None
    if a.dtype == np.float64:
        return a.ctypes.data_as(PD)
    if a.dtype == np.float32:
        return a.ctypes.data_as(PF)
    if a.dtype == np.int32:
        return a.ctypes.data_as(PI)
    if a.dtype == np.uint8:
        return a.ctypes.data_as(PU8)
    raise TypeError(a.dtype)
