"""Synthetic workloads with the shapes of the benchmark configurations.

Ring common to all (values as the reference's input.dat would hold them):
E = 6 GeV, C = 2304 m, h = 3840, nu_x = 135.18, nu_y = 86.27, chromaticity 2/2,
first-order amplitude-dependent tune shift 1e3 /m in both planes
(ringADTX = ringADTY = 1e3 1e3 0 0 0), alpha_c = 3.3e-5 / 1e-4 / 0, damping
times 20/20/10 ms in turns, U0 = 4.166343 MeV, V_RF = 8.2706 MV (the
reference's own formula gives nu_s = 0.0049), natural emittance 24 pm with
coupling 0.2 (eps_x = 20 pm, eps_y = 4 pm), sigma_z = 2.5 mm, sigma_dp = 9e-4.

  plain_single   1 bunch x 1e5, 1 section, broadband-resonator short-range
                 wake (Rs = 5 kOhm, R_perp = 2 MOhm/m, 30 GHz, Q = 1), 100 bins,
                 synchrotron radiation with quantum excitation.
  fast_ion       80 bunches x 2e4 in consecutive 2 ns buckets, 20 sections
                 (beta = 10 m, L = C/20, phase advance 2 pi nu / 20 each), CO
                 (A = 28, 2.0 Mb) at 1e-9 Pa and 300 K, one macro-ion per bunch
                 passage per section, exact Bassetti-Erskine kicks both ways.
  batched_uneven 900 bunches in 1000 buckets, macroparticles log-uniform in
                 [5e3, 5e4], 50 sections, long-range HOM (1.2 GHz, 1 MOhm/m,
                 Q = 1e4), 9-tap FIR feedback.
  large_trapping 1000 uniformly filled bunches x 5e4: h = 4000 with a bunch
                 in every 4th bucket (8 ns), V_RF re-solved so that the
                 reference's formula still gives nu_s = 0.0049; 50 sections,
                 clouds of 2e5 macro-ions per section pre-loaded
                 (preload_clouds), short-range wake as plain_single, HOM and
                 FIR as batched_uneven.

Beam current is not part of those shapes: 1 mA for the single bunch,
0.125 mA per bunch in the 2 ns trains (fast_ion, batched_uneven) and 0.03 mA
per bunch in large_trapping.  The last is the trapping regime the config is
named for: with 8 ns spacing CO (A = 28) is trapped when the critical mass
number N r_p L / (2 sigma_y (sigma_x + sigma_y)) is below 28, which needs
N <~ 2e9 electrons per bunch (0.03 mA gives 21; at 0.125 mA it is 86 and the
pre-loaded clouds are over-focused out of the beam within a few passages).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi

C_LIGHT = 299792458.0
E_CHARGE = 1.602017733e-19

# 9-tap FIR filter of the reference's example input (fbFircoeffx / y)
FIR9_X = [0.5865, 0.5254, -0.0959, -0.3964, -0.2094, -0.0695, -0.2310, -0.2686, 0.1589]
FIR9_Y = [0.7383, -0.2091, -0.4253, 0.1469, 0.1190, 0.0087, 0.0508, -0.3009, -0.1284]


def rf_voltage_for_nus(nus: float, harmonics: int, energy: float = 6.0e9, u0: float = 4.166343e6,
                       alphac1: float = 3.3e-5) -> float:
    """V_RF that gives synchrotron tune nus through the reference's formula
    nu_s^2 = -eta h V cos(phi_s) / (2 pi beta E) with phi_s = pi - asin(U0/V)
    (ReadInputSettings.cpp:1024-1027): V^2 = (2 pi beta E nu_s^2 / (eta h))^2 + U0^2."""
    gamma = energy / 0.51099906e6
    beta = math.sqrt(1.0 - gamma ** -2)
    eta = alphac1 - 1.0 / gamma ** 2
    a = 2 * math.pi * beta * energy * nus ** 2 / (eta * harmonics)
    return math.sqrt(a * a + u0 * u0)


def base_ring(n_sections: int) -> _abi.Ring:
    r = _abi.Ring()
    r.circ_ring = 2304.0
    r.work_qx, r.work_qy = 135.18, 86.27
    r.chrom[:] = [2.0, 2.0]
    r.alphac[:] = [3.3e-5, 1e-4, 0.0]
    r.adtx[:] = [1e3, 1e3, 0, 0, 0]
    r.adty[:] = [1e3, 1e3, 0, 0, 0]
    gamma = 6.0e9 / 0.51099906e6
    t0 = r.circ_ring / C_LIGHT / math.sqrt(1.0 - gamma ** -2)  # revolution time
    r.synch_rad_damp_time[:] = [20e-3 / t0, 20e-3 / t0, 10e-3 / t0]  # in turns
    r.pipe_aperture_x, r.pipe_aperture_y = 0.15, 0.10
    r.electron_energy = 6.0e9
    r.sdelta0 = 9.0e-4
    r.natural_emit = 24e-12
    r.coupling = 0.2
    r.u0 = 4.166343e6
    r.skew_quad_k = 0.0
    r.harmonics = 3840
    r.n_cav = 1
    r.cav_harm[0] = 1
    r.cav_vol[0] = 8.2706e6
    r.cav_phase[0] = 0.0
    return r


def ring_sections(ring: _abi.Ring, n: int, beta: float = 10.0, pressure_pa: float = 1e-9,
                  temperature: float = 300.0, aperture: float = 0.1):
    secs = (_abi.Section * n)()
    for k in range(n):
        s = secs[k]
        s.s = k * ring.circ_ring / n
        s.beta_x = s.beta_y = beta
        s.alpha_x = s.alpha_y = 0.0
        s.psi_x = 2 * math.pi * ring.work_qx * k / n
        s.psi_y = 2 * math.pi * ring.work_qy * k / n
        s.eta_x = s.etap_x = s.eta_y = s.etap_y = 0.0
        s.aperture_x = s.aperture_y = aperture
        s.pressure = pressure_pa
        s.temperature = temperature
    return secs


def bbr(rows) -> _abi.Bbr:
    """rows of (lRs, lQ, lfr, txRs, txQ, txfr, tyRs, tyQ, tyfr), frequencies in
    Hz as in the BBR input file (WakeFunction.cpp:273-281 multiplies by 2 pi)."""
    b = _abi.Bbr()
    b.n = len(rows)
    for i, r in enumerate(rows):
        b.l_rs[i], b.l_q[i], b.l_omega[i] = r[0], r[1], r[2] * 2 * math.pi
        b.tx_rs[i], b.tx_q[i], b.tx_omega[i] = r[3], r[4], r[5] * 2 * math.pi
        b.ty_rs[i], b.ty_q[i], b.ty_omega[i] = r[6], r[7], r[8] * 2 * math.pi
    return b


class Workload:
    """A config plus its bunch layout (the arrays stay alive with the object)."""

    def __init__(self, name, cfg, sections, n_macro, harm, ne, gen):
        self.name = name
        self.cfg = cfg
        self.sections = sections
        self.n_macro = np.ascontiguousarray(n_macro, dtype=np.int32)
        self.harm = np.ascontiguousarray(harm, dtype=np.int32)
        self.ne = np.ascontiguousarray(ne, dtype=np.float64)
        self.gen = gen  # (emit_x, emit_y, sigma_z, sigma_dp)
        self.bbi_table = None

    def set_bbi(self, table, time_domain: int, sim=(1, 1, 1, 1, 1)) -> None:
        """Broadband impedance: `table` is the impedance file's rows (11
        columns, time_domain 0) or the wake file's rows (6 columns,
        time_domain 1); the array stays alive with the workload."""
        cols = 6 if time_domain else 11
        t = np.ascontiguousarray(table, dtype=np.float64).reshape(-1, cols)
        self.bbi_table = t
        b = self.cfg.bbi
        b.flag = 1
        b.time_domain = int(time_domain)
        for i in range(5):
            b.sim[i] = int(sim[i])
        b.n_rows = t.shape[0]
        b.table = t.ctypes.data_as(C.POINTER(C.c_double))

    @property
    def n_bunches(self) -> int:
        return len(self.n_macro)

    @property
    def n_particles(self) -> int:
        return int(self.n_macro.sum())


def make(name: str, n_scale: float = 1.0, turns_lr: int = 10, lib=None, seed: int = 1234,
         derive=None, lattice_init=None, bunch_current: float | None = None) -> Workload:
    """Builds a workload.  `n_scale` scales macroparticle counts (tests use
    small values); `derive(cfg_ref)` / `lattice_init(ring_ref, sections, n)`
    default to the library's own cg_config_derive / cg_lattice_init (the
    oracle's or_config_derive / or_lattice_init take the same arguments, so a
    process that must not load the library passes those)."""
    if derive is None or lattice_init is None:
        L = lib or _abi.load()
        derive = derive or L.cg_config_derive
        lattice_init = lattice_init or L.cg_lattice_init
    if name == "plain_single":
        K, M = 1, 1
        n_macro = [max(1, int(1e5 * n_scale))]
        harm = [0]
    elif name == "fast_ion":
        K, M = 20, 80
        n_macro = [max(1, int(2e4 * n_scale))] * M
        harm = list(range(M))
    elif name == "batched_uneven":
        K, M = 50, 900
        rng = np.random.default_rng(seed)
        n_macro = [max(1, int(v * n_scale)) for v in np.exp(rng.uniform(math.log(5e3), math.log(5e4), M))]
        harm = list(range(M))
    elif name == "large_trapping":
        K, M = 50, 1000
        n_macro = [max(1, int(5e4 * n_scale))] * M
        harm = [4 * j for j in range(M)]
    else:
        raise KeyError(name)
    cfg = _abi.Config()
    cfg.ring = base_ring(K)
    if name == "large_trapping":
        cfg.ring.harmonics = 4000
        cfg.ring.cav_vol[0] = rf_voltage_for_nus(0.0049, 4000)
    if derive(C_ref(cfg)) != 0:
        raise RuntimeError("cg_config_derive failed")
    secs = ring_sections(cfg.ring, K)
    if lattice_init(C_ref(cfg.ring), secs, K) != 0:
        raise RuntimeError("cg_lattice_init failed")
    cfg.n_sections = K
    cfg.sections = C_cast(secs)
    cfg.flag_synrad = 1
    cfg.seed = seed
    if name in ("plain_single", "large_trapping"):
        cfg.flag_sr_wake = 1
        cfg.sr_bins = 100
        cfg.sr_bbr = bbr([(5e3, 1.0, 30e9, 2e6, 1.0, 30e9, 2e6, 1.0, 30e9)])
    if name in ("fast_ion", "batched_uneven", "large_trapping"):
        cfg.flag_beam_ion = 1
        ion = cfg.ion
        ion.n_species = 1
        ion.mass_number[0] = 28.0
        ion.cross_section[0] = 2.0e-22
        ion.gas_percent[0] = 1.0
        ion.loss_boundary = 10.0
        ion.max_ions = 100000 if name != "large_trapping" else 400000
        ion.macro_ions_per_ip = 1
    if name in ("batched_uneven", "large_trapping"):
        cfg.flag_lr_wake = 1
        cfg.lr_turns = turns_lr + 1
        cfg.lr_bbr = bbr([(0.0, 1.0, 1.2e9, 1e6, 1e4, 1.2e9, 1e6, 1e4, 1.2e9)])
        cfg.flag_fir = 1
        f = cfg.fir
        f.mode = 1
        f.delay, f.taps = 1, 9
        f.gain = 1.0
        f.kick_strength[:] = [2e-4, 2e-4, 0.0]
        f.power_limit = 1e6
        f.kicker_imped = 123e3
        for q in range(10):
            f.coeff_x[q] = 0.0 if q < 1 else FIR9_X[q - 1]
            f.coeff_y[q] = 0.0 if q < 1 else FIR9_Y[q - 1]
            f.coeff_z[q] = 0.0
        f.n_sections = 1
        f.start[0], f.end[0] = 0, 1 << 30
    f0 = cfg.ring.f0
    # 1 mA for the single bunch; 0.125 mA per bunch in the trains (N_e = 6e9,
    # the regime where CO ions are trapped inside the train: critical mass
    # number ~23 < 28 for 2 ns spacing)
    current = {"plain_single": 1e-3, "large_trapping": 0.03e-3}.get(name, 0.125e-3)
    if bunch_current is not None:
        current = bunch_current
    ne = [current / f0 / E_CHARGE] * M
    eps_x = cfg.ring.natural_emit / (1 + cfg.ring.coupling)
    eps_y = eps_x * cfg.ring.coupling
    return Workload(name, cfg, secs, n_macro, harm, ne, (eps_x, eps_y, 2.5e-3, 9.0e-4))


def preload_clouds(wl: Workload, n_ions: int = 200000, seed: int = 4321):
    """Accumulated clouds for every section (species 0): n_ions macro-ions at
    rest, Gaussian with the beam's transverse sizes at the section
    (sqrt(eps beta)) about the axis, from a seeded generator.  Returns a list
    of (x, y, vx, vy) per section."""
    rng = np.random.default_rng(seed)
    ex, ey = wl.gen[0], wl.gen[1]
    out = []
    for k in range(wl.cfg.n_sections):
        s = wl.sections[k]
        x = rng.normal(0.0, math.sqrt(ex * s.beta_x), n_ions)
        y = rng.normal(0.0, math.sqrt(ey * s.beta_y), n_ions)
        out.append((x, y, np.zeros(n_ions), np.zeros(n_ions)))
    return out


def C_ref(x):
    import ctypes
    return ctypes.byref(x)


def C_cast(secs):
    import ctypes
    return ctypes.cast(secs, ctypes.POINTER(_abi.Section))
