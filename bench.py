"""Benchmark: multi-particle tracking turns (MPBeam::Run order,
MPBeam.cpp:1010-1102) on B200.  One step = one full turn of the workload.

Workloads (--workload; default batched_uneven, the shape the surrogate
target is stated on):
  plain_single    config 0: 1 bunch x 1e5, 1 IP, short-range BBR wake (100
                  bins), synchrotron radiation with quantum excitation
  fast_ion        config 1: 80 bunches x 2e4, 20 IPs, CO ions, exact
                  Bassetti-Erskine kicks both ways
  batched_uneven  config 3: 900 of 1000 buckets filled, 5e3-5e4 macroparticles
                  per bunch (log-uniform), 50 IPs, CO ions, long-range HOM
                  wake, 9-tap FIR; the learned-field arm ("surrogate") beside
                  the exact path
  large_trapping  config 4: 1000 bunches x 5e4 (every 4th bucket of h = 4000),
                  clouds of 2e5 macro-ions per IP pre-loaded, 50 IPs, short-
                  range wake, HOM, FIR

  value     macroparticle-turns/s of the exact path with the beam resident in
            HBM (device time of K turns by CUDA events on the library's
            stream, L2 flushed before every turn)
  e2e       the same through the C ABI with the beam uploaded from pinned host
            memory and the per-bunch moments read back every turn
  roofline  every kernel of the turn with its own bound; the one with the
            largest share of the turn first
  cpu_baseline  the reference's own build (oracle/_ref) on the host cores

--impl reference times the reference's own CPU code (its src/*.cpp built in
oracle/_ref) on the same workload at full particle counts, one process per
host core, each holding a contiguous slice of the train: a step is one
interaction point of the turn loop over the whole train, and a turn is
extrapolated as (IPs x step) + the once-per-turn stages, both measured.
Multi-GPU: one process per GPU (torchrun), each an independent replica
(weak scaling) or, with --shard, one beam split by bunches; timing is the
max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DESC = {
    "plain_single": ("config 0 plain_single: 1 bunch x 1e5 FP64 macroparticles, 1 IP, short-range "
                     "BBR wake (5 kOhm / 2 MOhm/m, 30 GHz, Q = 1, 100 bins), synchrotron radiation "
                     "with quantum excitation"),
    "fast_ion": ("config 1 fast_ion: 80 bunches x 2e4 FP64 macroparticles, 2 ns spacing, 20 IPs, "
                 "CO at 1e-9 Pa, 1 macro-ion/bunch/IP, exact Bassetti-Erskine both ways, "
                 "synchrotron radiation with quantum excitation"),
    "batched_uneven": ("config 3 batched_uneven: 900 of 1000 buckets filled, 5e3-5e4 FP64 "
                       "macroparticles per bunch (log-uniform), 50 IPs, CO ions, long-range HOM "
                       "wake (1.2 GHz, 1 MOhm/m, Q = 1e4), 9-tap FIR, synchrotron radiation with "
                       "quantum excitation; value = exact Bassetti-Erskine path, learned-field arm "
                       "in 'surrogate'"),
    "large_trapping": ("config 4 large_trapping: 1000 bunches x 5e4 FP64 macroparticles (every 4th "
                       "bucket of h = 4000), 2e5 pre-loaded macro-ions per IP, 50 IPs, short-range "
                       "wake, long-range HOM wake, 9-tap FIR, synchrotron radiation with quantum "
                       "excitation, exact Bassetti-Erskine both ways"),
}


# the kick kernel's shapes in the order of cg_autotune's timings
KICK_SHAPES = ["256 thr x3/SM", "256 thr x4/SM", "128 thr x4/SM", "128 thr x6/SM",
               "256 thr x3/SM, 4 tiles per CTA", "128 thr x6/SM, 2 tiles per CTA",
               "128 thr x6/SM, 4 tiles per CTA", "256 thr x3/SM, 8 tiles per CTA"]


class ClockSampler:
    """Clock and throttle-reason samples while the timed region runs: NVML
    polled every 5 ms (read-only), or nvidia-smi every 200 ms where NVML is
    not available."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.source = "nvidia-smi"
        self._stop = threading.Event()
        self._t = None

    def _nvml(self):
        """The NVML handle of this process's CUDA device, or None."""
        try:
            import pynvml
            pynvml.nvmlInit()
            try:  # the CUDA device by its PCI address (NVML's indices may differ)
                import torch
                pr = torch.cuda.get_device_properties(self.index)
                bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
                return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            except Exception:
                return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)
        except Exception:
            return None

    def _run_nvml(self, nv, h):
        bits = [getattr(nv, "nvmlClocksEventReason" + n) for n in
                ("HwSlowdown", "HwThermalSlowdown", "SwThermalSlowdown", "SwPowerCap")]
        reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons",
                          getattr(nv, "nvmlDeviceGetCurrentClocksThrottleReasons", None))
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self._stop.is_set():
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            r = reasons(h)
            flags = ["Active" if r & b else "Not Active" for b in bits]
            self.samples.append([str(self.index), str(sm), str(mx), "", hex(r)] + flags)
            self._stop.wait(0.005)

    def _run(self):
        got = self._nvml()
        if got is not None:
            try:
                self.source = "nvml"
                self._run_nvml(*got)
                return
            except Exception:
                self.samples.clear()
                self.source = "nvidia-smi"
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([s.strip() for s in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 5 + i and s[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples), "source": self.source}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _ref_gen(wl, j, seed):
    """Seeded Gaussian macroparticles of bunch j (the same for any slicing)."""
    rng = np.random.default_rng([seed, j])
    ex, ey, sz, sdp = wl.gen
    s0 = wl.sections[0]
    n = int(wl.n_macro[j])
    c = np.empty((6, n))
    for d, sig in enumerate((np.sqrt(ex * s0.beta_x), np.sqrt(ex / s0.beta_x), np.sqrt(ey * s0.beta_y),
                             np.sqrt(ey / s0.beta_y), sz, sdp)):
        c[d] = rng.normal(0.0, sig, n)
    return c


def _ref_slice(spec):
    """One worker of the reference arm: the reference's own MP code
    (oracle/_ref/libcetasim_ref.so) on bunches [a, b) of the workload at full
    particle counts.  Times `nsteps` IP sections of the turn loop
    (MPBeam.cpp:1059-1070: moments, ion chain, map, moments) and once the
    per-turn stages (RF, drift, energy loss, damping, wakes, FIR, losses)."""
    import tempfile
    sys.path.insert(0, ROOT)
    import oracle
    from cetasim_b200 import configs, input_dat
    from oracle import ref
    name, n_scale, a, b, nsteps, seed = spec
    wl = configs.make(name, n_scale=n_scale, derive=oracle.config_derive,
                      lattice_init=oracle.lattice_init)
    cl = configs.preload_clouds(wl) if name == "large_trapping" else None
    parts = [_ref_gen(wl, j, seed) for j in range(a, b)]
    wl.n_macro, wl.harm, wl.ne = wl.n_macro[a:b].copy(), wl.harm[a:b].copy(), wl.ne[a:b].copy()
    with tempfile.TemporaryDirectory() as d:
        path = input_dat.write_case(d, wl, n_turns=1)
        r = ref.RefBeam(path, seed=seed)
        for j, c in enumerate(parts):
            r.upload(j, c)
        del parts
        if cl is not None:
            for k, (x, y, vx, vy) in enumerate(cl):
                r.upload_ions(k, 0, x, y, vx, vy)
        K = wl.cfg.n_sections
        times = []
        for s in range(nsteps):
            k = s % K
            t = time.perf_counter()
            r.MPBeamRMSCal(k)
            if wl.cfg.flag_beam_ion:
                r.SSBeamIonEffectOneInteractionPoint(0, k)
            r.BeamTransferPerInteractionPointDueToLatticeT(k)
            r.stage(ref.ST_RMS_ONLY, 0, k)
            times.append(time.perf_counter() - t)
        t = time.perf_counter()
        r.BeamMomtumUpdateDueToRFTest()
        r.BeamLongiPosTransferOneTurn()
        r.BeamEnergyLossOneTurn()
        if wl.cfg.flag_synrad:
            r.BeamSynRadDamping(0)
        if wl.cfg.flag_lr_wake:
            r.LRWakeBeamIntaction()
        if wl.cfg.flag_sr_wake:
            r.SRWakeBeamIntaction(1)
        r.stage(ref.ST_RMS_ONLY, 0, 0)
        if wl.cfg.flag_fir:
            r.FIRBunchByBunchFeedback(0)
        r.MarkParticleLostInBunch()
        tail = time.perf_counter() - t
        r.close()
    return times, tail, int(wl.n_macro.sum())


def reference_cpu(workload, n_scale, nsteps, workers=None, seed=7):
    """The reference's own CPU code on the workload: P processes (one per
    host core, at most one per bunch), slices balanced by macroparticle
    count.  Returns a dict with the extrapolated turn time and
    macroparticle-turns/s (total particles / turn), or None when the
    reference build is absent."""
    import multiprocessing as mp
    from oracle import ref
    if not ref.available():
        return None
    sys.path.insert(0, ROOT)
    from cetasim_b200 import configs
    import oracle
    wl = configs.make(workload, n_scale=n_scale, derive=oracle.config_derive,
                      lattice_init=oracle.lattice_init)
    M, K = wl.n_bunches, wl.cfg.n_sections
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    P = max(1, min(workers or cores, M))
    cum = np.concatenate([[0], np.cumsum(wl.n_macro)])
    cuts = [0] + [int(np.searchsorted(cum, cum[-1] * i / P)) for i in range(1, P)] + [M]
    cuts = sorted(set(cuts))
    specs = [(workload, n_scale, cuts[i], cuts[i + 1], nsteps, seed) for i in range(len(cuts) - 1)]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(len(specs)) as pool:
        res = pool.map(_ref_slice, specs)
    wall = time.perf_counter() - t0
    step = np.max(np.array([r[0] for r in res]), axis=0)  # the slowest slice of each step
    tail = max(r[1] for r in res)
    n = sum(r[2] for r in res)
    turn_s = K * float(np.mean(step)) + tail
    return {"value": n / turn_s, "turn_s": turn_s, "step_s": [float(x) for x in step],
            "tail_s": tail, "processes": len(specs), "particles": n, "wall_s": wall,
            "sample": (f"reference build (its src/*.cpp, oracle/_ref) on all {M} bunches at full "
                       f"particle counts in {len(specs)} processes (contiguous bunch slices); "
                       f"{nsteps} IP sections of the turn loop timed (slowest slice each), turn = "
                       f"{K} x mean IP section + the once-per-turn stages, measured")}


def run_reference(args, rank):
    if rank != 0:
        return
    r = reference_cpu(args.workload, args.n_scale, args.warmup + args.steps)
    if r is None:
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libcetasim_ref.so (the reference's own "
                                         "sources) is not built"}), flush=True)
        return
    # the turn from the timed steps only (the warm-up steps are dropped)
    steps = r["step_s"][args.warmup:]
    K = {"plain_single": 1, "fast_ion": 20}.get(args.workload, 50)
    turn_s = K * float(np.mean(steps)) + r["tail_s"]
    value = r["particles"] / turn_s
    line = {"impl": "reference", "metric": "macroparticle-turns/s", "value": value,
            "unit": "macroparticle-turns/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(steps)),
            "ms_per_turn": 1e3 * turn_s, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": DESC[args.workload], "macroparticles": r["particles"],
                       "turns_per_step": "one IP section of the turn per step (extrapolated turn in "
                                         "ms_per_turn)", "sample": r["sample"]},
            "cpu_baseline": {"value": value, "unit": "macroparticle-turns/s", "cores": r["processes"],
                             "kind": "reference", "sample": r["sample"]},
            "e2e": {"value": value, "unit": "macroparticle-turns/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n-scale", type=float, default=1.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="N > 1: one beam split by bunches over the ranks (strong scaling; "
                         "moments all-gathered over NCCL) instead of N replicas")
    ap.add_argument("--no-widened", action="store_true",
                    help="skip the broadband-impedance and space-charge stage timings")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="skip the surrogate measurement (training + surrogate turns)")
    ap.add_argument("--kick-variant", type=int, default=None, metavar="V",
                    help="kick shape V (0-3; 4-7: the same inside the map pass) instead of "
                         "the kick autotuner")
    ap.add_argument("--map-async", type=int, default=0, choices=[0, 1],
                    help="with --kick-variant: the map-pass form (1 = next chunk in flight)")
    ap.add_argument("--pipeline", default=None, metavar="G:IONS:RAMP",
                    help="pipeline shape (walk segments, ions per walk CTA, ramp 0/1) instead "
                         "of the whole-turn pipeline autotuner")
    ap.add_argument("--workload", default="batched_uneven", choices=list(DESC),
                    help="; ".join(f"{k}: {v}" for k, v in DESC.items()))
    args = ap.parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    from cetasim_b200 import _abi, configs
    from cetasim_b200.beam import MPBeam

    lib = _abi.load()
    wl = configs.make(args.workload, n_scale=args.n_scale, seed=1234 + rank)
    shard = None
    if args.shard and world > 1:
        nid = torch.zeros(128, dtype=torch.uint8, device="cuda")
        if rank == 0:
            nid.copy_(torch.frombuffer(bytearray(MPBeam.nccl_unique_id()), dtype=torch.uint8))
        pg.broadcast(nid, 0)
        shard = (rank, world, bytes(nid.cpu().numpy().tobytes()))
        wl = configs.make(args.workload, n_scale=args.n_scale, seed=1234)  # one beam
    beam = MPBeam(wl, device=local, shard=shard)
    beam.generate(seed=99 if shard else 99 + rank)
    if args.workload == "large_trapping":
        for k, (x, y, vx, vy) in enumerate(configs.preload_clouds(wl)):
            beam.upload_ions(k, 0, x, y, vx, vy)
    copies = 1 if shard else world  # independent beams the ranks advance
    stream = torch.cuda.ExternalStream(lib.cg_stream(beam.h))
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    # one turn to fill the ion records, the kick-shape autotuner on this beam
    # (it leaves the beam as it was), then the warm-up turns (the first one
    # instantiates the turn graph with the chosen shape)
    beam.Run(0, 1)
    ions = bool(wl.cfg.flag_beam_ion)
    if args.kick_variant is not None:
        beam.set_kick_variant(args.kick_variant)
        beam.set_map_async(args.map_async)
        tune = (args.kick_variant, None)
    elif ions:
        tune = beam.autotune(0, reps=10)
    else:
        tune = (0, None)
    t_first = 1
    # pipeline shape (walk segments x walk CTA size) over whole turns; the
    # beam is restored after each trial
    pipe = None
    if args.pipeline:
        g_, w_, r_ = (int(x) for x in args.pipeline.split(":"))
        beam.set_pipeline(g_, w_, bool(r_))
        pipe = ((g_, w_, r_), None)  # given, not tuned
    elif wl.cfg.flag_beam_ion:
        pipe = beam.autotune_pipeline(t_first, reps=3)
    launches = C.c_int()  # of the turn graph as tuned
    lib.cg_turn_launches(beam.h, C.byref(launches))
    beam.Run(t_first, args.warmup)
    barrier()
    times = []
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()  # evict the (L2-resident) beam between turns
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            beam.Run(t_first + args.warmup + s, 1)
            e1.record(stream)
            times.append((e0, e1))
        torch.cuda.synchronize()
    barrier()
    ms = [a.elapsed_time(b) for a, b in times]
    tot_ms = float(sum(ms))
    if pg:
        t = torch.tensor([tot_ms], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        tot_ms = float(t.item())
    n_part = wl.n_particles
    value = copies * n_part * args.steps / (tot_ms * 1e-3)

    # e2e through the C ABI: pinned host beam uploaded every turn, moments read back
    hbufs = []
    for j in beam.local:
        n = int(wl.n_macro[j])
        p = lib.cg_host_alloc(6 * 8 * n)
        arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(6, n))
        c, _ = beam.download(j)
        arr[:] = c
        hbufs.append((p, arr))
    table = (C.c_void_p * (6 * wl.n_bunches))()
    for j, (p, arr) in zip(beam.local, hbufs):
        for d in range(6):
            table[6 * j + d] = arr[d].ctypes.data
    mom = (_abi.BunchMoments * wl.n_bunches)()
    e2e_steps = max(3, args.steps // 2)
    barrier()
    ev = []
    for s in range(e2e_steps + 1):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        beam._check(lib.cg_upload_beam(beam.h, table, None))
        beam.Run(t_first + args.warmup + args.steps + s, 1)
        beam._check(lib.cg_beam_rms(beam.h, 0))
        beam._check(lib.cg_get_moments(beam.h, mom))
        e1.record(stream)
        if s > 0:
            ev.append((e0, e1))
    torch.cuda.synchronize()
    e2e_ms = float(sum(a.elapsed_time(b) for a, b in ev))
    if pg:
        t = torch.tensor([e2e_ms], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = copies * n_part * len(ev) / (e2e_ms * 1e-3)
    h2d = sum(int(wl.n_macro[j]) for j in beam.local) * 48
    d2h = wl.n_bunches * C.sizeof(_abi.BunchMoments)
    for p, _ in hbufs:
        lib.cg_host_free(p)

    # per-kernel device times on the live beam (cg_time_stage: one stage
    # launched `reps` times on the library stream, CUDA events around it)
    def stage_ms(st, reps):
        v = C.c_double()
        beam._check(lib.cg_time_stage(beam.h, st, 0, reps, C.byref(v)))
        return v.value
    K = wl.cfg.n_sections
    beam.MPBeamRMSCal(0)
    if ions:
        beam.SSBeamIonEffectOneInteractionPoint(10 ** 6, 0)
    kms = {"map_moments_pass": stage_ms(5, 20), "moments": stage_ms(3, 20),
           "section_map": stage_ms(0, 20), "longitudinal_tail": stage_ms(4, 5)}
    if ions:
        kms["ion_field_kick"] = stage_ms(1, 20)
        kms["ion_chain"] = stage_ms(2, 5)
    peak64 = C.c_double()
    lib.cg_fp64_peak(C.byref(peak64))
    hbm = measured_peak("hbm_gbs")
    n_part = wl.n_particles
    kernels = []
    # the map + moments pass: 6 FP64 read + written and the survival byte
    # read once per particle (97 B), HBM-bound
    mp_bytes = 97.0 * n_part
    kernels.append({"kernel": "k_map_pass (section map + next IP's moments)", "bound": "hbm",
                    "per_turn_ms": K * kms["map_moments_pass"],
                    "achieved": mp_bytes / (kms["map_moments_pass"] * 1e-3) / 1e9,
                    "peak": hbm[0], "unit": "GB/s", "peak_source": hbm[1],
                    "algorithmic_bytes": mp_bytes})
    if ions:
        fl = FLOPS_PER_KICK * n_part
        kernels.append({"kernel": "k_ion_kick (electron-side Bassetti-Erskine)", "bound": "fp64",
                        "per_turn_ms": K * kms["ion_field_kick"],
                        "achieved": fl / (kms["ion_field_kick"] * 1e-3) / 1e12,
                        "peak": peak64.value / 1e12, "unit": "TFLOP/s",
                        "peak_source": "FP64 FMA throughput measured by cg_fp64_peak",
                        "algorithmic_flops": fl})
        lat = C.c_double()
        beam._check(lib.cg_field_chain_latency(C.byref(lat)))
        steps = wl.n_bunches
        # ion-side field evaluations of one IP: the ions alive at each bunch
        # step (the cloud records of IP 0 left by the timed chain)
        ion_kicks = float(beam.cloud_record(0)[:, :, 5].sum())
        chain_fl = FLOPS_PER_KICK * ion_kicks / (kms["ion_chain"] * 1e-3)
        entry = {"kernel": "ion chain (k_ion_prep/walk/records/compact)",
                 "per_turn_ms": K * kms["ion_chain"], "ion_kicks_per_ip": ion_kicks,
                 "bunch_steps_per_ip": steps, "us_per_bunch_step": 1e3 * kms["ion_chain"] / steps,
                 "latency_floor_us": lat.value,
                 "latency_floor_source": "the walk's own step arithmetic for one ion, "
                                         "measured by cg_field_chain_latency",
                 "fp64_tflops": chain_fl / 1e12}
        if chain_fl > 0.2 * peak64.value:
            # many ions per step: the chain is a throughput kernel
            entry.update({"bound": "fp64", "achieved": chain_fl / 1e12, "peak": peak64.value / 1e12,
                          "unit": "TFLOP/s",
                          "peak_source": "FP64 FMA throughput measured by cg_fp64_peak"})
        else:
            # few ions per step: one dependent field evaluation per bunch step
            entry.update({"bound": "latency", "achieved": 1e3 * kms["ion_chain"] / steps,
                          "peak": lat.value, "unit": "us per bunch step (lower is better)",
                          "peak_source": entry["latency_floor_source"]})
        kernels.append(entry)
    # the once-per-turn longitudinal tail: RF, drift, loss, damping, wakes,
    # FIR, losses; one read and write of the state
    kernels.append({"kernel": "longitudinal tail (k_long, wakes, FIR, k_mark_lost)", "bound": "hbm",
                    "per_turn_ms": kms["longitudinal_tail"],
                    "achieved": mp_bytes / (kms["longitudinal_tail"] * 1e-3) / 1e9,
                    "peak": hbm[0], "unit": "GB/s", "peak_source": hbm[1],
                    "algorithmic_bytes": mp_bytes})
    for kk in kernels:
        a_, p_ = kk["achieved"], kk["peak"]
        kk["frac"] = (p_ / a_ if kk["bound"] == "latency" else a_ / p_) if a_ and p_ else None
    kernels.sort(key=lambda kk: -kk["per_turn_ms"])
    top = dict(kernels[0])
    top["traffic"] = kernel_traffic(args.workload, top["kernel"])
    top["kernels"] = kernels
    sur = None
    if world == 1 and ions and not args.no_surrogate:
        sur = surrogate_leg(args, beam, lib, stream, flush, kms["ion_field_kick"], tot_ms / args.steps,
                            clk.summary().get("sm_max_mhz"))

    widened = None
    if world == 1 and not args.no_widened:
        try:
            widened = widened_leg(measured_peak("hbm_gbs"))
        except Exception as e:  # reported, never required
            widened = {"failed": str(e)}

    result = None
    if rank == 0:
        cpu = None
        if not args.no_cpu and world == 1:
            try:
                r = reference_cpu(args.workload, args.n_scale, 4)
                if r is not None:
                    cpu = {"value": r["value"], "unit": "macroparticle-turns/s",
                           "cores": r["processes"], "kind": "reference",
                           "sample": r["sample"] + f"; {r['wall_s']:.1f} s wall"}
            except Exception as e:  # the baseline is reported, never required
                cpu = {"value": None, "unit": "macroparticle-turns/s", "cores": 0,
                       "kind": "reference", "sample": f"failed: {e}"}
        result = {
            "metric": "macroparticle-turns/s", "value": value, "unit": "macroparticle-turns/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if shard else "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": DESC[args.workload], "bunches": wl.n_bunches,
                       "macroparticles": n_part, "interaction_points": K,
                       "turns_per_step": 1, "l2": "flushed between turns (512 MB write)",
                       "parallelism": (f"bunch-sharded x{world} (moments all-gathered per IP)"
                                       if shard else f"replica x{world}")},
            "ion_kicks_per_s": (copies * n_part * K * args.steps / (tot_ms * 1e-3)) if ions else None,
            "kernels_ms": kms,
            "roofline": top,
            "cpu_baseline": cpu,
            "autotune": {"kick_shapes_ms": None if tune[1] is None else
                         [round(float(x), 5) for x in tune[1][:-4]],
                         "map_pass_ms": None if tune[1] is None else round(float(tune[1][-4]), 5),
                         "map_pass_with_kick_ms": None if tune[1] is None else
                         round(float(tune[1][-3]), 5),
                         "map_pass_async_ms": None if tune[1] is None else
                         round(float(tune[1][-2]), 5),
                         "map_pass_async_with_kick_ms": None if tune[1] is None else
                         round(float(tune[1][-1]), 5),
                         "map_async": beam.map_async(),
                         "chosen_shape": int(tune[0]) % len(KICK_SHAPES),
                         "kick_in_map_pass": bool(tune[0] >= len(KICK_SHAPES)),
                         "shapes": KICK_SHAPES,
                         "pipeline": None if pipe is None else {
                             "segments": pipe[0][0], "walk_ions": pipe[0][1],
                             "ramp": bool(pipe[0][2]),
                             "turn_ms": None if pipe[1] is None else {
                                 f"{g}x{w}{'r' if r else ''}": round(float(m), 4)
                                 for (g, w, r), m in zip(_abi.PIPE_SHAPES, pipe[1])}}},
            "surrogate": sur,
            "widened_stages": widened,
            "e2e": {"value": e2e_value, "unit": "macroparticle-turns/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches.value * args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(result), flush=True)
    beam.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return result


# FP64 operations of one electron-side kick (two w(z) through the Weideman
# series evaluated by Knuth's real recurrence, the exp of the Gaussian factor
# counted as one operation, and the field algebra), counted from
# be_field.cuh / faddeeva.cuh: per w(z) 3 (branch test) + 24 (Z and the Newton
# reciprocal) + 4 (r, s) + 150 (38 recurrence steps) + 5 (p) + 20 (w from p);
# 2 x 203 + 32.
FLOPS_PER_KICK = 438


def measured_peak(key):
    """(value, source) of a peak from MEASURED_PEAKS.json beside this file,
    else the pool's earlier measurement."""
    fallback = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            v = json.load(f).get(key)
        if v:
            return float(v), f"measured ({key}, MEASURED_PEAKS.json)"
    except (OSError, ValueError):
        pass
    return fallback[key], f"fallback ({key} of an earlier measurement on this pool)"


def widened_leg(hbm):
    """The stages beyond the ion hot path on the 80-bunch fast-ion train at
    full size (80 x 2e4 macroparticles): the broadband-impedance kick
    (frequency domain, 640 impedance samples to 300 GHz; time domain, a
    400-sample wake table) and the space charge at one section (2.5-D PIC on
    32 x 32 x 33, and the Bassetti-Erskine slices).  Each is the time of one
    host-synchronous C-ABI call (launches and the status read included),
    averaged over 20 after 3 warm-up calls; achieved = the stage's algorithmic
    bytes (read z, x, y and read-write px, py, dp: 72 B per macroparticle)
    over that time, against the measured copy bandwidth."""
    from cetasim_b200 import configs
    from cetasim_b200.beam import MPBeam

    def resonators(n, fmax):
        f = np.arange(n) * (fmax / (n - 1))
        t = np.zeros((n, 11))
        t[:, 0] = f
        with np.errstate(divide="ignore", invalid="ignore"):
            for p, (rs, fr) in enumerate(((2e4, 40e9), (4e5, 30e9), (4e5, 30e9), (1e5, 30e9), (1e5, 30e9))):
                z = rs / (1 + 1j * (fr / f - f / fr)) * (fr / f if p else 1.0)
                z[0] = 0
                t[:, 1 + p], t[:, 6 + p] = z.real, z.imag
        return t

    def wake(nw, dzw, cen):
        z = (np.arange(nw) - cen) * dzw
        env = np.exp(-0.5 * (z / 1.5e-3) ** 2) + np.where(z > 0, np.exp(-z / 20e-3), 0.0)
        t = np.zeros((nw, 6))
        t[:, 0] = z
        for p, a in enumerate((3e13, 2e15, 2e15, 5e14, 5e14)):
            t[:, 1 + p] = a * env * np.cos(2 * np.pi * z / 6e-3 + 0.3 * p)
        t[cen, 0] = 0.0
        return t

    def timed(fn, reps=20):
        for _ in range(3):
            fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        return (time.perf_counter() - t0) / reps * 1e3

    out = {"workload": "fast_ion train at full size: 80 bunches x 2e4 macroparticles",
           "timing": "host-synchronous C-ABI call, mean of 20 after 3 warm-up",
           "peak_gbs": hbm[0], "peak_source": hbm[1]}
    cases = [("bbi_frequency_domain", "bbi", 0, resonators(640, 300e9)),
             ("bbi_time_domain", "bbi", 1, wake(400, 0.5e-3, 40)),
             ("space_charge_pic_32x32x33", "sc", 2, None),
             ("space_charge_bassetti_erskine", "sc", 1, None)]
    for name, kind, mode, table in cases:
        wl = configs.make("fast_ion", n_scale=1.0)
        wl.cfg.flag_beam_ion = 0
        if kind == "bbi":
            wl.set_bbi(table, mode)
        else:
            wl.cfg.flag_sc = mode
            for i, v in enumerate((32, 32, 33)):
                wl.cfg.sc_mesh[i] = v
        b = MPBeam(wl)
        b.generate(seed=3)
        b.MPBeamRMSCal(0)
        ms = timed(b.BBImpBeamInteraction if kind == "bbi" else (lambda: b.BeamTransferDueToSpaceCharge(0)))
        gbs = 72.0 * wl.n_particles / (ms * 1e-3) / 1e9
        out[name] = {"ms": ms, "achieved_gbs": gbs, "frac": gbs / hbm[0] if hbm[0] else None}
        b.close()
    return out


def surrogate_leg(args, beam, lib, stream, flush, exact_kick_ms, exact_turn_ms, sm_mhz):
    """The learned field in place of the exact one: trains the surrogate on the
    GPU (2^20 exact-field samples), then times its kick kernel and whole turns
    with it, the same way as the exact path, and audits it against the exact
    field on the live beam."""
    import torch
    from cetasim_b200 import surrogate as S
    w, st = S.train()
    beam.set_surrogate(w)
    k_ms = C.c_double()
    beam._check(lib.cg_time_stage(beam.h, 6, 0, 20, C.byref(k_ms)))
    t0 = 10 ** 6
    beam.Run(t0, 2)
    ev = []
    for s in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        beam.Run(t0 + 2 + s, 1)
        e1.record(stream)
        ev.append((e0, e1))
    torch.cuda.synchronize()
    turn_ms = sum(a.elapsed_time(b) for a, b in ev) / len(ev)
    audit = beam.surrogate_audit(beam.wl.cfg.n_sections - 1)
    beam.set_surrogate(None)
    n = beam.wl.n_particles
    K = beam.wl.cfg.n_sections
    peak = measured_peak("bf16_tflops")
    bf16 = 17024.0 * n / (k_ms.value * 1e-3) / 1e12
    # the unit that bounds the network: every SiLU takes an exponential and a
    # reciprocal on the multi-function unit (16 results per clock per SM), 192
    # SiLU per sample
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mufu_ms = 384.0 * n / (16.0 * sms * (sm_mhz or 1965.0) * 1e6) * 1e3
    return {"network": "3-64-64-64-2 SiLU, BF16 weights, FP32 accumulation, tcgen05",
            "holdout_rms_rel": st[1], "holdout_max_rel": st[2], "train_s": st[3],
            "field_error_target": 1e-3,
            "audit_max_field_err_rel": audit[0] / audit[1] if audit[1] else None,
            "kick_ms": k_ms.value, "exact_kick_ms": exact_kick_ms,
            "ion_kicks_per_s_kernel": n / (k_ms.value * 1e-3),
            "exact_ion_kicks_per_s_kernel": n / (exact_kick_ms * 1e-3),
            "kick_speedup": exact_kick_ms / k_ms.value,
            "ion_kicks_per_s": n * K / (turn_ms * 1e-3),
            "exact_ion_kicks_per_s": n * K / (exact_turn_ms * 1e-3),
            "ms_per_turn": turn_ms, "exact_ms_per_turn": exact_turn_ms,
            "turn_speedup": exact_turn_ms / turn_ms, "target_speedup": 5.0,
            "kick_bf16_tflops": bf16, "kick_bf16_frac": bf16 / peak[0],
            "bf16_peak_source": peak[1],
            "roofline": {"bound": "mufu", "unit": "ms per kick launch (lower is better)",
                         "achieved": k_ms.value, "peak": mufu_ms, "frac": mufu_ms / k_ms.value,
                         "peak_source": "384 MUFU operations per sample (192 SiLU x (exp, rcp)) "
                                        "at 16 per clock per SM, SM count and max SM clock"}}


def kernel_traffic(workload, kernel):
    """DRAM bytes per launch of a kernel from the committed ncu summary of
    that kernel on that workload (profiles/<kernel>_<workload>.md, the line
    'dram bytes read / written per launch | R MB / W MB'), or None."""
    import re
    name = kernel.split()[0]
    if name == "ion":
        name = "k_ion_walk"
    try:
        txt = open(os.path.join(ROOT, "profiles", f"{name}_{workload}.md")).read()
    except OSError:
        return None
    m = re.findall(r"dram bytes read / written per launch \| ([\d.]+) MB / ([\d.]+) MB", txt)
    return (float(m[-1][0]) + float(m[-1][1])) * 1e6 if m else None


if __name__ == "__main__":
    main()
