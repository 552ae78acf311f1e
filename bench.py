"""Benchmark: fast-ion multi-particle tracking turns on B200.

Workload (one step = one full turn of MPBeam::Run order, MPBeam.cpp:1010-1102):
80 bunches x 2e4 FP64 macroparticles in consecutive 2 ns buckets, 20
interaction points (beta = 10 m), CO ions at 1e-9 Pa with one macro-ion per
bunch passage per IP, exact Bassetti-Erskine kicks both ways through the
FP64 Faddeeva kernel, synchrotron radiation with quantum excitation.

  value  macroparticle-turns/s with the beam resident in HBM (device time of
         K turns by CUDA events on the library's stream, L2 flushed between
         turns: the 77 MB state would otherwise stay in the 126 MB L2)
  e2e    the same through the C ABI with the beam uploaded from pinned host
         memory and the per-bunch moments read back every turn
  roofline  the electron-side field-kick kernel (the largest FP64 kernel of
         the turn) against the FP64 FMA throughput measured on this GPU
  cpu_baseline  the CPU oracle (OpenMP over particles) on a bounded sample

--impl reference times the reference algorithm on the host cores (the oracle
restatement; the reference's own tracking sources do not build here).
Multi-GPU: one process per GPU (torchrun), each an independent replica of the
workload (weak scaling); timing is the max over ranks.
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

BATCHED_DESC = ("batched_uneven: 900 of 1000 buckets filled, 5e3-5e4 FP64 macroparticles "
                "per bunch (log-uniform), 50 IPs, CO ions, exact Bassetti-Erskine both ways, "
                "long-range HOM wake, 9-tap FIR, synchrotron radiation with quantum excitation")
WORKLOAD_DESC = ("fast_ion: 80 bunches x 2e4 FP64 macroparticles, 2 ns spacing, 20 IPs, "
                 "CO at 1e-9 Pa, 1 macro-ion/bunch/IP, exact Bassetti-Erskine both ways, "
                 "synchrotron radiation with quantum excitation")


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


def cpu_sample(turns: int = 1, n_scale: float = 0.025, threads: int | None = None):
    """Oracle timing on a bounded sample of the workload: 80 bunches x 500
    macroparticles, all 20 IPs, `turns` turns.  Returns (value, seconds, n)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(threads or os.cpu_count() or 1))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    from helpers import particles, small
    wl = small("fast_ion", n_scale)
    o = oracle.OracleBeam(wl)
    for j, c in enumerate(particles(wl, seed=3, spread=2.0)):
        o.upload(j, c)
    t = time.perf_counter()
    o.Run(0, turns)
    dt = time.perf_counter() - t
    return wl.n_particles * turns / dt, dt, wl.n_particles


def run_reference(args, rank):
    if rank != 0:
        return
    from cetasim_b200 import build
    build.build_oracle()
    vals = []
    n = 0
    for s in range(args.warmup + args.steps):
        v, dt, n = cpu_sample(turns=1)
        if s >= args.warmup:
            vals.append(dt)
    tot = sum(vals)
    value = n * len(vals) / tot
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    sample = (f"80 bunches x {n // 80} macroparticles (of 2e4), 20 IPs, 1 turn per step; "
              "oracle restatement in C with OpenMP over particles")
    line = {"impl": "reference", "metric": "macroparticle-turns/s", "value": value,
            "unit": "macroparticle-turns/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(vals), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_DESC, "sample": sample},
            "cpu_baseline": {"value": value, "unit": "macroparticle-turns/s", "cores": cores,
                             "kind": "port", "sample": sample},
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
    ap.add_argument("--no-surrogate", action="store_true",
                    help="skip the surrogate measurement (training + surrogate turns)")
    ap.add_argument("--kick-variant", type=int, default=None, metavar="V",
                    help="kick shape V (0-3; 4-7: the same inside the map pass) instead of "
                         "the kick autotuner")
    ap.add_argument("--pipeline", default=None, metavar="G:IONS:RAMP",
                    help="pipeline shape (walk segments, ions per walk CTA, ramp 0/1) instead "
                         "of the whole-turn pipeline autotuner")
    ap.add_argument("--workload", default="fast_ion", choices=["fast_ion", "batched_uneven"],
                    help="batched_uneven: 900 bunches of 5e3-5e4, 50 IPs, LR wake + FIR")
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
    if args.kick_variant is not None:
        beam.set_kick_variant(args.kick_variant)
        tune = (args.kick_variant, None)
    else:
        tune = beam.autotune(0, reps=10)
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
    ion_kicks_turn = n_part * wl.cfg.n_sections  # electron-side kicks (dominant)

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

    # dominant FP64 kernel: electron-side ion kick at IP 0, timed alone
    beam.MPBeamRMSCal(0)
    beam.SSBeamIonEffectOneInteractionPoint(10**6, 0)
    kick_ms = C.c_double()
    beam._check(lib.cg_time_stage(beam.h, 1, 0, 20, C.byref(kick_ms)))
    map_ms = C.c_double()
    beam._check(lib.cg_time_stage(beam.h, 0, 0, 20, C.byref(map_ms)))
    chain_ms = C.c_double()
    beam._check(lib.cg_time_stage(beam.h, 2, 0, 5, C.byref(chain_ms)))
    mom_ms = C.c_double()
    beam._check(lib.cg_time_stage(beam.h, 3, 0, 20, C.byref(mom_ms)))
    pass_ms = C.c_double()
    beam._check(lib.cg_time_stage(beam.h, 5, 0, 20, C.byref(pass_ms)))
    tail_ms = C.c_double()
    beam._check(lib.cg_time_stage(beam.h, 4, 0, 5, C.byref(tail_ms)))
    peak = C.c_double()
    lib.cg_fp64_peak(C.byref(peak))
    flops_per_kick = FLOPS_PER_KICK
    achieved = n_part * flops_per_kick / (kick_ms.value * 1e-3)
    traffic = kick_traffic() if args.workload == "fast_ion" else None
    sur = None
    if world == 1 and not args.no_surrogate:
        sur = surrogate_leg(args, beam, lib, stream, flush, kick_ms.value, tot_ms / args.steps)

    result = None
    if rank == 0:
        cpu = None
        if not args.no_cpu and world == 1 and args.workload == "fast_ion":
            try:
                v, dt, n = cpu_sample(turns=1)
                cpu = {"value": v, "unit": "macroparticle-turns/s",
                       "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
                       "kind": "port",
                       "sample": f"80 bunches x {n // 80} macroparticles, 20 IPs, 1 turn "
                                 f"({dt:.1f} s); C oracle, OpenMP over particles"}
            except Exception as e:  # the baseline is reported, never required
                cpu = {"value": None, "unit": "macroparticle-turns/s", "cores": 0, "kind": "port",
                       "sample": f"failed: {e}"}
        result = {
            "metric": "macroparticle-turns/s", "value": value, "unit": "macroparticle-turns/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if shard else "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_DESC if args.workload == "fast_ion" else
                       BATCHED_DESC, "bunches": wl.n_bunches,
                       "macroparticles": n_part, "interaction_points": wl.cfg.n_sections,
                       "turns_per_step": 1, "l2": "flushed between turns (512 MB write)",
                       "parallelism": (f"bunch-sharded x{world} (moments all-gathered per IP)"
                                       if shard else f"replica x{world}")},
            "ion_kicks_per_s": copies * ion_kicks_turn * args.steps / (tot_ms * 1e-3),
            "kernels_ms": {"ion_field_kick": kick_ms.value, "section_map": map_ms.value,
                           "moments": mom_ms.value, "ion_chain": chain_ms.value,
                           "map_moments_pass": pass_ms.value,
                           "longitudinal_tail": tail_ms.value},
            "roofline": {"bound": "fp64", "kernel": "k_ion_kick (electron-side Bassetti-Erskine)",
                         "achieved": achieved / 1e12, "peak": peak.value / 1e12, "unit": "TFLOP/s",
                         "frac": achieved / peak.value if peak.value else None,
                         "peak_source": "measured FP64 FMA throughput (cg_fp64_peak)",
                         "algorithmic_flops_per_kick": flops_per_kick, "traffic": traffic,
                         "traffic_source": "profiles/k_ion_kick_fast_ion.md (ncu, one segment launch scaled to the full beam by tiles)"},
            "ion_chain": {"us_per_ip": 1e3 * chain_ms.value,
                          "us_per_bunch_step": 1e3 * chain_ms.value / wl.n_bunches,
                          "bound": "latency (one field evaluation per bunch step)"},
            "cpu_baseline": cpu,
            "autotune": {"kick_shapes_ms": None if tune[1] is None else
                         [round(float(x), 5) for x in tune[1][:-2]],
                         "map_pass_ms": None if tune[1] is None else round(float(tune[1][-2]), 5),
                         "map_pass_with_kick_ms": None if tune[1] is None else
                         round(float(tune[1][-1]), 5),
                         "chosen_shape": int(tune[0]) % 4,
                         "kick_in_map_pass": bool(tune[0] >= 4),
                         "shapes": ["256 thr x3/SM", "256 thr x4/SM", "128 thr x4/SM",
                                    "128 thr x6/SM"],
                         "pipeline": None if pipe is None else {
                             "segments": pipe[0][0], "walk_ions": pipe[0][1],
                             "ramp": bool(pipe[0][2]),
                             "turn_ms": None if pipe[1] is None else {
                                 f"{g}x{w}{'r' if r else ''}": round(float(m), 4)
                                 for (g, w, r), m in zip(_abi.PIPE_SHAPES, pipe[1])}}},
            "surrogate": sur,
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


def surrogate_leg(args, beam, lib, stream, flush, exact_kick_ms, exact_turn_ms):
    """The learned field in place of the exact one: trains the surrogate on the
    GPU (2^20 exact-field samples), then times its kick kernel and whole turns
    with it, the same way as the exact path."""
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
    return {"network": "3-64-64-64-2 SiLU, BF16 weights, FP32 accumulation, tcgen05",
            "holdout_rms_rel": st[1], "holdout_max_rel": st[2], "train_s": st[3],
            "kick_ms": k_ms.value, "exact_kick_ms": exact_kick_ms,
            "kick_speedup": exact_kick_ms / k_ms.value,
            "ion_kicks_per_s_kernel": n / (k_ms.value * 1e-3),
            "ms_per_turn": turn_ms, "exact_ms_per_turn": exact_turn_ms,
            "turn_speedup": exact_turn_ms / turn_ms,
            "audit_max_field_err_rel": audit[0] / audit[1] if audit[1] else None}


def kick_traffic():
    """DRAM bytes per k_ion_kick launch from the committed ncu summary."""
    import re
    try:
        txt = open(os.path.join(ROOT, "profiles", "k_ion_kick_fast_ion.md")).read()
    except OSError:
        return None
    # the full-beam line (the last one of the summary)
    m = re.findall(r"dram bytes read / written per launch \| ([\d.]+) MB / ([\d.]+) MB", txt)
    return (float(m[-1][0]) + float(m[-1][1])) * 1e6 if m else None

if __name__ == "__main__":
    main()
