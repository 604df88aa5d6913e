#!/usr/bin/env python
"""Benchmark of the B200 interpolated mode sum (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision faithful|exact]
    python bench.py --impl reference ...      # the reference's CPU path, timed on the host cores

Workload (one "step" = one waveform through InterpolatedModeSum): the plain
FP64 one-year waveform, K=3843 modes (l=2..10, m=0..l, n=-30..30), N=1000
knots on [0, 3.15e7] s, dt=10 s, 3,150,001 complex128 samples, seeded
synthetic inputs (fastemriwaveforms_b200.synthetic.plain_full).  The working
set (amplitudes 61 MB, spline coefficients 246 MB, folded coefficients 82 MB,
output 50 MB) exceeds the 126 MB L2, so no flush is needed between steps.

Metric: mode-samples/s = K * samples / time.
  value  -- inputs already in HBM, device time of K steps (CUDA events, max over ranks)
  e2e    -- the same call from pinned host inputs, host<-device copy of the waveform, per step
With N > 1 ranks (torchrun), every rank computes its own waveform (independent
seeds): per-GPU work is fixed ("weak" scaling) and no collective touches the
data path.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "mode-samples/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["faithful", "exact"], default="faithful")
    ap.add_argument("--workload", choices=["plain_full", "plain_small"], default="plain_full")
    ap.add_argument("--cpu-samples", type=int, default=60000,
                    help="output samples of the bounded single-core reference run (cpu_baseline)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="only run warmup + steps forward calls (for ncu captures); prints no JSON line")
    return ap.parse_args()


def workload(name: str, seed_offset: int = 0):
    from fastemriwaveforms_b200 import synthetic as S

    if name == "plain_full":
        return S.plain_full(seed=2 + seed_offset)
    return S.plain_small(seed=1 + seed_offset)


def config_of(inp, args, extra=None):
    cfg = {"workload": f"{inp.name}: 1 waveform, K={inp.num_modes} modes, N={inp.num_knots} knots, "
                       f"T={inp.out_len} samples, dt={inp.dt:g} s, complex128",
           "modes": inp.num_modes, "knots": inp.num_knots, "samples": inp.out_len,
           "precision": args.precision, "l2": "working set > L2 (126 MB); no flush",
           "parallelism": f"waveform-parallel x{args.gpus}"}
    if extra:
        cfg.update(extra)
    return cfg


# ------------------------------------------------------------------------------------------
# clocks
# ------------------------------------------------------------------------------------------
class ClockSampler:
    """SM clock and throttle reasons sampled through NVML (read-only) every
    5 ms on a background thread while the timed region runs."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, device):
        import threading

        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml as nv
            import torch

            nv.nvmlInit()
            h = None
            bus = getattr(torch.cuda.get_device_properties(device), "pci_bus_id", None)
            if bus is not None:
                try:
                    busid = "%08x:%02x:%02x.0" % (getattr(torch.cuda.get_device_properties(device), "pci_domain_id", 0),
                                                  bus, getattr(torch.cuda.get_device_properties(device),
                                                               "pci_device_id", 0))
                    h = nv.nvmlDeviceGetHandleByPciBusId(busid)
                except Exception:
                    h = None
            if h is None:
                h = nv.nvmlDeviceGetHandleByIndex(device.index or 0)
            self.nv, self.h = nv, h
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self._get_reasons = get_reasons
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        except Exception:
            self._thread = None

    def _run(self):
        nv, h = self.nv, self.h
        while not self._stop.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                bits = int(self._get_reasons(h))
                for bit, name in self.REASONS.items():
                    if bits & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            self._stop.wait(0.005)

    def stop(self):
        if self._thread is None:
            return None
        self._stop.set()
        self._thread.join(timeout=2)
        if not self.samples:
            return None
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples), "source": "NVML, 5 ms"}


# ------------------------------------------------------------------------------------------
# CPU baseline: the reference's own CPU path on a bounded window of the same workload
# ------------------------------------------------------------------------------------------
def _cpu_impl():
    from oracle import oracle as O

    if O.have_ref():
        return "ref", "reference"
    O.build(ref=False)
    return "oracle", "port"


def cpu_baseline(inp, samples: int):
    """Single-threaded: the reference's spline build of all 2K amplitude series
    plus its sum over the first `samples` output samples."""
    from oracle import oracle as O

    impl, kind = _cpu_impl()
    K = inp.num_modes
    t0 = time.perf_counter()
    y_all, pc, ylms = O.prepare_sum(inp)
    coeffs = O.spline_coeffs(inp.t, y_all, impl=impl)
    t1 = time.perf_counter()
    prob = O.window_problem(inp, coeffs, 0, samples)
    O.run_window(prob, impl)
    t2 = time.perf_counter()
    value = K * samples / (t2 - t1)
    return {"value": value, "unit": METRIC, "cores": 1, "kind": kind,
            "sample": f"{samples} output samples x {K} modes of the same waveform (first samples); "
                      f"sum {t2 - t1:.2f} s, spline build of all {2 * K} series {t1 - t0:.3f} s (not in value)",
            "cpu": _cpu_model()}


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _ref_worker(args):
    """One process of the reference arm: window problems at its segment offset."""
    impl, seed_off, j0, samples, steps = args
    from oracle import oracle as O

    inp = workload("plain_full", seed_off)
    y_all, pc, ylms = O.prepare_sum(inp)
    coeffs = O.spline_coeffs(inp.t, y_all, impl=impl)
    prob = O.window_problem(inp, coeffs, j0, samples)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        O.run_window(prob, impl)
        times.append(time.perf_counter() - t0)
    return times


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp

    impl, kind = _cpu_impl()
    inp = workload(args.workload)
    K = inp.num_modes
    procs = os.cpu_count() or 1
    samples = 20000 if args.workload == "plain_full" else 5000
    from oracle import oracle as O

    start, nseg = O.find_start_inds(inp.t, inp.dt, inp.out_len)
    # spread the windows over the waveform, one per process, each at a segment start
    js = [int(j) for j in np.linspace(0, nseg - 1, procs, endpoint=False)]
    steps = args.warmup + args.steps
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(impl, 0, j, samples, steps) for j in js])
    wall = time.perf_counter() - t0
    # per step: the slowest process bounds the step
    per_step = [max(r[s] for r in res) for s in range(args.warmup, steps)]
    step_s = statistics.mean(per_step)
    value = K * samples * procs / step_s
    line = {"metric": METRIC, "value": value, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(inp, args, {"reference_window": f"{procs} processes x {samples} samples"}),
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": procs, "kind": kind,
                             "sample": f"{procs} windows of {samples} samples x {K} modes at spread knot segments, "
                                       f"one process each (the reference path is single-threaded)",
                             "cpu": _cpu_model()},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------
def fp64_peak(device) -> float:
    """Measured FP64 FMA throughput (TFLOP/s) of this GPU: few_probe_fp64_fma."""
    import torch

    from fastemriwaveforms_b200 import _lib

    sms = torch.cuda.get_device_properties(device).multi_processor_count
    blocks = sms * 8
    iters = 4096
    out = torch.empty(blocks * 256, dtype=torch.float64, device=device)
    st = torch.cuda.current_stream(device).cuda_stream
    for _ in range(2):
        _lib.call("few_probe_fp64_fma", out.data_ptr(), blocks, iters, st)
    best = 0.0
    for _ in range(5):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        _lib.call("few_probe_fp64_fma", out.data_ptr(), blocks, iters, st)
        b.record()
        b.synchronize()
        flops = blocks * 256 * iters * 16
        best = max(best, flops / (a.elapsed_time(b) * 1e-3) / 1e12)
    return best


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    from fastemriwaveforms_b200 import InterpolatedModeSum

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    inp = workload(args.workload, seed_offset=rank)
    K, T = inp.num_modes, inp.out_len
    ims = InterpolatedModeSum(precision=args.precision)
    teuk_d = torch.from_numpy(inp.teuk_modes).to(dev)
    ylms_d = torch.from_numpy(inp.ylms).to(dev)
    pc_d = torch.from_numpy(inp.phase_coeffs).to(dev)
    call_args = (inp.t, teuk_d, ylms_d, inp.phase_t, pc_d, inp.l, inp.m, inp.k, inp.n)

    if args.profile:
        for _ in range(args.warmup + args.steps):
            ims(*call_args, T=inp.T, dt=inp.dt)
        torch.cuda.synchronize()
        return 0

    fp64_tflops = fp64_peak(dev)

    for _ in range(max(args.warmup, 3)):
        ims(*call_args, T=inp.T, dt=inp.dt)
    torch.cuda.synchronize()

    # ---- device-resident timed region -------------------------------------------------
    ims.record_stages = True
    clocks = ClockSampler(dev)
    stage_events = []
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        ims(*call_args, T=inp.T, dt=inp.dt)
        stage_events.append(ims._stage_events)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        tm = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        ms = float(tm.item())
    ims.record_stages = False
    ms_step = ms / args.steps
    value = world * K * T / (ms_step * 1e-3)
    stage = {name: statistics.mean(
        ev[i].elapsed_time(ev[i + 1]) for ev in stage_events) for i, name in enumerate(("spline", "fold", "sum"))}
    fold, seg = ims._last_plan
    gpu_launches = 3 * args.steps

    # ---- end to end: pinned host inputs, waveform back to the host ---------------------
    e2e = None
    if not args.no_e2e:
        teuk_h = torch.from_numpy(inp.teuk_modes).pin_memory()
        ylms_h = torch.from_numpy(inp.ylms).pin_memory()
        pc_h = torch.from_numpy(inp.phase_coeffs).pin_memory()
        out_h = torch.empty(T, dtype=torch.complex128).pin_memory()
        host_args = (inp.t, teuk_h, ylms_h, inp.phase_t, pc_h, inp.l, inp.m, inp.k, inp.n)
        for _ in range(2):
            wf = ims(*host_args, T=inp.T, dt=inp.dt)
            out_h.copy_(wf, non_blocking=True)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            wf = ims(*host_args, T=inp.T, dt=inp.dt)
            out_h.copy_(wf, non_blocking=True)
        b.record()
        torch.cuda.synchronize()
        barrier()
        ems = a.elapsed_time(b)
        if world > 1:
            tm = torch.tensor([ems], dtype=torch.float64, device=dev)
            dist.all_reduce(tm, op=dist.ReduceOp.MAX)
            ems = float(tm.item())
        h2d = (inp.teuk_modes.nbytes + inp.ylms.nbytes + inp.phase_coeffs.nbytes + inp.t.nbytes
               + seg.seg_info_host.nbytes + seg.units_host.nbytes)
        e2e = {"value": world * K * T / (ems / args.steps * 1e-3), "unit": METRIC,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(T * 16),
               "ms_per_step": ems / args.steps}

    # ---- roofline of the dominant kernel (the sum) ------------------------------------
    keys = fold.R * fold.NN
    flops_per_key_sample = 30 if args.precision == "faithful" else 20
    sum_flops = float(keys) * T * flops_per_key_sample
    achieved = sum_flops / (stage["sum"] * 1e-3) / 1e12
    pk, pk_kind = peaks()
    spline_bytes = 40.0 * inp.num_knots * 2 * K
    roofline = {"bound": "fp64", "kernel": "k_sum_folded", "achieved": achieved, "peak": fp64_tflops,
                "unit": "TFLOP/s", "frac": achieved / fp64_tflops, "traffic": None,
                "peak_source": "measured in this run: few_probe_fp64_fma (FP64 FMA pipe)",
                "algorithmic": f"{flops_per_key_sample} flop x {keys} keys x {T} samples per launch",
                "launch_ms": stage["sum"]}
    spline_roof = {"bound": "hbm", "kernel": "k_spline_build", "achieved": spline_bytes / (stage["spline"] * 1e-3) / 1e9,
                   "peak": pk["hbm_gbs"], "unit": "GB/s",
                   "frac": spline_bytes / (stage["spline"] * 1e-3) / 1e9 / pk["hbm_gbs"],
                   "peak_source": f"{pk_kind} hbm_gbs", "algorithmic": "40 B per (knot, series)",
                   "launch_ms": stage["spline"]}

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(inp, min(args.cpu_samples, T) if args.workload == "plain_full" else min(5000, T))
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config_of(inp, args),
            "e2e": e2e, "gpu_launches": gpu_launches, "roofline": roofline, "roofline_spline": spline_roof,
            "stage_ms": stage, "cpu_baseline": cpu, "clocks": clk,
            "device": torch.cuda.get_device_name(dev)}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
