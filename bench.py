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
With N > 1 ranks (torchrun) the default (--mode split) splits the one
waveform across the ranks (ShardedInterpolatedModeSum: contiguous sample
ranges, splines and fold built redundantly, the slices assembled by one NCCL
all_gather, gradients summed by one all_reduce): total work is fixed
("strong" scaling).  --mode replicas runs an independent waveform per rank
instead ("weak" scaling, no collective on the data path).
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
    ap.add_argument("--precision", choices=["faithful", "exact", "mixed"], default="faithful")
    ap.add_argument("--workload", choices=["plain_full", "plain_small"], default="plain_full")
    ap.add_argument("--cpu-samples", type=int, default=60000,
                    help="output samples of the bounded single-core reference run (cpu_baseline)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-window", type=int, default=32768,
                    help="--impl reference: output samples per process per step")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--mode", choices=["split", "replicas"], default=None,
                    help="with N > 1 ranks: split one waveform across the ranks (strong scaling, the default) or "
                         "run an independent waveform per rank (weak scaling); --mode split on one GPU runs the "
                         "split path in a one-rank group")
    ap.add_argument("--batch-count", type=int, default=256,
                    help="waveforms of the uneven batch (T ~ logU[1e5, 3.15e6], N ~ U[50, 2000], K ~ U[200, 3843])")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-fd", action="store_true", help="skip the frequency-domain sum measurement")
    ap.add_argument("--no-aak", action="store_true", help="skip the AAK summation measurement")
    ap.add_argument("--profile", action="store_true",
                    help="only run warmup + steps calls (for ncu captures); prints no JSON line")
    ap.add_argument("--profile-form", choices=["forward", "fwd_bwd", "fd", "aak", "amplitude"], default="forward",
                    help="with --profile: forward calls, forward+backward through autograd, the "
                         "frequency-domain sum, the AAK summation, or the amplitude grids")
    ap.add_argument("--fd-modes", type=int, default=3843,
                    help="with --profile-form fd: the first modes of the one-year FD trajectory")
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
    plus its sum over the first `samples` output samples.  The spline build
    serves the whole waveform, so `value` charges it pro rata (its time x
    samples / T): the rate a whole-waveform call would have."""
    from oracle import oracle as O

    impl, kind = _cpu_impl()
    K, T = inp.num_modes, inp.out_len
    t0 = time.perf_counter()
    y_all, pc, ylms = O.prepare_sum(inp)
    coeffs = O.spline_coeffs(inp.t, y_all, impl=impl)
    t1 = time.perf_counter()
    prob = O.window_problem(inp, coeffs, 0, samples)
    O.run_window(prob, impl)
    t2 = time.perf_counter()
    spline_share = (t1 - t0) * samples / T
    value = K * samples / (t2 - t1 + spline_share)
    return {"value": value, "unit": METRIC, "cores": 1, "kind": kind,
            "sample": f"{samples} output samples x {K} modes of the same waveform (first samples); "
                      f"sum {t2 - t1:.2f} s plus the spline build of all {2 * K} series ({t1 - t0:.3f} s) "
                      f"charged pro rata ({spline_share:.4f} s)",
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
    """One process of the reference arm: the reference's spline build of the
    whole waveform (timed once), then one window of its own sample range per
    step (windows tile the range and repeat once it is covered)."""
    impl, windows, steps = args
    from oracle import oracle as O

    inp = workload("plain_full")
    t0 = time.perf_counter()
    y_all, pc, ylms = O.prepare_sum(inp)
    coeffs = O.spline_coeffs(inp.t, y_all, impl=impl)
    spline_s = time.perf_counter() - t0
    probs = [O.window_problem(inp, coeffs, j0, n) for j0, n in windows]
    times = []
    for s in range(steps):
        t0 = time.perf_counter()
        O.run_window(probs[s % len(probs)], impl)
        times.append(time.perf_counter() - t0)
    return spline_s, times


def reference_windows(inp, procs: int, window: int):
    """Splits the waveform's knot segments into `procs` contiguous ranges of
    about equal sample counts, and each range into windows of about `window`
    samples that start at segment starts and tile the range exactly.
    Returns [(share, [(j0, samples), ...])] per process."""
    from oracle import oracle as O

    start, nseg = O.find_start_inds(inp.t, inp.dt, inp.out_len)
    start = [int(v) for v in start[:nseg + 1]]
    T = start[nseg]
    bounds = [0]
    for p in range(1, procs):
        target = p * T / procs
        j = max(bounds[-1] + 1, min(nseg - (procs - p), next(j for j in range(nseg + 1) if start[j] >= target)))
        bounds.append(j)
    bounds.append(nseg)
    out = []
    for p in range(procs):
        a, b = bounds[p], bounds[p + 1]
        wins, j = [], a
        while j < b:
            k = j + 1
            while k < b and start[k] - start[j] < window:
                k += 1
            wins.append((j, start[k] - start[j]))
            j = k
        out.append((start[b] - start[a], wins))
    return out


def run_reference(args):
    """The reference's own CPU path (its interpolate.cu built from source) on
    every host core, one process per core, over the same one-year workload.
    The path is single-threaded, so the harness splits the waveform: process p
    owns a contiguous range of knot segments (~T/P samples) and, per step,
    runs the reference's get_waveform on the next window of that range
    (windows tile the range; the whole waveform is covered every few steps).
    Each process builds the whole spline once; its time is charged to every
    step pro rata (window samples / the process's share), so the per-step rate
    is that of a whole-waveform call split P ways."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp

    impl, kind = _cpu_impl()
    inp = workload(args.workload)
    K = inp.num_modes
    procs = os.cpu_count() or 1
    window = args.ref_window if args.workload == "plain_full" else 5000
    plan = reference_windows(inp, procs, window)
    steps = args.warmup + args.steps
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(impl, wins, steps) for _, wins in plan])
    wall = time.perf_counter() - t0
    total_s, total_ms = 0.0, 0.0
    covered = set()
    for s in range(args.warmup, steps):
        step_s, step_samples = 0.0, 0
        for (share, wins), (spline_s, times) in zip(plan, res):
            j0, n = wins[s % len(wins)]
            covered.add(j0)
            step_s = max(step_s, times[s] + spline_s * n / share)
            step_samples += n
        total_s += step_s
        total_ms += K * step_samples
    value = total_ms / total_s
    nwin = sum(len(w) for _, w in plan)
    spline_mean = statistics.mean(r[0] for r in res)
    line = {"metric": METRIC, "value": value, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_s / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(inp, args),
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": procs, "kind": kind,
                             "sample": f"the whole waveform split into {procs} contiguous segment ranges, one "
                                       f"process per core; per step every process runs the reference's "
                                       f"get_waveform on the next ~{window}-sample window of its range "
                                       f"({nwin} windows tile the waveform; {len(covered)} run in the timed "
                                       f"steps); its whole-spline build ({spline_mean:.2f} s) charged pro rata",
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


def time_forward(ims, call_args, inp, steps, warmup):
    """Device time per forward (ms) and mean per-stage kernel times."""
    import torch

    for _ in range(warmup):
        ims(*call_args, T=inp.T, dt=inp.dt)
    torch.cuda.synchronize()
    ims.record_stages = True
    evs = []
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        ims(*call_args, T=inp.T, dt=inp.dt)
        evs.append(ims._stage_events)
    b.record()
    torch.cuda.synchronize()
    ims.record_stages = False
    stage = {name: statistics.mean(ev[i].elapsed_time(ev[i + 1]) for ev in evs)
             for i, name in enumerate(("spline", "fold", "sum"))}
    return a.elapsed_time(b) / steps, stage


def time_fwd_bwd(precision, inp, dev, steps, warmup, backward=None):
    """Forward + backward through torch.autograd (dL/d amplitude knots and
    dL/d phase coefficients), upstream gradient conj(h_ref + w) with w white,
    sigma = 0.1 rms(h_ref).  Device time per step (ms)."""
    import torch

    from fastemriwaveforms_b200 import InterpolatedModeSum

    ims = InterpolatedModeSum(precision=precision, backward=backward)
    teuk = torch.from_numpy(inp.teuk_modes).to(dev).requires_grad_(True)
    pc = torch.from_numpy(inp.phase_coeffs).to(dev).requires_grad_(True)
    ylms = torch.from_numpy(inp.ylms).to(dev)
    with torch.no_grad():
        h_ref = InterpolatedModeSum(precision="exact")(inp.t, teuk.detach(), ylms, inp.phase_t, pc.detach(), inp.l,
                                                       inp.m, inp.k, inp.n, T=inp.T, dt=inp.dt)
        gen = torch.Generator(device=dev).manual_seed(11)
        rms = torch.sqrt(torch.mean(torch.abs(h_ref) ** 2))
        w = torch.complex(torch.randn(h_ref.shape, generator=gen, device=dev, dtype=torch.float64),
                          torch.randn(h_ref.shape, generator=gen, device=dev, dtype=torch.float64))
        upstream = torch.conj(h_ref + 0.1 * rms * w / np.sqrt(2.0))

    def step():
        teuk.grad = None
        pc.grad = None
        h = ims(inp.t, teuk, ylms, inp.phase_t, pc, inp.l, inp.m, inp.k, inp.n, T=inp.T, dt=inp.dt)
        h.backward(upstream)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        step()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps, teuk.grad.detach().clone(), pc.grad.detach().clone()


def time_forward_form(precision, inp, dev, steps, warmup):
    """Forward only, inputs on the device: device time per call (ms)."""
    import torch

    from fastemriwaveforms_b200 import InterpolatedModeSum

    ims = InterpolatedModeSum(precision=precision)
    args = [inp.t, torch.from_numpy(inp.teuk_modes).to(dev), torch.from_numpy(inp.ylms).to(dev), inp.phase_t,
            torch.from_numpy(inp.phase_coeffs).to(dev), inp.l, inp.m, inp.k, inp.n]
    for _ in range(warmup):
        ims(*args, T=inp.T, dt=inp.dt)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        ims(*args, T=inp.T, dt=inp.dt)
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def cpu_batch_subset(cases, samples: int):
    """The reference's CPU path (one core) on the first waveforms of the batch,
    each on its first `samples` output samples with its whole spline build
    charged pro rata (as cpu_baseline): aggregate mode-samples/s."""
    ms, sec = 0.0, 0.0
    for c in cases:
        n = min(samples, c.out_len)
        r = cpu_baseline(c, n)
        ms += c.num_modes * n
        sec += c.num_modes * n / r["value"]
    return {"value": ms / sec, "unit": METRIC, "cores": 1, "kind": r["kind"],
            "sample": f"{len(cases)} waveforms of the batch (K {min(c.num_modes for c in cases)}-"
                      f"{max(c.num_modes for c in cases)}), the first {samples} samples of each, "
                      f"their spline builds charged pro rata ({sec:.2f} s)"}


def bench_batched(count: int, dev, steps: int, cpu: bool = False):
    """Uneven batch (T ~ logU[1e5, 3.15e6] samples, N ~ U[50, 2000], K ~ U[200, 3843]):
    looping InterpolatedModeSum (plain FP64, one call per waveform; forward, and
    forward + backward through autograd) vs the persistent batched launch in a
    CUDA graph (mixed form with the tensor-core adjoint), upstream gradient
    conj(h) per waveform; with cpu, the reference's CPU path on an 8-waveform
    subset (cpu_batch_subset)."""
    import torch

    from fastemriwaveforms_b200 import InterpolatedModeSum
    from fastemriwaveforms_b200 import synthetic as S
    from fastemriwaveforms_b200.batched import BatchedInterpolatedModeSum

    cases = S.batch_cases(count=count, seed=5)
    ms_total = sum(c.num_modes * c.out_len for c in cases)
    cpu_subset = cpu_batch_subset(cases[:8], 20000) if cpu else None
    loop = InterpolatedModeSum(precision="faithful")
    loop_fb = InterpolatedModeSum(precision="exact", backward="fp64")
    dev_args = []
    for c in cases:
        dev_args.append([c.t, torch.from_numpy(c.teuk_modes).to(dev), torch.from_numpy(c.ylms).to(dev), c.phase_t,
                         torch.from_numpy(c.phase_coeffs).to(dev), c.l, c.m, c.k, c.n])

    def fwd(a_, c):
        loop(*a_, T=c.T, dt=c.dt)

    def fwd_bwd(a_, c):
        a_[1].grad = None
        a_[4].grad = None
        h = loop_fb(*a_, T=c.T, dt=c.dt)
        h.backward(torch.conj(h.detach()))

    def timed(fn):
        for a_, c in zip(dev_args[:2], cases[:2]):
            fn(a_, c)
        torch.cuda.synchronize()
        per = []
        ea = torch.cuda.Event(enable_timing=True)
        eb = torch.cuda.Event(enable_timing=True)
        ea.record()
        for a_, c in zip(dev_args, cases):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            fn(a_, c)
            e1.record()
            per.append((e0, e1))
        eb.record()
        torch.cuda.synchronize()
        total = ea.elapsed_time(eb)
        pw = sorted(e0.elapsed_time(e1) for e0, e1 in per)
        return {"ms_total": total, "value": ms_total / (total * 1e-3), "p50_ms": pw[len(pw) // 2],
                "p99_ms": pw[min(len(pw) - 1, int(0.99 * len(pw)))]}

    out = {"waveforms": count, "mode_samples": ms_total, "loop_plain_fp64": timed(fwd)}
    if cpu_subset:
        out["cpu_subset"] = cpu_subset
    for a_ in dev_args:
        a_[1].requires_grad_(True)
        a_[4].requires_grad_(True)
    out["loop_plain_fp64_fwd_bwd"] = timed(fwd_bwd)
    del dev_args
    torch.cuda.empty_cache()

    # batched mixed: forward graph, then forward + backward graph
    b = BatchedInterpolatedModeSum(precision="mixed").setup(cases, requires_grad=True)
    outs = b.forward()
    grads = [torch.conj(o).clone() for o in outs]
    ea = torch.cuda.Event(enable_timing=True)
    eb = torch.cuda.Event(enable_timing=True)
    b.capture(backward=False)
    b.replay()
    torch.cuda.synchronize()
    ea.record()
    for _ in range(steps):
        b.replay()
    eb.record()
    torch.cuda.synchronize()
    fwd_ms = ea.elapsed_time(eb) / steps
    fwd_lat, _ = b.latencies()  # per-waveform completion times of the last replay
    b.capture(backward=True, grads=grads)
    b.replay()
    torch.cuda.synchronize()
    ea.record()
    for _ in range(steps):
        b.replay()
    eb.record()
    torch.cuda.synchronize()
    fb_ms = ea.elapsed_time(eb) / steps
    _, fb_lat = b.latencies()
    # gradients of two waveforms against the FP64 backward with the same upstream gradient
    errs = []
    for i in range(min(2, count)):
        c = cases[i]
        teuk = torch.from_numpy(c.teuk_modes).to(dev).requires_grad_(True)
        pc = torch.from_numpy(c.phase_coeffs).to(dev).requires_grad_(True)
        h = InterpolatedModeSum(precision="exact", backward="fp64")(c.t, teuk, torch.from_numpy(c.ylms).to(dev),
                                                                    c.phase_t, pc, c.l, c.m, c.k, c.n, T=c.T, dt=c.dt)
        h.backward(b.grad_in[i])
        gt, gp = b.grad_out[i]
        errs.append({"amplitude_knots": float(torch.linalg.norm(gt - teuk.grad) / torch.linalg.norm(teuk.grad)),
                     "phase_coeffs": float(torch.linalg.norm(gp - pc.grad) / torch.linalg.norm(pc.grad))})
    def pct(x, q):
        return float(np.percentile(x, q)) if x is not None else None

    out["batched_mixed_graph"] = {"fwd_ms": fwd_ms, "fwd_value": ms_total / (fwd_ms * 1e-3),
                                  "fwd_p50_ms": pct(fwd_lat, 50), "fwd_p99_ms": pct(fwd_lat, 99),
                                  "fwd_bwd_p50_ms": pct(fb_lat, 50), "fwd_bwd_p99_ms": pct(fb_lat, 99),
                                  "latency_note": "per-waveform completion time from the start of the graph "
                                                  "(all waveforms run concurrently in one launch)",
                                  "fwd_ms_per_waveform": fwd_ms / count, "fwd_bwd_ms": fb_ms,
                                  "fwd_bwd_value": ms_total / (fb_ms * 1e-3), "fwd_bwd_ms_per_waveform": fb_ms / count,
                                  "grad_rel_l2_vs_fp64": errs, "tuning": b.tuning,
                                  "chunk": b.chunk, "ctas_per_sm": b.ctas_per_sm, "mixed_error": b.mixed_error()}
    del b, outs, grads
    torch.cuda.empty_cache()
    return out


def bench_amplitude(dev, steps: int, pk, pk_kind, cpu: bool):
    """Amplitude grids (AmpInterp2D): 3843 modes x (real, imaginary) bicubic
    grids of 40 x 40 knots evaluated at 1000 trajectory points into the mode
    sum's (points, modes) layout; device time of few_amp_interp2d with inputs in
    HBM, HBM roofline on the algorithmic bytes (every coefficient read once,
    the output written once), and the reference's CPU interp2D on a sample."""
    import time

    import torch

    from fastemriwaveforms_b200 import _lib
    from fastemriwaveforms_b200 import synthetic as S
    from fastemriwaveforms_b200.summation import _ptr, _stream

    K, N, nw = 3843, 1000, 40
    tw, tu, coeff = S.amplitude_grids(K, nw=nw, nu=nw)
    w, u = S.amplitude_points(N)
    d = {k: torch.tensor(np.ascontiguousarray(v), dtype=torch.float64, device=dev)
         for k, v in (("tw", tw), ("tu", tu), ("c", coeff), ("w", w), ("u", u))}
    out = torch.empty((N, K), dtype=torch.complex128, device=dev)
    nc = coeff.shape[2]

    def run():
        _lib.call("few_amp_interp2d", _ptr(out), _ptr(d["tw"]), nw, _ptr(d["tu"]), nw, _ptr(d["c"]), 3, 3,
                  _ptr(d["w"]), _ptr(d["u"]), N, None, K, nc, _stream(dev))

    for _ in range(3):
        run()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(max(steps, 5)):
        run()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / max(steps, 5)
    nbytes = coeff.nbytes + out.numel() * 16
    entry = {"workload": f"{K} modes x 2 grids of {nw} x {nw} knots (bicubic), {N} points", "ms": ms,
             "value": K * N / (ms * 1e-3), "unit": "mode-points/s",
             "roofline": {"bound": "hbm", "kernel": "k_amp_interp2d", "achieved": nbytes / (ms * 1e-3) / 1e9,
                          "peak": pk["hbm_gbs"], "unit": "GB/s",
                          "frac": nbytes / (ms * 1e-3) / 1e9 / pk["hbm_gbs"], "peak_source": f"{pk_kind} hbm_gbs",
                          "algorithmic": "coefficients read once + output written once"}}
    if cpu:
        from oracle import oracle as O

        if O.have_ref():
            Ks = K  # every mode at every point (about a second on one core)
            cs = np.ascontiguousarray(coeff[:Ks].reshape(2 * Ks, -1))
            t0 = time.perf_counter()
            O.interp2d(tw, tu, cs, 3, 3, w, u, impl="ref")
            dt = time.perf_counter() - t0
            entry["cpu_baseline"] = {"value": Ks * N / dt, "unit": "mode-points/s", "cores": 1, "kind": "reference",
                                     "sample": f"{Ks} modes x {N} points ({dt:.2f} s)"}
    return entry


def bench_fd(dev, steps: int, fp64_tflops: float, cpu: bool):
    """Frequency-domain sum (FDInterpolatedModeSum): one year at dt = 10 s,
    3843 modes (l = 2..10, m = 0..l, n = -30..30), 1000 knots, M = 1e6,
    a = 0.5 prograde equatorial, p 12 -> 7.4, e 0.4 -> 0.2, phases integrated
    from the geodesic frequencies.  Device time of the whole call (geodesic
    frequencies, splines, plan, sum, (h+, hx)) with inputs in HBM, the sum
    kernel alone, the end-to-end call from host arrays with the (2, L) result
    copied back, and the reference's CPU kernel on a sample of the modes."""
    import time

    import torch

    from fastemriwaveforms_b200 import FDInterpolatedModeSum, get_fundamental_frequencies
    from fastemriwaveforms_b200 import synthetic as S
    from fastemriwaveforms_b200.geodesic import MTSUN_SI

    def gpu_freqs(M, a, p, e, x):
        o = get_fundamental_frequencies(a, p, e, x)
        den = 2 * np.pi * M * MTSUN_SI
        return np.stack([np.abs(o[0].cpu().numpy() / den), o[1].cpu().numpy() / den, o[2].cpu().numpy() / den])

    inp, tr = S.fd_full(frequencies=gpu_freqs)
    host_args = inp.call_args() + (tr.M, tr.a, tr.p, tr.e, tr.xI)
    dev_args = tuple(torch.tensor(np.ascontiguousarray(v), device=dev) if isinstance(v, np.ndarray) else v
                     for v in host_args)
    fd = FDInterpolatedModeSum(pad_output=True)
    ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    for _ in range(2):
        fd(*dev_args, T=inp.T, dt=inp.dt)
    torch.cuda.synchronize()
    n = max(steps, 3)
    call_ms, sum_ms = [], []
    for _ in range(n):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        fd.sum_events = ev
        a.record()
        out = fd(*dev_args, T=inp.T, dt=inp.dt)
        b.record()
        torch.cuda.synchronize()
        call_ms.append(a.elapsed_time(b))
        sum_ms.append(ev[0].elapsed_time(ev[1]))
    fd.sum_events = None
    bins = int(fd.total_bins.item())
    L = out.shape[1]
    # end to end: host inputs in, (2, L) waveform out to pinned host memory
    h = torch.empty(tuple(out.shape), dtype=torch.complex128).pin_memory()
    e2e_ms = []
    for _ in range(n):
        a = time.perf_counter()
        fd(*host_args, T=inp.T, dt=inp.dt, host_out=h)
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - a) * 1e3)
    h2d = sum(v.nbytes for v in host_args if isinstance(v, np.ndarray))
    ms, kms, ems = float(np.median(call_ms)), float(np.median(sum_ms)), float(np.median(e2e_ms))
    entry = {"workload": "one year at dt=10 s, K=3843 (l=2..10, m=0..l, n=-30..30), N=1000 knots, "
                         f"M=1e6, a=0.5 prograde equatorial; L={L} frequency bins, {bins} (mode, bin) evaluations",
             "ms": ms, "sum_kernel_ms": kms, "value": bins / (kms * 1e-3), "unit": "mode-bins/s (sum kernel)",
             "call_value": bins / (ms * 1e-3),
             "e2e": {"ms": ems, "value": bins / (ems * 1e-3), "unit": "mode-bins/s", "h2d_bytes_per_step": int(h2d),
                     "d2h_bytes_per_step": int(h.numel() * 16)},
             "fp64_peak_tflops": fp64_tflops}
    # FP64 work per (mode, bin) evaluation from an ncu capture of k_fd_sum on the one-year
    # trajectory (DFMA x 2 + DADD + DMUL per bin visited)
    flops_per_bin = 786.0
    entry["roofline"] = {"bound": "fp64", "kernel": "k_fd_sum", "achieved": bins * flops_per_bin / (kms * 1e-3) / 1e12,
                         "peak": fp64_tflops, "unit": "TFLOP/s",
                         "frac": bins * flops_per_bin / (kms * 1e-3) / 1e12 / fp64_tflops,
                         "peak_source": "measured in this run: few_probe_fp64_fma (FP64 FMA pipe)",
                         "algorithmic": f"{flops_per_bin:.0f} FP64 flop per (mode, bin) evaluation (ncu count) x {bins}",
                         "traffic": {"bytes_per_launch_300_modes": 70.5e6,
                                     "source": "ncu capture of k_fd_sum, first 300 modes of the one-year case"}}
    if cpu:
        from oracle import oracle as O

        if O.have_ref():
            # the reference's get_waveform_generic_fd (single core) on the first Ks modes, with this
            # run's own bin plan and the reference's spline of those modes' amplitudes + frequencies
            Ks = 40
            fk = gpu_freqs(tr.M, tr.a, tr.p, tr.e, tr.xI)
            y = np.concatenate([inp.teuk_modes[:, :Ks].T.real, inp.teuk_modes[:, :Ks].T.imag, fk], axis=0)
            interp = O.interpolate_arrays(inp.t, y, impl="ref")
            s32 = fd.seg_start_inds[:Ks].cpu().numpy()
            e32 = fd.seg_end_inds[:Ks].cpu().numpy()
            freq = fd.frequency.cpu().numpy()
            lo = np.clip(s32.astype(np.int64), 0, None)
            hi = np.clip(e32.astype(np.int64), None, len(freq) - 1)
            sample_bins = int(np.clip(hi - lo + 1, 0, None).sum())
            pc = np.transpose(inp.phase_coeffs, (2, 1, 0))
            yl = np.concatenate([inp.ylms[:Ks], inp.ylms[3843:3843 + Ks] * (-1.0) ** inp.l[:Ks]])
            t0 = time.perf_counter()
            O.fd_kernel(interp, inp.phase_t, pc, inp.m[:Ks], inp.k[:Ks], inp.n[:Ks], inp.t, freq, s32, e32, yl,
                        L // 2, True, impl="ref")
            dt = time.perf_counter() - t0
            entry["cpu_baseline"] = {"value": sample_bins / dt, "unit": "mode-bins/s", "cores": 1,
                                     "kind": "reference",
                                     "sample": f"the reference's FD kernel on the first {Ks} modes: {sample_bins} "
                                               f"(mode, bin) evaluations in {dt:.1f} s"}
    return entry


def bench_aak(dev, steps: int, cpu: bool, fp64_tflops: float | None = None):
    """AAK summation (AAKSummation): one year at dt = 10 s (3,150,001 samples),
    a 1000-knot trajectory with e 0.6 -> 0.35, 18 harmonics (the reference's
    int(30 e0)); device time of the call with the coefficients in HBM, and the
    reference's CPU AAK kernel on the first 20,000 samples."""
    import time

    import torch

    from fastemriwaveforms_b200 import AAKSummation
    from fastemriwaveforms_b200 import synthetic as S

    inp = S.aak_case(N=1000, span=3.15e7, seed=55)
    args = list(inp.call_args())
    args[11] = torch.tensor(inp.interp_coeffs, device=dev)
    aak = AAKSummation()
    for _ in range(2):
        out = aak(*args, T=inp.T, dt=inp.dt)
    torch.cuda.synchronize()
    n = max(steps, 3)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(n):
        out = aak(*args, T=inp.T, dt=inp.dt)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / n
    L = out.numel()
    entry = {"workload": f"one year at dt=10 s: {L} samples, N={len(inp.t)} knots, {inp.nmodes} harmonics, "
                         "plain polarisations (mich=False)",
             "ms": ms, "value": L / (ms * 1e-3), "unit": "samples/s",
             "harmonic_value": L * inp.nmodes / (ms * 1e-3)}
    if fp64_tflops:
        # FP64 work per sample at 18 harmonics from an ncu capture of k_aak (one-year case)
        flops_per_sample = 8792.0
        ach = L * flops_per_sample / (ms * 1e-3) / 1e12
        entry["roofline"] = {"bound": "fp64", "kernel": "k_aak", "achieved": ach, "peak": fp64_tflops,
                             "unit": "TFLOP/s", "frac": ach / fp64_tflops,
                             "peak_source": "measured in this run: few_probe_fp64_fma (FP64 FMA pipe)",
                             "algorithmic": f"{flops_per_sample:.0f} FP64 flop per sample (ncu count, 18 harmonics)"}
    if cpu:
        from oracle import oracle as O

        if O.have_ref():
            Ls = 20000
            t0 = time.perf_counter()
            O.aak_waveform(inp.t, inp.interp_coeffs, inp.m1, inp.a, inp.m2, inp.qS, inp.phiS, inp.qK, inp.phiK,
                           inp.dist, inp.nmodes, False, Ls, inp.dt, impl="ref")
            dt = time.perf_counter() - t0
            entry["cpu_baseline"] = {"value": Ls / dt, "unit": "samples/s", "cores": 1, "kind": "reference",
                                     "sample": f"the reference's AAK kernel on the first {Ls} samples ({dt:.2f} s)"}
    return entry


def _sig(x, digits: int = 4):
    """Floats rounded to `digits` significant digits, recursively."""
    if isinstance(x, float):
        return float(f"{x:.{digits}g}")
    if isinstance(x, dict):
        return {k: _sig(v, digits) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_sig(v, digits) for v in x]
    return x


def summary(faithful_ms, forms, fb, fb_adj, batched):
    """The mixed-vs-FP64 figures in short form (ms per waveform, accuracy)."""
    mixed = forms["mixed"]
    out = {"forms": {"faithful": {"ms": faithful_ms}, "exact": {"ms": forms["exact"]["ms_per_step"]},
                     "mixed": {"ms": mixed["ms_per_step"], "mismatch": mixed["mismatch_vs_faithful"],
                               "rel_l2": mixed["rel_l2_vs_faithful"], "max_rel": mixed["max_rel_vs_faithful"],
                               "tensor_frac": mixed["roofline"]["frac"]}},
           "fwd_bwd": {k: {"ms": v["ms_per_step"], **({"grad_rel_l2_vs_exact": v["grad_rel_l2_vs_exact"]}
                                                       if "grad_rel_l2_vs_exact" in v else {})}
                       for k, v in fb.items()},
           "fwd_bwd_adjoint_case": {k: v["ms_per_step"] for k, v in fb_adj.items()
                                    if isinstance(v, dict) and "ms_per_step" in v},
           "fwd_adjoint_case": dict(fb_adj["forward_ms"],
                                    **({"cpu_1core_ms": fb_adj["cpu_forward_ms_whole"]}
                                       if "cpu_forward_ms_whole" in fb_adj else {}))}
    if batched:
        loop, bm = batched["loop_plain_fp64"], batched["batched_mixed_graph"]
        loop_fb = batched["loop_plain_fp64_fwd_bwd"]
        out["batched"] = {"waveforms": batched["waveforms"], "mode_samples": float(batched["mode_samples"]),
                          "loop_fp64": {"fwd_ms": loop["ms_total"], "fwd_p50_ms": loop["p50_ms"],
                                        "fwd_p99_ms": loop["p99_ms"], "fwd_bwd_ms": loop_fb["ms_total"],
                                        "fwd_bwd_p50_ms": loop_fb["p50_ms"], "fwd_bwd_p99_ms": loop_fb["p99_ms"]},
                          "graph_mixed": {k: bm[k] for k in ("fwd_ms", "fwd_bwd_ms", "fwd_value", "fwd_bwd_value")
                                          if k in bm}}
        for k in ("fwd_p50_ms", "fwd_p99_ms", "fwd_bwd_p50_ms", "fwd_bwd_p99_ms"):
            if k in bm:
                out["batched"]["graph_mixed"][k] = bm[k]
        if "cpu_subset" in batched:
            out["batched"]["cpu_1core_subset_value"] = batched["cpu_subset"]["value"]
    return _sig(out)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def run_split(args, world: int, rank: int, dev) -> int:
    """One waveform split across `world` ranks: forward (slices gathered on
    every rank), end to end from pinned host inputs, and forward + backward
    (gradients all-reduced).  Device time, max over ranks."""
    import torch
    import torch.distributed as dist

    from fastemriwaveforms_b200.distributed import ShardedInterpolatedModeSum

    inp = workload(args.workload)
    K, T = inp.num_modes, inp.out_len
    ims = ShardedInterpolatedModeSum(precision=args.precision, gather=True)
    teuk_d = torch.from_numpy(inp.teuk_modes).to(dev)
    ylms_d = torch.from_numpy(inp.ylms).to(dev)
    pc_d = torch.from_numpy(inp.phase_coeffs).to(dev)
    call_args = (inp.t, teuk_d, ylms_d, inp.phase_t, pc_d, inp.l, inp.m, inp.k, inp.n)

    def timed(step, n):
        dist.barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            step()
        b.record()
        torch.cuda.synchronize()
        dist.barrier()
        tm = torch.tensor([a.elapsed_time(b) / n], dtype=torch.float64, device=dev)
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        return float(tm.item())

    def fwd():
        ims(*call_args, T=inp.T, dt=inp.dt)

    for _ in range(max(args.warmup, 3)):
        fwd()
    clocks = ClockSampler(dev)
    ms = timed(fwd, args.steps)
    clk = clocks.stop()
    e2e = None
    if not args.no_e2e:
        teuk_h = torch.from_numpy(inp.teuk_modes).pin_memory()
        ylms_h = torch.from_numpy(inp.ylms).pin_memory()
        pc_h = torch.from_numpy(inp.phase_coeffs).pin_memory()
        out_h = torch.empty(T, dtype=torch.complex128).pin_memory()
        host_args = (inp.t, teuk_h, ylms_h, inp.phase_t, pc_h, inp.l, inp.m, inp.k, inp.n)

        def e2e_step():
            h = ims(*host_args, T=inp.T, dt=inp.dt)
            if rank == 0:
                out_h.copy_(h[:T], non_blocking=True)

        for _ in range(max(args.warmup, 3)):
            e2e_step()
        ems = timed(e2e_step, args.steps)
        h2d = inp.teuk_modes.nbytes + inp.ylms.nbytes + inp.phase_coeffs.nbytes + inp.t.nbytes
        e2e = {"value": K * T / (ems * 1e-3), "unit": METRIC, "ms_per_step": ems,
               "h2d_bytes_per_step": int(h2d * world), "d2h_bytes_per_step": int(T * 16)}
    teuk_g = teuk_d.clone().requires_grad_(True)
    pc_g = pc_d.clone().requires_grad_(True)
    with torch.no_grad():
        h_ref = ims(*call_args, T=inp.T, dt=inp.dt).clone()
    upstream = torch.conj(h_ref)

    def fwd_bwd():
        teuk_g.grad = None
        pc_g.grad = None
        h = ims(inp.t, teuk_g, ylms_d, inp.phase_t, pc_g, inp.l, inp.m, inp.k, inp.n, T=inp.T, dt=inp.dt)
        h.backward(upstream)

    for _ in range(3):
        fwd_bwd()
    fb_ms = timed(fwd_bwd, max(2, args.steps // 2))
    if rank == 0:
        line = {"metric": METRIC, "value": K * T / (ms * 1e-3), "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {**config_of(inp, args),
                           "parallelism": f"split x{world}: contiguous sample ranges per rank, splines and fold "
                                          f"built on every rank, NCCL all_gather of the slices, gradient all_reduce"},
                "e2e": e2e, "gpu_launches": 3 * args.steps * world, "cpu_baseline": None, "clocks": clk,
                "device": torch.cuda.get_device_name(dev),
                "fwd_bwd": {"ms_per_step": fb_ms, "value": K * T / (fb_ms * 1e-3),
                            "note": "forward + backward through autograd, gradients all-reduced"}}
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()
    return 0


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
        if args.mode in (None, "split"):
            return run_split(args, world, rank, dev)
    elif args.mode == "split":
        import socket

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if "MASTER_PORT" not in os.environ:
            with socket.socket() as sk:
                sk.bind(("127.0.0.1", 0))
                os.environ["MASTER_PORT"] = str(sk.getsockname()[1])
        dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120), device_id=dev)
        return run_split(args, 1, 0, dev)

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
        if args.profile_form == "fd":
            # the frequency-domain sum on the one-year trajectory, first --fd-modes modes
            from fastemriwaveforms_b200 import FDInterpolatedModeSum
            from fastemriwaveforms_b200 import synthetic as S

            fin, ftr = S.fd_full()
            Kf = min(args.fd_modes, fin.num_modes)
            sel = np.r_[0:Kf, fin.num_modes:fin.num_modes + Kf]
            fargs = (fin.t, np.ascontiguousarray(fin.teuk_modes[:, :Kf]), fin.ylms[sel], fin.phase_t,
                     fin.phase_coeffs, fin.l[:Kf], fin.m[:Kf], fin.k[:Kf], fin.n[:Kf], ftr.M, ftr.a, ftr.p, ftr.e,
                     ftr.xI)
            fd = FDInterpolatedModeSum(pad_output=True)
            for _ in range(args.warmup + args.steps):
                fd(*fargs, T=fin.T, dt=fin.dt)
            torch.cuda.synchronize()
            return 0
        if args.profile_form == "amplitude":
            # AmpInterp2D: 3843 modes x 2 bicubic grids of 40 x 40 knots at 1000 points
            from fastemriwaveforms_b200 import AmpInterp2D
            from fastemriwaveforms_b200 import synthetic as S

            tw, tu, coeff = S.amplitude_grids(3843, nw=40, nu=40)
            w, u = S.amplitude_points(1000)
            amp = AmpInterp2D(tw, tu, coeff, None, None, None, None)
            w_d = torch.tensor(w, device=dev)
            u_d = torch.tensor(u, device=dev)
            for _ in range(args.warmup + args.steps):
                amp(w_d, u_d)
            torch.cuda.synchronize()
            return 0
        if args.profile_form == "aak":
            # the AAK summation on a 3e6 s trajectory (300,001 samples, 18 harmonics)
            from fastemriwaveforms_b200 import AAKSummation
            from fastemriwaveforms_b200 import synthetic as S

            ain = S.aak_case(N=100, span=3e6, seed=55)
            aak = AAKSummation()
            for _ in range(args.warmup + args.steps):
                aak(*ain.call_args(), T=ain.T, dt=ain.dt)
            torch.cuda.synchronize()
            return 0
        if args.profile_form == "fwd_bwd":
            time_fwd_bwd(args.precision, inp, dev, args.steps, args.warmup)
        else:
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
    def time_e2e(module):
        """ms per call through the public API from pinned host inputs, the
        waveform copied back to pinned host memory every step (``host_out``)."""
        teuk_h = torch.from_numpy(inp.teuk_modes).pin_memory()
        ylms_h = torch.from_numpy(inp.ylms).pin_memory()
        pc_h = torch.from_numpy(inp.phase_coeffs).pin_memory()
        out_h = torch.empty(T, dtype=torch.complex128).pin_memory()
        host_args = (inp.t, teuk_h, ylms_h, inp.phase_t, pc_h, inp.l, inp.m, inp.k, inp.n)
        for _ in range(max(args.warmup, 3)):
            module(*host_args, T=inp.T, dt=inp.dt, host_out=out_h)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            # the waveform streams to pinned host memory while the sum runs
            module(*host_args, T=inp.T, dt=inp.dt, host_out=out_h)
        b.record()
        torch.cuda.synchronize()
        barrier()
        ems = a.elapsed_time(b)
        if world > 1:
            tm = torch.tensor([ems], dtype=torch.float64, device=dev)
            dist.all_reduce(tm, op=dist.ReduceOp.MAX)
            ems = float(tm.item())
        return ems / args.steps

    e2e = None
    h2d = (inp.teuk_modes.nbytes + inp.ylms.nbytes + inp.phase_coeffs.nbytes + inp.t.nbytes
           + seg.seg_info_host.nbytes + seg.units_host.nbytes)
    if not args.no_e2e:
        ems = time_e2e(ims)
        e2e = {"value": world * K * T / (ems * 1e-3), "unit": METRIC,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(T * 16),
               "ms_per_step": ems}

    # ---- the other forms on the same waveform ----------------------------------------
    from fastemriwaveforms_b200 import get_mismatch

    forms = {}
    ref_wf = ims(*call_args, T=inp.T, dt=inp.dt).clone()
    pk, pk_kind = peaks()
    for prec in ("exact", "mixed"):
        other = InterpolatedModeSum(precision=prec)
        ms_o, st_o = time_forward(other, call_args, inp, args.steps, 2)
        wf_o = other(*call_args, T=inp.T, dt=inp.dt)
        torch.cuda.synchronize()
        d = (wf_o - ref_wf)
        entry = {"ms_per_step": ms_o, "value": world * K * T / (ms_o * 1e-3), "stage_ms": st_o,
                 "mismatch_vs_faithful": get_mismatch(wf_o, ref_wf),
                 "rel_l2_vs_faithful": float(torch.linalg.norm(d) / torch.linalg.norm(ref_wf)),
                 "max_rel_vs_faithful": float(d.abs().max() / ref_wf.abs().max())}
        if prec == "mixed":
            f_ = other._last_plan[0]
            kdim = 2 * ((f_.NN + 15) // 16 * 16)  # K: (n', re/im)
            nb = (8 * f_.R + 15) // 16 * 16       # N: 8 columns per (m', k') row
            tflop = 2.0 * kdim * nb * 3 * T / 1e12
            entry["mixed_error"] = other.mixed_error()
            if not args.no_e2e:
                ems_m = time_e2e(other)
                entry["e2e"] = {"value": world * K * T / (ems_m * 1e-3), "unit": METRIC, "ms_per_step": ems_m,
                                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(T * 16)}
            entry["roofline"] = {"bound": "tensor", "kernel": "k_sum_mixed (+ k_fold_mixed)",
                                 "achieved": tflop / (st_o["sum"] * 1e-3), "peak": pk["bf16_tflops"],
                                 "unit": "TFLOP/s", "frac": tflop / (st_o["sum"] * 1e-3) / pk["bf16_tflops"],
                                 "peak_source": f"{pk_kind} bf16_tflops (burst)",
                                 "algorithmic": f"MMA work issued: 2 x K {kdim} x N {nb} x 3 split products per sample"}
        forms[prec] = entry
    fb = {}
    # exact: FP64 forward and adjoint; mixed: tensor-core forward and adjoint;
    # mixed_fp64_adjoint: tensor-core forward, FP64 adjoint
    for name, prec, bwd in (("exact", "exact", "fp64"), ("mixed", "mixed", "mixed"),
                            ("mixed_fp64_adjoint", "mixed", "fp64")):
        ms_fb, gt, gp = time_fwd_bwd(prec, inp, dev, max(2, args.steps // 2), 3, backward=bwd)
        fb[name] = {"ms_per_step": ms_fb}
        if name == "exact":
            g_ref = (gt, gp)
        else:
            fb[name]["grad_rel_l2_vs_exact"] = {
                "amplitude_knots": float(torch.linalg.norm(gt - g_ref[0]) / torch.linalg.norm(g_ref[0])),
                "phase_coeffs": float(torch.linalg.norm(gp - g_ref[1]) / torch.linalg.norm(g_ref[1]))}
    del g_ref
    # the adjoint workload: K=1000, N=500, 1,000,000 samples
    from fastemriwaveforms_b200 import synthetic as S

    adj = S.adjoint_case(seed=4 + rank)
    fb_adj = {"workload": f"K={adj.num_modes}, N={adj.num_knots}, T={adj.out_len}"}
    for name, prec, bwd in (("exact", "exact", "fp64"), ("mixed", "mixed", "mixed"),
                            ("mixed_fp64_adjoint", "mixed", "fp64")):
        fb_adj[name] = {"ms_per_step": time_fwd_bwd(prec, adj, dev, max(2, args.steps // 2), 3, backward=bwd)[0]}
    fb_adj["forward_ms"] = {p: time_forward_form(p, adj, dev, max(3, args.steps), 3)
                            for p in ("faithful", "exact", "mixed")}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        c = cpu_baseline(adj, 60000)
        fb_adj["cpu_forward"] = c
        fb_adj["cpu_forward_ms_whole"] = adj.num_modes * adj.out_len / c["value"] * 1e3  # rate x whole waveform

    batched = None if args.no_batch else bench_batched(args.batch_count, dev, max(2, args.steps // 2),
                                                       cpu=(rank == 0 and world == 1 and not args.no_cpu_baseline))
    amplitude = bench_amplitude(dev, args.steps, pk, pk_kind, cpu=(rank == 0 and not args.no_cpu_baseline))
    fdsum = None if args.no_fd else bench_fd(dev, args.steps, fp64_tflops,
                                             cpu=(rank == 0 and not args.no_cpu_baseline))
    aakw = None if args.no_aak else bench_aak(dev, args.steps, cpu=(rank == 0 and not args.no_cpu_baseline),
                                              fp64_tflops=fp64_tflops)

    # ---- roofline of the dominant kernel (the sum) ------------------------------------
    keys = fold.R * fold.NN
    flops_per_key_sample = 30 if args.precision == "faithful" else 20
    sum_flops = float(keys) * T * flops_per_key_sample
    achieved = sum_flops / (stage["sum"] * 1e-3) / 1e12
    spline_bytes = 40.0 * inp.num_knots * 2 * K
    # DRAM bytes of one launch at this workload from an ncu capture (dram__bytes_read.sum +
    # dram__bytes_write.sum); null for workloads not captured
    captured = args.workload == "plain_full" and args.precision == "faithful"
    traffic = {"bytes_per_launch": 161.0e6, "source": "ncu capture of k_sum_folded (faithful, one-year workload)",
               "algorithmic_bytes": float(keys) * 64.0 * seg.nseg + 2.0 * 16.0 * T} if captured else None
    roofline = {"bound": "fp64", "kernel": "k_sum_folded", "achieved": achieved, "peak": fp64_tflops,
                "unit": "TFLOP/s", "frac": achieved / fp64_tflops, "traffic": traffic,
                "peak_source": "measured in this run: few_probe_fp64_fma (FP64 FMA pipe)",
                "algorithmic": f"{flops_per_key_sample} flop x {keys} keys x {T} samples per launch",
                "launch_ms": stage["sum"]}
    spline_roof = {"bound": "hbm", "kernel": "k_spline_build", "achieved": spline_bytes / (stage["spline"] * 1e-3) / 1e9,
                   "peak": pk["hbm_gbs"], "unit": "GB/s",
                   "frac": spline_bytes / (stage["spline"] * 1e-3) / 1e9 / pk["hbm_gbs"],
                   "peak_source": f"{pk_kind} hbm_gbs", "algorithmic": "40 B per (knot, series)",
                   "traffic": ({"bytes_per_launch": 423.9e6,
                                "source": "ncu capture of k_spline_build_factored (one-year workload)"}
                               if args.workload == "plain_full" else None),
                   "launch_ms": stage["spline"]}

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(inp, min(args.cpu_samples, T) if args.workload == "plain_full" else min(5000, T))
    # Key order: the contract's keys, then the rows around the path (long),
    # then the full per-form records, and last a compact summary of the mixed
    # and forward+backward figures, so that the end of the line carries them.
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config_of(inp, args),
            "e2e": e2e, "gpu_launches": gpu_launches, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
            "device": torch.cuda.get_device_name(dev),
            "around_path": {"amplitude": amplitude, "fd": fdsum, "aak": aakw},
            "roofline_spline": spline_roof, "stage_ms": stage,
            "detail": {"forms": forms, "fwd_bwd": fb, "fwd_bwd_adjoint_case": fb_adj, "batched": batched}}
    line.update(summary(ms_step, forms, fb, fb_adj, batched))
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
