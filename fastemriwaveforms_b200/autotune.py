"""Autotuner for the persistent (batched) mode-sum launch.

Tunable shape: the work-unit length (output samples per unit, which sets how
often a CTA reloads a segment's folded coefficients and how evenly the units
spread), the number of persistent CTAs per SM and, for the tensor-core sum, the
shape of its operand pipeline: A stages per producer half (with two, a half
writes its next chunk while the tensor cores read the previous one) and B
bulk-copy slots the MMA warp keeps in flight ahead of the MMAs.  Deeper
pipelines hide more latency but take shared memory that a second CTA per SM
needs.  Each candidate is timed with CUDA events on
the caller's real batch (the sum kernel only; the rest of the forward does not
depend on the choice) and the fastest is cached in a JSON file keyed by GPU
name, precision and the batch's shape buckets.

Cache location: $FEW_B200_TUNE_CACHE, else ~/.cache/fastemriwaveforms_b200/tune.json.
"""
from __future__ import annotations

import json
import math
import os
import threading

import torch

CHUNKS = (256, 512, 1024)
CTAS_PER_SM = (1, 2, 3)
MIXED_CHUNKS = (512, 1024)
MIXED_CTAS_PER_SM = (1, 2)   # 288-thread CTAs of ~100 KB shared memory: at most two resident per SM
A_STAGES = (1, 2)
B_STAGES = (2, 3, 4)
_lock = threading.Lock()


def cache_path() -> str:
    p = os.environ.get("FEW_B200_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "fastemriwaveforms_b200", "tune.json")


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(table: dict) -> None:
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + f".tmp{os.getpid()}"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home keeps the choice in memory only


def bucket(x: float) -> int:
    """Power-of-two bucket of a positive size."""
    return 1 << max(0, int(math.ceil(math.log2(max(x, 1.0)))))


def key_of(device, precision: str, max_R: int, max_NN: int, mean_seg_len: float, n_wave: int) -> str:
    name = torch.cuda.get_device_name(device).replace(" ", "_")
    return (f"{name}|{precision}|R{bucket(max_R)}|NN{bucket(max_NN)}|L{bucket(mean_seg_len)}"
            f"|W{bucket(n_wave)}")


def lookup(key: str):
    with _lock:
        return _load().get(key)


def record(key: str, choice: dict) -> None:
    with _lock:
        table = _load()
        table[key] = choice
        _store(table)


def time_ms(fn, reps: int = 3) -> float:
    """Median device time (ms) of fn() on the current stream."""
    fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b))
    times.sort()
    return times[len(times) // 2]


def candidates_for(precision: str) -> list:
    """The shapes tried for a precision: dicts of make_runner's keyword arguments."""
    if precision == "mixed":
        return [{"chunk": c, "ctas_per_sm": m, "astages": a, "bstages": b} for c in MIXED_CHUNKS
                for m in MIXED_CTAS_PER_SM for a in A_STAGES for b in B_STAGES]
    return [{"chunk": c, "ctas_per_sm": m} for c in CHUNKS for m in CTAS_PER_SM]


def tune(key: str, make_runner, candidates) -> dict:
    """Time make_runner(**shape)() for every candidate shape and cache the best."""
    results = []
    for shape in candidates:
        run = make_runner(**shape)
        results.append((time_ms(run), shape))
    results.sort(key=lambda r: r[0])
    best_ms, best = results[0]
    choice = dict(best, ms=best_ms, tried=[dict(sh, ms=t) for t, sh in results])
    record(key, choice)
    return choice
