"""Autotuner for the persistent (batched) mode-sum launch.

Tunable shape: the work-unit length (output samples per unit, which sets how
often a CTA reloads a segment's folded coefficients and how evenly the units
spread) and the number of persistent CTAs per SM.  Each candidate is timed with
CUDA events on the caller's real batch (the sum kernel only; the rest of the
forward does not depend on the choice) and the fastest is cached in a JSON file
keyed by GPU name, precision and the batch's shape buckets.

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


def tune(key: str, make_runner, candidates=None) -> dict:
    """Time make_runner(chunk, ctas_per_sm)() for every candidate and cache the best."""
    if candidates is None:
        candidates = [(c, m) for c in CHUNKS for m in CTAS_PER_SM]
    results = []
    for chunk, per_sm in candidates:
        run = make_runner(chunk, per_sm)
        results.append((time_ms(run), chunk, per_sm))
    results.sort()
    best_ms, chunk, per_sm = results[0]
    choice = {"chunk": chunk, "ctas_per_sm": per_sm, "ms": best_ms,
              "tried": [{"chunk": c, "ctas_per_sm": m, "ms": t} for t, c, m in results]}
    record(key, choice)
    return choice
