"""Tile-shape autotuner with a cached JSON table.

`tune_strip` times the strike-strip kernel for each candidate number of
samples in flight per thread (ILP); `tune_book` times the persistent book
kernel for candidate (threads per block, samples per thread per tile).  Each
candidate is a prepared plan (CUDA graph) replayed a few times on the
engine's stream and timed with CUDA events; the fastest wins.  Results are
cached per device name and workload signature in a JSON file
(OF_AUTOTUNE_CACHE, default ~/.cache/openferric_b200/autotune.json) and
reused by `best_strip_ilp` / `best_book_tile` without re-timing.
"""
from __future__ import annotations

import json
import os
import threading
from typing import Dict, List, Optional, Sequence, Tuple

from ._lib import context

_LOCK = threading.Lock()


def cache_path() -> str:
    return os.environ.get("OF_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "openferric_b200", "autotune.json"))


def _load() -> Dict[str, dict]:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(table: Dict[str, dict]) -> None:
    path = cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _device_name(device: int) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def _time_launches(ctx, launch, reps: int) -> float:
    """Median milliseconds of `reps` launches on the engine's stream (CUDA events)."""
    import statistics
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    launch()
    stream.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for s, e in ev:
        s.record(stream)
        launch()
        e.record(stream)
    stream.synchronize()
    return statistics.median(s.elapsed_time(e) for s, e in ev)


def _strip_key(device: int, generator, n_strikes: int, antithetic: bool) -> str:
    steps_bucket = 1 << max(0, int(generator.steps - 1).bit_length())
    kpl = (n_strikes + 31) // 32
    return f"strip|{_device_name(device)}|model={generator.to_abi().kind}|steps<={steps_bucket}|kpl={kpl}|anti={int(antithetic)}"


def tune_strip(generator, strikes: Sequence[float], num_paths: int, antithetic: bool = False, device: int = 0,
               candidates: Sequence[int] = (1, 2), reps: int = 5) -> Tuple[int, Dict[int, float]]:
    """Times the strip for each ILP candidate; stores and returns the best."""
    from .core import OptionType
    from .engines import StripPlan
    ctx = context(device)
    times = {}
    for ilp in candidates:
        plan = StripPlan(generator, OptionType.Call, strikes, num_paths, 1, 1.0, antithetic, device, tile_ilp=ilp)
        try:
            times[ilp] = _time_launches(ctx, plan.launch, reps)
        finally:
            plan.close()
    best = min(times, key=times.get)
    with _LOCK:
        table = _load()
        table[_strip_key(device, generator, len(strikes), antithetic)] = {
            "ilp": best, "ms": {str(k): v for k, v in times.items()}, "paths": num_paths}
        _store(table)
    return best, times


def best_strip_ilp(generator, n_strikes: int, antithetic: bool = False, device: int = 0) -> int:
    """The cached ILP for this workload signature, 0 (library default) if untuned."""
    entry = _load().get(_strip_key(device, generator, n_strikes, antithetic))
    return int(entry["ilp"]) if entry else 0


def tune_book(entries, seed: int = 1, device: int = 0,
              candidates: Sequence[Tuple[int, int]] = ((256, 4), (256, 2), (256, 8), (128, 4), (128, 8)),
              reps: int = 3) -> Tuple[Tuple[int, int], Dict[str, float]]:
    """Times the persistent book kernel for each (block, paths_per_thread)."""
    from .book import BookPlan
    ctx = context(device)
    times = {}
    for block, ppt in candidates:
        plan = BookPlan(entries, seed, block=block, paths_per_thread=ppt, use_graph=True, device=device)
        try:
            times[(block, ppt)] = _time_launches(ctx, plan.launch, reps)
        finally:
            plan.close()
    best = min(times, key=times.get)
    key = f"book|{_device_name(device)}|n={len(entries)}"
    with _LOCK:
        table = _load()
        table[key] = {"block": best[0], "paths_per_thread": best[1],
                      "ms": {f"{b}x{p}": v for (b, p), v in times.items()}}
        _store(table)
    return best, {f"{b}x{p}": v for (b, p), v in times.items()}


def best_book_tile(n_entries: int, device: int = 0) -> Optional[Tuple[int, int]]:
    entry = _load().get(f"book|{_device_name(device)}|n={n_entries}")
    return (int(entry["block"]), int(entry["paths_per_thread"])) if entry else None
