"""Tile-shape autotuner with a cached JSON table.

`tune_strip` times the strike-strip kernel for each candidate number of
samples in flight per thread (ILP); `tune_book` times the persistent book
kernel for candidate (threads per block, samples per thread per tile).  The
timing is native (of_autotune_strip / of_autotune_book): each candidate is a
prepared plan (CUDA graph) replayed a few times on the engine's stream and
timed with CUDA events; the fastest wins.  Results are
cached per device name and workload signature in a JSON file
(OF_AUTOTUNE_CACHE, default ~/.cache/openferric_b200/autotune.json) and
reused by `best_strip_ilp` / `best_book_tile` without re-timing.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import threading
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

from . import _abi as A
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


def _store(table: Dict[str, dict]) -> bool:
    """Writes the table; False (and the tuning result still returned to the
    caller) when the cache location is not writable."""
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp"  # one per process: ranks of a job may write at once
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
        return True
    except OSError:
        return False


def _device_name(device: int) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def _candidates(shapes: Sequence[Tuple[int, int]]):
    arr = (A.OfTuneCandidate * len(shapes))()
    for i, (block, ppt) in enumerate(shapes):
        arr[i].block, arr[i].paths_per_thread = int(block), int(ppt)
    return arr


def _strip_key(device: int, generator, n_strikes: int, antithetic: bool) -> str:
    steps_bucket = 1 << max(0, int(generator.steps - 1).bit_length())
    kpl = (n_strikes + 31) // 32
    return f"strip|{_device_name(device)}|model={generator.to_abi().kind}|steps<={steps_bucket}|kpl={kpl}|anti={int(antithetic)}"


def tune_strip(generator, strikes: Sequence[float], num_paths: int, antithetic: bool = False, device: int = 0,
               candidates: Sequence[int] = (1, 2), reps: int = 5) -> Tuple[int, Dict[int, float]]:
    """Times the strip for each tile shape (1 or 2 samples in flight per
    thread; 3 = warp-specialised producer/consumer warps, measured slower on
    the B200 and therefore not a default candidate); stores and returns the
    best."""
    from .core import OptionType
    ctx = context(device)
    ks = np.ascontiguousarray(strikes, dtype=np.float64)
    model = generator.to_abi()
    cfg = A.OfMcConfig(num_paths=int(num_paths), seed=1, antithetic=int(antithetic),
                       precision=A.OF_PREC_FP32_PHILOX, discount_factor=1.0)
    cands = _candidates([(0, ilp) for ilp in candidates])
    best_i = C.c_int32()
    with ctx.lock:
        ctx.check(ctx._L.of_autotune_strip(ctx.handle, C.byref(model), OptionType.Call.value,
                                           ks.ctypes.data_as(C.POINTER(C.c_double)), len(ks), C.byref(cfg),
                                           cands, len(cands), int(reps), C.byref(best_i)))
    times = {c.paths_per_thread: c.ms for c in cands}
    best = cands[best_i.value].paths_per_thread
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
    from .book import book_entries_abi
    ctx = context(device)
    arr, _keep, _ = book_entries_abi(entries)
    cfg = A.OfBookConfig(seed=int(seed) & 0xFFFFFFFFFFFFFFFF, use_graph=1)
    cands = _candidates(candidates)
    best_i = C.c_int32()
    with ctx.lock:
        ctx.check(ctx._L.of_autotune_book(ctx.handle, arr, len(arr), C.byref(cfg), cands, len(cands), int(reps),
                                          C.byref(best_i)))
    times = {(c.block, c.paths_per_thread): c.ms for c in cands}
    best = (cands[best_i.value].block, cands[best_i.value].paths_per_thread)
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
