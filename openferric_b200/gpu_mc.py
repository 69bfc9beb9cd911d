"""engines::gpu::mc_european_gpu (src/engines/gpu/gpu_mc.rs:322-349) on CUDA:
the reference's WGSL European kernel semantics (f32 paths, xoshiro128++,
Box-Muller, per-block reduction), without a graphics API."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from ._lib import context


@dataclass
class GpuMcResult:
    price: float
    stderr: float


def mc_european_gpu(spot: float, strike: float, rate: float, vol: float, expiry: float, num_paths: int,
                    num_steps: int, seed: int, is_call: bool, device: int = 0) -> GpuMcResult:
    ctx = context(device)
    p, s = C.c_double(), C.c_double()
    with ctx.lock:
        ctx.check(ctx._L.of_mc_european_gpu(ctx.handle, spot, strike, rate, vol, expiry, int(num_paths),
                                            int(num_steps), int(seed) & 0xFFFFFFFF, int(bool(is_call)),
                                            C.byref(p), C.byref(s)))
    return GpuMcResult(p.value, s.value)
