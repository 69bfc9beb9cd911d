"""engines::gpu::mc_european_gpu (src/engines/gpu/gpu_mc.rs:322-349) on the GPU.

stream="philox" (the default) prices the European on this engine's own GBM
path: the FP32 Philox strike-strip kernel with one strike (of_mc_strip),
log-Euler steps with Box-Muller normals in registers, compensated FP32 into
FP64 sums.  stream="xoshiro128" runs the reference's WGSL kernel semantics
instead (of_mc_european_gpu: f32 paths, xoshiro128++ seeded from the path
index, Box-Muller, per-block reduction), for callers that want the
reference shader's numbers without a graphics API.  Both estimate the same
discretised price; only the draws differ.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

from ._lib import context
from .core import OptionType, PricingError


@dataclass
class GpuMcResult:
    price: float
    stderr: float


def mc_european_gpu(spot: float, strike: float, rate: float, vol: float, expiry: float, num_paths: int,
                    num_steps: int, seed: int, is_call: bool, device: int = 0, stream: str = "philox") -> GpuMcResult:
    if stream == "philox":
        from .engines import Gbm, GbmPathGenerator, price_strike_strip
        if num_paths <= 0 or num_steps <= 0:
            raise PricingError.InvalidInput("num_paths and num_steps must be > 0")
        gen = GbmPathGenerator(Gbm(rate, vol), spot, expiry, int(num_steps))
        (p, s), = price_strike_strip(gen, OptionType.Call if is_call else OptionType.Put, [strike], int(num_paths),
                                     int(seed), math.exp(-rate * expiry), device=device)
        return GpuMcResult(p, s)
    if stream != "xoshiro128":
        raise PricingError.InvalidInput(f"unknown stream {stream!r} (philox or xoshiro128)")
    ctx = context(device)
    p, s = C.c_double(), C.c_double()
    with ctx.lock:
        ctx.check(ctx._L.of_mc_european_gpu(ctx.handle, spot, strike, rate, vol, expiry, int(num_paths),
                                            int(num_steps), int(seed) & 0xFFFFFFFF, int(bool(is_call)),
                                            C.byref(p), C.byref(s)))
    return GpuMcResult(p.value, s.value)
