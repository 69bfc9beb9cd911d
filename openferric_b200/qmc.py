"""Sobol quasi-Monte Carlo, mirroring openferric's engines::monte_carlo::mc_qmc
(src/engines/monte_carlo/mc_qmc.rs:27-150) on the GPU (of_mc_european_qmc).

The point set is the reference's SobolSequence (src/math/sobol.rs); FP64
reference mode keeps its arithmetic, FP32 mode walks the same points with
FP32 paths."""
from __future__ import annotations

import ctypes as C
import math

from . import _abi as A
from ._lib import context
from .core import Diagnostics, OptionType, PricingResult
from .engines import Precision
from .instruments import VanillaOption
from .market import Market


def _intrinsic(opt: OptionType, spot: float, strike: float) -> float:
    return max(spot - strike, 0.0) if opt is OptionType.Call else max(strike - spot, 0.0)


def mc_european_qmc_with_seed(instrument: VanillaOption, market: Market, n_paths: int, n_steps: int, seed: int,
                              precision: Precision = Precision.Fp64Reference, device: int = 0) -> PricingResult:
    """mc_european_qmc_with_seed (mc_qmc.rs:39-150): NaN without a stderr for
    no paths/steps, a non-European exercise or a non-positive vol; the
    intrinsic value for expiry <= 0."""
    nan = PricingResult(price=math.nan, stderr=None)
    if n_paths == 0 or n_steps == 0:
        return nan
    if not instrument.exercise.is_european:
        return nan
    if instrument.expiry <= 0.0:
        return PricingResult(price=_intrinsic(instrument.option_type, market.spot, instrument.strike), stderr=0.0)
    vol = market.vol_for(instrument.strike, instrument.expiry)
    if vol <= 0.0 or not math.isfinite(vol):
        return nan
    p = A.OfQmcParams(option_type=instrument.option_type.value, precision=precision.value, spot=market.spot,
                      strike=instrument.strike, rate=market.rate,
                      dividend_yield=market.effective_dividend_yield(instrument.expiry), vol=vol,
                      expiry=instrument.expiry, num_paths=int(n_paths), num_steps=int(n_steps),
                      seed=int(seed) & 0xFFFFFFFFFFFFFFFF)
    out = A.OfMcResult()
    ctx = context(device)
    with ctx.lock:
        ctx.check(ctx._L.of_mc_european_qmc(ctx.handle, C.byref(p), C.byref(out)))
    d = Diagnostics()
    d.insert("num_paths", float(n_paths))
    d.insert("num_steps", float(n_steps))
    d.insert("vol", vol)
    return PricingResult(price=out.price, stderr=out.stderr_, diagnostics=d)


def mc_european_qmc(instrument: VanillaOption, market: Market, n_paths: int, n_steps: int,
                    precision: Precision = Precision.Fp64Reference, device: int = 0) -> PricingResult:
    """mc_european_qmc (mc_qmc.rs:27-36): seed 0."""
    return mc_european_qmc_with_seed(instrument, market, n_paths, n_steps, 0, precision, device)
