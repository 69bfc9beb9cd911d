"""B200-native Monte Carlo pricing engine behind openferric's PricingEngine API.

The engines here price through libofgpu.so (include/of_gpu.h); there is no CPU
fallback.  Names follow the openferric crate: `MonteCarloPricingEngine`,
`ArithmeticAsianMC`, `MonteCarloEngine`, `LongstaffSchwartzEngine`, with the
same instruments, `Market` and `PricingResult`.
"""
from ._lib import GpuUnavailable, OfGpuError, context
from .core import (AsianSpec, Averaging, BarrierDirection, BarrierSpec, BarrierStyle, Diagnostics, ExerciseStyle,
                   Greeks, OptionType, PricingError, PricingResult, StrikeType)
from .engines import (ArithmeticAsianMC, ControlVariate, ControlVariateKind, FastRngKind, Gbm, GbmPathGenerator,
                      Heston, HestonPathGenerator, MonteCarloEngine, MonteCarloPricingEngine, Precision,
                      VarianceReduction, price_strike_strip)
from .gpu_mc_engine import GpuMcEngine
from .instruments import AsianOption, BarrierOption, BermudanOption, VanillaOption, daily_fixings
from .market import DividendEvent, DividendKind, DividendSchedule, Market, MarketBuilder, SampledVolSurface

__all__ = [
    "GpuUnavailable", "OfGpuError", "context", "AsianSpec", "Averaging", "BarrierDirection", "BarrierSpec",
    "BarrierStyle", "Diagnostics", "ExerciseStyle", "Greeks", "OptionType", "PricingError", "PricingResult",
    "StrikeType", "ArithmeticAsianMC", "ControlVariate", "ControlVariateKind", "FastRngKind", "Gbm",
    "GbmPathGenerator", "Heston", "HestonPathGenerator", "MonteCarloEngine", "MonteCarloPricingEngine", "Precision",
    "VarianceReduction", "price_strike_strip", "SampledVolSurface", "DividendEvent", "DividendKind",
    "DividendSchedule", "AsianOption", "BarrierOption", "BermudanOption", "VanillaOption",
    "daily_fixings", "Market", "MarketBuilder", "GpuMcEngine",
]
