"""GpuMcEngine: the Monte Carlo engine class of openferric's Python module
(`McEngine`, python/src/engines.rs:1230-1438) on the GPU.

The static methods keep the reference's names, argument order, defaults,
string options and error behaviour:
- invalid strings raise ValueError with the reference's messages
  (engines.rs:33-105);
- a market the builder rejects raises ValueError("invalid market inputs")
  (engines.rs:53-55; the flat vol is floored at 1e-8, python/src/helpers.rs:60-67);
- a PricingError from the engine raises ValueError with the error's Debug
  form, e.g. `InvalidInput("num_paths must be > 0")` (engines.rs:57-59).

Each method builds the same instrument and market as the reference and prices
them with this package's engines (MonteCarloPricingEngine, ArithmeticAsianMC,
MonteCarloGreeksEngine).  One keyword is added, `precision`:
- "fp64" (the default): the reference's xoshiro256++ streams;
- "fp32": Philox.

`accuracy_tier` is validated and has no effect: it selects the CPU's SIMD
approximations in the reference.  Only the reproducible xoshiro256++ stream is
available on the GPU; other `rng_kind`s and `reproducible=False` are rejected
by the engine, with a ValueError.  Spread options are not on the GPU path.
Drop-in use: `from openferric_b200 import GpuMcEngine as McEngine`.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence, TypeVar

from .core import AsianSpec, Averaging, ExerciseStyle, Greeks, OptionType, PricingError, PricingResult, StrikeType
from .engines import ArithmeticAsianMC, FastRngKind, MonteCarloPricingEngine, Precision, VarianceReduction
from .greeks import MonteCarloGreeksEngine
from .instruments import AsianOption, VanillaOption
from .market import Market

T = TypeVar("T")


def _option_type(value: str) -> OptionType:
    v = value.lower()
    if v == "call":
        return OptionType.Call
    if v == "put":
        return OptionType.Put
    raise ValueError("option_type must be 'call' or 'put'")


def _exercise(style: Optional[str], bermudan_dates: Optional[Sequence[float]]) -> ExerciseStyle:
    s = (style if style is not None else "european").lower()
    if s == "european":
        return ExerciseStyle.european()
    if s == "american":
        return ExerciseStyle.american()
    if s == "bermudan":
        return ExerciseStyle.bermudan(list(bermudan_dates) if bermudan_dates is not None else [])
    raise ValueError(f"unsupported exercise style '{s}'")


def _market(spot: float, rate: float, dividend_yield: float, vol: float) -> Market:
    try:
        return (Market.builder().spot(spot).rate(rate).dividend_yield(dividend_yield).flat_vol(max(vol, 1e-8))
                .build())
    except PricingError:
        raise ValueError("invalid market inputs") from None


def _accuracy_tier(value: Optional[str]) -> Optional[str]:
    if value is None:
        return None
    v = value.lower()
    if v in ("high", "fast"):
        return v
    raise ValueError(f"unsupported accuracy tier '{v}'")


def _variance_reduction(value: Optional[str]) -> VarianceReduction:
    v = (value if value is not None else "none").lower()
    if v == "none":
        return VarianceReduction.None_
    if v == "antithetic":
        return VarianceReduction.Antithetic
    if v in ("control_variate", "control-variate"):
        return VarianceReduction.ControlVariate
    raise ValueError(f"unsupported variance reduction '{v}'")


def _rng_kind(value: Optional[str]) -> FastRngKind:
    v = (value if value is not None else "xoshiro256plusplus").lower()
    if v in ("xoshiro256plusplus", "xoshiro256_plus_plus", "xoshiro"):
        return FastRngKind.Xoshiro256PlusPlus
    if v in ("pcg64", "pcg"):
        return FastRngKind.Pcg64
    if v in ("threadrng", "thread_rng", "thread"):
        return FastRngKind.ThreadRng
    if v in ("stdrng", "std_rng", "std"):
        return FastRngKind.StdRng
    raise ValueError(f"unsupported rng kind '{v}'")


def _precision(value: Optional[str]) -> Precision:
    v = (value if value is not None else "fp64").lower()
    if v == "fp64":
        return Precision.Fp64Reference
    if v == "fp32":
        return Precision.Fp32Philox
    raise ValueError(f"unsupported precision '{v}'")


def _priced(fn: Callable[[], T]) -> T:
    """Runs an engine call; a PricingError becomes ValueError(Debug form)."""
    try:
        return fn()
    except PricingError as e:
        raise ValueError(f'{e.kind}("{e.message}")') from None


def _gpu_stream_only(rng: FastRngKind, reproducible: Optional[bool]) -> None:
    # MonteCarloGreeksEngine has no stream options of its own; the same rule
    # as the pricing engine's
    if rng is not FastRngKind.Xoshiro256PlusPlus or reproducible is False:
        raise ValueError('InvalidInput("the GPU engine supports the reproducible Xoshiro256PlusPlus stream only")')


class GpuMcEngine:
    """McEngine (python/src/engines.rs:1230-1438) with GPU engines behind it."""

    def __init__(self):
        pass

    @staticmethod
    def vanilla_price(option_type: str, spot: float, strike: float, expiry: float, rate: float,
                      dividend_yield: float, vol: float, num_paths: int, num_steps: int, seed: int,
                      variance_reduction: Optional[str] = None, rng_kind: Optional[str] = None,
                      reproducible: Optional[bool] = None, accuracy_tier: Optional[str] = None,
                      exercise_style: Optional[str] = None, bermudan_dates: Optional[Sequence[float]] = None,
                      precision: Optional[str] = None, device: int = 0) -> PricingResult:
        """MonteCarloPricingEngine::price of a vanilla (engines.rs:1241-1279)."""
        market = _market(spot, rate, dividend_yield, vol)
        instrument = VanillaOption(_option_type(option_type), float(strike), float(expiry),
                                   _exercise(exercise_style, bermudan_dates))
        engine = MonteCarloPricingEngine(num_paths, num_steps, seed, device) \
            .with_variance_reduction(_variance_reduction(variance_reduction)) \
            .with_rng_kind(_rng_kind(rng_kind)).with_precision(_precision(precision))
        if reproducible is False:
            engine = engine.with_randomized_streams()
        _accuracy_tier(accuracy_tier)
        return _priced(lambda: engine.price(instrument, market))

    @staticmethod
    def arithmetic_asian_price(option_type: str, spot: float, strike: float, expiry: float, rate: float,
                               dividend_yield: float, vol: float, observation_times: Sequence[float], paths: int,
                               steps: int, seed: int, control_variate: Optional[bool] = None,
                               rng_kind: Optional[str] = None, reproducible: Optional[bool] = None,
                               precision: Optional[str] = None, device: int = 0) -> PricingResult:
        """ArithmeticAsianMC::price, fixed strike (engines.rs:1281-1316)."""
        market = _market(spot, rate, dividend_yield, vol)
        instrument = AsianOption(_option_type(option_type), float(strike), float(expiry),
                                 AsianSpec(Averaging.Arithmetic, StrikeType.Fixed,
                                           [float(t) for t in observation_times]))
        engine = ArithmeticAsianMC(paths, steps, seed, device) \
            .with_control_variate(True if control_variate is None else bool(control_variate)) \
            .with_precision(_precision(precision))
        _gpu_stream_only(_rng_kind(rng_kind), reproducible)
        return _priced(lambda: engine.price(instrument, market))

    @staticmethod
    def _greeks_engine(option_type: str, spot: float, strike: float, expiry: float, rate: float,
                       dividend_yield: float, vol: float, num_paths: int, seed: int, antithetic: Optional[bool],
                       spot_bump_rel: Optional[float], rng_kind: Optional[str], reproducible: Optional[bool],
                       device: int):
        market = _market(spot, rate, dividend_yield, vol)
        ot = _option_type(option_type)
        instrument = VanillaOption.european_call(strike, expiry) if ot is OptionType.Call \
            else VanillaOption.european_put(strike, expiry)
        engine = MonteCarloGreeksEngine(num_paths, seed, device) \
            .with_antithetic(True if antithetic is None else bool(antithetic)) \
            .with_spot_bump_rel(1.0e-2 if spot_bump_rel is None else float(spot_bump_rel))
        _gpu_stream_only(_rng_kind(rng_kind), reproducible)
        return engine, instrument, market

    @staticmethod
    def greeks_pathwise(option_type: str, spot: float, strike: float, expiry: float, rate: float,
                        dividend_yield: float, vol: float, num_paths: int, seed: int,
                        antithetic: Optional[bool] = None, spot_bump_rel: Optional[float] = None,
                        rng_kind: Optional[str] = None, reproducible: Optional[bool] = None,
                        device: int = 0) -> Greeks:
        """MonteCarloGreeksEngine::estimate_pathwise (engines.rs:1318-1350)."""
        engine, instrument, market = GpuMcEngine._greeks_engine(
            option_type, spot, strike, expiry, rate, dividend_yield, vol, num_paths, seed, antithetic, spot_bump_rel,
            rng_kind, reproducible, device)
        return _priced(lambda: engine.estimate_pathwise(instrument, market))

    @staticmethod
    def greeks_likelihood_ratio(option_type: str, spot: float, strike: float, expiry: float, rate: float,
                                dividend_yield: float, vol: float, num_paths: int, seed: int,
                                antithetic: Optional[bool] = None, spot_bump_rel: Optional[float] = None,
                                rng_kind: Optional[str] = None, reproducible: Optional[bool] = None,
                                device: int = 0) -> Greeks:
        """MonteCarloGreeksEngine::estimate_likelihood_ratio (engines.rs:1352-1384)."""
        engine, instrument, market = GpuMcEngine._greeks_engine(
            option_type, spot, strike, expiry, rate, dividend_yield, vol, num_paths, seed, antithetic, spot_bump_rel,
            rng_kind, reproducible, device)
        return _priced(lambda: engine.estimate_likelihood_ratio(instrument, market))

    @staticmethod
    def spread_price(s1: float, s2: float, k: float, vol1: float, vol2: float, rho: float, q1: float, q2: float,
                     rate: float, expiry: float, num_paths: int, seed: int, antithetic: Optional[bool] = None,
                     rng_kind: Optional[str] = None, reproducible: Optional[bool] = None) -> PricingResult:
        """SpreadMonteCarloEngine (engines.rs:1386-1425) is not on the GPU path."""
        raise ValueError('InvalidInput("spread options are not priced by the GPU engine")')
