"""GPU Monte Carlo pricing engines behind openferric's `PricingEngine` API.

Mirrors, name for name:
  mc::MonteCarloEngine, GbmPathGenerator, HestonPathGenerator, ControlVariate
      (src/mc/simulation.rs:20-348)
  engines::monte_carlo::{MonteCarloPricingEngine, ArithmeticAsianMC, VarianceReduction}
      (src/engines/monte_carlo/mc_engine.rs:31-988)
Every price is computed by libofgpu (include/of_gpu.h); the host side only
validates, resolves the volatility and computes control-variate means, as the
reference's engines do before their simulation loop.
"""
from __future__ import annotations

import ctypes as C
import enum
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

from . import _abi as A
from ._lib import context
from .analytic import bs_price, geometric_asian_discrete_fixed
from .core import (Averaging, BarrierDirection, BarrierStyle, Diagnostics, OptionType, PricingError,
                   PricingResult, StrikeType)
from .instruments import AsianOption, BarrierOption, VanillaOption
from .market import Market


class VarianceReduction(enum.Enum):
    """engines::monte_carlo::VarianceReduction (mc_engine.rs:31-41)."""

    None_ = 0
    Antithetic = 1
    ControlVariate = 2


class Precision(enum.Enum):
    """Arithmetic mode of the device engine.

    Fp64Reference: openferric's own draws (xoshiro256++ per sample, Acklam
    inverse, FP64 paths); results match the reference run for run.
    Fp32Philox: Philox4x32-10 normals, FP32 register-resident paths,
    compensated FP32 per-thread sums, FP64 reductions."""

    Fp64Reference = A.OF_PREC_FP64_REFERENCE
    Fp32Philox = A.OF_PREC_FP32_PHILOX


class FastRngKind(enum.Enum):
    """math::fast_rng::FastRngKind (src/math/fast_rng.rs:20-27).  The device
    engine implements the two reproducible kinds, Xoshiro256PlusPlus (the
    default) and Pcg64, in its FP64 reference mode; ThreadRng and StdRng
    (the rand crate's generators) are not available."""

    Xoshiro256PlusPlus = 0
    Pcg64 = 1
    ThreadRng = 2
    StdRng = 3


# ---------------------------------------------------------------------------
# Models and path generators (src/models/stochastic.rs, src/mc/simulation.rs)
# ---------------------------------------------------------------------------
@dataclass
class Gbm:
    mu: float
    sigma: float


@dataclass
class Heston:
    mu: float
    kappa: float
    theta: float
    xi: float
    rho: float
    v0: float

    def validate(self) -> bool:
        """Heston::validate (src/models/stochastic.rs:47-54)."""
        return (self.kappa > 0.0 and self.theta >= 0.0 and self.xi >= 0.0 and self.v0 >= 0.0
                and -1.0 < self.rho < 1.0)


@dataclass
class GbmPathGenerator:
    """GbmPathGenerator (simulation.rs:39-78); with a dividend schedule it is
    DiscreteDividendGbmPathGenerator (mc_engine.rs:123-175)."""

    model: Gbm
    s0: float
    maturity: float
    steps: int
    dividends: Optional[object] = None  # market.DividendSchedule

    def num_normal_streams(self) -> int:
        return 1

    def to_abi(self) -> A.OfModel:
        """The model struct; a dividend array stays referenced by this generator."""
        m = A.OfModel(kind=A.OF_MODEL_GBM, s0=self.s0, mu=self.model.mu, sigma=self.model.sigma,
                      maturity=self.maturity, steps=int(self.steps))
        arr = self.dividends.to_abi() if self.dividends is not None else None
        if arr is not None:
            self._abi_dividends = arr
            m.dividends = C.cast(arr, C.POINTER(A.OfDividendEvent))
            m.n_dividends = len(arr)
        return m


@dataclass
class HestonPathGenerator:
    """HestonPathGenerator (simulation.rs:80-117).  scheme "euler" is the
    reference's Euler step with the variance floored at 0 after every step;
    "qe" is Andersen's quadratic-exponential scheme (Fp32Philox only)."""

    model: Heston
    s0: float
    maturity: float
    steps: int
    scheme: str = "euler"

    def num_normal_streams(self) -> int:
        return 2

    def to_abi(self) -> A.OfModel:
        kind = A.OF_MODEL_HESTON_QE if self.scheme == "qe" else A.OF_MODEL_HESTON_EULER
        m = self.model
        return A.OfModel(kind=kind, s0=self.s0, mu=m.mu, sigma=0.0, maturity=self.maturity, steps=int(self.steps),
                         kappa=m.kappa, theta=m.theta, xi=m.xi, rho=m.rho, v0=m.v0)


PathGenerator = Union[GbmPathGenerator, HestonPathGenerator]


class ControlVariateKind(enum.Enum):
    VanillaTerminal = A.OF_CV_VANILLA_TERMINAL
    GeometricAsian = A.OF_CV_GEOMETRIC_ASIAN
    TerminalSpot = A.OF_CV_TERMINAL_SPOT


@dataclass
class ControlVariate:
    """mc::ControlVariate (simulation.rs:120-124).  The reference carries a
    closure; the device engine carries one of the evaluators the reference's
    instruments build (mc_engine.rs:458-485, 546-583) or the terminal spot."""

    expected: float
    kind: ControlVariateKind


# ---------------------------------------------------------------------------
# Payoff descriptors (MonteCarloInstrument, mc_engine.rs:44-584)
# ---------------------------------------------------------------------------
def _payoff_abi(instrument) -> Tuple[A.OfPayoff, Optional[np.ndarray]]:
    p = A.OfPayoff()
    p.option_type = instrument.option_type.value
    p.strike = float(instrument.strike)
    p.expiry = float(instrument.expiry)
    keep = None
    if isinstance(instrument, VanillaOption):
        p.kind = A.OF_PAYOFF_VANILLA
    elif isinstance(instrument, BarrierOption):
        p.kind = A.OF_PAYOFF_BARRIER
        b = instrument.barrier
        p.barrier_direction = A.OF_BARRIER_UP if b.direction is BarrierDirection.Up else A.OF_BARRIER_DOWN
        p.barrier_style = A.OF_BARRIER_IN if b.style is BarrierStyle.In else A.OF_BARRIER_OUT
        p.barrier_level = float(b.level)
        p.rebate = float(b.rebate)
    elif isinstance(instrument, AsianOption):
        p.kind = A.OF_PAYOFF_ASIAN
        s = instrument.asian
        p.averaging = A.OF_AVG_ARITHMETIC if s.averaging is Averaging.Arithmetic else A.OF_AVG_GEOMETRIC
        p.strike_type = A.OF_STRIKE_FIXED if s.strike_type is StrikeType.Fixed else A.OF_STRIKE_FLOATING
        keep = np.ascontiguousarray(s.observation_times, dtype=np.float64)
        p.observation_times = keep.ctypes.data_as(C.POINTER(C.c_double))
        p.n_observations = len(keep)
    else:
        raise PricingError.InvalidInput(f"unsupported instrument {type(instrument).__name__}")
    return p, keep


def _vanilla(option_type: OptionType, spot: float, strike: float) -> float:
    v = spot - strike if option_type is OptionType.Call else strike - spot
    return v if v > 0.0 else 0.0


def payoff_from_path(instrument, path: Sequence[float]) -> float:
    """Host evaluation of MonteCarloInstrument::payoff_from_path on a short
    path (used for the maturity == 0 branch, mc_engine.rs:896-904)."""
    st = path[-1]
    if isinstance(instrument, VanillaOption):
        return _vanilla(instrument.option_type, st, instrument.strike)
    if isinstance(instrument, BarrierOption):
        b = instrument.barrier
        hit = any(s >= b.level for s in path) if b.direction is BarrierDirection.Up else any(
            s <= b.level for s in path)
        active = hit if b.style is BarrierStyle.In else not hit
        return _vanilla(instrument.option_type, st, instrument.strike) if active else b.rebate
    if isinstance(instrument, AsianOption):
        avg = st  # average_for_observations with maturity <= 0 (mc_engine.rs:92-94)
        if instrument.asian.strike_type is StrikeType.Fixed:
            return _vanilla(instrument.option_type, avg, instrument.strike)
        return _vanilla(instrument.option_type, st, avg)
    raise PricingError.InvalidInput(f"unsupported instrument {type(instrument).__name__}")


def reference_strike(instrument, spot: float) -> float:
    """MonteCarloInstrument::reference_strike (mc_engine.rs:449-451, 496-498, 524-529)."""
    if isinstance(instrument, AsianOption) and instrument.asian.strike_type is StrikeType.Floating:
        return spot
    return instrument.strike


def instrument_control_variate(instrument, market: Market, vol: float,
                               exact_order: bool = True) -> Optional[ControlVariate]:
    """MonteCarloInstrument::control_variate (mc_engine.rs:458-485, 546-583).
    exact_order=False computes the geometric-Asian mean's covariance sum in
    O(n log n) instead of the reference's order (see
    geometric_asian_discrete_fixed)."""
    if market.has_discrete_dividends():
        return None
    if isinstance(instrument, VanillaOption):
        if not instrument.exercise.is_european:
            return None
        adjusted = market.spot * math.exp(-market.dividend_yield * instrument.expiry)
        expected_disc = bs_price(instrument.option_type, adjusted, instrument.strike, market.rate, 0.0, vol,
                                 instrument.expiry)
        df = math.exp(-market.rate * instrument.expiry)
        return ControlVariate(expected_disc / df, ControlVariateKind.VanillaTerminal)
    if isinstance(instrument, AsianOption):
        s = instrument.asian
        if s.averaging is not Averaging.Arithmetic or s.strike_type is not StrikeType.Fixed:
            return None
        expected_disc = geometric_asian_discrete_fixed(instrument.option_type, market.spot, instrument.strike,
                                                       market.rate, market.dividend_yield, vol,
                                                       s.observation_times, exact_order=exact_order)
        df = math.exp(-market.rate * instrument.expiry)
        return ControlVariate(expected_disc / df, ControlVariateKind.GeometricAsian)
    return None


# ---------------------------------------------------------------------------
# mc::MonteCarloEngine
# ---------------------------------------------------------------------------
class MonteCarloEngine:
    """mc::MonteCarloEngine (simulation.rs:126-348) on the GPU.  `run` takes
    an instrument (its built-in payoff) where the reference takes a closure."""

    def __init__(self, num_paths: int, seed: int, device: int = 0):
        self.num_paths = int(num_paths)
        self.antithetic = False
        self.control_variate: Optional[ControlVariate] = None
        self.seed = int(seed)
        self.rng_kind = FastRngKind.Xoshiro256PlusPlus
        self.reproducible = True
        self.precision = Precision.Fp64Reference
        self.device = device
        self.injected_normals: Optional[np.ndarray] = None
        self.last_kernel_ms = 0.0

    @staticmethod
    def new(num_paths: int, seed: int) -> "MonteCarloEngine":
        return MonteCarloEngine(num_paths, seed)

    def with_antithetic(self, antithetic: bool) -> "MonteCarloEngine":
        self.antithetic = bool(antithetic)
        return self

    def with_control_variate(self, cv: ControlVariate) -> "MonteCarloEngine":
        self.control_variate = cv
        return self

    def with_seed(self, seed: int) -> "MonteCarloEngine":
        self.seed = int(seed)
        self.reproducible = True
        return self

    def with_rng_kind(self, kind: FastRngKind) -> "MonteCarloEngine":
        self.rng_kind = kind
        return self

    def with_precision(self, precision: Precision) -> "MonteCarloEngine":
        self.precision = precision
        return self

    def with_injected_normals(self, normals: Optional[np.ndarray]) -> "MonteCarloEngine":
        """Test hook: use these normals ([sample][step][stream]) instead of the
        device stream (PathGenerator::generate_from_normals, simulation.rs:22)."""
        self.injected_normals = None if normals is None else np.ascontiguousarray(normals, dtype=np.float64)
        return self

    def run_full(self, generator: PathGenerator, instrument, discount_factor: float) -> A.OfMcResult:
        if self.num_paths <= 0:
            raise PricingError.InvalidInput("num_paths must be > 0")
        if self.rng_kind not in (FastRngKind.Xoshiro256PlusPlus, FastRngKind.Pcg64) or not self.reproducible:
            raise PricingError.InvalidInput(
                "the GPU engine supports the reproducible Xoshiro256PlusPlus and Pcg64 streams only")
        ctx = context(self.device)
        model = generator.to_abi()
        payoff, keep = _payoff_abi(instrument)
        cfg = A.OfMcConfig(num_paths=self.num_paths, seed=self.seed & 0xFFFFFFFFFFFFFFFF,
                           rng_kind=A.OF_RNG_PCG64 if self.rng_kind is FastRngKind.Pcg64 else A.OF_RNG_XOSHIRO256PP,
                           antithetic=int(self.antithetic), precision=self.precision.value,
                           discount_factor=float(discount_factor))
        if self.control_variate is not None:
            cfg.control_variate = self.control_variate.kind.value
            cfg.cv_expected = float(self.control_variate.expected)
        if self.injected_normals is not None:
            cfg.injected_normals = self.injected_normals.ctypes.data_as(C.POINTER(C.c_double))
            cfg.n_injected = self.injected_normals.size
        out = A.OfMcResult()
        with ctx.lock:
            ctx.check(ctx._L.of_mc_run(ctx.handle, C.byref(model), C.byref(payoff), C.byref(cfg), C.byref(out)))
        del keep
        self.last_kernel_ms = out.kernel_ms
        return out

    def run(self, generator: PathGenerator, instrument, discount_factor: float) -> Tuple[float, float]:
        out = self.run_full(generator, instrument, discount_factor)
        return out.price, out.stderr_


# ---------------------------------------------------------------------------
# engines::monte_carlo::MonteCarloPricingEngine
# ---------------------------------------------------------------------------
def _check_mc_instrument(instrument):
    if not isinstance(instrument, (VanillaOption, BarrierOption, AsianOption)):
        raise PricingError.InvalidInput(f"unsupported instrument {type(instrument).__name__}")
    instrument.validate()


class MonteCarloPricingEngine:
    """engines::monte_carlo::MonteCarloPricingEngine (mc_engine.rs:588-988) on the GPU."""

    def __init__(self, num_paths: int, num_steps: int, seed: int, device: int = 0):
        self.num_paths = int(num_paths)
        self.num_steps = int(num_steps)
        self.seed = int(seed)
        self.rng_kind = FastRngKind.Xoshiro256PlusPlus
        self.reproducible = True
        self.variance_reduction = VarianceReduction.None_
        self.precision = Precision.Fp64Reference
        self.device = device
        self.last_kernel_ms = 0.0

    @staticmethod
    def new(num_paths: int, num_steps: int, seed: int) -> "MonteCarloPricingEngine":
        return MonteCarloPricingEngine(num_paths, num_steps, seed)

    def with_variance_reduction(self, vr: VarianceReduction) -> "MonteCarloPricingEngine":
        self.variance_reduction = vr
        return self

    def with_rng_kind(self, kind: FastRngKind) -> "MonteCarloPricingEngine":
        self.rng_kind = kind
        if kind is FastRngKind.ThreadRng:
            self.reproducible = False
        return self

    def with_seed(self, seed: int) -> "MonteCarloPricingEngine":
        self.seed = int(seed)
        self.reproducible = True
        return self

    def with_randomized_streams(self) -> "MonteCarloPricingEngine":
        self.reproducible = False
        return self

    def with_precision(self, precision: Precision) -> "MonteCarloPricingEngine":
        self.precision = precision
        return self

    # The per-instrument setup of MonteCarloPricingEngine::price (mc_engine.rs:875-975).
    def _setup(self, instrument, market: Market):
        _check_mc_instrument(instrument)
        if self.num_paths == 0:
            raise PricingError.InvalidInput("num_paths must be > 0")
        if self.num_steps == 0:
            raise PricingError.InvalidInput("num_steps must be > 0")
        maturity = instrument.expiry
        if maturity < 0.0:
            raise PricingError.InvalidInput("instrument maturity must be >= 0")
        if maturity == 0.0:
            return None, PricingResult(price=payoff_from_path(instrument, [market.spot]), stderr=0.0)
        ref_k = max(reference_strike(instrument, market.spot), 1e-12)
        vol = market.vol_for(ref_k, maturity)
        if vol <= 0.0:
            raise PricingError.InvalidInput("market volatility must be > 0")
        gen = GbmPathGenerator(Gbm(market.rate - market.dividend_yield, vol), market.spot, maturity, self.num_steps,
                               market.dividend_schedule if market.has_discrete_dividends() else None)
        anti = self.variance_reduction is VarianceReduction.Antithetic
        cv = instrument_control_variate(instrument, market, vol) \
            if self.variance_reduction is VarianceReduction.ControlVariate else None
        df = math.exp(-market.rate * maturity)
        return (gen, anti, cv, df, vol), None

    def _diagnostics(self, vol: float) -> Diagnostics:
        d = Diagnostics()
        d.insert("num_paths", float(self.num_paths))
        d.insert("num_steps", float(self.num_steps))
        d.insert("vol", vol)
        return d

    def price(self, instrument, market: Market) -> PricingResult:
        setup, early = self._setup(instrument, market)
        if early is not None:
            return early
        gen, anti, cv, df, vol = setup
        eng = MonteCarloEngine(self.num_paths, self.seed, self.device).with_antithetic(anti) \
            .with_rng_kind(self.rng_kind).with_precision(self.precision)
        eng.reproducible = self.reproducible
        if cv is not None:
            eng.with_control_variate(cv)
        price, stderr = eng.run(gen, instrument, df)
        self.last_kernel_ms = eng.last_kernel_ms
        return PricingResult(price=price, stderr=stderr, greeks=None, diagnostics=self._diagnostics(vol))

    def price_batch(self, items: Sequence[Tuple[object, Market]], block: int = 0, paths_per_thread: int = 0,
                    use_graph: bool = True) -> List[PricingResult]:
        """Prices many (instrument, market) pairs in one persistent launch
        (FP32 Philox mode), with this engine's paths, steps and variance
        reduction applied to each."""
        entries, early, vols = [], {}, []
        keep = []
        for idx, (inst, mkt) in enumerate(items):
            setup, res = self._setup(inst, mkt)
            if res is not None:
                early[idx] = res
                continue
            gen, anti, cv, df, vol = setup
            payoff, k = _payoff_abi(inst)
            keep.append(k)
            keep.append(gen)  # holds the dividend array the model points to
            e = A.OfBookEntry(model=gen.to_abi(), payoff=payoff, num_paths=self.num_paths, antithetic=int(anti),
                              discount_factor=df)
            if cv is not None:
                e.control_variate = cv.kind.value
                e.cv_expected = cv.expected
            entries.append((idx, e, vol))
        out: List[Optional[PricingResult]] = [None] * len(items)
        for idx, r in early.items():
            out[idx] = r
        if entries:
            results = price_book_entries([e for _, e, _ in entries], seed=self.seed, block=block,
                                         paths_per_thread=paths_per_thread, use_graph=use_graph,
                                         device=self.device)
            for (idx, _, vol), r in zip(entries, results):
                out[idx] = PricingResult(price=r.price, stderr=r.stderr_, diagnostics=self._diagnostics(vol))
        del keep
        return out  # type: ignore[return-value]

    def price_with_greeks_aad(self, instrument, market: Market) -> PricingResult:
        """PricingEngine::price_with_greeks_aad (mc_engine.rs:977-987):
        pathwise adjoint Greeks for European vanillas, plain price otherwise."""
        if isinstance(instrument, VanillaOption):
            from .greeks import mc_european_pathwise_aad
            return mc_european_pathwise_aad(self, instrument, market)
        return self.price(instrument, market)


# ---------------------------------------------------------------------------
# engines::monte_carlo::ArithmeticAsianMC
# ---------------------------------------------------------------------------
class ArithmeticAsianMC:
    """ArithmeticAsianMC (mc_engine.rs:671-869): antithetic always on, geometric
    Asian control variate by default."""

    def __init__(self, paths: int, steps: int, seed: int, device: int = 0):
        self.paths = int(paths)
        self.steps = int(steps)
        self.seed = int(seed)
        self.control_variate = True
        self.rng_kind = FastRngKind.Xoshiro256PlusPlus
        self.reproducible = True
        self.precision = Precision.Fp64Reference
        self.device = device

    @staticmethod
    def new(paths: int, steps: int, seed: int) -> "ArithmeticAsianMC":
        return ArithmeticAsianMC(paths, steps, seed)

    def with_control_variate(self, on: bool) -> "ArithmeticAsianMC":
        self.control_variate = bool(on)
        return self

    def with_seed(self, seed: int) -> "ArithmeticAsianMC":
        self.seed = int(seed)
        self.reproducible = True
        return self

    def with_precision(self, precision: Precision) -> "ArithmeticAsianMC":
        self.precision = precision
        return self

    def price(self, instrument: AsianOption, market: Market) -> PricingResult:
        instrument.validate()
        if instrument.asian.averaging is not Averaging.Arithmetic:
            raise PricingError.InvalidInput("ArithmeticAsianMC requires Averaging::Arithmetic")
        if instrument.asian.strike_type is not StrikeType.Fixed:
            raise PricingError.InvalidInput("ArithmeticAsianMC currently supports StrikeType::Fixed only")
        if self.paths == 0:
            raise PricingError.InvalidInput("arithmetic asian mc paths must be > 0")
        if self.steps == 0:
            raise PricingError.InvalidInput("arithmetic asian mc steps must be > 0")
        maturity = instrument.expiry
        vol = market.vol_for(instrument.strike, maturity)
        if vol <= 0.0 or not math.isfinite(vol):
            raise PricingError.InvalidInput("market volatility must be finite and > 0")
        gen = GbmPathGenerator(Gbm(market.rate - market.dividend_yield, vol), market.spot, maturity, self.steps,
                               market.dividend_schedule if market.has_discrete_dividends() else None)
        eng = MonteCarloEngine(self.paths, self.seed, self.device).with_antithetic(True).with_precision(self.precision)
        if self.control_variate and not market.has_discrete_dividends():  # mc_engine.rs:791
            expected_disc = geometric_asian_discrete_fixed(instrument.option_type, market.spot, instrument.strike,
                                                           market.rate, market.dividend_yield, vol,
                                                           instrument.asian.observation_times)
            df = math.exp(-market.rate * maturity)
            eng.with_control_variate(ControlVariate(expected_disc / df, ControlVariateKind.GeometricAsian))
        price, stderr = eng.run(gen, instrument, math.exp(-market.rate * maturity))
        d = Diagnostics()
        d.insert("num_paths", float(self.paths))
        d.insert("num_steps", float(self.steps))
        d.insert("vol", vol)
        return PricingResult(price=price, stderr=stderr, diagnostics=d)


# ---------------------------------------------------------------------------
# Strike strip and batched book
# ---------------------------------------------------------------------------
def price_strike_strip(generator: PathGenerator, option_type: OptionType, strikes: Sequence[float], num_paths: int,
                       seed: int, discount_factor: float, antithetic: bool = False,
                       device: int = 0, tile_ilp: int = 0) -> List[Tuple[float, float]]:
    """European (price, stderr) for every strike from one shared FP32 Philox
    path set (of_mc_strip)."""
    ctx = context(device)
    model = generator.to_abi()
    ks = np.ascontiguousarray(strikes, dtype=np.float64)
    out = (A.OfMcResult * len(ks))()
    res: List[Tuple[float, float]] = []
    for lo in range(0, len(ks), 128):
        chunk = ks[lo:lo + 128]
        cfg = A.OfMcConfig(num_paths=int(num_paths), seed=int(seed) & 0xFFFFFFFFFFFFFFFF, antithetic=int(antithetic),
                           precision=A.OF_PREC_FP32_PHILOX, discount_factor=float(discount_factor),
                           tile_ilp=int(tile_ilp))
        part = (A.OfMcResult * len(chunk))()
        with ctx.lock:
            ctx.check(ctx._L.of_mc_strip(ctx.handle, C.byref(model), option_type.value,
                                         chunk.ctypes.data_as(C.POINTER(C.c_double)), len(chunk), C.byref(cfg),
                                         part))
        res.extend((r.price, r.stderr_) for r in part)
    del out
    return res


class StripPlan:
    """A strike strip prepared once (device buffers + captured CUDA graph);
    `launch` enqueues one replay on the context stream without a host sync,
    `results` waits and returns (price, stderr) per strike."""

    def __init__(self, generator: PathGenerator, option_type: OptionType, strikes: Sequence[float], num_paths: int,
                 seed: int, discount_factor: float, antithetic: bool = False, device: int = 0, tile_ilp: int = 0):
        self.ctx = context(device)
        self.n = len(strikes)
        self.path_steps = float(num_paths) * float(generator.steps)
        ks = np.ascontiguousarray(strikes, dtype=np.float64)
        model = generator.to_abi()
        cfg = A.OfMcConfig(num_paths=int(num_paths), seed=int(seed) & 0xFFFFFFFFFFFFFFFF, antithetic=int(antithetic),
                           precision=A.OF_PREC_FP32_PHILOX, discount_factor=float(discount_factor),
                           tile_ilp=int(tile_ilp))
        h = C.c_void_p()
        L = self.ctx._L
        with self.ctx.lock:
            self.ctx.check(L.of_strip_plan_create(self.ctx.handle, C.byref(model), option_type.value,
                                                  ks.ctypes.data_as(C.POINTER(C.c_double)), len(ks), C.byref(cfg),
                                                  C.byref(h)))
        self.handle = h

    def launch(self):
        self.ctx.check(self.ctx._L.of_strip_plan_launch(self.handle))

    def results(self) -> List[Tuple[float, float]]:
        out = (A.OfMcResult * self.n)()
        self.ctx.check(self.ctx._L.of_strip_plan_results(self.handle, out))
        return [(r.price, r.stderr_) for r in out]

    def close(self):
        if self.handle and self.handle.value:
            self.ctx._L.of_strip_plan_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def price_book_entries(entries: Sequence[A.OfBookEntry], seed: int, block: int = 0, paths_per_thread: int = 0,
                       use_graph: bool = True, device: int = 0) -> List[A.OfMcResult]:
    ctx = context(device)
    arr = (A.OfBookEntry * len(entries))(*entries)
    cfg = A.OfBookConfig(seed=int(seed) & 0xFFFFFFFFFFFFFFFF, block=block, paths_per_thread=paths_per_thread,
                         use_graph=int(use_graph))
    out = (A.OfMcResult * len(entries))()
    with ctx.lock:
        ctx.check(ctx._L.of_mc_price_book(ctx.handle, arr, len(entries), C.byref(cfg), out))
    return list(out)
