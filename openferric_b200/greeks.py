"""Monte Carlo Greeks on the GPU, mirroring openferric's
engines::monte_carlo::{mc_aad, mc_greeks} (src/engines/monte_carlo/mc_aad.rs,
mc_greeks.rs): same entry points, validation and estimator definitions, on the
reference's own random streams (FP64)."""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Tuple

from . import _abi as A
from ._lib import context
from .core import Diagnostics, Greeks, OptionType, PricingError, PricingResult
from .engines import FastRngKind, Heston, MonteCarloPricingEngine, VarianceReduction
from .instruments import VanillaOption
from .market import Market


def _call(name: str, p: A.OfGreeksParams, device: int = 0) -> A.OfGreeksResult:
    ctx = context(device)
    out = A.OfGreeksResult()
    with ctx.lock:
        ctx.check(getattr(ctx._L, name)(ctx.handle, C.byref(p), C.byref(out)))
    return out


def mc_european_pathwise_aad(engine: MonteCarloPricingEngine, instrument: VanillaOption,
                             market: Market) -> PricingResult:
    """mc_european_pathwise_aad (mc_aad.rs:75-219)."""
    instrument.validate()
    if not instrument.exercise.is_european:
        raise PricingError.InvalidInput("mc pathwise AAD supports European exercise only")
    if engine.num_paths == 0:
        raise PricingError.InvalidInput("num_paths must be > 0")
    if engine.num_steps == 0:
        raise PricingError.InvalidInput("num_steps must be > 0")
    if instrument.expiry <= 0.0:
        v = market.spot - instrument.strike if instrument.option_type is OptionType.Call else \
            instrument.strike - market.spot
        return PricingResult(price=max(v, 0.0), stderr=0.0, greeks=Greeks(0.0, 0.0, 0.0, 0.0, 0.0))
    vol = market.vol_for(instrument.strike, instrument.expiry)
    if vol <= 0.0 or not math.isfinite(vol):
        raise PricingError.InvalidInput("market volatility must be finite and > 0")
    if engine.rng_kind is not FastRngKind.Xoshiro256PlusPlus or not engine.reproducible:
        raise PricingError.InvalidInput("the GPU engine supports the reproducible Xoshiro256PlusPlus stream only")
    p = A.OfGreeksParams(option_type=instrument.option_type.value,
                         antithetic=int(engine.variance_reduction is VarianceReduction.Antithetic),
                         spot=market.spot, strike=instrument.strike, rate=market.rate,
                         dividend_yield=market.effective_dividend_yield(instrument.expiry), vol=vol,
                         expiry=instrument.expiry, num_paths=engine.num_paths, num_steps=engine.num_steps,
                         seed=engine.seed & 0xFFFFFFFFFFFFFFFF)
    r = _call("of_mc_european_pathwise_aad", p, engine.device)
    d = Diagnostics()
    d.insert("num_paths", float(engine.num_paths))
    d.insert("num_steps", float(engine.num_steps))
    d.insert("vol", vol)
    return PricingResult(price=r.price, stderr=r.stderr_, greeks=Greeks(r.delta, 0.0, r.vega, r.theta, r.rho),
                         diagnostics=d)


@dataclass
class HestonAadConfig:
    """HestonAadConfig (mc_aad.rs:222-237)."""

    num_paths: int
    num_steps: int
    seed: int


def heston_price_delta_aad(option_type: OptionType, strike: float, maturity: float, spot: float, rate: float,
                           model: Heston, config: HestonAadConfig, device: int = 0) -> Tuple[float, float]:
    """heston_price_delta_aad (mc_aad.rs:280-342): (mean price, mean delta)."""
    if config.num_paths == 0:
        raise PricingError.InvalidInput("num_paths must be > 0")
    if config.num_steps == 0:
        raise PricingError.InvalidInput("num_steps must be > 0")
    if maturity <= 0.0:
        v = spot - strike if option_type is OptionType.Call else strike - spot
        return max(v, 0.0), 0.0
    if not model.validate():
        raise PricingError.InvalidInput("invalid Heston parameters")
    p = A.OfGreeksParams(option_type=option_type.value, spot=spot, strike=strike, rate=rate, expiry=maturity,
                         num_paths=config.num_paths, num_steps=config.num_steps,
                         seed=config.seed & 0xFFFFFFFFFFFFFFFF, mu=model.mu, kappa=model.kappa, theta=model.theta,
                         xi=model.xi, rho=model.rho, v0=model.v0)
    r = _call("of_heston_price_delta_aad", p, device)
    return r.price, r.delta


class MonteCarloGreeksEngine:
    """MonteCarloGreeksEngine (mc_greeks.rs:20-95)."""

    def __init__(self, num_paths: int, seed: int, device: int = 0):
        self.num_paths = int(num_paths)
        self.seed = int(seed)
        self.antithetic = True
        self.spot_bump_rel = 1.0e-2
        self.rng_kind = FastRngKind.Xoshiro256PlusPlus
        self.reproducible = True
        self.device = device

    @staticmethod
    def new(num_paths: int, seed: int) -> "MonteCarloGreeksEngine":
        return MonteCarloGreeksEngine(num_paths, seed)

    def with_antithetic(self, on: bool) -> "MonteCarloGreeksEngine":
        self.antithetic = bool(on)
        return self

    def with_spot_bump_rel(self, rel: float) -> "MonteCarloGreeksEngine":
        self.spot_bump_rel = max(float(rel), 1.0e-6)
        return self

    def with_seed(self, seed: int) -> "MonteCarloGreeksEngine":
        self.seed = int(seed)
        self.reproducible = True
        return self

    def _run(self, instrument: VanillaOption, market: Market) -> A.OfGreeksResult:
        instrument.validate()
        if not instrument.exercise.is_european:
            raise PricingError.InvalidInput("MonteCarloGreeksEngine supports European exercise only")
        if self.num_paths == 0:
            raise PricingError.InvalidInput("num_paths must be > 0")
        if self.spot_bump_rel <= 0.0 or not math.isfinite(self.spot_bump_rel):
            raise PricingError.InvalidInput("spot_bump_rel must be finite and > 0")
        if instrument.expiry <= 0.0:
            return A.OfGreeksResult()
        vol = market.vol_for(instrument.strike, instrument.expiry)
        if vol <= 0.0 or not math.isfinite(vol):
            raise PricingError.InvalidInput("market volatility must be finite and > 0")
        p = A.OfGreeksParams(option_type=instrument.option_type.value, antithetic=int(self.antithetic),
                             spot=market.spot, strike=instrument.strike, rate=market.rate,
                             dividend_yield=market.effective_dividend_yield(instrument.expiry), vol=vol,
                             expiry=instrument.expiry, num_paths=self.num_paths,
                             seed=self.seed & 0xFFFFFFFFFFFFFFFF, spot_bump_rel=self.spot_bump_rel)
        return _call("of_mc_greek_estimators", p, self.device)

    def estimate_pathwise(self, instrument: VanillaOption, market: Market) -> Greeks:
        r = self._run(instrument, market)
        return Greeks(r.delta, r.gamma, 0.0, 0.0, 0.0)

    def estimate_likelihood_ratio(self, instrument: VanillaOption, market: Market) -> Greeks:
        r = self._run(instrument, market)
        return Greeks(r.lr_delta, r.lr_gamma, r.lr_vega, 0.0, 0.0)
