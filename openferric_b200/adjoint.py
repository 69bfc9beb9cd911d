"""Heston pathwise adjoint Greeks (of_heston_price_adjoint) and their
torch.autograd.Function.

`price_with_adjoint` prices a European or daily-fixing arithmetic Asian option
under Heston (Andersen QE, FP32 paths) and returns the price with
d/d(S0, r, v0, kappa, theta, xi, rho) from one forward pass and one backward
sweep.  `HestonAdjointFunction.apply(params, spec)` exposes the same call to
autograd: the forward returns the price, the backward multiplies the incoming
gradient by the adjoint Greeks computed in the forward.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Dict, Optional

from . import _abi as A
from ._lib import context
from .core import Averaging, OptionType, PricingError, StrikeType
from .engines import Heston
from .instruments import AsianOption, VanillaOption
from .market import Market


@dataclass
class AdjointResult:
    price: float
    stderr: float
    greeks: Dict[str, float]
    greeks_stderr: Dict[str, float]
    kernel_ms: float = 0.0


@dataclass
class HestonAdjointSpec:
    """Contract and simulation settings that stay fixed under differentiation."""

    strike: float
    expiry: float
    num_paths: int
    num_steps: int
    seed: int
    option_type: OptionType = OptionType.Call
    asian: bool = True
    dividend_yield: float = 0.0
    checkpoint_every: int = 32
    # Half-width of the smoothed QE branch switch around psi_c = 1.5 (0 = hard switch,
    # whose jump a pathwise derivative cannot see; see include/of_gpu.h).
    qe_switch_band: float = 0.05


def _params(spec: HestonAdjointSpec, spot, rate, v0, kappa, theta, xi, rho, forward_only=False):
    return A.OfHestonAdjointParams(
        spot=float(spot), strike=float(spec.strike), rate=float(rate), dividend_yield=float(spec.dividend_yield),
        expiry=float(spec.expiry), kappa=float(kappa), theta=float(theta), xi=float(xi), rho=float(rho),
        v0=float(v0), num_paths=int(spec.num_paths), num_steps=int(spec.num_steps),
        seed=int(spec.seed) & 0xFFFFFFFFFFFFFFFF, option_type=spec.option_type.value,
        payoff=A.OF_PAYOFF_ASIAN if spec.asian else A.OF_PAYOFF_VANILLA, scheme=A.OF_MODEL_HESTON_QE,
        checkpoint_every=int(spec.checkpoint_every), forward_only=int(forward_only),
        qe_switch_band=float(spec.qe_switch_band))


def heston_adjoint(spec: HestonAdjointSpec, spot: float, rate: float, v0: float, kappa: float, theta: float,
                   xi: float, rho: float, forward_only: int = 0, device: int = 0) -> AdjointResult:
    """forward_only: 0 price + adjoint Greeks, 1 price only (FP32), 2 price
    only in FP64 on the same draws (for bump-and-revalue with common random
    numbers)."""
    ctx = context(device)
    p = _params(spec, spot, rate, v0, kappa, theta, xi, rho, forward_only)
    out = A.OfAdjointResult()
    with ctx.lock:
        ctx.check(ctx._L.of_heston_price_adjoint(ctx.handle, C.byref(p), C.byref(out)))
    return AdjointResult(out.price, out.stderr_, dict(zip(A.OF_ADJ_NAMES, list(out.greeks))),
                         dict(zip(A.OF_ADJ_NAMES, list(out.greeks_stderr))), out.kernel_ms)


def price_with_adjoint(instrument, market: Market, model: Heston, num_paths: int, num_steps: int, seed: int,
                       device: int = 0) -> AdjointResult:
    """Price and Heston sensitivities of a European vanilla or a daily-fixing
    fixed-strike arithmetic Asian (observation at every simulation step)."""
    if isinstance(instrument, VanillaOption):
        instrument.validate()
        if not instrument.exercise.is_european:
            raise PricingError.InvalidInput("adjoint pricing supports European exercise only")
        asian = False
    elif isinstance(instrument, AsianOption):
        instrument.validate()
        s = instrument.asian
        if s.averaging is not Averaging.Arithmetic or s.strike_type is not StrikeType.Fixed:
            raise PricingError.InvalidInput("adjoint pricing supports fixed-strike arithmetic Asians")
        expected = [instrument.expiry * (j / num_steps) for j in range(1, num_steps + 1)]
        if len(s.observation_times) != num_steps or any(
                abs(a - b) > 1e-12 * max(1.0, instrument.expiry) for a, b in zip(s.observation_times, expected)):
            raise PricingError.InvalidInput("adjoint Asian pricing needs a fixing at every simulation step")
        asian = True
    else:
        raise PricingError.InvalidInput(f"unsupported instrument {type(instrument).__name__}")
    spec = HestonAdjointSpec(strike=instrument.strike, expiry=instrument.expiry, num_paths=num_paths,
                             num_steps=num_steps, seed=seed, option_type=instrument.option_type, asian=asian,
                             dividend_yield=market.dividend_yield)
    return heston_adjoint(spec, market.spot, market.rate, model.v0, model.kappa, model.theta, model.xi, model.rho,
                          device=device)


try:
    import torch

    class HestonAdjointFunction(torch.autograd.Function):
        """price = HestonAdjointFunction.apply(params, spec) with params =
        tensor([S0, r, v0, kappa, theta, xi, rho]); backward returns
        grad * (d price / d params) from the adjoint kernel."""

        @staticmethod
        def forward(ctx, params, spec: HestonAdjointSpec):
            vals = [float(x) for x in params.detach().cpu().double().tolist()]
            res = heston_adjoint(spec, *vals)
            g = torch.tensor([res.greeks[n] for n in A.OF_ADJ_NAMES], dtype=params.dtype, device=params.device)
            ctx.save_for_backward(g)
            return torch.tensor(res.price, dtype=params.dtype, device=params.device)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g, None

except ImportError:  # pragma: no cover - torch is part of the image
    HestonAdjointFunction = None
