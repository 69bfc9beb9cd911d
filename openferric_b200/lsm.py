"""Longstaff-Schwartz on the GPU, mirroring openferric's
engines::lsm::LongstaffSchwartzEngine (src/engines/lsm/longstaff_schwartz.rs:66-630).

`price` keeps the reference's semantics (same validation messages, same draws
in FP64 reference mode, basis {1,S,S^2}); `with_precision(Fp32Philox)` and
`with_basis_degree(3)` select the FP32 Philox path store and the cubic basis
{1,x,x^2,x^3} (x = S/K) solved by Cholesky; `price_batch` prices many
contracts through one date loop.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _abi as A
from ._lib import context
from .core import Diagnostics, Greeks, OptionType, PricingError, PricingResult
from .engines import Precision
from .instruments import VanillaOption
from .market import Market


class LongstaffSchwartzEngine:
    """LongstaffSchwartzEngine (longstaff_schwartz.rs:66-112) with GBM dynamics."""

    def __init__(self, num_paths: int, num_steps: int, seed: int, device: int = 0):
        self.num_paths = int(num_paths)
        self.num_steps = int(num_steps)
        self.seed = int(seed)
        self.precision = Precision.Fp64Reference
        self.basis_degree = 2
        self.device = device
        self.injected_normals: Optional[np.ndarray] = None
        self.last_kernel_ms = 0.0

    @staticmethod
    def new(num_paths: int, num_steps: int, seed: int) -> "LongstaffSchwartzEngine":
        return LongstaffSchwartzEngine(num_paths, num_steps, seed)

    def with_precision(self, precision: Precision) -> "LongstaffSchwartzEngine":
        self.precision = precision
        return self

    def with_basis_degree(self, degree: int) -> "LongstaffSchwartzEngine":
        if degree not in (2, 3):
            raise PricingError.InvalidInput("basis degree must be 2 or 3")
        self.basis_degree = degree
        return self

    def with_injected_normals(self, normals: Optional[np.ndarray]) -> "LongstaffSchwartzEngine":
        """Test hook: [contract][path][step] normals instead of the device stream."""
        self.injected_normals = None if normals is None else np.ascontiguousarray(normals, dtype=np.float64)
        return self

    def _contract(self, instrument: VanillaOption, market: Market) -> Tuple[A.OfLsmContract, Optional[np.ndarray],
                                                                          float]:
        instrument.validate()
        if self.num_steps < 2:
            raise PricingError.InvalidInput("num_steps must be >= 2 for Longstaff-Schwartz")
        if self.num_paths < 3:
            raise PricingError.InvalidInput("num_paths must be >= 3 for Longstaff-Schwartz")
        vol = market.vol_for(instrument.strike, instrument.expiry) if instrument.expiry > 0.0 else 0.0
        if instrument.expiry > 0.0 and vol <= 0.0:
            raise PricingError.InvalidInput("market volatility must be > 0")
        ex = instrument.exercise
        kind = A.OF_EXERCISE_EUROPEAN if ex.is_european else (
            A.OF_EXERCISE_AMERICAN if ex.is_american else A.OF_EXERCISE_BERMUDAN)
        dates = np.ascontiguousarray(ex.dates, dtype=np.float64) if ex.is_bermudan else None
        k = A.OfLsmContract(option_type=instrument.option_type.value, exercise=kind, spot=market.spot,
                            strike=instrument.strike, rate=market.rate,
                            dividend_yield=market.effective_dividend_yield(instrument.expiry), vol=vol,
                            expiry=instrument.expiry, num_steps=self.num_steps)
        if dates is not None:
            k.exercise_dates = dates.ctypes.data_as(C.POINTER(C.c_double))
            k.n_exercise_dates = len(dates)
        return k, dates, vol

    def _run(self, items: Sequence[Tuple[VanillaOption, Market]], want_delta: bool) -> List[A.OfLsmResult]:
        ctx = context(self.device)
        built = [self._contract(i, m) for i, m in items]
        arr = (A.OfLsmContract * len(built))(*[b[0] for b in built])
        cfg = A.OfLsmConfig(num_paths=self.num_paths, seed=self.seed & 0xFFFFFFFFFFFFFFFF,
                            precision=self.precision.value, basis_degree=self.basis_degree,
                            want_delta=int(want_delta))
        if self.injected_normals is not None:
            cfg.injected_normals = self.injected_normals.ctypes.data_as(C.POINTER(C.c_double))
            cfg.n_injected = self.injected_normals.size
        out = (A.OfLsmResult * len(built))()
        with ctx.lock:
            ctx.check(ctx._L.of_lsm_price(ctx.handle, arr, len(built), C.byref(cfg), out))
        self.last_kernel_ms = out[0].kernel_ms if len(built) else 0.0
        self._vols = [b[2] for b in built]
        return list(out)

    def _result(self, r: A.OfLsmResult, vol: float, with_delta: bool) -> PricingResult:
        d = Diagnostics()
        d.insert("num_paths", float(self.num_paths))
        d.insert("num_steps", float(self.num_steps))
        d.insert("vol", vol)
        g = Greeks(r.delta, 0.0, 0.0, 0.0, 0.0) if with_delta else None
        return PricingResult(price=r.price, stderr=r.stderr_, greeks=g, diagnostics=d)

    def price(self, instrument: VanillaOption, market: Market) -> PricingResult:
        """PricingEngine<VanillaOption>::price (longstaff_schwartz.rs:421-618)."""
        if instrument.expiry == 0.0:
            instrument.validate()
            v = market.spot - instrument.strike if instrument.option_type is OptionType.Call else \
                instrument.strike - market.spot
            return PricingResult(price=max(v, 0.0), stderr=0.0)
        r = self._run([(instrument, market)], False)[0]
        return self._result(r, self._vols[0], False)

    def price_with_delta(self, instrument: VanillaOption, market: Market) -> PricingResult:
        """Price plus the pathwise (adjoint) delta under the fitted exercise
        policy: d/dS0 of the realised discounted cash flow, S_tau/S0 per path."""
        r = self._run([(instrument, market)], True)[0]
        return self._result(r, self._vols[0], True)

    def price_batch(self, items: Sequence[Tuple[VanillaOption, Market]], with_delta: bool = False) -> List[
            PricingResult]:
        rs = self._run(items, with_delta)
        return [self._result(r, v, with_delta) for r, v in zip(rs, self._vols)]


def xoshiro_jump_states(seed: int, draws: Sequence[int], device: int = 0) -> List[List[int]]:
    """States of the xoshiro256++ stream seeded with `seed` after each entry of
    `draws` next_u64 calls (device GF(2) jump-ahead)."""
    ctx = context(device)
    d = np.ascontiguousarray(draws, dtype=np.uint64)
    out = np.zeros(len(d) * 4, dtype=np.uint64)
    with ctx.lock:
        ctx.check(ctx._L.of_xoshiro_jump(ctx.handle, seed & 0xFFFFFFFFFFFFFFFF,
                                         d.ctypes.data_as(C.POINTER(C.c_uint64)), len(d),
                                         out.ctypes.data_as(C.POINTER(C.c_uint64))))
    return out.reshape(-1, 4).tolist()
