"""Longstaff-Schwartz on the GPU, mirroring openferric's
engines::lsm::LongstaffSchwartzEngine (src/engines/lsm/longstaff_schwartz.rs:66-630).

`price` keeps the reference's semantics (same validation messages, same draws
in FP64 reference mode, basis {1,S,S^2}); `with_precision(Fp32Philox)` and
`with_basis_degree(3)` select the FP32 Philox path store and the cubic basis
{1,x,x^2,x^3} (x = S/K) solved by Cholesky; `price_batch` prices many
contracts through one date loop.  `price_bermudan_with_boundary` prices a
BermudanOption (a strike per exercise date) under GBM, local-vol Euler or
Heston Euler paths and returns the exercise boundary.  A BarrierOption is
priced by the engine's European barrier Monte Carlo on its single stream
(of_lsm_barrier).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _abi as A
from ._lib import context
from .core import BarrierDirection, BarrierStyle, Diagnostics, Greeks, OptionType, PricingError, PricingResult
from .engines import Precision
from .instruments import BarrierOption, BermudanOption, VanillaOption
from .market import Market


@dataclass(frozen=True)
class LsmDynamics:
    """LsmDynamics (longstaff_schwartz.rs:24-39): Gbm, LocalVolEuler or
    HestonEuler(kappa, theta, xi, rho, v0) for the Bermudan path simulation."""

    kind: int = A.OF_LSM_GBM
    kappa: float = 0.0
    theta: float = 0.0
    xi: float = 0.0
    rho: float = 0.0
    v0: float = 0.0


LsmDynamics.Gbm = LsmDynamics(A.OF_LSM_GBM)
LsmDynamics.LocalVolEuler = LsmDynamics(A.OF_LSM_LOCAL_VOL)


@dataclass
class ExerciseBoundaryPoint:
    """ExerciseBoundaryPoint (longstaff_schwartz.rs:42-55)."""

    time: float
    strike: float
    boundary_spot: Optional[float]
    itm_paths: int
    exercised_paths: int


@dataclass
class BermudanLsmOutput:
    """BermudanLsmOutput (longstaff_schwartz.rs:57-64)."""

    result: PricingResult
    exercise_boundary: List[ExerciseBoundaryPoint]


class LongstaffSchwartzEngine:
    """LongstaffSchwartzEngine (longstaff_schwartz.rs:66-112)."""

    def __init__(self, num_paths: int, num_steps: int, seed: int, device: int = 0):
        self.num_paths = int(num_paths)
        self.num_steps = int(num_steps)
        self.seed = int(seed)
        self.precision = Precision.Fp64Reference
        self.basis_degree = 2
        self.device = device
        self.dynamics = LsmDynamics.Gbm
        self.injected_normals: Optional[np.ndarray] = None
        self.batch_contracts = 0
        self.last_kernel_ms = 0.0

    @staticmethod
    def new(num_paths: int, num_steps: int, seed: int) -> "LongstaffSchwartzEngine":
        return LongstaffSchwartzEngine(num_paths, num_steps, seed)

    def with_local_vol_dynamics(self) -> "LongstaffSchwartzEngine":
        """Local-vol Euler paths for Bermudan pricing, sigma = market.vol_for(S, t) (:81-85)."""
        self.dynamics = LsmDynamics.LocalVolEuler
        return self

    def with_heston_dynamics(self, model) -> "LongstaffSchwartzEngine":
        """Heston Euler paths for Bermudan pricing; the drift is r - q, model.mu is ignored (:87-112)."""
        self.dynamics = LsmDynamics(A.OF_LSM_HESTON_EULER, model.kappa, model.theta, model.xi, model.rho, model.v0)
        return self

    def with_precision(self, precision: Precision) -> "LongstaffSchwartzEngine":
        self.precision = precision
        return self

    def with_basis_degree(self, degree: int) -> "LongstaffSchwartzEngine":
        if degree not in (2, 3):
            raise PricingError.InvalidInput("basis degree must be 2 or 3")
        self.basis_degree = degree
        return self

    def with_batch_contracts(self, n: int) -> "LongstaffSchwartzEngine":
        """At most this many contracts per date loop of price_batch (0 = as
        many as the path-store budget allows)."""
        if n < 0:
            raise PricingError.InvalidInput("batch_contracts must be >= 0")
        self.batch_contracts = int(n)
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
                            want_delta=int(want_delta), batch_contracts=self.batch_contracts)
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

    def price_bermudan_with_boundary(self, instrument: BermudanOption, market: Market) -> BermudanLsmOutput:
        """price_bermudan_with_boundary (longstaff_schwartz.rs:294-417): the
        price and the exercise boundary (largest exercised spot of a put,
        smallest of a call) at each scheduled step, then the terminal point."""
        instrument.validate()
        if self.num_steps < 2:
            raise PricingError.InvalidInput("num_steps must be >= 2 for Longstaff-Schwartz")
        if self.num_paths < 3:
            raise PricingError.InvalidInput("num_paths must be >= 3 for Longstaff-Schwartz")
        sched = instrument.effective_schedule()
        ts = np.ascontiguousarray([t for t, _ in sched], dtype=np.float64)
        ks = np.ascontiguousarray([k for _, k in sched], dtype=np.float64)
        terminal_strike = float(ks[-1])
        dyn = self.dynamics
        k = A.OfBermudanContract(option_type=instrument.option_type.value, dynamics=dyn.kind, spot=market.spot,
                                 rate=market.rate, dividend_yield=market.effective_dividend_yield(instrument.expiry),
                                 expiry=instrument.expiry, num_steps=self.num_steps,
                                 schedule_times=ts.ctypes.data_as(C.POINTER(C.c_double)),
                                 schedule_strikes=ks.ctypes.data_as(C.POINTER(C.c_double)), n_schedule=len(ts),
                                 kappa=dyn.kappa, theta=dyn.theta, xi=dyn.xi, rho=dyn.rho, v0=dyn.v0)
        keep = [ts, ks]
        vol = None
        if dyn.kind == A.OF_LSM_GBM:
            vol = market.vol_for(terminal_strike, instrument.expiry)
            k.vol = vol
        elif dyn.kind == A.OF_LSM_LOCAL_VOL:
            gk, gt, gv = (np.ascontiguousarray(a, dtype=np.float64) for a in market.vol.grid())
            keep += [gk, gt, gv]
            k.lv_strikes = gk.ctypes.data_as(C.POINTER(C.c_double))
            k.lv_n_strikes = len(gk)
            k.lv_expiries = gt.ctypes.data_as(C.POINTER(C.c_double))
            k.lv_n_expiries = len(gt)
            k.lv_vols = gv.ctypes.data_as(C.POINTER(C.c_double))
        cfg = A.OfLsmConfig(num_paths=self.num_paths, seed=self.seed & 0xFFFFFFFFFFFFFFFF,
                            precision=self.precision.value, basis_degree=self.basis_degree, want_delta=0)
        if self.injected_normals is not None:
            cfg.injected_normals = self.injected_normals.ctypes.data_as(C.POINTER(C.c_double))
            cfg.n_injected = self.injected_normals.size
        cap = len(sched) + 1
        pts = (A.OfBoundaryPoint * cap)()
        nb = C.c_int64()
        out = A.OfLsmResult()
        ctx = context(self.device)
        with ctx.lock:
            ctx.check(ctx._L.of_lsm_bermudan(ctx.handle, C.byref(k), C.byref(cfg), C.byref(out), pts, cap,
                                             C.byref(nb)))
        del keep
        self.last_kernel_ms = out.kernel_ms
        d = Diagnostics()
        d.insert("num_paths", float(self.num_paths))
        d.insert("num_steps", float(self.num_steps))
        d.insert("exercise_dates", float(len(sched)))
        if vol is not None:
            d.insert("vol", vol)
        boundary = [ExerciseBoundaryPoint(p.time, p.strike, p.boundary_spot if p.has_boundary else None,
                                          int(p.itm_paths), int(p.exercised_paths)) for p in pts[:nb.value]]
        return BermudanLsmOutput(PricingResult(price=out.price, stderr=out.stderr_, diagnostics=d), boundary)

    def price_barrier(self, instrument: BarrierOption, market: Market) -> PricingResult:
        """PricingEngine<BarrierOption>::price (longstaff_schwartz.rs:632-736):
        the engine's single xoshiro256++ stream, path-major, log-Euler steps,
        the barrier monitored on every point of the path including the spot,
        the vanilla payoff when active and the rebate otherwise, discounted by
        exp(-r T).  FP64 reference draws only."""
        instrument.validate()
        if self.num_steps == 0:
            raise PricingError.InvalidInput("num_steps must be > 0")
        if self.num_paths == 0:
            raise PricingError.InvalidInput("num_paths must be > 0")
        vol = market.vol_for(instrument.strike, instrument.expiry)
        if vol <= 0.0:
            raise PricingError.InvalidInput("market volatility must be > 0")
        b = instrument.barrier
        k = A.OfLsmBarrierContract(
            option_type=instrument.option_type.value,
            barrier_direction=A.OF_BARRIER_UP if b.direction is BarrierDirection.Up else A.OF_BARRIER_DOWN,
            barrier_style=A.OF_BARRIER_IN if b.style is BarrierStyle.In else A.OF_BARRIER_OUT,
            spot=market.spot, strike=instrument.strike, rate=market.rate,
            dividend_yield=market.effective_dividend_yield(instrument.expiry), vol=vol, expiry=instrument.expiry,
            barrier_level=b.level, rebate=b.rebate, num_steps=self.num_steps)
        cfg = A.OfLsmConfig(num_paths=self.num_paths, seed=self.seed & 0xFFFFFFFFFFFFFFFF,
                            precision=self.precision.value, basis_degree=self.basis_degree, want_delta=0)
        if self.injected_normals is not None:
            cfg.injected_normals = self.injected_normals.ctypes.data_as(C.POINTER(C.c_double))
            cfg.n_injected = self.injected_normals.size
        out = A.OfLsmResult()
        ctx = context(self.device)
        with ctx.lock:
            ctx.check(ctx._L.of_lsm_barrier(ctx.handle, C.byref(k), C.byref(cfg), C.byref(out)))
        self.last_kernel_ms = out.kernel_ms
        d = Diagnostics()
        d.insert("num_paths", float(self.num_paths))
        d.insert("num_steps", float(self.num_steps))
        d.insert("vol", vol)
        return PricingResult(price=out.price, stderr=out.stderr_, diagnostics=d)

    def price(self, instrument, market: Market) -> PricingResult:
        """PricingEngine<VanillaOption>::price (longstaff_schwartz.rs:421-618);
        a BermudanOption goes through price_bermudan_with_boundary (:620-630),
        a BarrierOption through price_barrier (:632-736)."""
        if isinstance(instrument, BermudanOption):
            return self.price_bermudan_with_boundary(instrument, market).result
        if isinstance(instrument, BarrierOption):
            return self.price_barrier(instrument, market)
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
