"""Market snapshot, mirroring openferric's `market::Market` (src/market/market.rs:180-415)."""
from __future__ import annotations

from dataclasses import dataclass, field
import math
from typing import Callable, Optional, Sequence

from .core import PricingError


class SampledVolSurface:
    """market::SampledVolSurface (src/market/market.rs:52-175): vols on a
    strictly increasing strike x expiry grid, looked up bilinearly
    (strike first, then expiry), flat outside the grid."""

    # The grids MarketBuilder samples a non-parametric surface onto
    # (market.rs:93-102): strikes are spot times these multipliers.
    DEFAULT_MONEYNESS = (0.5, 0.6, 0.7, 0.8, 0.9, 0.95, 1.0, 1.05, 1.1, 1.15, 1.2, 1.3, 1.4, 1.5, 1.7, 1.9, 2.1)
    DEFAULT_EXPIRIES = (1.0 / 52.0, 1.0 / 12.0, 0.25, 0.5, 1.0, 2.0, 3.0, 5.0, 10.0)

    def __init__(self, strikes: Sequence[float], expiries: Sequence[float], vols: Sequence[Sequence[float]]):
        self.strikes = [float(k) for k in strikes]
        self.expiries = [float(t) for t in expiries]
        self.vols = [[float(v) for v in row] for row in vols]

    @staticmethod
    def new(strikes, expiries, vols) -> "SampledVolSurface":
        """SampledVolSurface::new (market.rs:62-91), same messages (raised as InvalidInput)."""
        if len(strikes) < 2 or len(expiries) < 2:
            raise PricingError.InvalidInput("sampled surface requires >= 2 strikes and >= 2 expiries")
        if any(b <= a for a, b in zip(strikes, strikes[1:])):
            raise PricingError.InvalidInput("sampled surface strikes must be strictly increasing")
        if any(b <= a for a, b in zip(expiries, expiries[1:])):
            raise PricingError.InvalidInput("sampled surface expiries must be strictly increasing")
        if len(vols) != len(expiries):
            raise PricingError.InvalidInput("sampled surface row count must match expiries")
        if any(len(row) != len(strikes) for row in vols):
            raise PricingError.InvalidInput("sampled surface each row must match strike count")
        if any((not math.isfinite(v)) or v <= 0.0 for row in vols for v in row):
            raise PricingError.InvalidInput("sampled surface vols must be finite and > 0")
        return SampledVolSurface(strikes, expiries, vols)

    @staticmethod
    def from_surface(surface: Callable[[float, float], float], spot: float) -> "SampledVolSurface":
        """SampledVolSurface::from_surface (market.rs:127-146)."""
        spot = max(spot, 1.0e-8)
        strikes = [max(spot * m, 1.0e-8) for m in SampledVolSurface.DEFAULT_MONEYNESS]
        rows = []
        for t in SampledVolSurface.DEFAULT_EXPIRIES:
            row = []
            for k in strikes:
                v = float(surface(k, t))
                row.append(max(v, 1.0e-8) if math.isfinite(v) else 1.0e-8)
            rows.append(row)
        return SampledVolSurface(strikes, list(SampledVolSurface.DEFAULT_EXPIRIES), rows)

    @staticmethod
    def _locate(grid, x):
        if x <= grid[0]:
            return 0, 0, 0.0
        last = len(grid) - 1
        if x >= grid[last]:
            return last, last, 0.0
        lo = 0
        for i in range(last):
            if grid[i] <= x <= grid[i + 1]:
                lo = i
                break
        return lo, lo + 1, (x - grid[lo]) / (grid[lo + 1] - grid[lo])

    def vol(self, strike: float, expiry: float) -> float:
        e0, e1, ew = self._locate(self.expiries, max(expiry, self.expiries[0]))
        s0, s1, sw = self._locate(self.strikes, max(strike, self.strikes[0]))
        v = self.vols
        if e0 == e1 and s0 == s1:
            return v[e0][s0]
        if e0 == e1:
            return v[e0][s0] + (v[e0][s1] - v[e0][s0]) * sw
        if s0 == s1:
            return v[e0][s0] + (v[e1][s0] - v[e0][s0]) * ew
        a = v[e0][s0] + (v[e0][s1] - v[e0][s0]) * sw
        b = v[e1][s0] + (v[e1][s1] - v[e1][s0]) * sw
        return a + (b - a) * ew

    def grid(self):
        """(strikes, expiries, vols[expiry][strike]) as float64 arrays."""
        import numpy as np
        return (np.asarray(self.strikes, dtype=np.float64), np.asarray(self.expiries, dtype=np.float64),
                np.asarray(self.vols, dtype=np.float64))


class VolSource:
    """market::VolSource (src/market/market.rs:179-198): a flat vol, or a
    sampled surface (MarketBuilder samples a callable surface onto the
    default grid, as the reference does for non-parametric surfaces)."""

    def __init__(self, flat: Optional[float] = None, sampled: Optional[SampledVolSurface] = None,
                 surface: Optional[Callable[[float, float], float]] = None):
        self.flat = flat
        self.sampled = sampled
        self.surface = surface

    def vol(self, strike: float, expiry: float) -> float:
        if self.sampled is not None:
            return self.sampled.vol(strike, expiry)
        if self.surface is not None:
            return float(self.surface(strike, expiry))
        return float(self.flat)

    def grid(self):
        """The source as a sampled grid (a flat vol is a 1 x 1 grid)."""
        import numpy as np
        if self.sampled is not None:
            return self.sampled.grid()
        if self.surface is not None:
            raise PricingError.InvalidInput("an unsampled vol surface has no grid")
        one = np.ones(1, dtype=np.float64)
        return one, one, np.full((1, 1), float(self.flat))


class DividendKind:
    """DividendKind (src/market/dividends.rs:16-43)."""

    CASH = 0
    PROPORTIONAL = 1


@dataclass(frozen=True)
class DividendEvent:
    """DividendEvent (src/market/dividends.rs:45-92): a cash amount or a
    proportional ratio at an ex-dividend time (years)."""

    time: float
    kind: int
    amount: float

    @staticmethod
    def cash(time: float, amount: float) -> "DividendEvent":
        e = DividendEvent(float(time), DividendKind.CASH, float(amount))
        e.validate()
        return e

    @staticmethod
    def proportional(time: float, ratio: float) -> "DividendEvent":
        e = DividendEvent(float(time), DividendKind.PROPORTIONAL, float(ratio))
        e.validate()
        return e

    def apply_jump(self, pre_div_spot: float) -> float:
        if self.kind == DividendKind.CASH:
            return max(pre_div_spot - self.amount, 0.0)
        return pre_div_spot * (1.0 - self.amount)

    def validate(self) -> None:
        if not math.isfinite(self.time) or self.time <= 0.0:
            raise PricingError.InvalidInput("dividend event time must be finite and > 0")
        if self.kind == DividendKind.CASH:
            if not math.isfinite(self.amount) or self.amount < 0.0:
                raise PricingError.InvalidInput("cash dividend amount must be finite and >= 0")
        elif not math.isfinite(self.amount) or not 0.0 <= self.amount < 1.0:
            raise PricingError.InvalidInput("proportional dividend ratio must be finite and in [0, 1)")


class DividendSchedule:
    """DividendSchedule (src/market/dividends.rs:93-228): events sorted by
    time, strictly increasing."""

    def __init__(self, events=()):
        self._events = tuple(sorted(events, key=lambda e: e.time))

    @staticmethod
    def new(events) -> "DividendSchedule":
        s = DividendSchedule(events)
        s.validate()
        return s

    @staticmethod
    def empty() -> "DividendSchedule":
        return DividendSchedule(())

    def is_empty(self) -> bool:
        return not self._events

    def events(self):
        return self._events

    def events_until(self, maturity: float):
        return [e for e in self._events if e.time <= maturity]

    def validate(self) -> None:
        prev = 0.0
        for e in self._events:
            e.validate()
            if e.time <= prev:
                raise PricingError.InvalidInput("dividend event times must be strictly increasing")
            prev = e.time

    def forward_price(self, spot: float, rate: float, q: float, maturity: float) -> float:
        """Forward with deterministic jumps (dividends.rs:145-184)."""
        if maturity <= 0.0:
            return spot
        if not math.isfinite(spot) or spot <= 0.0:
            return 0.0
        carry = rate - q
        fwd = spot * math.exp(carry * maturity)
        for e in self.events_until(maturity):
            if e.kind == DividendKind.CASH:
                fwd -= e.amount * math.exp(carry * (maturity - e.time))
            else:
                fwd *= 1.0 - e.amount
        return max(fwd, 0.0)

    def prepaid_forward_spot(self, spot: float, rate: float, q: float, maturity: float) -> float:
        return self.forward_price(spot, rate, q, maturity) * math.exp(-rate * maturity)

    def escrowed_spot_adjustment(self, spot: float, rate: float, maturity: float) -> float:
        return self.prepaid_forward_spot(spot, rate, 0.0, maturity)

    def effective_dividend_yield(self, spot: float, rate: float, q: float, maturity: float) -> float:
        """dividends.rs:203-218."""
        if maturity <= 0.0 or spot <= 0.0:
            return q
        ratio = max(self.forward_price(spot, rate, q, maturity) / spot, 1.0e-16)
        return rate - math.log(ratio) / maturity

    def apply_jumps_until(self, spot: float, time: float) -> float:
        for e in self.events_until(time):
            spot = e.apply_jump(spot)
        return spot

    def to_abi(self):
        """The events as an of_dividend_event array (None when empty)."""
        from . import _abi as A
        if not self._events:
            return None
        return (A.OfDividendEvent * len(self._events))(
            *[A.OfDividendEvent(time=e.time, kind=e.kind, amount=e.amount) for e in self._events])


@dataclass
class Market:
    """market::Market (src/market/market.rs:201-302)."""

    spot: float
    rate: float
    dividend_yield: float
    vol: VolSource
    reference_date: Optional[str] = None
    dividend_schedule: "DividendSchedule" = field(default_factory=lambda: DividendSchedule.empty())

    @staticmethod
    def builder() -> "MarketBuilder":
        return MarketBuilder()

    def has_discrete_dividends(self) -> bool:
        return not self.dividend_schedule.is_empty()

    def forward_price(self, maturity: float) -> float:
        return self.dividend_schedule.forward_price(self.spot, self.rate, self.dividend_yield, maturity)

    def prepaid_forward_spot(self, maturity: float) -> float:
        return self.dividend_schedule.prepaid_forward_spot(self.spot, self.rate, self.dividend_yield, maturity)

    def effective_dividend_yield(self, maturity: float) -> float:
        return self.dividend_schedule.effective_dividend_yield(self.spot, self.rate, self.dividend_yield, maturity)

    def vol_for(self, strike: float, expiry: float) -> float:
        return self.vol.vol(strike, expiry)


class MarketBuilder:
    """market::MarketBuilder (src/market/market.rs:305-415), same validation messages."""

    def __init__(self):
        self._spot = None
        self._rate = None
        self._q = None
        self._flat = None
        self._surface = None
        self._ref = None
        self._divs = None

    def dividend_schedule(self, schedule: DividendSchedule) -> "MarketBuilder":
        """Sets a deterministic discrete dividend schedule (market.rs:340-343)."""
        self._divs = schedule
        return self

    def spot(self, spot: float) -> "MarketBuilder":
        self._spot = float(spot)
        return self

    def rate(self, rate: float) -> "MarketBuilder":
        self._rate = float(rate)
        return self

    def dividend_yield(self, q: float) -> "MarketBuilder":
        self._q = float(q)
        return self

    def flat_vol(self, vol: float) -> "MarketBuilder":
        self._flat = float(vol)
        self._surface = None
        return self

    def vol_surface(self, surface) -> "MarketBuilder":
        """A SampledVolSurface, or a callable vol(strike, expiry) that build()
        samples onto the default grid (market.rs:385-391)."""
        self._surface = surface
        self._flat = None
        return self

    def reference_date(self, d: str) -> "MarketBuilder":
        self._ref = d
        return self

    def build(self) -> Market:
        if self._spot is None:
            raise PricingError.InvalidInput("market spot is required")
        if self._spot <= 0.0:
            raise PricingError.InvalidInput("market spot must be > 0")
        if self._surface is not None:
            if isinstance(self._surface, SampledVolSurface):
                vol = VolSource(sampled=self._surface)
            else:
                vol = VolSource(sampled=SampledVolSurface.from_surface(self._surface, self._spot))
        else:
            if self._flat is None:
                raise PricingError.InvalidInput("either market flat_vol or vol_surface is required")
            if self._flat <= 0.0:
                raise PricingError.InvalidInput("market flat_vol must be > 0")
            vol = VolSource(flat=self._flat)
        sched = self._divs if self._divs is not None else DividendSchedule.empty()
        sched.validate()
        return Market(spot=self._spot, rate=self._rate or 0.0, dividend_yield=self._q or 0.0, vol=vol,
                      reference_date=self._ref, dividend_schedule=sched)
