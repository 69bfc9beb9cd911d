"""Market snapshot, mirroring openferric's `market::Market` (src/market/market.rs:180-415)."""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Optional

from .core import PricingError


class VolSource:
    """market::VolSource (src/market/market.rs:179-198): a flat vol or a surface
    callable `vol(strike, expiry)`."""

    def __init__(self, flat: Optional[float] = None, surface: Optional[Callable[[float, float], float]] = None):
        self.flat = flat
        self.surface = surface

    def vol(self, strike: float, expiry: float) -> float:
        if self.surface is not None:
            return float(self.surface(strike, expiry))
        return float(self.flat)


@dataclass
class Market:
    """market::Market (src/market/market.rs:201-302).  Discrete dividend
    schedules are not supported by the GPU engines (an empty schedule is the
    only accepted value)."""

    spot: float
    rate: float
    dividend_yield: float
    vol: VolSource
    reference_date: Optional[str] = None
    dividend_schedule: tuple = field(default_factory=tuple)

    @staticmethod
    def builder() -> "MarketBuilder":
        return MarketBuilder()

    def has_discrete_dividends(self) -> bool:
        return len(self.dividend_schedule) > 0

    def effective_dividend_yield(self, maturity: float) -> float:
        # With no discrete schedule the effective yield is the continuous one
        # (market/dividends.rs effective_dividend_yield).
        return self.dividend_yield

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

    def vol_surface(self, surface: Callable[[float, float], float]) -> "MarketBuilder":
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
            vol = VolSource(surface=self._surface)
        else:
            if self._flat is None:
                raise PricingError.InvalidInput("either market flat_vol or vol_surface is required")
            if self._flat <= 0.0:
                raise PricingError.InvalidInput("market flat_vol must be > 0")
            vol = VolSource(flat=self._flat)
        return Market(spot=self._spot, rate=self._rate or 0.0, dividend_yield=self._q or 0.0, vol=vol,
                      reference_date=self._ref)
