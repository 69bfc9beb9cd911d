"""Instruments on the Monte Carlo path, mirroring openferric's `instruments`
module (src/instruments/{vanilla,asian,barrier,bermudan}.rs) with the same
constructors and validation messages."""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from .core import (AsianSpec, Averaging, BarrierDirection, BarrierSpec, BarrierStyle, ExerciseStyle, OptionType,
                   PricingError, StrikeType)


@dataclass
class VanillaOption:
    """instruments::VanillaOption (src/instruments/vanilla.rs:16-102)."""

    option_type: OptionType
    strike: float
    expiry: float
    exercise: ExerciseStyle = ExerciseStyle.European

    @staticmethod
    def european_call(strike: float, expiry: float) -> "VanillaOption":
        return VanillaOption(OptionType.Call, float(strike), float(expiry), ExerciseStyle.European)

    @staticmethod
    def european_put(strike: float, expiry: float) -> "VanillaOption":
        return VanillaOption(OptionType.Put, float(strike), float(expiry), ExerciseStyle.European)

    @staticmethod
    def american_call(strike: float, expiry: float) -> "VanillaOption":
        return VanillaOption(OptionType.Call, float(strike), float(expiry), ExerciseStyle.American)

    @staticmethod
    def american_put(strike: float, expiry: float) -> "VanillaOption":
        return VanillaOption(OptionType.Put, float(strike), float(expiry), ExerciseStyle.American)

    def instrument_type(self) -> str:
        return "VanillaOption"

    def validate(self) -> None:
        if self.strike <= 0.0:
            raise PricingError.InvalidInput("vanilla strike must be > 0")
        if self.expiry < 0.0:
            raise PricingError.InvalidInput("vanilla expiry must be >= 0")
        if self.exercise.is_bermudan:
            if not self.exercise.dates:
                raise PricingError.InvalidInput("bermudan exercise dates cannot be empty")
            if any(d <= 0.0 or d > self.expiry for d in self.exercise.dates):
                raise PricingError.InvalidInput("bermudan exercise dates must lie in (0, expiry]")


@dataclass
class AsianOption:
    """instruments::AsianOption (src/instruments/asian.rs:16-63)."""

    option_type: OptionType
    strike: float
    expiry: float
    asian: AsianSpec

    @staticmethod
    def new(option_type: OptionType, strike: float, expiry: float, asian: AsianSpec) -> "AsianOption":
        return AsianOption(option_type, float(strike), float(expiry), asian)

    def instrument_type(self) -> str:
        return "AsianOption"

    def validate(self) -> None:
        if self.expiry < 0.0:
            raise PricingError.InvalidInput("asian expiry must be >= 0")
        if self.strike <= 0.0:
            raise PricingError.InvalidInput("asian strike must be > 0")
        if not self.asian.observation_times:
            raise PricingError.InvalidInput("asian observation_times cannot be empty")
        obs = np.asarray(self.asian.observation_times, dtype=np.float64)
        if np.any((obs < 0.0) | (obs > self.expiry)):  # asian.rs:55-64; NaN compares false there too
            raise PricingError.InvalidInput("asian observation_times must lie in [0, expiry]")


@dataclass
class BarrierOption:
    """instruments::BarrierOption (src/instruments/barrier.rs:17-65)."""

    option_type: OptionType
    strike: float
    expiry: float
    barrier: BarrierSpec

    def instrument_type(self) -> str:
        return "BarrierOption"

    def validate(self) -> None:
        if self.strike <= 0.0:
            raise PricingError.InvalidInput("barrier strike must be > 0")
        if self.expiry < 0.0:
            raise PricingError.InvalidInput("barrier expiry must be >= 0")
        if self.barrier.level <= 0.0:
            raise PricingError.InvalidInput("barrier level must be > 0")
        if self.barrier.rebate < 0.0:
            raise PricingError.InvalidInput("barrier rebate must be >= 0")

    @staticmethod
    def builder() -> "BarrierOptionBuilder":
        return BarrierOptionBuilder()


class BarrierOptionBuilder:
    """instruments::BarrierOptionBuilder (src/instruments/barrier.rs:67-140)."""

    def __init__(self):
        self._type = None
        self._strike = None
        self._expiry = None
        self._dir = None
        self._style = None
        self._level = None
        self._rebate = 0.0

    def call(self):
        self._type = OptionType.Call
        return self

    def put(self):
        self._type = OptionType.Put
        return self

    def strike(self, k):
        self._strike = float(k)
        return self

    def expiry(self, t):
        self._expiry = float(t)
        return self

    def up_and_out(self, level):
        self._dir, self._style, self._level = BarrierDirection.Up, BarrierStyle.Out, float(level)
        return self

    def up_and_in(self, level):
        self._dir, self._style, self._level = BarrierDirection.Up, BarrierStyle.In, float(level)
        return self

    def down_and_out(self, level):
        self._dir, self._style, self._level = BarrierDirection.Down, BarrierStyle.Out, float(level)
        return self

    def down_and_in(self, level):
        self._dir, self._style, self._level = BarrierDirection.Down, BarrierStyle.In, float(level)
        return self

    def rebate(self, r):
        self._rebate = float(r)
        return self

    def build(self) -> BarrierOption:
        if self._type is None:
            raise PricingError.InvalidInput("barrier option_type is required")
        if self._strike is None:
            raise PricingError.InvalidInput("barrier strike is required")
        if self._expiry is None:
            raise PricingError.InvalidInput("barrier expiry is required")
        if self._dir is None:
            raise PricingError.InvalidInput("barrier specification is required")
        opt = BarrierOption(self._type, self._strike, self._expiry,
                            BarrierSpec(self._dir, self._style, self._level, self._rebate))
        opt.validate()
        return opt


@dataclass
class BermudanOption:
    """instruments::BermudanOption (src/instruments/bermudan.rs:19-150): exercise
    dates with a strike per date."""

    option_type: OptionType
    expiry: float
    exercise_dates: List[float]
    strike_schedule: List[float]

    @staticmethod
    def new(option_type: OptionType, expiry: float, exercise_dates: Sequence[float],
            strike_schedule: Sequence[float]) -> "BermudanOption":
        return BermudanOption(option_type, float(expiry), [float(t) for t in exercise_dates],
                              [float(k) for k in strike_schedule])

    @staticmethod
    def with_constant_strike(option_type: OptionType, strike: float, expiry: float,
                             exercise_dates: Sequence[float]) -> "BermudanOption":
        return BermudanOption.new(option_type, expiry, exercise_dates, [float(strike)] * len(exercise_dates))

    def instrument_type(self) -> str:
        return "BermudanOption"

    def validate(self) -> None:
        import math
        if self.expiry <= 0.0 or not math.isfinite(self.expiry):
            raise PricingError.InvalidInput("bermudan expiry must be finite and > 0")
        if not self.exercise_dates:
            raise PricingError.InvalidInput("bermudan exercise_dates cannot be empty")
        if len(self.exercise_dates) != len(self.strike_schedule):
            raise PricingError.InvalidInput("bermudan strike_schedule must match exercise_dates length")
        if any((not math.isfinite(t)) or t <= 0.0 or t > self.expiry for t in self.exercise_dates):
            raise PricingError.InvalidInput("bermudan exercise_dates must be finite and in (0, expiry]")
        if any(b <= a for a, b in zip(self.exercise_dates, self.exercise_dates[1:])):
            raise PricingError.InvalidInput("bermudan exercise_dates must be strictly increasing")
        if any((not math.isfinite(k)) or k <= 0.0 for k in self.strike_schedule):
            raise PricingError.InvalidInput("bermudan strike_schedule entries must be finite and > 0")

    def effective_schedule(self) -> List[Tuple[float, float]]:
        """(time, strike) pairs, with (expiry, last strike) appended when the
        last date is before expiry (bermudan.rs:82-101)."""
        self.validate()
        out = list(zip(self.exercise_dates, self.strike_schedule))
        if self.expiry - out[-1][0] > 1.0e-12:
            out.append((self.expiry, out[-1][1]))
        return out


def daily_fixings(expiry: float, steps: int) -> List[float]:
    """Observation times at every simulation step 1..steps (daily fixings);
    the last one is the expiry exactly."""
    return [expiry * (j / steps) for j in range(1, steps + 1)]


__all__ = ["VanillaOption", "AsianOption", "BarrierOption", "BarrierOptionBuilder", "BermudanOption", "AsianSpec",
           "BarrierSpec", "Averaging", "StrikeType", "BarrierDirection", "BarrierStyle", "daily_fixings"]
