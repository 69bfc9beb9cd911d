"""Contract types of the pricing API, mirroring openferric's `core` module.

openferric (Rust) defines these in src/core/types.rs and src/core/engine.rs; the
names, fields, validation messages and error kinds are kept so that code (and
tests) written against the reference read the same here.
"""
from __future__ import annotations

import enum
import math
from dataclasses import dataclass, field
from typing import Dict, Iterator, List, Optional, Tuple


class OptionType(enum.Enum):
    """core::OptionType (src/core/types.rs:13-19)."""

    Call = 0
    Put = 1

    def sign(self) -> float:
        return 1.0 if self is OptionType.Call else -1.0


class BarrierDirection(enum.Enum):
    """core::BarrierDirection (src/core/types.rs:52-58)."""

    Up = 0
    Down = 1


class BarrierStyle(enum.Enum):
    """core::BarrierStyle (src/core/types.rs:61-67)."""

    In = 0
    Out = 1


class Averaging(enum.Enum):
    """core::Averaging (src/core/types.rs:94-100)."""

    Arithmetic = 0
    Geometric = 1


class StrikeType(enum.Enum):
    """core::StrikeType (src/core/types.rs:103-109)."""

    Fixed = 0
    Floating = 1


@dataclass(frozen=True)
class ExerciseStyle:
    """core::ExerciseStyle (src/core/types.rs:41-49): European, American or
    Bermudan{dates}."""

    kind: str
    dates: Tuple[float, ...] = ()

    @staticmethod
    def european() -> "ExerciseStyle":
        return ExerciseStyle("European")

    @staticmethod
    def american() -> "ExerciseStyle":
        return ExerciseStyle("American")

    @staticmethod
    def bermudan(dates) -> "ExerciseStyle":
        return ExerciseStyle("Bermudan", tuple(float(d) for d in dates))

    @property
    def is_european(self) -> bool:
        return self.kind == "European"

    @property
    def is_american(self) -> bool:
        return self.kind == "American"

    @property
    def is_bermudan(self) -> bool:
        return self.kind == "Bermudan"


ExerciseStyle.European = ExerciseStyle.european()
ExerciseStyle.American = ExerciseStyle.american()


@dataclass
class BarrierSpec:
    """core::BarrierSpec (src/core/types.rs:70-91)."""

    direction: BarrierDirection
    style: BarrierStyle
    level: float
    rebate: float = 0.0


@dataclass
class AsianSpec:
    """core::AsianSpec (src/core/types.rs:112-120)."""

    averaging: Averaging
    strike_type: StrikeType
    observation_times: List[float]


@dataclass
class Greeks:
    """core::Greeks (src/core/engine.rs:17-28)."""

    delta: float
    gamma: float
    vega: float
    theta: float
    rho: float


# DiagKey names (src/core/engine.rs:56-185).
DIAG_KEYS = (
    "barrier_level", "conversion_value", "credit_spread", "d", "d1", "d2", "delta", "discount_factor",
    "double_knockout_base", "effective_vol", "exercise_dates", "fair_variance", "fair_volatility", "inside_barriers",
    "integral", "max_exercises", "min_exercises", "npv", "num_paths", "num_threads", "observation_count",
    "num_space_steps", "num_steps", "num_time_steps", "pd", "pm", "pu", "pv_forward", "rho", "rho_domestic",
    "rho_foreign", "s_max", "series_terms", "survival_digital", "u", "var_of_var", "vol", "vol_adj",
)


class Diagnostics:
    """Fixed 8-slot diagnostics map (core::Diagnostics, src/core/engine.rs:193-274).
    Inserting an unknown key or a ninth key raises, as the reference panics."""

    CAPACITY = 8

    def __init__(self):
        self._entries: Dict[str, float] = {}

    def insert(self, key: str, value: float) -> Optional[float]:
        if key not in DIAG_KEYS:
            raise KeyError(f"unsupported diagnostics key `{key}`; add it to core::DiagKey")
        prev = self._entries.get(key)
        if prev is None and len(self._entries) >= self.CAPACITY:
            raise OverflowError(f"diagnostics capacity exceeded ({self.CAPACITY})")
        self._entries[key] = float(value)
        return prev

    def get(self, key: str) -> Optional[float]:
        return self._entries.get(key)

    def contains_key(self, key: str) -> bool:
        return key in self._entries

    def __len__(self) -> int:
        return len(self._entries)

    def is_empty(self) -> bool:
        return not self._entries

    def iter(self) -> Iterator[Tuple[str, float]]:
        return iter(self._entries.items())

    def __repr__(self) -> str:
        return f"Diagnostics({self._entries})"


@dataclass
class PricingResult:
    """core::PricingResult (src/core/engine.rs:278-287)."""

    price: float
    stderr: Optional[float] = None
    greeks: Optional[Greeks] = None
    diagnostics: Diagnostics = field(default_factory=Diagnostics)


class PricingError(Exception):
    """core::PricingError (src/core/engine.rs:293-316).  `kind` is one of
    InvalidInput, ConvergenceFailure, MarketDataMissing, NumericalError."""

    _PREFIX = {
        "InvalidInput": "invalid input",
        "ConvergenceFailure": "convergence failure",
        "MarketDataMissing": "market data missing",
        "NumericalError": "numerical error",
    }

    def __init__(self, kind: str, message: str):
        if kind not in self._PREFIX:
            raise ValueError(f"unknown PricingError kind {kind}")
        self.kind = kind
        self.message = message
        super().__init__(f"{self._PREFIX[kind]}: {message}")

    @classmethod
    def InvalidInput(cls, message: str) -> "PricingError":
        return cls("InvalidInput", message)

    @classmethod
    def ConvergenceFailure(cls, message: str) -> "PricingError":
        return cls("ConvergenceFailure", message)

    @classmethod
    def MarketDataMissing(cls, message: str) -> "PricingError":
        return cls("MarketDataMissing", message)

    @classmethod
    def NumericalError(cls, message: str) -> "PricingError":
        return cls("NumericalError", message)


def is_finite(x: float) -> bool:
    return math.isfinite(x)
