"""Batched book pricing: many instruments, each with its own paths and steps,
in one persistent kernel launch (of_mc_price_book / of_book_plan_*).

`BookEntry` carries what MonteCarloPricingEngine::price derives per instrument
(src/engines/monte_carlo/mc_engine.rs:875-975); `price_book` returns one
PricingResult per entry.  `price_book_greeks` is
MonteCarloPricingEngine::price_with_greeks_aad (mc_engine.rs:977-987) for a
whole book: price, delta, vega, rho and theta of every GBM option from the
same launch (of_mc_price_book_greeks).  `BookPlan` keeps the device tables and
the captured CUDA graph for repeated launches.  `synthetic_book` builds the
seeded mixed book (European / daily-fixing arithmetic Asian / up-and-out call)
used by the benchmarks.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _abi as A
from ._lib import context
from .core import (AsianSpec, Averaging, BarrierDirection, BarrierSpec, BarrierStyle, Diagnostics, Greeks,
                   OptionType, PricingResult, StrikeType)
from .engines import (Gbm, GbmPathGenerator, VarianceReduction, _payoff_abi, instrument_control_variate,
                      reference_strike)
from .instruments import AsianOption, BarrierOption, VanillaOption
from .market import Market


@dataclass
class BookEntry:
    instrument: object
    market: Market
    num_paths: int
    num_steps: int
    variance_reduction: VarianceReduction = VarianceReduction.None_


def book_entries_abi(entries: Sequence[BookEntry]):
    """The of_book_entry array of a book, the objects its pointers refer to
    (keep them alive while the array is in use) and each entry's volatility."""
    arr = (A.OfBookEntry * len(entries))()
    keep, vols = [], []
    for k, e in enumerate(entries):
        inst, m = e.instrument, e.market
        inst.validate()
        vol = m.vol_for(max(reference_strike(inst, m.spot), 1e-12), inst.expiry)
        gen = GbmPathGenerator(Gbm(m.rate - m.dividend_yield, vol), m.spot, inst.expiry, e.num_steps,
                               m.dividend_schedule if m.has_discrete_dividends() else None)
        payoff, held = _payoff_abi(inst)
        keep.append(held)
        keep.append(gen)  # holds the dividend array the model points to
        vols.append(vol)
        # the FP32 book needs no bit-level parity of the control-variate mean
        # with the reference's summation order: the O(n log n) covariance sum
        cv = instrument_control_variate(inst, m, vol, exact_order=False) \
            if e.variance_reduction is VarianceReduction.ControlVariate else None
        arr[k] = A.OfBookEntry(model=gen.to_abi(), payoff=payoff, num_paths=int(e.num_paths),
                               antithetic=int(e.variance_reduction is VarianceReduction.Antithetic),
                               discount_factor=math.exp(-m.rate * inst.expiry))
        if cv is not None:
            arr[k].control_variate = cv.kind.value
            arr[k].cv_expected = cv.expected
    return arr, keep, vols


@dataclass
class BookGreeksResult:
    """One option of `price_book_greeks`: its PricingResult with `greeks`
    filled (gamma = 0, as the reference's pathwise AAD returns it) and the
    Monte Carlo standard error of each Greek."""
    result: PricingResult
    greeks_stderr: Greeks


def _greeks_of(g: A.OfBookGreeks):
    return (Greeks(delta=g.delta, gamma=g.gamma, vega=g.vega, theta=g.theta, rho=g.rho),
            Greeks(delta=g.delta_se, gamma=g.gamma_se, vega=g.vega_se, theta=g.theta_se, rho=g.rho_se))


def _diagnostics(paths, steps, vol):
    d = Diagnostics()
    d.insert("num_paths", float(paths))
    d.insert("num_steps", float(steps))
    d.insert("vol", vol)
    return d


class BookPlan:
    """Device tables + CUDA graph for a book; launch() replays without a host sync.

    mode: A.OF_BOOK_PRICE (prices), A.OF_BOOK_GREEKS (prices and pathwise
    Greeks; `greeks_results()` reads them), A.OF_BOOK_PRICE_FP64 (the Greeks
    mode's prices in FP64 on the same draws, for bump-and-revalue checks) or
    A.OF_BOOK_GREEKS_FP64 (its prices and Greeks in FP64 on the same draws)."""

    def __init__(self, entries: Sequence[BookEntry], seed: int, block: int = 0, paths_per_thread: int = 0,
                 use_graph: bool = True, device: int = 0, mode: int = A.OF_BOOK_PRICE):
        self.ctx = context(device)
        self.n = len(entries)
        self.mode = int(mode)
        arr, self._keep, self._vols = book_entries_abi(entries)
        cfg = A.OfBookConfig(seed=int(seed) & 0xFFFFFFFFFFFFFFFF, block=block, paths_per_thread=paths_per_thread,
                             use_graph=int(use_graph), mode=self.mode)
        h = C.c_void_p()
        with self.ctx.lock:
            self.ctx.check(self.ctx._L.of_book_plan_create(self.ctx.handle, arr, self.n, C.byref(cfg), C.byref(h)))
        self.handle = h
        self.entries = list(entries)

    def info(self):
        b, p, nt, ps = C.c_int32(), C.c_int32(), C.c_int64(), C.c_double()
        self.ctx.check(self.ctx._L.of_book_plan_info(self.handle, C.byref(b), C.byref(p), C.byref(nt), C.byref(ps)))
        return {"block": b.value, "paths_per_thread": p.value, "tiles": nt.value, "path_steps": ps.value}

    def launch(self):
        self.ctx.check(self.ctx._L.of_book_plan_launch(self.handle))

    def raw_results(self) -> List[A.OfMcResult]:
        out = (A.OfMcResult * self.n)()
        self.ctx.check(self.ctx._L.of_book_plan_results(self.handle, out))
        return list(out)

    def results(self) -> List[PricingResult]:
        return [PricingResult(price=r.price, stderr=r.stderr_, diagnostics=_diagnostics(e.num_paths, e.num_steps, vol))
                for e, r, vol in zip(self.entries, self.raw_results(), self._vols)]

    def raw_greeks(self) -> List[A.OfBookGreeks]:
        out = (A.OfBookGreeks * self.n)()
        self.ctx.check(self.ctx._L.of_book_plan_greeks(self.handle, out))
        return list(out)

    def greeks_results(self) -> List[BookGreeksResult]:
        """Prices and Greeks of the last launch (mode OF_BOOK_GREEKS or OF_BOOK_GREEKS_FP64)."""
        out = []
        for r, g in zip(self.results(), self.raw_greeks()):
            r.greeks, se = _greeks_of(g)
            out.append(BookGreeksResult(r, se))
        return out

    def close(self):
        if self.handle and self.handle.value:
            self.ctx._L.of_book_plan_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def price_book(entries: Sequence[BookEntry], seed: int, block: int = 0, paths_per_thread: int = 0,
               device: int = 0) -> List[PricingResult]:
    plan = BookPlan(entries, seed, block, paths_per_thread, use_graph=False, device=device)
    try:
        plan.launch()
        return plan.results()
    finally:
        plan.close()


def price_book_greeks(entries: Sequence[BookEntry], seed: int, block: int = 0, paths_per_thread: int = 0,
                      device: int = 0) -> List[BookGreeksResult]:
    """Price and pathwise Greeks (delta, vega, rho, theta) of every entry in
    one persistent launch (of_mc_price_book_greeks).  GBM options without
    discrete dividends; barrier options are priced by one-step survival (no
    control variate), the other payoffs by the book's own estimator."""
    plan = BookPlan(entries, seed, block, paths_per_thread, use_graph=False, device=device, mode=A.OF_BOOK_GREEKS)
    try:
        plan.launch()
        return plan.greeks_results()
    finally:
        plan.close()


def price_book_greeks_fp64(entries: Sequence[BookEntry], seed: int, block: int = 0, paths_per_thread: int = 0,
                           device: int = 0) -> List[BookGreeksResult]:
    """The prices and pathwise Greeks of `price_book_greeks` in FP64 path
    arithmetic on the same draws (mode OF_BOOK_GREEKS_FP64): the same
    estimator without the FP32 rounding."""
    plan = BookPlan(entries, seed, block, paths_per_thread, use_graph=False, device=device,
                    mode=A.OF_BOOK_GREEKS_FP64)
    try:
        plan.launch()
        return plan.greeks_results()
    finally:
        plan.close()


def price_book_fp64(entries: Sequence[BookEntry], seed: int, block: int = 0, paths_per_thread: int = 0,
                    device: int = 0) -> List[PricingResult]:
    """The prices of `price_book_greeks` in FP64 path arithmetic on the same
    draws (same seed, entries and path counts): the revaluations of a
    bump-and-revalue check with common random numbers."""
    plan = BookPlan(entries, seed, block, paths_per_thread, use_graph=False, device=device,
                    mode=A.OF_BOOK_PRICE_FP64)
    try:
        plan.launch()
        return plan.results()
    finally:
        plan.close()


@dataclass
class StderrRound:
    """One book launch of `price_book_to_stderr`: how many options it priced,
    their total paths and path-steps, how many met the target, the
    launch's device time and the round's host wall clock (planning, uploads,
    launch and readback)."""
    options: int
    paths: int
    path_steps: float
    converged: int
    kernel_ms: float = 0.0
    wall_ms: float = 0.0


def paths_for_stderr(paths: int, stderr: float, target: float, margin: float = 1.05, granule: int = 256) -> int:
    """Paths that bring a standard error measured with `paths` down to
    `target` (stderr scales as paths^-1/2), with a safety margin, rounded up to
    a multiple of `granule`; never fewer than `paths`: the total that
    of_book_price_to_stderr aims at for an option after a round (where the
    follow-up launch runs the difference), for planning a book's cost on the
    host."""
    if not (stderr > target):
        return paths
    need = paths * (stderr / target) ** 2 * margin
    return max(paths, int(math.ceil(need / granule)) * granule)


def price_book_to_stderr(entries: Sequence[BookEntry], seed: int, se_rel: float = 1e-4, pilot_paths: int = 8192,
                         max_rounds: int = 4, device: int = 0, greeks: bool = False, margin: float = 0.0):
    """Prices every entry to a standard error of at most `se_rel` x its spot
    (of_book_price_to_stderr).

    A pilot launch of the whole book with `pilot_paths` per option estimates
    each option's standard error; every option above its target gets more
    paths, in one book launch (its total scaled by (SE/target)^2 x `margin`,
    0 = the default 1.05), and so
    on until all meet the target or `max_rounds` launches have run.  Each round
    draws from its own seed (seed + round), and an option's result pools the
    samples of all its rounds (its diagnostics carry their total path count).
    Returns the results and the rounds.

    greeks=True prices every launch with the pathwise Greeks
    (of_book_price_to_stderr_greeks): the results are then BookGreeksResult,
    each option's Greeks pooled over the same launches as its price."""
    ctx = context(device)
    n = len(entries)
    arr, keep, vols = book_entries_abi(entries)
    cfg = A.OfBookConfig(seed=int(seed) & 0xFFFFFFFFFFFFFFFF)
    tgt = A.OfStderrTarget(se_rel=float(se_rel), pilot_paths=int(pilot_paths), max_rounds=int(max_rounds),
                           margin=float(margin))
    out = (A.OfMcResult * n)()
    paths = (C.c_int64 * n)()
    rounds = (A.OfStderrRound * max(1, int(max_rounds)))()
    n_rounds = C.c_int32()
    gr = (A.OfBookGreeks * n)() if greeks else None
    with ctx.lock:
        if greeks:
            ctx.check(ctx._L.of_book_price_to_stderr_greeks(ctx.handle, arr, n, C.byref(cfg), C.byref(tgt), out, gr,
                                                            paths, rounds, C.byref(n_rounds)))
        else:
            ctx.check(ctx._L.of_book_price_to_stderr(ctx.handle, arr, n, C.byref(cfg), C.byref(tgt), out, paths,
                                                     rounds, C.byref(n_rounds)))
    del keep
    results = []
    for k, (e, r, p, vol) in enumerate(zip(entries, out, paths, vols)):
        res = PricingResult(price=r.price, stderr=r.stderr_, diagnostics=_diagnostics(p, e.num_steps, vol))
        if greeks:
            res.greeks, se = _greeks_of(gr[k])
            res = BookGreeksResult(res, se)
        results.append(res)
    return results, [StderrRound(rd.options, rd.paths, rd.path_steps, rd.converged, rd.kernel_ms, rd.wall_ms)
                     for rd in rounds[:n_rounds.value]]


def synthetic_book(n: int = 4096, seed: int = 20261203, steps_per_year: int = 252, min_log2_paths: int = 14,
                   max_log2_paths: int = 18, variance_reduction: VarianceReduction = VarianceReduction.None_
                   ) -> List[BookEntry]:
    """Seeded mixed book: one third each European call, daily-fixing
    arithmetic Asian call, discretely monitored up-and-out call;
    S0~U[50,150], K=S0 U[0.8,1.2], sigma~U[0.1,0.6], r~U[0,0.06],
    T~U[0.1,5], steps = round(252 T), paths log-uniform in [2^14, 2^18]
    rounded to a multiple of 256, barrier = S0 U[1.1,1.5]."""
    rng = np.random.default_rng(seed)
    s0 = rng.uniform(50.0, 150.0, n)
    k = s0 * rng.uniform(0.8, 1.2, n)
    vol = rng.uniform(0.10, 0.60, n)
    r = rng.uniform(0.0, 0.06, n)
    T = rng.uniform(0.1, 5.0, n)
    logp = rng.uniform(min_log2_paths, max_log2_paths, n)
    bar = s0 * rng.uniform(1.1, 1.5, n)
    out = []
    for i in range(n):
        steps = max(1, int(round(steps_per_year * T[i])))
        paths = max(256, int(round(2.0 ** logp[i] / 256.0)) * 256)
        m = Market.builder().spot(s0[i]).rate(r[i]).dividend_yield(0.0).flat_vol(vol[i]).build()
        kind = i % 3
        if kind == 0:
            inst = VanillaOption.european_call(k[i], T[i])
        elif kind == 1:
            obs = [T[i] * (j / steps) for j in range(1, steps + 1)]  # last fixing == T exactly
            inst = AsianOption(OptionType.Call, k[i], T[i], AsianSpec(Averaging.Arithmetic, StrikeType.Fixed, obs))
        else:
            inst = BarrierOption(OptionType.Call, k[i], T[i],
                                 BarrierSpec(BarrierDirection.Up, BarrierStyle.Out, bar[i], 0.0))
        out.append(BookEntry(inst, m, paths, steps, variance_reduction))
    return out
