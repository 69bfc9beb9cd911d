"""The batched book's pathwise Greeks (of_mc_price_book_greeks).

Checks, each through the C ABI:
- every Greek (delta, vega, rho, theta) of every payoff kind against central
  bump-and-revalue with common random numbers: the revaluations are the same
  launch in FP64 path arithmetic on the same draws (of_book_plan mode
  OF_BOOK_PRICE_FP64), bumps of 1e-4 relative;
- the European Greeks against the reference's own estimator,
  mc_european_pathwise_aad (src/engines/monte_carlo/mc_aad.rs:75-219) on the
  reference streams, within combined standard errors;
- the prices of the Greeks mode against the book's price mode: the same draws
  for Europeans and Asians, and for barriers (priced by one-step survival)
  within combined standard errors of the plain estimator;
- the standard-error target with Greeks.
"""
import math

import pytest

from openferric_b200 import (AsianOption, AsianSpec, Averaging, BarrierDirection, BarrierOption, BarrierSpec,
                             BarrierStyle, Market, MonteCarloPricingEngine, OptionType, PricingError, StrikeType,
                             VanillaOption, VarianceReduction)
from openferric_b200.book import (BookEntry, price_book, price_book_fp64, price_book_greeks, price_book_to_stderr,
                                  synthetic_book)

pytestmark = pytest.mark.gpu

BASE = dict(spot=100.0, vol=0.3, rate=0.03, q=0.01)


def _instrument(kind, T, steps):
    if kind == "euro_call":
        return VanillaOption.european_call(105.0, T)
    if kind == "euro_put":
        return VanillaOption.european_put(95.0, T)
    if kind == "asian_daily":
        obs = [T * j / steps for j in range(1, steps + 1)]
        return AsianOption(OptionType.Call, 100.0, T, AsianSpec(Averaging.Arithmetic, StrikeType.Fixed, obs))
    if kind == "asian_monthly_put":
        obs = [T * j / 12.0 for j in range(1, 13)]
        return AsianOption(OptionType.Put, 102.0, T, AsianSpec(Averaging.Arithmetic, StrikeType.Fixed, obs))
    if kind == "asian_geometric":
        obs = [T * j / steps for j in range(1, steps + 1)]
        return AsianOption(OptionType.Call, 98.0, T, AsianSpec(Averaging.Geometric, StrikeType.Fixed, obs))
    if kind == "asian_floating":
        obs = [T * j / 12.0 for j in range(0, 13)]
        return AsianOption(OptionType.Call, 1.0, T, AsianSpec(Averaging.Arithmetic, StrikeType.Floating, obs))
    if kind == "up_out_call":
        return BarrierOption(OptionType.Call, 100.0, T, BarrierSpec(BarrierDirection.Up, BarrierStyle.Out, 135.0, 0.0))
    if kind == "down_out_put":
        return BarrierOption(OptionType.Put, 100.0, T, BarrierSpec(BarrierDirection.Down, BarrierStyle.Out, 75.0, 1.5))
    if kind == "up_in_call":
        return BarrierOption(OptionType.Call, 100.0, T, BarrierSpec(BarrierDirection.Up, BarrierStyle.In, 125.0, 0.5))
    if kind == "down_in_put":
        return BarrierOption(OptionType.Put, 100.0, T, BarrierSpec(BarrierDirection.Down, BarrierStyle.In, 85.0, 0.0))
    raise ValueError(kind)


KINDS = ["euro_call", "euro_put", "asian_daily", "asian_monthly_put", "asian_geometric", "asian_floating",
         "up_out_call", "down_out_put", "up_in_call", "down_in_put"]


def _entry(kind, spot, vol, rate, T, steps=48, paths=1 << 16, anti=False):
    m = Market.builder().spot(spot).rate(rate).dividend_yield(BASE["q"]).flat_vol(vol).build()
    vr = VarianceReduction.Antithetic if anti else VarianceReduction.None_
    return BookEntry(_instrument(kind, T, steps), m, paths, steps, vr)


def _book(params, anti):
    spot, vol, rate, T = params
    return [_entry(k, spot, vol, rate, T, anti=anti) for k in KINDS]


@pytest.mark.parametrize("anti", [False, True])
def test_book_greeks_match_fp64_crn_central_differences(anti):
    base = (BASE["spot"], BASE["vol"], BASE["rate"], 1.25)
    seed = 20261204
    got = price_book_greeks(_book(base, anti), seed)
    h = 1e-4
    fds = []
    for t in range(4):  # spot, vol, rate, expiry
        up, dn = list(base), list(base)
        up[t] *= 1.0 + h
        dn[t] *= 1.0 - h
        pu = price_book_fp64(_book(tuple(up), anti), seed)
        pd = price_book_fp64(_book(tuple(dn), anti), seed)
        fds.append([(a.price - b.price) / (2.0 * h * base[t]) for a, b in zip(pu, pd)])
    p64 = price_book_fp64(_book(base, anti), seed)
    for k, kind in enumerate(KINDS):
        g = got[k].result.greeks
        # the Greeks mode's FP32 price against its FP64 revaluation on the same draws
        assert abs(got[k].result.price - p64[k].price) <= 2e-5 * abs(p64[k].price) + 1e-6, kind
        for name, value, fd in (("delta", g.delta, fds[0][k]), ("vega", g.vega, fds[1][k]),
                                ("rho", g.rho, fds[2][k]), ("theta", g.theta, -fds[3][k])):
            tol = max(1e-3 * abs(fd), 2e-4)
            assert abs(value - fd) <= tol, (kind, name, value, fd)
        assert g.gamma == 0.0


@pytest.mark.parametrize("option_type", [OptionType.Call, OptionType.Put])
def test_book_european_greeks_match_reference_pathwise_aad(option_type):
    """Independent streams of the same estimator: each Greek within 4
    combined standard errors (the reference-side error from the book's
    per-sample spread and the reference's path count)."""
    m = Market.builder().spot(100.0).rate(0.03).dividend_yield(0.01).flat_vol(0.25).build()
    opt = VanillaOption(option_type, 105.0, 1.3)
    n_book, n_ref, steps = 1 << 20, 200_000, 37
    book = price_book_greeks([BookEntry(opt, m, n_book, steps)], seed=5)[0]
    ref = MonteCarloPricingEngine(n_ref, steps, 42).price_with_greeks_aad(opt, m)
    g, se, rg = book.result.greeks, book.greeks_stderr, ref.greeks
    scale = math.sqrt(1.0 + n_book / n_ref)
    for name in ("delta", "vega", "rho", "theta"):
        a, b, s = getattr(g, name), getattr(rg, name), getattr(se, name) * scale
        assert abs(a - b) <= 4.0 * s, (name, a, b, s)
    assert abs(book.result.price - ref.price) <= 4.0 * math.hypot(book.result.stderr, ref.stderr)


def test_greeks_mode_prices_agree_with_price_mode():
    book = synthetic_book(n=30, seed=11, min_log2_paths=15, max_log2_paths=16)
    plain = price_book(book, seed=3)
    gm = price_book_greeks(book, seed=3)
    for e, p, g in zip(book, plain, gm):
        if isinstance(e.instrument, BarrierOption):
            # one-step survival vs the plain estimator: independent estimators of one price
            assert abs(g.result.price - p.price) <= 4.0 * math.hypot(g.result.stderr, p.stderr) + 1e-9
            # conditioning on survival removes the knock-out variance
            assert g.result.stderr <= p.stderr * 1.02 + 1e-12
        else:  # same draws, same payoff: FP32 rounding only
            assert abs(g.result.price - p.price) <= 1e-4 * abs(p.price) + 1e-6, (g.result.price, p.price)
        for name in ("delta", "vega", "rho", "theta"):
            assert math.isfinite(getattr(g.result.greeks, name))


def test_book_greeks_to_stderr_target():
    book = synthetic_book(n=9, seed=3, min_log2_paths=14, max_log2_paths=15)
    res, rounds = price_book_to_stderr(book, seed=7, se_rel=2e-4, greeks=True)
    assert len(rounds) >= 1
    for e, r in zip(book, res):
        assert r.result.stderr <= 2e-4 * e.market.spot
        assert r.result.greeks is not None and r.greeks_stderr.delta >= 0.0
        if not isinstance(e.instrument, BarrierOption):  # long calls; a knock-out's vega may be negative
            assert r.result.greeks.vega > 0.0 and r.result.greeks.delta > 0.0


def test_greeks_mode_rejects_what_it_cannot_differentiate():
    import ctypes as C
    from openferric_b200 import _abi as A
    from openferric_b200._lib import context
    from openferric_b200.book import book_entries_abi
    from openferric_b200.market import DividendEvent, DividendSchedule
    m = Market.builder().spot(100.0).rate(0.03).flat_vol(0.2).build()
    bar = BarrierOption(OptionType.Call, 100.0, 1.0, BarrierSpec(BarrierDirection.Up, BarrierStyle.Out, 130.0, 0.0))
    arr, keep, _ = book_entries_abi([BookEntry(bar, m, 4096, 16)])
    arr[0].control_variate = A.OF_CV_TERMINAL_SPOT  # the survival-weighted path has no plain terminal spot
    ctx = context(0)
    out, gr = (A.OfMcResult * 1)(), (A.OfBookGreeks * 1)()
    st = ctx._L.of_mc_price_book_greeks(ctx.handle, arr, 1, C.byref(A.OfBookConfig(seed=1)), out, gr)
    assert st == A.OF_ERR_UNSUPPORTED and "control variate" in ctx._L.of_ctx_last_error(ctx.handle).decode()
    md = Market.builder().spot(100.0).rate(0.03).flat_vol(0.2).dividend_schedule(
        DividendSchedule([DividendEvent.cash(0.5, 1.0)])).build()
    with pytest.raises(PricingError):
        price_book_greeks([BookEntry(VanillaOption.european_call(100.0, 1.0), md, 4096, 16)], seed=1)


def _oracle_option(kind, k, steps=48, anti=False):
    from oracle.book_oracle import GreekOption
    base = dict(s0=BASE["spot"], r=BASE["rate"], q=BASE["q"], sigma=BASE["vol"], T=1.25, steps=steps, stream=k,
                antithetic=anti)
    daily = [0.0] + [1.0] * steps
    monthly = [0.0] * (steps + 1)
    for j in range(1, 13):
        monthly[round(j / 12.0 * steps)] += 1.0
    monthly0 = list(monthly)
    monthly0[0] += 1.0
    return {
        "euro_call": GreekOption("vanilla", True, strike=105.0, **base),
        "euro_put": GreekOption("vanilla", False, strike=95.0, **base),
        "asian_daily": GreekOption("asian", True, strike=100.0, weights=daily, **base),
        "asian_monthly_put": GreekOption("asian", False, strike=102.0, weights=monthly, **base),
        "asian_geometric": GreekOption("asian", True, strike=98.0, weights=daily, geometric=True, **base),
        "asian_floating": GreekOption("asian", True, strike=1.0, weights=monthly0, floating=True, **base),
        "up_out_call": GreekOption("barrier", True, strike=100.0, up=True, barrier=135.0, **base),
        "down_out_put": GreekOption("barrier", False, strike=100.0, up=False, barrier=75.0, rebate=1.5, **base),
        "up_in_call": GreekOption("barrier", True, strike=100.0, up=True, knock_in=True, barrier=125.0, rebate=0.5,
                                  **base),
        "down_in_put": GreekOption("barrier", False, strike=100.0, up=False, knock_in=True, barrier=85.0, **base),
    }[kind]


@pytest.mark.parametrize("anti", [False, True])
def test_book_greeks_mode_matches_the_oracle_on_the_same_draws(anti):
    """The CPU restatement (oracle/book_oracle.py) draws the kernel's own
    Philox blocks: the FP64 mode equals it to FP64 rounding, and the FP32
    Greeks mode's price and Greeks to FP32 path precision."""
    from oracle.book_oracle import book_greeks
    paths, seed = 4096, 77
    base = (BASE["spot"], BASE["vol"], BASE["rate"], 1.25)
    book = [_entry(k, *base, paths=paths, anti=anti) for k in KINDS]
    g32 = price_book_greeks(book, seed)
    p64 = price_book_fp64(book, seed)
    for k, kind in enumerate(KINDS):
        price, g = book_greeks(_oracle_option(kind, k, anti=anti), paths, seed)
        assert abs(p64[k].price - price) <= 1e-9 * abs(price) + 1e-12, (kind, p64[k].price, price)
        assert abs(g32[k].result.price - price) <= 2e-5 * abs(price) + 1e-6, (kind, g32[k].result.price, price)
        gg = g32[k].result.greeks
        for name, value, ref in zip(("delta", "vega", "rho", "theta"), (gg.delta, gg.vega, gg.rho, gg.theta), g):
            assert abs(value - ref) <= 1e-4 * abs(ref) + 2e-5, (kind, name, value, ref)


@pytest.mark.parametrize("anti", [False, True])
def test_price_mode_geometric_control_variate_matches_fp64_same_draws(anti):
    """Daily-fixing arithmetic Asians priced with the geometric-Asian control
    variate take a step loop specialised for them in the price mode (the
    fixings' compensated sum and the log-spots' sum); the FP64 mode prices the
    same draws with the same estimator, so the two agree to FP32 rounding, the
    control-variate adjustment included."""
    from dataclasses import replace
    from openferric_b200.engines import VarianceReduction
    from openferric_b200.instruments import AsianOption
    book = [e for e in synthetic_book(n=30, seed=12, min_log2_paths=13, max_log2_paths=14)
            if isinstance(e.instrument, AsianOption)]
    book = [replace(e, variance_reduction=VarianceReduction.ControlVariate) for e in book]
    if anti:  # the reference's ArithmeticAsianMC: antithetic pairs and the control variate
        book = [replace(e, variance_reduction=VarianceReduction.Antithetic) for e in book[:3]] + book[3:]
    p32 = price_book(book, seed=5)
    p64 = price_book_fp64(book, seed=5)
    for e, a, b in zip(book, p32, p64):
        assert abs(a.price - b.price) <= 1e-4 * abs(b.price) + 1e-6, (e.instrument.strike, a.price, b.price)
        assert abs(a.stderr - b.stderr) <= 1e-3 * b.stderr + 1e-8, (a.stderr, b.stderr)


@pytest.mark.parametrize("anti", [False, True])
def test_fp64_greeks_mode_is_the_derivative_of_the_fp64_prices(anti):
    """Mode OF_BOOK_GREEKS_FP64 runs the Greeks mode's estimator in FP64 on the
    same draws: its pathwise Greeks are the derivatives of the FP64 prices
    (central differences with common random numbers), to the differences'
    own truncation and rounding, for every payoff kind; and the FP32 Greeks
    are those numbers up to FP32 rounding."""
    from openferric_b200.book import price_book_greeks_fp64
    base = (BASE["spot"], BASE["vol"], BASE["rate"], 1.25)
    seed = 20261205
    g64 = price_book_greeks_fp64(_book(base, anti), seed)
    g32 = price_book_greeks(_book(base, anti), seed)
    h = 1e-5
    for t, name in enumerate(("delta", "vega", "rho", "theta")):
        up, dn = list(base), list(base)
        up[t] *= 1.0 + h
        dn[t] *= 1.0 - h
        pu = price_book_fp64(_book(tuple(up), anti), seed)
        pd = price_book_fp64(_book(tuple(dn), anti), seed)
        for k, kind in enumerate(KINDS):
            fd = (pu[k].price - pd[k].price) / (2.0 * h * base[t])
            fd = -fd if name == "theta" else fd
            v64, v32 = getattr(g64[k].result.greeks, name), getattr(g32[k].result.greeks, name)
            # the payoff's kink crossed within the bump: O(h) in the difference
            assert abs(v64 - fd) <= 1e-4 * abs(fd) + 1e-5, (kind, name, v64, fd)
            assert abs(v32 - v64) <= 1e-3 * abs(v64) + 2e-4, (kind, name, v32, v64)
    for k in range(len(KINDS)):
        assert abs(g32[k].result.price - g64[k].result.price) <= 2e-5 * abs(g64[k].result.price) + 1e-6
