"""Batched persistent book kernel (of_mc_price_book): each option against the
oracle's FP64 Monte Carlo of the same instrument (independent draws, same
scheme), and invariance of the per-sample streams to the tile shape and to
CUDA-graph replay."""
import math

import pytest

from openferric_b200 import VarianceReduction
from openferric_b200 import _abi as A
from openferric_b200.book import BookEntry, BookPlan, price_book, synthetic_book
from openferric_b200.instruments import VanillaOption
from openferric_b200.engines import Gbm, GbmPathGenerator, _payoff_abi, instrument_control_variate

pytestmark = pytest.mark.gpu


def oracle_price(orc, e: BookEntry, paths, seed=5):
    inst, m = e.instrument, e.market
    vol = m.vol_for(inst.strike, inst.expiry)
    gen = GbmPathGenerator(Gbm(m.rate - m.dividend_yield, vol), m.spot, inst.expiry, e.num_steps)
    payoff, keep = _payoff_abi(inst)
    cfg = A.OfMcConfig(num_paths=paths, seed=seed, discount_factor=math.exp(-m.rate * inst.expiry))
    return orc.mc_run(gen.to_abi(), payoff, cfg, threads=8)


def test_small_book_matches_oracle_per_option(orc):
    book = synthetic_book(n=24, seed=11, min_log2_paths=14, max_log2_paths=15)
    res = price_book(book, seed=3)
    for e, r in zip(book, res):
        ref = oracle_price(orc, e, 1 << 13)
        se = math.hypot(r.stderr, ref.stderr_)
        assert abs(r.price - ref.price) <= 4.5 * se + 1e-4 * e.market.spot, (e.instrument, r.price, ref.price, se)


def test_tile_shape_does_not_change_the_paths():
    book = synthetic_book(n=12, seed=5, min_log2_paths=12, max_log2_paths=14)
    a = price_book(book, seed=9, block=256, paths_per_thread=4)
    b = price_book(book, seed=9, block=128, paths_per_thread=1)
    c = price_book(book, seed=9, block=64, paths_per_thread=8)
    # same per-sample draws; only the compensated-FP32 per-thread partial sums
    # regroup, which moves the result at the FP32 rounding level
    for x, y, z in zip(a, b, c):
        assert abs(x.price - y.price) <= 1e-6 * abs(x.price) + 1e-9
        assert abs(x.price - z.price) <= 1e-6 * abs(x.price) + 1e-9


def test_graph_replay_is_deterministic():
    book = synthetic_book(n=30, seed=7, min_log2_paths=12, max_log2_paths=13)
    plan = BookPlan(book, seed=1, use_graph=True)
    plan.launch()
    r1 = [r.price for r in plan.results()]
    plan.launch()
    plan.launch()
    r2 = [r.price for r in plan.results()]
    plan.close()
    assert r1 == r2
    direct = [r.price for r in price_book(book, seed=1)]
    assert r1 == direct


def test_book_control_variate_and_antithetic():
    from openferric_b200.analytic import bs_price
    from openferric_b200.core import OptionType
    book = synthetic_book(n=9, seed=4, min_log2_paths=15, max_log2_paths=15)
    plain = price_book(book, seed=2)
    anti = price_book([BookEntry(e.instrument, e.market, e.num_paths, e.num_steps, VarianceReduction.Antithetic)
                       for e in book], seed=2)
    for p, r in zip(plain, anti):
        assert abs(p.price - r.price) <= 5 * math.hypot(p.stderr, r.stderr) + 1e-3
    cv = price_book([BookEntry(e.instrument, e.market, e.num_paths, e.num_steps, VarianceReduction.ControlVariate)
                     for e in book], seed=2)
    for k, (e, p, r) in enumerate(zip(book, plain, cv)):
        if k % 3 == 0:
            # The European's control variate is its own payoff (mc_engine.rs:458-485): the
            # estimate collapses to the closed form and the variance to rounding level.
            m = e.market
            bs = bs_price(OptionType.Call, m.spot, e.instrument.strike, m.rate, 0.0,
                          m.vol_for(e.instrument.strike, e.instrument.expiry), e.instrument.expiry)
            assert abs(r.price - bs) <= 1e-6 * bs + 1e-9
            assert math.isnan(r.stderr) or r.stderr <= 1e-4 * max(bs, 1.0)
        elif k % 3 == 1:
            # Asian: geometric control variate, much tighter than plain
            assert abs(p.price - r.price) <= 5 * math.hypot(p.stderr, r.stderr) + 1e-3
            assert r.stderr < 0.5 * p.stderr
        else:
            # the barrier option has no control variate: same draws, same estimate
            assert r.price == p.price


def test_full_book_plan_info():
    book = synthetic_book()
    plan = BookPlan(book, seed=20261203)
    info = plan.info()
    plan.close()
    assert info["path_steps"] == pytest.approx(sum(float(e.num_paths) * e.num_steps for e in book))
    assert info["tiles"] > 4096


@pytest.mark.parametrize("vr", [VarianceReduction.None_, VarianceReduction.Antithetic])
def test_specialised_step_loops_match_the_general_loop(vr):
    """Vanilla, daily-fixing Asian and barrier options take step loops
    specialised at compile time.  A 0 % proportional dividend (a jump that
    adds log(1) = 0 to the log-spot) sends the same options through the
    general loop.  The Asian and barrier loops must give the same numbers
    bit for bit: same draws, same arithmetic.  The vanilla loop sums the
    same draws and adds the drift once (y_T = steps drift + diff sum z), so
    its numbers differ from the stepwise sum by FP32 rounding only."""
    from dataclasses import replace
    from openferric_b200 import Market
    from openferric_b200.market import DividendEvent, DividendSchedule
    book = synthetic_book(n=18, seed=4, min_log2_paths=11, max_log2_paths=12, variance_reduction=vr)
    general = []
    for e in book:
        m = e.market
        sched = DividendSchedule.new([DividendEvent.proportional(0.5 * e.instrument.expiry, 0.0)])
        m2 = (Market.builder().spot(m.spot).rate(m.rate).dividend_yield(m.dividend_yield)
              .flat_vol(m.vol_for(m.spot, e.instrument.expiry)).dividend_schedule(sched).build())
        general.append(replace(e, market=m2))
    a = price_book(book, seed=21)
    b = price_book(general, seed=21)
    for e, x, y in zip(book, a, b):
        if isinstance(e.instrument, VanillaOption):
            assert abs(x.price - y.price) <= 1e-5 * abs(y.price) + 1e-6, (e.instrument, x.price, y.price)
            assert abs(x.stderr - y.stderr) <= 1e-4 * y.stderr + 1e-9, (e.instrument, x.stderr, y.stderr)
        else:
            assert x.price == y.price and x.stderr == y.stderr, (e.instrument, x.price, y.price)


@pytest.mark.parametrize("mixed_vr", [False, True])
def test_price_book_to_stderr_meets_the_target(mixed_vr):
    from openferric_b200.book import price_book_to_stderr
    from openferric_b200.instruments import AsianOption
    book = synthetic_book(n=12, seed=8, min_log2_paths=10, max_log2_paths=11)
    if mixed_vr:  # geometric control variate for the Asians, antithetic pairs elsewhere
        book = [BookEntry(e.instrument, e.market, e.num_paths, e.num_steps,
                          VarianceReduction.ControlVariate if isinstance(e.instrument, AsianOption)
                          else VarianceReduction.Antithetic) for e in book]
    res, rounds = price_book_to_stderr(book, seed=3, se_rel=2e-3, pilot_paths=2048)
    for e, r in zip(book, res):
        assert r.stderr <= 2e-3 * e.market.spot, (e.instrument, r.stderr)
    assert rounds[0].options == len(book) and rounds[0].paths == 2048 * len(book)
    assert sum(r.converged for r in rounds) == len(book)
    assert all(later.options < earlier.options for earlier, later in zip(rounds, rounds[1:]))
    for r in res:  # each result's path count: the pilot's, or a larger multiple of 256
        p = int(r.diagnostics.get("num_paths"))
        assert p >= 2048 and p % 256 == 0
    from openferric_b200 import PricingError
    with pytest.raises(PricingError, match="max_rounds"):
        price_book_to_stderr(book, seed=3, max_rounds=0)
    with pytest.raises(PricingError, match="margin"):
        price_book_to_stderr(book, seed=3, margin=0.5)
    # the same pilot (same seed) sends the same options to the first follow-up;
    # a larger margin gives them more paths
    _, wide = price_book_to_stderr(book, seed=3, se_rel=2e-3, pilot_paths=2048, margin=1.5)
    assert wide[0].paths == rounds[0].paths and wide[1].options == rounds[1].options
    assert wide[1].paths > rounds[1].paths


def test_price_book_to_stderr_pools_its_rounds():
    """Each round draws from its own seed and an option's result pools the
    running sums of all its rounds: replaying the rounds with plain book
    launches (the same sub-books, seeds and path counts) and adding their sums
    gives the driver's results."""
    import math
    from dataclasses import replace
    from openferric_b200.book import BookPlan, price_book_to_stderr
    book = synthetic_book(n=8, seed=8, min_log2_paths=10, max_log2_paths=11)
    se_rel, pilot, seed, margin = 2e-3, 2048, 3, 1.1
    res, rounds = price_book_to_stderr(book, seed=seed, se_rel=se_rel, pilot_paths=pilot, margin=margin)
    assert len(rounds) >= 2  # the test needs at least one follow-up round
    sums = [[0.0] * 5 for _ in book]
    samples, paths = [0] * len(book), [0] * len(book)
    pending, nxt = list(range(len(book))), {i: pilot for i in range(len(book))}
    for r in range(len(rounds)):
        sub = [replace(book[i], num_paths=nxt[i]) for i in pending]
        plan = BookPlan(sub, seed + r, block=256, paths_per_thread=4, use_graph=False)  # the driver's tile shape here
        try:
            plan.launch()
            raw = plan.raw_results()
        finally:
            plan.close()
        still = []
        for i, o in zip(pending, raw):
            for k, f in enumerate(("sum_x", "sum_x2", "sum_y", "sum_xy", "sum_y2")):
                sums[i][k] += getattr(o, f)
            samples[i] += o.samples
            paths[i] += nxt[i]
            n = samples[i]
            df = math.exp(-book[i].market.rate * book[i].instrument.expiry)
            var = (sums[i][1] - sums[i][0] ** 2 / n) / (n - 1)
            se = df * math.sqrt(var / n)
            tgt = se_rel * book[i].market.spot
            if se > tgt:
                need = paths[i] * (se / tgt) ** 2 * margin
                nxt[i] = max(256, math.ceil((need - paths[i]) / 256.0) * 256)
                still.append(i)
        pending = still
    for i, (e, got) in enumerate(zip(book, res)):
        n = samples[i]
        df = math.exp(-e.market.rate * e.instrument.expiry)
        price = df * sums[i][0] / n
        assert abs(got.price - price) <= 1e-9 * abs(price) + 1e-12, (i, got.price, price)
        assert int(got.diagnostics.get("num_paths")) == paths[i]
