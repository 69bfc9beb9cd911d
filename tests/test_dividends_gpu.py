"""Discrete dividends on GBM paths (DiscreteDividendGbmPathGenerator,
mc_engine.rs:123-175) through of_mc_run (FP64 reference stream and FP32
Philox) and the batched book, against the oracle and the reference's
dividend tests (tests/dividend_modelling_issue58.rs)."""
import math

import pytest

import openferric_b200 as of
from openferric_b200 import (ArithmeticAsianMC, AsianOption, AsianSpec, Averaging, BarrierOption, DividendEvent,
                             DividendSchedule, StrikeType,
                             MonteCarloPricingEngine, OptionType, Precision, PricingError, VanillaOption,
                             VarianceReduction)
from openferric_b200.engines import GbmPathGenerator, Gbm, price_strike_strip

pytestmark = pytest.mark.gpu

MIXED = DividendSchedule.new([DividendEvent.cash(0.25, 1.5), DividendEvent.proportional(0.5, 0.02),
                              DividendEvent.cash(0.75, 2.0), DividendEvent.cash(1.5, 9.0)])


def _arith(opt, k, expiry, steps):
    return AsianOption(opt, k, expiry, AsianSpec(Averaging.Arithmetic, StrikeType.Fixed, of.daily_fixings(expiry, steps)))


def _market(sched, spot=100.0, r=0.04, q=0.01, vol=0.25):
    return of.Market.builder().spot(spot).rate(r).dividend_yield(q).dividend_schedule(sched).flat_vol(vol).build()


@pytest.mark.parametrize("vr", [VarianceReduction.None_, VarianceReduction.Antithetic,
                                VarianceReduction.ControlVariate])
@pytest.mark.parametrize("kind", ["vanilla", "barrier", "asian"])
def test_fp64_dividends_match_oracle(orc, vr, kind):
    from test_mc_gpu import _oracle_run, close, PRICE_RTOL
    m = _market(MIXED)
    if kind == "vanilla":
        inst = VanillaOption.european_put(100.0, 1.0)
    elif kind == "barrier":
        inst = BarrierOption.builder().put().strike(100.0).expiry(1.0).down_and_in(90.0).rebate(0.5).build()
    else:
        inst = _arith(OptionType.Call, 100.0, 1.0, 50)
    eng = MonteCarloPricingEngine(20000, 50, 11).with_variance_reduction(vr)
    res = eng.price(inst, m)
    gen = GbmPathGenerator(Gbm(m.rate - m.dividend_yield, 0.25), 100.0, 1.0, 50, m.dividend_schedule)
    # control variates are off with a discrete schedule (mc_engine.rs:462-464, 552-554)
    ref = _oracle_run(orc, gen, inst, vr is VarianceReduction.Antithetic, None, math.exp(-0.04), 20000, 11)
    assert close(res.price, ref.price, PRICE_RTOL), (res.price, ref.price)


def test_terminal_mean_is_the_dividend_forward():
    """E[S_T] of the simulated paths is the schedule's forward (dividends.rs:145-184)."""
    m = _market(MIXED, q=0.0)
    fwd = m.forward_price(1.0)
    call0 = VanillaOption.european_call(1e-9, 1.0)  # payoff = S_T
    for prec in (Precision.Fp64Reference, Precision.Fp32Philox):
        r = MonteCarloPricingEngine(1 << 18, 64, 3).with_precision(prec).price(call0, m)
        est = r.price / math.exp(-0.04)
        assert abs(est - fwd) <= 4.0 * r.stderr / math.exp(-0.04) + 1e-6, (prec, est, fwd)


def test_barrier_knocks_in_on_the_ex_dividend_jump():
    """dividend_modelling_issue58.rs:57-112: a 10 cash dividend at t=0.5 on a
    near-deterministic path knocks in a 95 down-and-in put (price ~ 10)."""
    barrier = BarrierOption.builder().put().strike(100.0).expiry(1.0).down_and_in(95.0).rebate(0.0).build()
    base = of.Market.builder().spot(100.0).rate(0.0).dividend_yield(0.0).flat_vol(1.0e-8).build()
    with_div = _market(DividendSchedule.new([DividendEvent.cash(0.5, 10.0)]), r=0.0, q=0.0, vol=1.0e-8)
    for prec in (Precision.Fp64Reference, Precision.Fp32Philox):
        eng = MonteCarloPricingEngine(20_000, 252, 42).with_variance_reduction(
            VarianceReduction.Antithetic).with_precision(prec)
        assert eng.price(barrier, base).price <= 1.0e-3
        assert abs(eng.price(barrier, with_div).price - 10.0) <= 1.0e-3


def test_fp32_book_with_dividends_agrees_with_oracle(orc):
    from test_mc_gpu import _oracle_run
    m = _market(MIXED)
    insts = [VanillaOption.european_call(100.0, 1.0), VanillaOption.european_put(95.0, 2.0),
             _arith(OptionType.Put, 100.0, 1.0, 64)]
    eng = MonteCarloPricingEngine(1 << 18, 64, 5).with_precision(Precision.Fp32Philox)
    gpu = eng.price_batch([(i, m) for i in insts])
    for inst, g in zip(insts, gpu):
        gen = GbmPathGenerator(Gbm(m.rate - m.dividend_yield, 0.25), 100.0, inst.expiry, 64, m.dividend_schedule)
        ref = _oracle_run(orc, gen, inst, False, None, math.exp(-0.04 * inst.expiry), 1 << 16, 9)
        se = math.hypot(g.stderr, ref.stderr_)
        assert abs(g.price - ref.price) <= 4.0 * se + 1e-3, (inst, g.price, ref.price, se)


def test_arithmetic_asian_mc_runs_without_control_variate_under_dividends():
    m = _market(MIXED)
    inst = _arith(OptionType.Call, 100.0, 1.0, 32)
    r = ArithmeticAsianMC(50_000, 32, 7).price(inst, m)
    no_div = ArithmeticAsianMC(50_000, 32, 7).price(inst, _market(DividendSchedule.empty()))
    assert math.isfinite(r.price) and r.price < no_div.price  # dividends lower the call


def test_strip_rejects_dividends_and_bad_events_are_invalid():
    gen = GbmPathGenerator(Gbm(0.03, 0.2), 100.0, 1.0, 16, MIXED)
    with pytest.raises(PricingError):
        price_strike_strip(gen, OptionType.Call, [100.0], 1000, 1, 1.0)
    with pytest.raises(PricingError):
        DividendSchedule.new([DividendEvent.cash(0.5, 1.0), DividendEvent.cash(0.5, 2.0)])
    with pytest.raises(PricingError):
        DividendEvent.proportional(0.5, 1.0)
