"""GPU Bermudan Longstaff-Schwartz with the exercise boundary (of_lsm_bermudan)
against the oracle's restatement of price_bermudan_with_boundary
(longstaff_schwartz.rs:294-417) and the reference's Bermudan tests
(tests/bermudan_quantlib.rs)."""
import math

import numpy as np
import pytest

import openferric_b200 as of
from openferric_b200 import OptionType, Precision, PricingError
from openferric_b200.lsm import LongstaffSchwartzEngine
from openferric_b200 import Heston

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _market(spot, rate, q, vol):
    return of.Market.builder().spot(spot).rate(rate).dividend_yield(q).flat_vol(vol).build()


def _smile(k, t):
    return max(0.18 + 0.08 * abs(k / 100.0 - 1.0) + 0.03 * math.sqrt(max(t, 1e-6)), 0.05)


def _compare_to_oracle(gpu, ref, price_rel=1e-9):
    p, se, recs = ref
    assert abs(gpu.result.price - p) <= price_rel * max(1.0, abs(p)), (gpu.result.price, p)
    assert abs(gpu.result.stderr - se) <= 1e-6 * se + 1e-12
    assert len(gpu.exercise_boundary) == len(recs)
    for g, (t, k, b, itm, ex) in zip(gpu.exercise_boundary, recs):
        assert g.time == t and g.strike == k
        assert g.itm_paths == itm
        assert abs(g.exercised_paths - ex) <= 2
        assert (g.boundary_spot is None) == (b is None)
        if b is not None and g.exercised_paths == ex:
            assert g.boundary_spot == pytest.approx(b, rel=1e-12)


@pytest.mark.parametrize("opt", [OptionType.Put, OptionType.Call])
@pytest.mark.parametrize("degree", [2, 3])
def test_gbm_fp64_matches_oracle_stream(orc, opt, degree):
    dates = [0.1, 0.25, 0.4, 0.55, 0.8, 0.9]
    strikes = [100.0, 99.0, 98.0, 97.0, 96.0, 95.0]
    inst = of.BermudanOption.new(opt, 1.0, dates, strikes)
    m = _market(100.0, 0.04, 0.02, 0.25)
    eng = LongstaffSchwartzEngine(30000, 60, 17).with_basis_degree(degree)
    gpu = eng.price_bermudan_with_boundary(inst, m)
    ref = orc.lsm_bermudan(opt.value, 1.0, inst.effective_schedule(), 100.0, 0.04, 0.02, 30000, 60, 17, dynamics=0,
                           vol=0.25, degree=degree)
    _compare_to_oracle(gpu, ref)
    assert gpu.result.diagnostics.get("exercise_dates") == 7.0  # 6 dates + (expiry, last strike)


def test_local_vol_fp64_matches_oracle_stream(orc):
    inst = of.BermudanOption.with_constant_strike(OptionType.Put, 100.0, 1.0, [0.2, 0.4, 0.6, 0.8, 1.0])
    m = of.Market.builder().spot(100).rate(0.02).dividend_yield(0.01).vol_surface(_smile).build()
    eng = LongstaffSchwartzEngine(20000, 45, 123).with_local_vol_dynamics()
    gpu = eng.price_bermudan_with_boundary(inst, m)
    ref = orc.lsm_bermudan(1, 1.0, inst.effective_schedule(), 100.0, 0.02, 0.01, 20000, 45, 123, dynamics=1,
                           lv=m.vol.grid())
    _compare_to_oracle(gpu, ref)
    assert not gpu.result.diagnostics.contains_key("vol")


def test_heston_fp64_matches_oracle_stream(orc):
    inst = of.BermudanOption.with_constant_strike(OptionType.Put, 100.0, 1.0, [0.2, 0.4, 0.6, 0.8, 1.0])
    h = Heston(mu=0.0, kappa=2.0, theta=0.04, xi=0.6, rho=-0.5, v0=0.04)
    eng = LongstaffSchwartzEngine(20000, 50, 321).with_heston_dynamics(h)
    gpu = eng.price_bermudan_with_boundary(inst, _market(100.0, 0.02, 0.01, 0.2))
    ref = orc.lsm_bermudan(1, 1.0, inst.effective_schedule(), 100.0, 0.02, 0.01, 20000, 50, 321, dynamics=2,
                           heston=(2.0, 0.04, 0.6, -0.5, 0.04))
    _compare_to_oracle(gpu, ref)


def test_quantlib_fd_cases_at_reference_settings():
    """bermudan_quantlib.rs:207-239: LSM(450000, 120, 7) within 0.5 % of the
    QuantLib FD price on the put cases, in both precisions; every case has a
    populated boundary."""
    g = load_golden("bermudan_quantlib.json")
    e = g["lsm_engine"]
    for c in g["cases"]:
        opt = OptionType.Put if c["option_type"] == "Put" else OptionType.Call
        inst = of.BermudanOption.with_constant_strike(opt, c["strike"], c["expiry"], c["dates"])
        m = _market(c["spot"], c["rate"], c["dividend"], c["vol"])
        for prec in (Precision.Fp64Reference, Precision.Fp32Philox):
            eng = LongstaffSchwartzEngine(e["num_paths"], e["num_steps"], e["seed"]).with_precision(prec)
            out = eng.price_bermudan_with_boundary(inst, m)
            err = abs(out.result.price - c["quantlib_fd_price"]) / c["quantlib_fd_price"]
            tol = g["rel_tolerance"] if opt is OptionType.Put else 2 * g["rel_tolerance"]
            assert err <= tol, (c, prec, out.result.price, out.result.stderr)
            if opt is OptionType.Put:
                assert any(b.boundary_spot is not None for b in out.exercise_boundary)


def test_step_down_strike_prices_lower_than_constant():
    """bermudan_quantlib.rs:241-265."""
    dates = [0.25, 0.5, 0.75, 1.0]
    step = of.BermudanOption.new(OptionType.Put, 1.0, dates, [100.0, 97.5, 95.0, 92.5])
    const = of.BermudanOption.with_constant_strike(OptionType.Put, 100.0, 1.0, dates)
    m = _market(100.0, 0.03, 0.0, 0.25)
    lsm = LongstaffSchwartzEngine(250_000, 100, 42)
    assert lsm.price(step, m).price < lsm.price(const, m).price


def test_local_vol_and_heston_dynamics_at_reference_settings():
    """bermudan_quantlib.rs:267-335."""
    inst = of.BermudanOption.with_constant_strike(OptionType.Put, 100.0, 1.0, [0.2, 0.4, 0.6, 0.8, 1.0])
    lv_m = of.Market.builder().spot(100).rate(0.02).dividend_yield(0.01).vol_surface(_smile).build()
    out = LongstaffSchwartzEngine(200_000, 90, 123).with_local_vol_dynamics().price_bermudan_with_boundary(inst, lv_m)
    assert math.isfinite(out.result.price) and out.result.price > 0
    assert any(p.boundary_spot is not None for p in out.exercise_boundary)
    h = Heston(mu=0.0, kappa=2.0, theta=0.04, xi=0.6, rho=-0.5, v0=0.04)
    out = LongstaffSchwartzEngine(220_000, 100, 321).with_heston_dynamics(h).price_bermudan_with_boundary(
        inst, _market(100.0, 0.02, 0.01, 0.2))
    assert math.isfinite(out.result.price) and out.result.price > 0
    assert any(p.boundary_spot is not None for p in out.exercise_boundary)


def test_dense_schedule_approaches_american(orc):
    """bermudan_quantlib.rs:337-389: 52 dates, LSM(350000, 120, 11) within 3 %
    of the American price (CRR 2500 steps here)."""
    am = orc.crr_american(1, 100.0, 100.0, 0.05, 0.0, 0.2, 1.0, 2500)
    inst = of.BermudanOption.with_constant_strike(OptionType.Put, 100.0, 1.0, [i / 52 for i in range(1, 53)])
    p = LongstaffSchwartzEngine(350_000, 120, 11).price(inst, _market(100.0, 0.05, 0.0, 0.2))
    assert p.price <= am + 0.20
    assert abs(p.price - am) / am <= 0.03


def test_fp32_philox_agrees_with_fp64_within_stderr():
    inst = of.BermudanOption.with_constant_strike(OptionType.Put, 40.0, 1.0, [0.25, 0.5, 0.75, 1.0])
    m = _market(36.0, 0.06, 0.0, 0.2)
    for dyn in ("gbm", "heston", "lv"):
        e64 = LongstaffSchwartzEngine(1 << 18, 50, 5)
        e32 = LongstaffSchwartzEngine(1 << 18, 50, 6).with_precision(Precision.Fp32Philox)
        mm = m
        if dyn == "heston":
            h = Heston(mu=0.0, kappa=1.5, theta=0.04, xi=0.3, rho=-0.6, v0=0.04)
            e64.with_heston_dynamics(h)
            e32.with_heston_dynamics(h)
        elif dyn == "lv":
            mm = of.Market.builder().spot(36).rate(0.06).vol_surface(lambda k, t: 0.2 + 0.05 * abs(k / 40 - 1)).build()
            e64.with_local_vol_dynamics()
            e32.with_local_vol_dynamics()
        a = e64.price_bermudan_with_boundary(inst, mm).result
        b = e32.price_bermudan_with_boundary(inst, mm).result
        assert abs(a.price - b.price) <= 4.0 * math.hypot(a.stderr, b.stderr) + 2e-3, (dyn, a.price, b.price)


def test_bermudan_validation_messages():
    m = _market(100.0, 0.03, 0.0, 0.2)
    eng = LongstaffSchwartzEngine(1000, 1, 1)
    inst = of.BermudanOption.with_constant_strike(OptionType.Put, 100.0, 1.0, [0.5, 1.0])
    with pytest.raises(PricingError, match="num_steps must be >= 2"):
        eng.price_bermudan_with_boundary(inst, m)
    with pytest.raises(PricingError, match="strictly increasing"):
        LongstaffSchwartzEngine(1000, 10, 1).price(
            of.BermudanOption.with_constant_strike(OptionType.Put, 100.0, 1.0, [0.5, 0.5]), m)
    bad = Heston(mu=0.0, kappa=-1.0, theta=0.04, xi=0.3, rho=0.0, v0=0.04)
    with pytest.raises(PricingError, match="invalid Heston parameters"):
        LongstaffSchwartzEngine(1000, 10, 1).with_heston_dynamics(bad).price(inst, m)
