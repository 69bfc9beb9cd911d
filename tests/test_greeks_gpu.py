"""GPU Monte Carlo Greeks on the reference streams vs the oracle's restatement of
mc_aad.rs / mc_greeks.rs (same draws: agreement to ~1e-12 relative), plus the
reference's own known-answer tests run through the GPU engines."""
import math

import pytest
from scipy.special import ndtr

from openferric_b200 import (Heston, Market, MonteCarloPricingEngine, OptionType, PricingError, VanillaOption,
                             VarianceReduction)
from openferric_b200 import _abi as A
from openferric_b200.analytic import bs_greeks
from openferric_b200.greeks import HestonAadConfig, MonteCarloGreeksEngine, heston_price_delta_aad

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


@pytest.mark.parametrize("option_type", [OptionType.Call, OptionType.Put])
@pytest.mark.parametrize("anti", [False, True])
def test_pathwise_aad_matches_oracle(orc, option_type, anti):
    m = Market.builder().spot(100.0).rate(0.03).dividend_yield(0.01).flat_vol(0.25).build()
    opt = VanillaOption(option_type, 105.0, 1.3)
    vr = VarianceReduction.Antithetic if anti else VarianceReduction.None_
    res = MonteCarloPricingEngine(20001, 37, 42).with_variance_reduction(vr).price_with_greeks_aad(opt, m)
    ref = orc.gbm_pathwise_aad(option_type.value, 105.0, 100.0, 0.03, 0.01, 0.25, 1.3, 20001, 37, 42, anti)
    assert rel(res.price, ref["price"]) < 1e-12
    assert rel(res.stderr, ref["stderr"]) < 1e-10
    g = res.greeks
    assert rel(g.delta, ref["delta"]) < 1e-11
    assert rel(g.vega, ref["vega"]) < 1e-11
    assert rel(g.theta, ref["theta"]) < 1e-11
    assert rel(g.rho, ref["rho"]) < 1e-11
    assert g.gamma == 0.0


def test_pathwise_aad_recovers_bs_greeks():
    """mc_aad.rs:352-409 on the GPU engine (120k antithetic x 64, seed 42)."""
    m = Market.builder().spot(100.0).rate(0.03).dividend_yield(0.01).flat_vol(0.20).build()
    opt = VanillaOption.european_call(100.0, 1.0)
    res = MonteCarloPricingEngine(120_000, 64, 42).with_variance_reduction(
        VarianceReduction.Antithetic).price_with_greeks_aad(opt, m)
    ref = bs_greeks(OptionType.Call, 100.0, 100.0, 0.03, 0.01, 0.2, 1.0)
    g = res.greeks
    assert abs(g.delta - ref["delta"]) < 6e-3
    assert abs(g.vega - ref["vega"]) < 8e-2
    assert abs(g.rho - ref["rho"]) < 7e-2
    assert abs(g.theta - ref["theta"]) < 9e-2


def test_heston_delta_matches_oracle_and_crn_bump(orc):
    model = Heston(mu=0.03, kappa=1.8, theta=0.04, xi=0.6, rho=-0.5, v0=0.04)
    cfg = HestonAadConfig(60_000, 64, 7)
    price, delta = heston_price_delta_aad(OptionType.Call, 70.0, 1.0, 100.0, 0.03, model, cfg)
    rp, rd = orc.heston_price_delta(OF_CALL, 70.0, 1.0, 100.0, 0.03, 0.03, 1.8, 0.04, 0.6, -0.5, 0.04, 60_000, 64, 7)
    assert rel(price, rp) < 1e-12 and rel(delta, rd) < 1e-12
    up, _ = heston_price_delta_aad(OptionType.Call, 70.0, 1.0, 100.0 + 1e-3, 0.03, model, cfg)
    dn, _ = heston_price_delta_aad(OptionType.Call, 70.0, 1.0, 100.0 - 1e-3, 0.03, model, cfg)
    assert abs(delta - (up - dn) / 2e-3) < 1e-4  # mc_aad.rs:437-480


OF_CALL = A.OF_CALL


@pytest.mark.parametrize("anti", [False, True])
def test_greek_estimators_match_oracle(orc, anti):
    m = Market.builder().spot(100.0).rate(0.05).dividend_yield(0.0).flat_vol(0.2).build()
    opt = VanillaOption.european_put(95.0, 0.8)
    eng = MonteCarloGreeksEngine(50001, 9).with_antithetic(anti)
    pw, lr = eng.estimate_pathwise(opt, m), eng.estimate_likelihood_ratio(opt, m)
    ref = orc.mc_greek_estimators(A.OF_PUT, 95.0, 100.0, 0.05, 0.0, 0.2, 0.8, 50001, 9, anti)
    assert rel(pw.delta, ref["pathwise_delta"]) < 1e-12
    assert rel(pw.gamma, ref["pathwise_gamma"]) < 1e-12
    assert rel(lr.delta, ref["lr_delta"]) < 1e-12
    assert rel(lr.gamma, ref["lr_gamma"]) < 1e-12
    assert rel(lr.vega, ref["lr_vega"]) < 1e-12


def test_greek_estimators_reference_values():
    """mc_greeks.rs:361-418 through the GPU engine."""
    m = Market.builder().spot(100.0).rate(0.05).dividend_yield(0.0).flat_vol(0.2).build()
    opt = VanillaOption.european_call(100.0, 1.0)
    eng = MonteCarloGreeksEngine(100_000, 42)
    pw, lr = eng.estimate_pathwise(opt, m), eng.estimate_likelihood_ratio(opt, m)
    d1 = (0.05 + 0.02) / 0.2
    assert abs(pw.delta - ndtr(d1)) / ndtr(d1) <= 0.02
    assert abs(pw.delta - 0.6368) / 0.6368 < 0.02
    assert abs(pw.gamma - 0.01876) / 0.01876 < 0.20
    assert abs(lr.vega - 37.524) / 37.524 < 0.05


def test_greeks_validation():
    m = Market.builder().spot(100.0).rate(0.05).flat_vol(0.2).build()
    with pytest.raises(PricingError, match="European exercise only"):
        MonteCarloGreeksEngine(1000, 1).estimate_pathwise(VanillaOption.american_put(100, 1), m)
    with pytest.raises(PricingError, match="invalid Heston parameters"):
        heston_price_delta_aad(OptionType.Call, 100, 1.0, 100, 0.0, Heston(0.0, -1.0, 0.04, 0.5, 0.0, 0.04),
                               HestonAadConfig(10, 10, 1))
