"""GpuMcEngine (the reference Python module's McEngine surface) on the GPU:
each static method returns exactly what the engine it wraps returns for the
same instrument and market, and the reference's own known answers hold
(mc_engine.rs:998-1021: 100k x 252 paths, seed 42, within 1 % of Black-Scholes;
the arithmetic Asian of mc_engine.rs:1097-1132 within 2 % of 5.73)."""
import math

import pytest

from openferric_b200 import (ArithmeticAsianMC, AsianOption, AsianSpec, Averaging, GpuMcEngine, Market,
                             MonteCarloPricingEngine, OptionType, StrikeType, VanillaOption, VarianceReduction)
from openferric_b200.analytic import bs_price
from openferric_b200.greeks import MonteCarloGreeksEngine

pytestmark = pytest.mark.gpu


def _market(spot=100.0, rate=0.05, q=0.0, vol=0.2):
    return Market.builder().spot(spot).rate(rate).dividend_yield(q).flat_vol(vol).build()


def test_vanilla_price_is_the_engine_price_and_the_reference_known_answer():
    r = GpuMcEngine.vanilla_price("call", 100.0, 100.0, 1.0, 0.05, 0.0, 0.2, 100_000, 252, 42)
    direct = MonteCarloPricingEngine(100_000, 252, 42).price(VanillaOption.european_call(100.0, 1.0), _market())
    assert r.price == direct.price and r.stderr == direct.stderr
    bs = bs_price(OptionType.Call, 100.0, 100.0, 0.05, 0.0, 0.2, 1.0)
    assert abs(r.price - bs) <= 0.01 * bs
    assert r.diagnostics.get("num_paths") == 100_000.0


@pytest.mark.parametrize("vr", ["antithetic", "control_variate", "Control-Variate"])
def test_vanilla_price_variance_reduction_strings(vr):
    r = GpuMcEngine.vanilla_price("put", 100.0, 105.0, 0.5, 0.03, 0.01, 0.25, 50_000, 64, 7, variance_reduction=vr)
    kind = VarianceReduction.Antithetic if vr == "antithetic" else VarianceReduction.ControlVariate
    direct = MonteCarloPricingEngine(50_000, 64, 7).with_variance_reduction(kind).price(
        VanillaOption.european_put(105.0, 0.5), _market(rate=0.03, q=0.01, vol=0.25))
    assert r.price == direct.price and r.stderr == direct.stderr


def test_fp32_precision_agrees_with_fp64_statistically():
    a = GpuMcEngine.vanilla_price("call", 100.0, 100.0, 1.0, 0.05, 0.0, 0.2, 200_000, 64, 3)
    b = GpuMcEngine.vanilla_price("call", 100.0, 100.0, 1.0, 0.05, 0.0, 0.2, 200_000, 64, 4, precision="fp32")
    assert abs(a.price - b.price) <= 4.0 * math.hypot(a.stderr, b.stderr)


def test_arithmetic_asian_price_is_the_engine_price_and_the_reference_known_answer():
    obs = [m / 11.0 for m in range(12)]
    r = GpuMcEngine.arithmetic_asian_price("call", 100.0, 100.0, 1.0, 0.05, 0.0, 0.2, obs, 100_000, 252, 42)
    inst = AsianOption(OptionType.Call, 100.0, 1.0, AsianSpec(Averaging.Arithmetic, StrikeType.Fixed, obs))
    direct = ArithmeticAsianMC(100_000, 252, 42).price(inst, _market())
    assert r.price == direct.price and r.stderr == direct.stderr
    assert abs(r.price - 5.73) / 5.73 <= 0.02


def test_greeks_are_the_engine_estimates():
    g = GpuMcEngine.greeks_pathwise("call", 100.0, 100.0, 1.0, 0.05, 0.0, 0.2, 100_000, 5)
    l = GpuMcEngine.greeks_likelihood_ratio("call", 100.0, 100.0, 1.0, 0.05, 0.0, 0.2, 100_000, 5)
    eng = MonteCarloGreeksEngine(100_000, 5)
    inst, m = VanillaOption.european_call(100.0, 1.0), _market()
    assert g == eng.estimate_pathwise(inst, m)
    assert l == eng.estimate_likelihood_ratio(inst, m)
    assert 0.55 < g.delta < 0.7 and 0.55 < l.delta < 0.7
