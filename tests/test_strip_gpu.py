"""GPU strike strip (of_mc_strip): many European strikes from one shared FP32
Philox path set, checked against the oracle's FP64 Monte Carlo (independent
draws, same scheme) and the semi-analytic Heston / Black-Scholes prices."""
import math

import numpy as np
import pytest

from openferric_b200 import (Gbm, GbmPathGenerator, Heston, HestonPathGenerator, OptionType, PricingError,
                             price_strike_strip)
from openferric_b200 import _abi as A
from openferric_b200.analytic import bs_price

pytestmark = pytest.mark.gpu

HESTON = Heston(mu=0.03, kappa=2.0, theta=0.04, xi=0.5, rho=-0.7, v0=0.04)
STRIKES = [80.0 + k for k in range(41)]


@pytest.mark.parametrize("anti", [False, True])
@pytest.mark.parametrize("option_type", [OptionType.Call, OptionType.Put])
def test_heston_euler_strip_matches_oracle_mc(orc, anti, option_type):
    gen = HestonPathGenerator(HESTON, 100.0, 1.0, 64)
    df = math.exp(-0.03)
    gpu = price_strike_strip(gen, option_type, STRIKES, 1 << 18, 7, df, antithetic=anti)
    cfg = A.OfMcConfig(num_paths=1 << 15, seed=11, antithetic=int(anti), discount_factor=df)
    ref = orc.mc_strip(gen.to_abi(), option_type.value, STRIKES, cfg, threads=8)
    for k, ((p, s), r) in enumerate(zip(gpu, ref)):
        se = math.hypot(s, r.stderr_)
        assert abs(p - r.price) <= 4.0 * se + 1e-3, (STRIKES[k], p, r.price, se)


def test_gbm_strip_matches_black_scholes():
    gen = GbmPathGenerator(Gbm(0.05, 0.2), 100.0, 1.0, 32)
    res = price_strike_strip(gen, OptionType.Call, STRIKES, 1 << 20, 3, math.exp(-0.05), antithetic=True)
    for k, (p, s) in zip(STRIKES, res):
        bs = bs_price(OptionType.Call, 100, k, 0.05, 0.0, 0.2, 1.0)
        assert abs(p - bs) <= 4.0 * s + 1e-3, (k, p, bs, s)


def test_full_size_heston_strip_against_semi_analytic(orc):
    """The benchmark workload (2^20 paths x 256 steps, seed 7).  The Euler
    scheme has an O(dt) bias, so the check is on the step-doubling
    (Richardson) extrapolation 2 P(512) - P(256)."""
    df = math.exp(-0.03)
    p256 = price_strike_strip(HestonPathGenerator(HESTON, 100.0, 1.0, 256), OptionType.Call, STRIKES, 1 << 20, 7, df)
    p512 = price_strike_strip(HestonPathGenerator(HESTON, 100.0, 1.0, 512), OptionType.Call, STRIKES, 1 << 20, 7, df)
    worst = 0.0
    for k, (a, b) in zip(STRIKES, zip(p256, p512)):
        exact = orc.heston_call(100.0, k, 0.03, 0.0, 1.0, 0.04, 2.0, 0.04, 0.5, -0.7)
        extrap = 2.0 * b[0] - a[0]
        se = math.sqrt(4.0 * b[1] ** 2 + a[1] ** 2)
        worst = max(worst, abs(extrap - exact) / se)
        assert abs(extrap - exact) <= 5.0 * se + 5e-3, (k, a[0], b[0], extrap, exact, se)
        assert a[1] <= 0.02  # SE of the strip at 2^20 paths


def test_qe_strip_against_semi_analytic(orc):
    gen = HestonPathGenerator(HESTON, 100.0, 1.0, 256, scheme="qe")
    res = price_strike_strip(gen, OptionType.Call, STRIKES, 1 << 20, 7, math.exp(-0.03))
    for k, (p, s) in zip(STRIKES, res):
        exact = orc.heston_call(100.0, k, 0.03, 0.0, 1.0, 0.04, 2.0, 0.04, 0.5, -0.7)
        assert abs(p - exact) <= 4.0 * s + 0.01, (k, p, exact, s)


def test_strip_put_call_parity_on_shared_paths():
    gen = HestonPathGenerator(HESTON, 100.0, 1.0, 64)
    df = math.exp(-0.03)
    calls = price_strike_strip(gen, OptionType.Call, STRIKES, 1 << 18, 5, df)
    puts = price_strike_strip(gen, OptionType.Put, STRIKES, 1 << 18, 5, df)
    # same paths: C - P = df (E[S_T] - K) exactly in expectation; the MC
    # estimate of E[S_T] is common to all strikes
    fwd = [c[0] - p[0] + df * k for (c, p, k) in zip(calls, puts, STRIKES)]
    assert max(fwd) - min(fwd) < 1e-3
    assert abs(fwd[0] - 100.0) < 0.2


def test_strip_more_than_128_strikes_is_chunked():
    gen = GbmPathGenerator(Gbm(0.05, 0.2), 100.0, 1.0, 8)
    ks = list(np.linspace(50, 150, 300))
    res = price_strike_strip(gen, OptionType.Call, ks, 1 << 14, 3, 1.0)
    assert len(res) == 300 and all(np.isfinite(p) for p, _ in res)


def test_strip_rejects_bad_strikes():
    gen = GbmPathGenerator(Gbm(0.05, 0.2), 100.0, 1.0, 8)
    with pytest.raises(PricingError):
        price_strike_strip(gen, OptionType.Call, [100.0, -1.0], 1000, 3, 1.0)


@pytest.mark.parametrize("scheme", ["euler", "qe"])
@pytest.mark.parametrize("anti", [False, True])
@pytest.mark.parametrize("n_paths", [1 << 16, 100_003])
def test_strip_two_samples_in_flight_matches_one(scheme, anti, n_paths):
    """tile_ilp=2 walks the same Philox counters in a different order, so the
    prices agree with tile_ilp=1 up to the FP32 accumulation order; a ragged
    path count exercises the partial last warp round."""
    gen = HestonPathGenerator(HESTON, 100.0, 1.0, 63, scheme=scheme)
    one = price_strike_strip(gen, OptionType.Call, STRIKES[:37], n_paths, 9, 0.97, antithetic=anti, tile_ilp=1)
    two = price_strike_strip(gen, OptionType.Call, STRIKES[:37], n_paths, 9, 0.97, antithetic=anti, tile_ilp=2)
    for (p1, s1), (p2, s2) in zip(one, two):
        assert abs(p1 - p2) <= 2e-6 * max(1.0, abs(p1)), (p1, p2)
        assert abs(s1 - s2) <= 2e-6 * max(1.0, s1), (s1, s2)


def test_strip_gbm_two_samples_in_flight_matches_one():
    gen = GbmPathGenerator(Gbm(0.05, 0.2), 100.0, 1.0, 30)
    one = price_strike_strip(gen, OptionType.Put, STRIKES, 1 << 17, 4, 0.95, tile_ilp=1)
    two = price_strike_strip(gen, OptionType.Put, STRIKES, 1 << 17, 4, 0.95, tile_ilp=2)
    for (p1, _), (p2, _) in zip(one, two):
        assert abs(p1 - p2) <= 2e-6 * max(1.0, abs(p1)), (p1, p2)


@pytest.mark.parametrize("scheme", ["euler", "qe", "gbm"])
@pytest.mark.parametrize("anti", [False, True])
@pytest.mark.parametrize("n_paths,strikes", [(1 << 16, 37), (100_003, 41), (333, 64), (4099, 5)])
def test_strip_warp_specialised_matches_one_sample_per_thread(scheme, anti, n_paths, strikes):
    """tile_ilp=3: producer warps write the same Philox blocks to a shared-memory
    ring and consumer warps run the same steps and payoffs per sample, so the
    prices agree with tile_ilp=1 up to the FP32 accumulation order.  Odd step
    counts exercise the partial last Philox block, ragged path counts the
    partial last warp round, 64 strikes two strikes per lane, and 333 paths
    fewer samples than one block's round."""
    gen = GbmPathGenerator(Gbm(0.05, 0.2), 100.0, 1.0, 29) if scheme == "gbm" else \
        HestonPathGenerator(HESTON, 100.0, 1.0, 63, scheme=scheme)
    ks = [60.0 + 80.0 * k / max(1, strikes - 1) for k in range(strikes)]
    one = price_strike_strip(gen, OptionType.Call, ks, n_paths, 9, 0.97, antithetic=anti, tile_ilp=1)
    ws = price_strike_strip(gen, OptionType.Call, ks, n_paths, 9, 0.97, antithetic=anti, tile_ilp=3)
    for (p1, s1), (p3, s3) in zip(one, ws):
        assert abs(p1 - p3) <= 2e-6 * max(1.0, abs(p1)), (p1, p3)
        assert abs(s1 - s3) <= 2e-6 * max(1.0, s1), (s1, s3)


def test_strip_warp_specialised_plan_replays():
    """The plan (CUDA graph with the status-word reset) replays the
    warp-specialised kernel and returns the same prices every time."""
    from openferric_b200.engines import StripPlan
    gen = HestonPathGenerator(HESTON, 100.0, 1.0, 64)
    plan = StripPlan(gen, OptionType.Call, STRIKES, 1 << 16, 5, 0.97, tile_ilp=3)
    try:
        plan.launch()
        first = plan.results()
        for _ in range(3):
            plan.launch()
        assert plan.results() == first
    finally:
        plan.close()


def test_strip_rejects_bad_tile_ilp():
    gen = GbmPathGenerator(Gbm(0.05, 0.2), 100.0, 1.0, 8)
    with pytest.raises(PricingError):
        price_strike_strip(gen, OptionType.Call, [100.0], 1000, 3, 1.0, tile_ilp=4)
