"""Full-size workloads of the benchmark configurations, checked through
properties that do not depend on the path count:

- the 4096-option batched book (2.31e11 path-steps): each European call within
  5 standard errors of Black-Scholes; each daily-fixing arithmetic Asian call
  between the discrete geometric Asian closed form (AM >= GM on every path)
  and the European call (convex order for r >= 0); each up-and-out call below
  the European call (its payoff is smaller on every path);
- LSM in FP32 with the cubic basis at 2^20 paths and 50 dates a year: the
  Longstaff-Schwartz Table 1 known answers (tests/lsm_reference.rs, through
  the golden fixture), and, for the benchmark's 256 American puts, the bounds
  European <= LSM <= CRR American (the fitted policy is sub-optimal) and
  -1 <= delta <= 0;
- the Heston QE Asian adjoint at 2^20 paths x 512 steps: all seven Greeks
  against central bump-and-revalue with common random numbers."""
import math

import numpy as np
import pytest

from conftest import load_golden
from openferric_b200 import AsianOption, BarrierOption, Market, OptionType, Precision, VanillaOption
from openferric_b200 import _abi as A
from openferric_b200.analytic import bs_price, geometric_asian_cov_sum_sorted, hart_norm_cdf
from openferric_b200.book import price_book, synthetic_book
from openferric_b200.lsm import LongstaffSchwartzEngine

pytestmark = pytest.mark.gpu


def _geometric_asian_call(s0, k, r, sigma, obs):
    """Discrete geometric-average Asian call (the closed form of
    analytic.geometric_asian_discrete_fixed, q = 0) with the O(n log n)
    covariance sum, for fixing schedules of up to 1260 dates."""
    n = float(len(obs))
    var = sigma * sigma * geometric_asian_cov_sum_sorted(obs) / (n * n)
    m = math.log(s0) + (r - 0.5 * sigma * sigma) * (sum(obs) / n)
    sv = math.sqrt(var)
    d1 = (m - math.log(k) + var) / sv
    return math.exp(-r * max(obs)) * (math.exp(m + 0.5 * var) * hart_norm_cdf(d1) - k * hart_norm_cdf(d1 - sv))


def test_full_book_size_independent_bounds():
    book = synthetic_book()
    res = price_book(book, seed=20261203)
    kinds = {VanillaOption: 0, AsianOption: 0, BarrierOption: 0}
    for e, r in zip(book, res):
        inst, m = e.instrument, e.market
        assert math.isfinite(r.price) and r.price >= 0.0 and r.stderr >= 0.0
        vol = m.vol_for(m.spot, inst.expiry)
        bs = bs_price(OptionType.Call, m.spot, inst.strike, m.rate, 0.0, vol, inst.expiry)
        tol = 5.0 * r.stderr + 1e-4 * m.spot
        kinds[type(inst)] += 1
        if isinstance(inst, VanillaOption):
            assert abs(r.price - bs) <= tol, (inst, r.price, bs, r.stderr)
        elif isinstance(inst, AsianOption):
            geo = _geometric_asian_call(m.spot, inst.strike, m.rate, vol, inst.asian.observation_times)
            assert geo - tol <= r.price <= bs + tol, (inst.strike, r.price, geo, bs, r.stderr)
        else:
            assert r.price <= bs + tol, (inst.strike, r.price, bs, r.stderr)
    assert kinds == {VanillaOption: 1366, AsianOption: 1365, BarrierOption: 1365}


def test_full_size_fp32_lsm_reproduces_table1():
    g = load_golden("lsm_table1.json")
    by_t = {}
    for c in g["cases"]:
        m = Market.builder().spot(c["spot"]).rate(g["rate"]).flat_vol(c["sigma"]).build()
        by_t.setdefault(c["expiry"], []).append((c, VanillaOption.american_put(g["strike"], c["expiry"]), m))
    for T, group in by_t.items():
        eng = LongstaffSchwartzEngine(1 << 20, int(50 * T), 42).with_precision(Precision.Fp32Philox) \
            .with_basis_degree(3)
        res = eng.price_batch([(inst, m) for _, inst, m in group])
        for (c, _, _), r in zip(group, res):
            assert abs(r.price - c["expected"]) <= c["tolerance"], (c, r.price)


def test_full_lsm_workload_bounds(orc):
    """The benchmark's 256 American puts (S0 ~ U[30, 50], K = 40, r = 0.06,
    sigma in {0.2, 0.4}, T in {1, 2}, 2^20 paths, 50 dates a year)."""
    rng = np.random.default_rng(20261203)
    items = []
    for i in range(256):
        vol, T = (0.2, 0.4)[i % 2], (1.0, 2.0)[(i // 2) % 2]
        m = Market.builder().spot(rng.uniform(30.0, 50.0)).rate(0.06).flat_vol(vol).build()
        items.append((VanillaOption.american_put(40.0, T), m))
    for T in (1.0, 2.0):
        sub = [it for it in items if it[0].expiry == T]
        eng = LongstaffSchwartzEngine(1 << 20, int(50 * T), 42).with_precision(Precision.Fp32Philox) \
            .with_basis_degree(3)
        res = eng.price_batch(sub, with_delta=True)
        for (inst, m), r in zip(sub, res):
            vol = m.vol_for(40.0, T)
            euro = bs_price(OptionType.Put, m.spot, 40.0, 0.06, 0.0, vol, T)
            crr = orc.crr_american(A.OF_PUT, m.spot, 40.0, 0.06, 0.0, vol, T, 1000)
            tol = 5.0 * r.stderr + 2e-3
            assert euro - tol <= r.price <= crr + tol, (m.spot, vol, T, euro, r.price, crr, r.stderr)
            assert -1.0 <= r.greeks.delta <= 0.0, (m.spot, vol, T, r.greeks.delta)


def test_full_size_adjoint_matches_crn_bumps():
    from openferric_b200.adjoint import HestonAdjointSpec, heston_adjoint
    base = dict(spot=100.0, rate=0.03, v0=0.04, kappa=2.0, theta=0.04, xi=0.5, rho=-0.7)
    spec = HestonAdjointSpec(strike=100.0, expiry=2.0, num_paths=1 << 20, num_steps=512, seed=7, asian=True)
    res = heston_adjoint(spec, **base)
    assert res.stderr <= 1e-4 * base["spot"]  # the SE target of the priced+Greeks metric
    for name in A.OF_ADJ_NAMES:
        h = 1e-4 * abs(base[name])
        up, dn = dict(base), dict(base)
        up[name] += h
        dn[name] -= h
        fd = (heston_adjoint(spec, forward_only=2, **up).price - heston_adjoint(spec, forward_only=2, **dn).price) \
            / (2 * h)
        assert abs(res.greeks[name] - fd) <= max(1e-3 * abs(fd), 2e-4), (name, res.greeks[name], fd)
