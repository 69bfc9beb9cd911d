"""Heston pathwise adjoint (of_heston_price_adjoint): every sensitivity against
central bump-and-revalue with common random numbers (same seed, forward-only
kernel), the price against the semi-analytic Heston value, and the
torch.autograd.Function wrapper."""
import math

import pytest

from openferric_b200 import AsianOption, AsianSpec, Averaging, Heston, Market, OptionType, StrikeType, VanillaOption
from openferric_b200 import _abi as A
from openferric_b200.adjoint import HestonAdjointFunction, HestonAdjointSpec, heston_adjoint, price_with_adjoint

pytestmark = pytest.mark.gpu

BASE = dict(spot=100.0, rate=0.03, v0=0.04, kappa=2.0, theta=0.04, xi=0.5, rho=-0.7)


def crn_fd(spec, name, rel_bump=1e-4):
    """Central difference with common random numbers: the FP64 price-only pass
    on the same Philox draws (forward_only=2)."""
    p = dict(BASE)
    h = rel_bump * abs(p[name])
    up, dn = dict(p), dict(p)
    up[name] += h
    dn[name] -= h
    pu = heston_adjoint(spec, forward_only=2, **up).price
    pd = heston_adjoint(spec, forward_only=2, **dn).price
    return (pu - pd) / (2 * h)


@pytest.mark.parametrize("asian", [True, False])
def test_adjoint_greeks_match_crn_central_differences(asian):
    """2^20 paths: the pathwise derivative and the central difference differ
    only on the paths that cross the payoff's kink or the smoothed branch
    switch within the bump, a Monte Carlo average that shrinks as paths^-1/2
    (rho, the smallest relative sensitivity here, sat at 8e-4 of the 1e-3 bar
    with 2^18 paths)."""
    spec = HestonAdjointSpec(strike=100.0, expiry=2.0 if asian else 1.0, num_paths=1 << 20,
                             num_steps=512 if asian else 256, seed=7, asian=asian)
    res = heston_adjoint(spec, **BASE)
    fwd = heston_adjoint(spec, forward_only=1, **BASE)
    fwd64 = heston_adjoint(spec, forward_only=2, **BASE)
    assert res.price == fwd.price  # the adjoint run prices the same paths
    assert abs(fwd64.price - res.price) <= 1e-4 * abs(res.price)  # FP32 path error
    for name in A.OF_ADJ_NAMES:
        fd = crn_fd(spec, name)
        adj = res.greeks[name]
        # same draws, smoothed branch switch: the pathwise derivative and the central
        # difference of the same expectation agree to FP32 path precision
        assert abs(adj - fd) <= max(1e-3 * abs(fd), 2e-4), (name, adj, fd, abs(adj - fd) / abs(fd),
                                                             res.greeks_stderr[name])


def test_adjoint_european_price_near_semi_analytic(orc):
    spec = HestonAdjointSpec(strike=100.0, expiry=1.0, num_paths=1 << 20, num_steps=256, seed=3, asian=False)
    res = heston_adjoint(spec, **BASE)
    exact = orc.heston_call(100.0, 100.0, 0.03, 0.0, 1.0, 0.04, 2.0, 0.04, 0.5, -0.7)
    assert abs(res.price - exact) <= 4 * res.stderr + 0.01


def test_adjoint_delta_against_heston_semi_analytic_bump(orc):
    spec = HestonAdjointSpec(strike=100.0, expiry=1.0, num_paths=1 << 20, num_steps=256, seed=5, asian=False)
    res = heston_adjoint(spec, **BASE)
    h = 0.01
    exact = (orc.heston_call(100.0 + h, 100.0, 0.03, 0.0, 1.0, 0.04, 2.0, 0.04, 0.5, -0.7) -
             orc.heston_call(100.0 - h, 100.0, 0.03, 0.0, 1.0, 0.04, 2.0, 0.04, 0.5, -0.7)) / (2 * h)
    assert abs(res.greeks["spot"] - exact) <= 4 * res.greeks_stderr["spot"] + 2e-3


@pytest.mark.parametrize("option_type,strike", [(OptionType.Call, 100.0), (OptionType.Put, 95.0)])
def test_adjoint_delta_against_the_reference_heston_delta(option_type, strike):
    """The QE adjoint's delta against the reference's own Heston delta,
    heston_price_delta_aad (src/engines/monte_carlo/mc_aad.rs:239-342:
    forward-mode Euler on the reference streams, FP64): independent
    estimators of the same sensitivity from two discretisations at 256 steps.
    The reference returns a plain mean; its standard error is the adjoint's
    per-path spread at the reference's path count.  2e-3 covers the two
    schemes' discretisation biases."""
    from openferric_b200.greeks import HestonAadConfig, heston_price_delta_aad
    n_adj, n_ref, steps = 1 << 20, 1 << 18, 256
    spec = HestonAdjointSpec(strike=strike, expiry=1.0, num_paths=n_adj, num_steps=steps, seed=9, asian=False,
                             option_type=option_type)
    res = heston_adjoint(spec, **BASE)
    model = Heston(mu=BASE["rate"], kappa=BASE["kappa"], theta=BASE["theta"], xi=BASE["xi"], rho=BASE["rho"],
                   v0=BASE["v0"])
    price_ref, delta_ref = heston_price_delta_aad(option_type, strike, 1.0, BASE["spot"], BASE["rate"], model,
                                                  HestonAadConfig(n_ref, steps, 42))
    se = res.greeks_stderr["spot"] * math.sqrt(1.0 + n_adj / n_ref)
    assert abs(res.greeks["spot"] - delta_ref) <= 4.0 * se + 2e-3, (res.greeks["spot"], delta_ref, se)
    se_p = res.stderr * math.sqrt(1.0 + n_adj / n_ref)
    assert abs(res.price - price_ref) <= 4.0 * se_p + 0.01


def test_price_with_adjoint_instrument_api():
    m = Market.builder().spot(100.0).rate(0.03).flat_vol(0.2).build()
    h = Heston(0.03, 2.0, 0.04, 0.5, -0.7, 0.04)
    steps = 64
    obs = [2.0 * j / steps for j in range(1, steps + 1)]
    opt = AsianOption(OptionType.Call, 100.0, 2.0, AsianSpec(Averaging.Arithmetic, StrikeType.Fixed, obs))
    r = price_with_adjoint(opt, m, h, 1 << 16, steps, 11)
    spec = HestonAdjointSpec(strike=100.0, expiry=2.0, num_paths=1 << 16, num_steps=steps, seed=11, asian=True)
    r2 = heston_adjoint(spec, **BASE)
    assert r.price == r2.price and r.greeks == r2.greeks
    rv = price_with_adjoint(VanillaOption.european_put(95.0, 1.0), m, h, 1 << 16, 64, 11)
    assert rv.greeks["spot"] < 0.0 and rv.price > 0.0


def test_autograd_function_backward_returns_adjoint_greeks():
    import torch
    spec = HestonAdjointSpec(strike=100.0, expiry=1.0, num_paths=1 << 16, num_steps=64, seed=1, asian=True)
    params = torch.tensor([BASE[n] for n in A.OF_ADJ_NAMES], dtype=torch.float64, requires_grad=True)
    price = HestonAdjointFunction.apply(params, spec)
    price.backward()
    ref = heston_adjoint(spec, **BASE)
    assert abs(price.item() - ref.price) == 0.0
    for k, name in enumerate(A.OF_ADJ_NAMES):
        assert params.grad[k].item() == pytest.approx(ref.greeks[name], rel=1e-12, abs=1e-15)


def test_hard_switch_band_zero_is_andersen_qe():
    """band = 0 is Andersen's hard switch: the price agrees with the smoothed
    scheme to well within a standard error (the band only touches steps with
    psi within 0.05 of psi_c)."""
    hard = HestonAdjointSpec(strike=100.0, expiry=1.0, num_paths=1 << 18, num_steps=128, seed=2, asian=True,
                             qe_switch_band=0.0)
    soft = HestonAdjointSpec(strike=100.0, expiry=1.0, num_paths=1 << 18, num_steps=128, seed=2, asian=True)
    a = heston_adjoint(hard, forward_only=1, **BASE)
    b = heston_adjoint(soft, forward_only=1, **BASE)
    assert abs(a.price - b.price) <= 0.5 * a.stderr
