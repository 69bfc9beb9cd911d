"""GPU Sobol QMC (of_mc_european_qmc) against the oracle's restatement of
mc_european_qmc_with_seed (mc_qmc.rs:39-150) and the reference's QMC tests."""
import math

import pytest

import openferric_b200 as of
from openferric_b200 import OptionType, Precision, PricingError, VanillaOption
from openferric_b200.analytic import bs_price
from openferric_b200.qmc import mc_european_qmc, mc_european_qmc_with_seed

pytestmark = pytest.mark.gpu


def _market(spot=100.0, r=0.05, q=0.0, vol=0.2):
    return of.Market.builder().spot(spot).rate(r).dividend_yield(q).flat_vol(vol).build()


@pytest.mark.parametrize("opt", [OptionType.Call, OptionType.Put])
@pytest.mark.parametrize("paths,steps,seed", [(10000, 1, 11), (4097, 64, 3), (20000, 252, 0), (777, 5, 2 ** 63 + 9)])
def test_fp64_matches_oracle(orc, opt, paths, steps, seed):
    inst = VanillaOption.european_call(100.0, 1.0) if opt is OptionType.Call else VanillaOption.european_put(100.0, 1.0)
    m = _market(q=0.01)
    g = mc_european_qmc_with_seed(inst, m, paths, steps, seed)
    p, se = orc.mc_european_qmc(opt.value, 100.0, 100.0, 0.05, 0.01, 0.2, 1.0, paths, steps, seed)
    assert abs(g.price - p) <= 1e-12 * max(1.0, abs(p)), (g.price, p)
    assert abs(g.stderr - se) <= 1e-9 * se + 1e-15
    assert g.diagnostics.get("num_steps") == float(steps)


def test_fp32_mode_walks_the_same_points(orc):
    inst = VanillaOption.european_call(100.0, 1.0)
    m = _market()
    for paths, steps in ((1 << 16, 32), (100_003, 128)):
        a = mc_european_qmc_with_seed(inst, m, paths, steps, 5)
        b = mc_european_qmc_with_seed(inst, m, paths, steps, 5, precision=Precision.Fp32Philox)
        # same points, FP32 normals on the top 23 bits: differences far below the stderr
        assert abs(a.price - b.price) <= 0.05 * a.stderr, (a.price, b.price, a.stderr)


def test_reference_known_answers():
    """mc_qmc.rs:178-198 and :160-176."""
    inst = VanillaOption.european_call(100.0, 1.0)
    m = _market()
    q = mc_european_qmc_with_seed(inst, m, 10_000, 1, 11)
    bs = bs_price(OptionType.Call, 100.0, 100.0, 0.05, 0.0, 0.2, 1.0)
    assert abs(q.price - bs) / bs <= 0.001
    qmc = mc_european_qmc_with_seed(inst, m, 50_000, 1, 7)
    mc = of.MonteCarloPricingEngine(50_000, 1, 7).price(inst, m)
    assert qmc.stderr < 1.2 * mc.stderr


def test_large_point_set_converges_to_black_scholes():
    inst = VanillaOption.european_put(105.0, 2.0)
    m = _market(r=0.03, q=0.01, vol=0.3)
    bs = bs_price(OptionType.Put, 100.0, 105.0, 0.03, 0.01, 0.3, 2.0)
    for prec in (Precision.Fp64Reference, Precision.Fp32Philox):
        q = mc_european_qmc_with_seed(inst, m, 1 << 22, 64, 1, precision=prec)
        assert abs(q.price - bs) <= 3.0 * q.stderr + 0.02  # time-discretisation-free for GBM terminal payoffs


def test_reference_edge_results_and_validation():
    inst = VanillaOption.european_call(100.0, 1.0)
    assert math.isnan(mc_european_qmc(inst, _market(), 0, 10).price)
    assert mc_european_qmc(inst, _market(), 0, 10).stderr is None
    assert mc_european_qmc(VanillaOption.european_put(100.0, 0.0), _market(spot=90.0), 100, 10).price == 10.0
    assert math.isnan(mc_european_qmc(VanillaOption.american_put(100.0, 1.0), _market(), 100, 10).price)
    with pytest.raises(PricingError):
        mc_european_qmc(inst, _market(), 100, 30000)
