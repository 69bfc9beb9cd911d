"""GPU parity of the generic Monte Carlo path (of_mc_run) against the oracle.

FP64 reference mode: the device draws openferric's own streams, so prices
must equal the oracle's to 1e-12 relative (standard errors to 1e-10: they are
differences of sums).  FP32 Philox mode: independent draws, so prices must
agree within a few combined standard errors."""
import ctypes as C
import math

import numpy as np
import pytest

from openferric_b200 import (ArithmeticAsianMC, AsianOption, AsianSpec, Averaging, BarrierDirection, BarrierOption,
                             BarrierSpec, BarrierStyle, ControlVariate, ControlVariateKind, Gbm, GbmPathGenerator,
                             Heston, HestonPathGenerator, Market, MonteCarloEngine, MonteCarloPricingEngine,
                             OptionType, Precision, PricingError, StrikeType, VanillaOption, VarianceReduction)
from openferric_b200 import _abi as A
from openferric_b200.analytic import bs_price

pytestmark = pytest.mark.gpu

PRICE_RTOL = 1e-12
SE_RTOL = 1e-10


def close(a, b, rtol):
    return abs(a - b) <= rtol * max(abs(a), abs(b), 1e-300) or abs(a - b) <= 1e-300


def se_close(a, b, rtol, price):
    """Standard errors agree, or both are zero variance.  With a control
    variate identical to the payoff the adjusted variance is a difference of
    sums that cancels to rounding level (the reference returns NaN, 0 or a
    few 1e-9 there, depending on summation order): any NaN or value below
    1e-7 of the price on both sides is the same zero variance."""
    zero = 1e-7 * max(1.0, abs(price))
    za = math.isnan(a) or abs(a) <= zero
    zb = math.isnan(b) or abs(b) <= zero
    if za or zb:
        return za and zb
    return close(a, b, rtol)


def _market(spot=100.0, r=0.05, q=0.0, vol=0.2):
    return Market.builder().spot(spot).rate(r).dividend_yield(q).flat_vol(vol).build()


def _oracle_run(orc, gen, instrument, anti, cv, df, num_paths, seed, injected=None, rng_kind=A.OF_RNG_XOSHIRO256PP):
    from openferric_b200.engines import _payoff_abi
    payoff, keep = _payoff_abi(instrument)
    cfg = A.OfMcConfig(num_paths=num_paths, seed=seed, antithetic=int(anti), discount_factor=df, rng_kind=rng_kind)
    if cv is not None:
        cfg.control_variate = cv.kind.value
        cfg.cv_expected = cv.expected
    if injected is not None:
        cfg.injected_normals = injected.ctypes.data_as(C.POINTER(C.c_double))
        cfg.n_injected = injected.size
    r = orc.mc_run(gen.to_abi(), payoff, cfg, threads=8)
    del keep
    return r


def _instruments(expiry):
    obs = [expiry * k / 10 for k in range(1, 11)]
    return {
        "call": VanillaOption.european_call(100.0, expiry),
        "put": VanillaOption.european_put(105.0, expiry),
        "up_out_call": BarrierOption(OptionType.Call, 100.0, expiry,
                                     BarrierSpec(BarrierDirection.Up, BarrierStyle.Out, 125.0, 1.5)),
        "down_in_put": BarrierOption(OptionType.Put, 100.0, expiry,
                                     BarrierSpec(BarrierDirection.Down, BarrierStyle.In, 85.0, 0.0)),
        "asian_arith_call": AsianOption(OptionType.Call, 100.0, expiry,
                                        AsianSpec(Averaging.Arithmetic, StrikeType.Fixed, obs)),
        "asian_geo_put": AsianOption(OptionType.Put, 100.0, expiry,
                                     AsianSpec(Averaging.Geometric, StrikeType.Fixed, obs)),
        "asian_floating_call": AsianOption(OptionType.Call, 100.0, expiry,
                                           AsianSpec(Averaging.Arithmetic, StrikeType.Floating, obs)),
    }


GENS = {
    "gbm": lambda T, n: GbmPathGenerator(Gbm(0.03, 0.25), 100.0, T, n),
    "heston": lambda T, n: HestonPathGenerator(Heston(0.03, 2.0, 0.04, 0.5, -0.7, 0.04), 100.0, T, n),
}


def _cv_for(name, inst, gen):
    if name in ("call", "put"):
        return ControlVariate(10.0, ControlVariateKind.VanillaTerminal)
    if name == "asian_arith_call":
        return ControlVariate(5.0, ControlVariateKind.GeometricAsian)
    return ControlVariate(103.0, ControlVariateKind.TerminalSpot)


@pytest.mark.parametrize("model", ["gbm", "heston"])
@pytest.mark.parametrize("name", list(_instruments(1.0).keys()))
@pytest.mark.parametrize("anti", [False, True])
@pytest.mark.parametrize("use_cv", [False, True])
def test_fp64_reference_mode_matches_oracle(orc, model, name, anti, use_cv):
    T, steps, paths, seed = 1.0, 24, 3001, 1234
    gen = GENS[model](T, steps)
    inst = _instruments(T)[name]
    cv = _cv_for(name, inst, gen) if use_cv else None
    df = math.exp(-0.03 * T)
    eng = MonteCarloEngine(paths, seed).with_antithetic(anti)
    if cv is not None:
        eng.with_control_variate(cv)
    gpu = eng.run_full(gen, inst, df)
    ref = _oracle_run(orc, gen, inst, anti, cv, df, paths, seed)
    assert gpu.samples == ref.samples
    assert close(gpu.price, ref.price, PRICE_RTOL), (gpu.price, ref.price)
    assert se_close(gpu.stderr_, ref.stderr_, SE_RTOL, ref.price), (gpu.stderr_, ref.stderr_)
    for f in ("sum_x", "sum_x2", "sum_y", "sum_xy", "sum_y2"):
        assert close(getattr(gpu, f), getattr(ref, f), 1e-12), f


@pytest.mark.parametrize("model", ["gbm", "heston"])
def test_injected_normals_path_matches_oracle(orc, model):
    """The test hook: the oracle's normals injected into both engines."""
    T, steps, paths, seed = 0.75, 17, 777, 99
    gen = GENS[model](T, steps)
    inst = _instruments(T)["up_out_call"]
    streams = gen.num_normal_streams()
    z = orc.run_normals(seed, paths, steps, streams)
    gpu = MonteCarloEngine(paths, seed).with_injected_normals(z).run_full(gen, inst, 0.97)
    ref = _oracle_run(orc, gen, inst, False, None, 0.97, paths, seed, injected=z)
    own = MonteCarloEngine(paths, seed).run_full(gen, inst, 0.97)
    assert close(gpu.price, ref.price, PRICE_RTOL)
    assert close(gpu.price, own.price, PRICE_RTOL)
    # perturb one normal: the result must move (the hook is really used)
    z2 = z.copy()
    z2[0] += 3.0
    moved = MonteCarloEngine(paths, seed).with_injected_normals(z2).run_full(gen, inst, 0.97)
    assert moved.price != gpu.price


def test_injected_normals_too_short_is_invalid_input():
    gen = GENS["gbm"](1.0, 10)
    with pytest.raises(PricingError) as e:
        MonteCarloEngine(100, 1).with_injected_normals(np.zeros(999)).run(gen, VanillaOption.european_call(100, 1), 1)
    assert e.value.kind == "InvalidInput"


def test_odd_path_count_and_single_sample(orc):
    gen = GENS["gbm"](1.0, 8)
    inst = _instruments(1.0)["call"]
    for n, anti in ((1, False), (1, True), (2, True), (3, True), (5, False)):
        gpu = MonteCarloEngine(n, 3).with_antithetic(anti).run_full(gen, inst, 1.0)
        ref = _oracle_run(orc, gen, inst, anti, None, 1.0, n, 3)
        assert gpu.samples == ref.samples
        assert close(gpu.price, ref.price, PRICE_RTOL)
        assert gpu.stderr_ == ref.stderr_ or close(gpu.stderr_, ref.stderr_, SE_RTOL)


@pytest.mark.parametrize("model", ["gbm", "heston"])
@pytest.mark.parametrize("anti", [False, True])
@pytest.mark.parametrize("name", ["asian_arith_call", "put"])
def test_fp64_pcg64_streams_match_oracle(orc, model, anti, name):
    """with_rng_kind(FastRngKind::Pcg64): every sample draws from
    Pcg64::seed_from_u64(stream_seed(seed, i)) (fast_rng.rs:86-128,
    simulation.rs:215-216); the FP64 engine equals the oracle's restatement,
    and the xoshiro run of the same seed differs."""
    from openferric_b200.engines import FastRngKind
    T, steps, paths, seed = 1.0, 24, 3001, 1234
    gen = GENS[model](T, steps)
    inst = _instruments(T)[name]  # a GBM put takes the two-lanes-per-sample kernel
    gpu = MonteCarloEngine(paths, seed).with_antithetic(anti).with_rng_kind(FastRngKind.Pcg64).run_full(gen, inst, 0.97)
    ref = _oracle_run(orc, gen, inst, anti, None, 0.97, paths, seed, rng_kind=A.OF_RNG_PCG64)
    xo = MonteCarloEngine(paths, seed).with_antithetic(anti).run_full(gen, inst, 0.97)
    assert close(gpu.price, ref.price, PRICE_RTOL), (gpu.price, ref.price)
    assert se_close(gpu.stderr_, ref.stderr_, SE_RTOL, ref.price)
    assert gpu.price != xo.price


def test_pcg64_is_rejected_in_fp32_mode_and_thread_rng_everywhere():
    from openferric_b200.engines import FastRngKind, Precision
    gen = GENS["gbm"](1.0, 8)
    inst = _instruments(1.0)["call"]
    with pytest.raises(PricingError, match="Philox streams only"):
        MonteCarloEngine(1000, 1).with_rng_kind(FastRngKind.Pcg64).with_precision(Precision.Fp32Philox) \
            .run_full(gen, inst, 1.0)
    with pytest.raises(PricingError, match="Xoshiro256PlusPlus and Pcg64"):
        MonteCarloEngine(1000, 1).with_rng_kind(FastRngKind.ThreadRng).run_full(gen, inst, 1.0)


def test_large_seed_wraps_like_reference(orc):
    gen = GENS["gbm"](1.0, 12)
    inst = _instruments(1.0)["put"]
    seed = 2 ** 64 - 3
    gpu = MonteCarloEngine(5000, seed).run_full(gen, inst, 1.0)
    ref = _oracle_run(orc, gen, inst, False, None, 1.0, 5000, seed)
    assert close(gpu.price, ref.price, PRICE_RTOL)


# ---- the reference's own MonteCarloPricingEngine tests, on the GPU -------------
def test_gpu_mc_european_within_one_percent_of_bs(orc):
    """mc_engine.rs:998-1021, and the FP64 run equals the oracle run."""
    m = _market()
    opt = VanillaOption.european_call(100.0, 1.0)
    res = MonteCarloPricingEngine(100_000, 252, 42).price(opt, m)
    bs = bs_price(OptionType.Call, 100, 100, 0.05, 0.0, 0.2, 1.0)
    assert abs(res.price - bs) / bs <= 0.01
    ref = _oracle_run(orc, GbmPathGenerator(Gbm(0.05, 0.2), 100.0, 1.0, 252), opt, False, None, math.exp(-0.05),
                      100_000, 42)
    assert close(res.price, ref.price, PRICE_RTOL)
    assert res.diagnostics.get("num_paths") == 100_000.0 and res.diagnostics.get("vol") == 0.2


def test_gpu_antithetic_lower_stderr():
    m = _market()
    opt = VanillaOption.european_call(100.0, 1.0)
    plain = MonteCarloPricingEngine(100_000, 252, 42).price(opt, m)
    anti = MonteCarloPricingEngine(100_000, 252, 42).with_variance_reduction(VarianceReduction.Antithetic).price(opt, m)
    assert anti.stderr < plain.stderr


def test_gpu_control_variate_within_half_percent():
    m = _market()
    opt = VanillaOption.european_call(100.0, 1.0)
    res = MonteCarloPricingEngine(100_000, 252, 42).with_variance_reduction(VarianceReduction.ControlVariate).price(
        opt, m)
    bs = bs_price(OptionType.Call, 100, 100, 0.05, 0.0, 0.2, 1.0)
    assert abs(res.price - bs) / bs <= 0.005


def test_gpu_arithmetic_asian_within_two_percent():
    m = _market()
    obs = [k / 11.0 for k in range(12)]
    opt = AsianOption(OptionType.Call, 100.0, 1.0, AsianSpec(Averaging.Arithmetic, StrikeType.Fixed, obs))
    res = ArithmeticAsianMC(100_000, 252, 42).with_control_variate(True).price(opt, m)
    assert abs(res.price - 5.73) / 5.73 <= 0.02


def test_gpu_seeded_runs_are_bit_reproducible():
    m = _market()
    opt = VanillaOption.european_call(100.0, 1.0)
    a = MonteCarloPricingEngine(20_000, 64, 123).price(opt, m)
    b = MonteCarloPricingEngine(20_000, 64, 123).price(opt, m)
    assert a.price == b.price and a.stderr == b.stderr


def test_gpu_maturity_zero_returns_intrinsic():
    m = _market(spot=110)
    res = MonteCarloPricingEngine(1000, 10, 1).price(VanillaOption.european_call(100.0, 0.0), m)
    assert res.price == 10.0 and res.stderr == 0.0


def test_validation_messages_match_reference():
    m = _market()
    with pytest.raises(PricingError, match="num_paths must be > 0"):
        MonteCarloPricingEngine(0, 10, 1).price(VanillaOption.european_call(100, 1), m)
    with pytest.raises(PricingError, match="num_steps must be > 0"):
        MonteCarloPricingEngine(10, 0, 1).price(VanillaOption.european_call(100, 1), m)
    with pytest.raises(PricingError, match="vanilla strike must be > 0"):
        MonteCarloPricingEngine(10, 10, 1).price(VanillaOption.european_call(-1, 1), m)


# ---- FP32 Philox mode: statistical parity ---------------------------------------
@pytest.mark.parametrize("name", ["call", "put", "up_out_call", "down_in_put", "asian_arith_call", "asian_geo_put",
                                  "asian_floating_call"])
@pytest.mark.parametrize("model", ["gbm", "heston"])
def test_fp32_mode_agrees_with_oracle_within_4_se(orc, name, model):
    T, steps = 1.0, 64
    gen = GENS[model](T, steps)
    inst = _instruments(T)[name]
    df = math.exp(-0.03 * T)
    gpu = MonteCarloEngine(1 << 18, 11).with_antithetic(True).with_precision(Precision.Fp32Philox).run_full(
        gen, inst, df)
    ref = _oracle_run(orc, gen, inst, True, None, df, 1 << 16, 5)
    se = math.hypot(gpu.stderr_, ref.stderr_)
    assert abs(gpu.price - ref.price) <= 4.0 * se + 1e-4 * 100.0, (gpu.price, ref.price, se)


def test_fp32_mode_control_variate_tightens_error():
    m = _market()
    opt = VanillaOption.european_call(100.0, 1.0)
    e = MonteCarloPricingEngine(1 << 20, 64, 7).with_precision(Precision.Fp32Philox)
    plain = e.price(opt, m)
    cv = MonteCarloPricingEngine(1 << 20, 64, 7).with_precision(Precision.Fp32Philox).with_variance_reduction(
        VarianceReduction.ControlVariate).price(opt, m)
    bs = bs_price(OptionType.Call, 100, 100, 0.05, 0.0, 0.2, 1.0)
    assert cv.stderr < 0.5 * plain.stderr
    assert abs(plain.price - bs) <= 4 * plain.stderr
    assert abs(cv.price - bs) <= 4 * cv.stderr + 2e-3


def test_fp32_mode_is_deterministic():
    m = _market()
    opt = VanillaOption.european_put(100.0, 1.0)
    e = MonteCarloPricingEngine(1 << 16, 32, 9).with_precision(Precision.Fp32Philox)
    assert e.price(opt, m).price == e.price(opt, m).price


def test_fp32_qe_scheme_prices_near_semi_analytic(orc):
    h = Heston(0.03, 2.0, 0.04, 0.5, -0.7, 0.04)
    gen = HestonPathGenerator(h, 100.0, 1.0, 128, scheme="qe")
    df = math.exp(-0.03)
    r = MonteCarloEngine(1 << 20, 3).with_antithetic(True).with_precision(Precision.Fp32Philox).run_full(
        gen, VanillaOption.european_call(100.0, 1.0), df)
    exact = orc.heston_call(100.0, 100.0, 0.03, 0.0, 1.0, 0.04, 2.0, 0.04, 0.5, -0.7)
    assert abs(r.price - exact) <= 4 * r.stderr_ + 0.01, (r.price, exact, r.stderr_)


def test_qe_has_no_fp64_reference_mode():
    gen = HestonPathGenerator(Heston(0.03, 2.0, 0.04, 0.5, -0.7, 0.04), 100.0, 1.0, 8, scheme="qe")
    with pytest.raises(PricingError):
        MonteCarloEngine(100, 1).run(gen, VanillaOption.european_call(100, 1), 1.0)


def test_device_peak_probes_are_plausible():
    """The roofline denominators: MUFU results/s and FP32 flops/s of a B200
    (148 SMs, <= 2.1 GHz: nominal 16 MUFU and 256 FP32 flops per clock per SM)."""
    from openferric_b200._lib import context
    p = context(0).device_peaks()
    assert 1e12 < p["sfu_ops_per_s"] < 148 * 16 * 2.1e9 * 1.05
    assert 2e13 < p["fp32_flops_per_s"] < 148 * 256 * 2.1e9 * 1.05
    assert p["probe_ms"] > 0.0
