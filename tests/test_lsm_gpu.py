"""GPU Longstaff-Schwartz (of_lsm_price) against the oracle's restatement of
LongstaffSchwartzEngine::price and the CRR binomial tree.

FP64 reference mode draws the reference's single sequential xoshiro256++
stream (device GF(2) jump-ahead), so the price equals the oracle's to
1e-12 relative.  FP32 Philox mode with the cubic basis is checked against a
2000-step binomial tree."""
import math

import numpy as np
import pytest

from conftest import load_golden
from openferric_b200 import ExerciseStyle, Market, OptionType, Precision, PricingError, VanillaOption
from openferric_b200 import _abi as A
from openferric_b200.lsm import LongstaffSchwartzEngine, xoshiro_jump_states

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


def test_device_jump_ahead_matches_sequential_stream(orc):
    draws = [0, 1, 2, 63, 64, 65, 1000, 12345, 200_003]
    states = xoshiro_jump_states(42, draws)
    x = orc.Xoshiro(42)
    done = 0
    for d, st in zip(draws, states):
        while done < d:
            x.next_u64()
            done += 1
        assert st == x.state(), d


@pytest.mark.parametrize("case", [
    (OptionType.Put, ExerciseStyle.American, 36.0, 0.2, 1.0),
    (OptionType.Put, ExerciseStyle.American, 44.0, 0.4, 2.0),
    (OptionType.Call, ExerciseStyle.American, 40.0, 0.3, 1.0),
    (OptionType.Put, ExerciseStyle.European, 40.0, 0.2, 1.0),
    (OptionType.Put, ExerciseStyle.bermudan([0.25, 0.5, 0.75, 1.0]), 38.0, 0.25, 1.0),
])
def test_fp64_reference_stream_matches_oracle(orc, case):
    ot, ex, s0, vol, T = case
    m = Market.builder().spot(s0).rate(0.06).dividend_yield(0.01).flat_vol(vol).build()
    opt = VanillaOption(ot, 40.0, T, ex)
    gpu = LongstaffSchwartzEngine(20_003, 20, 42).price(opt, m)
    exercise = 0 if ex.is_european else (1 if ex.is_american else 2)
    dates = list(ex.dates) if ex.is_bermudan else None
    p, s = orc.lsm_price(ot.value, 40.0, T, exercise, s0, 0.06, 0.01, vol, 20_003, 20, 42, dates=dates)
    assert rel(gpu.price, p) < 1e-12, (gpu.price, p)
    assert rel(gpu.stderr, s) < 1e-10
    assert gpu.diagnostics.get("num_steps") == 20.0


def test_injected_normals_match_oracle(orc):
    m = Market.builder().spot(38.0).rate(0.06).flat_vol(0.3).build()
    opt = VanillaOption.american_put(40.0, 1.0)
    z = np.random.default_rng(3).standard_normal(4001 * 12)
    gpu = LongstaffSchwartzEngine(4001, 12, 0).with_injected_normals(z).price(opt, m)
    p, _ = orc.lsm_price(A.OF_PUT, 40.0, 1.0, 1, 38.0, 0.06, 0.0, 0.3, 4001, 12, 0, normals=z)
    assert rel(gpu.price, p) < 1e-12


def test_cubic_basis_fp64_matches_oracle(orc):
    m = Market.builder().spot(40.0).rate(0.06).flat_vol(0.4).build()
    opt = VanillaOption.american_put(40.0, 1.0)
    gpu = LongstaffSchwartzEngine(30_000, 25, 5).with_basis_degree(3).price(opt, m)
    p, _ = orc.lsm_price(A.OF_PUT, 40.0, 1.0, 1, 40.0, 0.06, 0.0, 0.4, 30_000, 25, 5, degree=3)
    assert rel(gpu.price, p) < 1e-11


def test_longstaff_schwartz_table1_on_gpu(orc):
    """tests/lsm_reference.rs:29-223 through the GPU engine, and run-for-run equal to the oracle."""
    g = load_golden("lsm_table1.json")
    e = g["engine"]
    eng = LongstaffSchwartzEngine(e["num_paths"], e["num_steps"], e["seed"])
    items = []
    for c in g["cases"]:
        m = Market.builder().spot(c["spot"]).rate(g["rate"]).flat_vol(c["sigma"]).build()
        items.append((VanillaOption.american_put(g["strike"], c["expiry"]), m))
    res = eng.price_batch(items)
    for c, r in zip(g["cases"], res):
        assert abs(r.price - c["expected"]) <= c["tolerance"], (c, r.price)
    c0 = g["cases"][0]
    p, _ = orc.lsm_price(A.OF_PUT, g["strike"], c0["expiry"], 1, c0["spot"], g["rate"], 0.0, c0["sigma"],
                         e["num_paths"], e["num_steps"], e["seed"])
    assert rel(res[0].price, p) < 1e-12


def test_fp32_cubic_basis_against_binomial(orc):
    eng = LongstaffSchwartzEngine(1 << 20, 50, 7).with_precision(Precision.Fp32Philox).with_basis_degree(3)
    cases = [(36.0, 0.2, 1.0), (40.0, 0.4, 1.0), (44.0, 0.2, 2.0)]
    items = []
    for s0, vol, T in cases:
        m = Market.builder().spot(s0).rate(0.06).flat_vol(vol).build()
        items.append((VanillaOption.american_put(40.0, T), m))
    res = eng.price_batch(items, with_delta=True)
    for (s0, vol, T), r in zip(cases, res):
        crr = orc.crr_american(A.OF_PUT, s0, 40.0, 0.06, 0.0, vol, T, 2000)
        # LSM is biased low by the sub-optimal fitted policy and the 50/yr grid
        assert crr - 0.06 - 4 * r.stderr <= r.price <= crr + 4 * r.stderr, (s0, vol, T, r.price, crr, r.stderr)
        h = 0.05
        crr_delta = (orc.crr_american(A.OF_PUT, s0 + h, 40.0, 0.06, 0.0, vol, T, 2000) -
                     orc.crr_american(A.OF_PUT, s0 - h, 40.0, 0.06, 0.0, vol, T, 2000)) / (2 * h)
        assert abs(r.greeks.delta - crr_delta) < 0.03, (r.greeks.delta, crr_delta)


def test_fp32_and_fp64_modes_agree_statistically(orc):
    m = Market.builder().spot(40.0).rate(0.06).flat_vol(0.2).build()
    opt = VanillaOption.american_put(40.0, 1.0)
    a = LongstaffSchwartzEngine(1 << 18, 50, 1).with_precision(Precision.Fp32Philox).price(opt, m)
    b = LongstaffSchwartzEngine(1 << 18, 50, 2).price(opt, m)
    assert abs(a.price - b.price) <= 4 * math.hypot(a.stderr, b.stderr) + 0.01


def test_fp32_flag_row_delta_agrees_with_fp64_payment_steps():
    """The FP32 mode takes each path's payment step from per-date exercise
    flag rows, the FP64 mode from a per-path array: on independent draws the
    two deltas agree statistically, for a put and a call, with padding paths
    (n not a multiple of the 1024-path chunk) and a batch of two contracts."""
    n = (1 << 18) + 333
    items = [(VanillaOption.american_put(40.0, 1.0), Market.builder().spot(38.0).rate(0.06).flat_vol(0.3).build()),
             (VanillaOption.american_call(40.0, 1.0),
              Market.builder().spot(42.0).rate(0.03).dividend_yield(0.08).flat_vol(0.3).build())]
    d32 = LongstaffSchwartzEngine(n, 50, 3).with_precision(Precision.Fp32Philox).price_batch(items, with_delta=True)
    d64 = LongstaffSchwartzEngine(n, 50, 4).price_batch(items, with_delta=True)
    for a, b in zip(d32, d64):
        # delta per path is bounded by S_tau/S0 (~1.5); its SE at n paths is below 2e-3
        assert abs(a.greeks.delta - b.greeks.delta) < 0.01, (a.greeks.delta, b.greeks.delta)
        assert abs(a.price - b.price) <= 4 * math.hypot(a.stderr, b.stderr) + 0.01
    assert d32[0].greeks.delta < -0.3 and d32[1].greeks.delta > 0.3


def test_lsm_validation_messages():
    m = Market.builder().spot(40.0).rate(0.06).flat_vol(0.2).build()
    with pytest.raises(PricingError, match="num_steps must be >= 2 for Longstaff-Schwartz"):
        LongstaffSchwartzEngine(100, 1, 1).price(VanillaOption.american_put(40, 1), m)
    with pytest.raises(PricingError, match="num_paths must be >= 3 for Longstaff-Schwartz"):
        LongstaffSchwartzEngine(2, 10, 1).price(VanillaOption.american_put(40, 1), m)
    r = LongstaffSchwartzEngine(100, 10, 1).price(VanillaOption.american_put(40, 0.0), m)
    assert r.price == 0.0 and r.stderr == 0.0


def test_fp32_batches_do_not_change_the_draws():
    """Each contract draws from its own Philox stream (its index in the list),
    whatever batch it lands in: batches of 1, 2 and the automatic sizes price
    the same paths.  The FP32 moment sums group the chunks by block, and the
    blocks per contract follow the batch size, so the fitted betas move by
    about the FP32 rounding of the moments, flip exercise decisions near the
    boundary, and the flips propagate through the later regressions: measured
    up to 0.07 standard errors at 2^17 paths.  Independent draws would differ
    by about 1.4 standard errors (rms)."""
    items = []
    for i, (s0, vol) in enumerate([(36.0, 0.2), (40.0, 0.4), (44.0, 0.2), (38.0, 0.3), (42.0, 0.25)]):
        m = Market.builder().spot(s0).rate(0.06).flat_vol(vol).build()
        items.append((VanillaOption.american_put(40.0, 1.0), m))
    runs = []
    for b in (0, 1, 2):
        eng = LongstaffSchwartzEngine(1 << 17, 50, 11).with_precision(Precision.Fp32Philox) \
            .with_basis_degree(3).with_batch_contracts(b)
        runs.append(eng.price_batch(items, with_delta=True))
    for k in range(len(items)):
        ref = runs[0][k]
        for other in runs[1:]:
            r = other[k]
            assert abs(r.price - ref.price) <= 0.25 * ref.stderr, (k, r.price, ref.price, ref.stderr)
            assert abs(r.stderr - ref.stderr) <= 0.01 * ref.stderr, (k, r.stderr, ref.stderr)
