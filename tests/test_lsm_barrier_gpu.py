"""LongstaffSchwartzEngine::price(BarrierOption) on the GPU (of_lsm_barrier)
against the oracle's restatement of src/engines/lsm/longstaff_schwartz.rs:632-736
(the engine's single xoshiro256++ stream, reproduced on the device by GF(2)
jump-ahead), and the reference's own barrier tests
(tests/lsm_reference.rs:466-582)."""
import math

import numpy as np
import pytest

from openferric_b200 import (BarrierDirection, BarrierOption, BarrierSpec, BarrierStyle, Market, OptionType,
                             PricingError, VanillaOption)
from openferric_b200 import _abi as A
from openferric_b200.engines import Precision
from openferric_b200.lsm import LongstaffSchwartzEngine

pytestmark = pytest.mark.gpu

CASES = [  # option type, direction, style, strike, barrier, rebate, expiry
    (OptionType.Call, BarrierDirection.Up, BarrierStyle.Out, 100.0, 130.0, 0.0, 1.0),
    (OptionType.Call, BarrierDirection.Up, BarrierStyle.In, 95.0, 120.0, 1.5, 0.75),
    (OptionType.Put, BarrierDirection.Down, BarrierStyle.Out, 105.0, 90.0, 0.0, 0.5),
    (OptionType.Put, BarrierDirection.Down, BarrierStyle.In, 105.0, 90.0, 0.7, 0.5),
    (OptionType.Put, BarrierDirection.Up, BarrierStyle.Out, 100.0, 101.0, 0.0, 1.0),  # barrier near the spot
    (OptionType.Call, BarrierDirection.Down, BarrierStyle.Out, 100.0, 100.0, 2.0, 1.0),  # knocked at path[0]
]


def _barrier(c):
    ot, d, st, k, b, r, T = c
    return BarrierOption(ot, k, T, BarrierSpec(d, st, b, r))


@pytest.mark.parametrize("case", CASES)
def test_lsm_barrier_matches_oracle_on_the_reference_stream(orc, case):
    m = Market.builder().spot(100.0).rate(0.04).dividend_yield(0.01).flat_vol(0.3).build()
    inst = _barrier(case)
    paths, steps, seed = 20011, 40, 7
    got = LongstaffSchwartzEngine(paths, steps, seed).price(inst, m)
    ot, d, st, k, b, r, T = case
    ref_p, ref_s = orc.lsm_barrier(ot.value, k, T, d is BarrierDirection.Up, st is BarrierStyle.In, b, r, 100.0,
                                   0.04, 0.01, 0.3, paths, steps, seed)
    assert abs(got.price - ref_p) <= 1e-12 * max(abs(ref_p), 1e-300), (got.price, ref_p)
    # a payoff that is the same on every path (knocked out at the spot) has a
    # variance that is a cancellation residue of order 1e-16 x the mean squared
    assert abs(got.stderr - ref_s) <= 1e-10 * ref_s + 1e-7 * abs(ref_p)
    assert got.diagnostics.get("num_paths") == paths and got.diagnostics.get("vol") == 0.3


def test_lsm_barrier_injected_normals_match_oracle(orc):
    rng = np.random.default_rng(3)
    z = rng.standard_normal((512, 16))
    m = Market.builder().spot(100.0).rate(0.02).flat_vol(0.25).build()
    case = CASES[1]
    got = LongstaffSchwartzEngine(512, 16, 1).with_injected_normals(z).price(_barrier(case), m)
    ot, d, st, k, b, r, T = case
    ref_p, _ = orc.lsm_barrier(ot.value, k, T, True, True, b, r, 100.0, 0.02, 0.0, 0.25, 512, 16, 1, normals=z)
    assert abs(got.price - ref_p) <= 1e-12 * abs(ref_p)


def test_lsm_barrier_knockin_plus_knockout_approx_plain():
    """tests/lsm_reference.rs:517-582 at the reference's settings (100k paths,
    50 steps, seed 42); on one stream the sum equals the European exactly."""
    m = Market.builder().spot(100.0).rate(0.05).flat_vol(0.25).build()
    eng = LongstaffSchwartzEngine(100_000, 50, 42)
    ko = eng.price(BarrierOption(OptionType.Put, 105.0, 0.5,
                                 BarrierSpec(BarrierDirection.Down, BarrierStyle.Out, 90.0, 0.0)), m).price
    ki = eng.price(BarrierOption(OptionType.Put, 105.0, 0.5,
                                 BarrierSpec(BarrierDirection.Down, BarrierStyle.In, 90.0, 0.0)), m).price
    plain = eng.price(VanillaOption.european_put(105.0, 0.5), m).price
    assert abs(ki + ko - plain) <= 0.50
    assert abs(ki + ko - plain) <= 1e-11 * plain


def test_lsm_barrier_knockout_leq_plain_american():
    """tests/lsm_reference.rs:466-511 (100k paths, 50 steps, seed 42)."""
    m = Market.builder().spot(100.0).rate(0.05).flat_vol(0.25).build()
    eng = LongstaffSchwartzEngine(100_000, 50, 42)
    vanilla = eng.price(VanillaOption.american_put(100.0, 1.0), m).price
    barrier = eng.price(BarrierOption(OptionType.Put, 100.0, 1.0,
                                      BarrierSpec(BarrierDirection.Down, BarrierStyle.Out, 80.0, 0.0)), m).price
    assert barrier <= vanilla + 0.15


def test_lsm_barrier_rejects_fp32_and_bad_input():
    m = Market.builder().spot(100.0).rate(0.05).flat_vol(0.25).build()
    inst = _barrier(CASES[0])
    with pytest.raises(PricingError):
        LongstaffSchwartzEngine(1000, 10, 1).with_precision(Precision.Fp32Philox).price(inst, m)
    with pytest.raises(PricingError, match="num_steps must be > 0"):
        LongstaffSchwartzEngine(1000, 0, 1).price(inst, m)
    with pytest.raises(PricingError, match="num_paths must be > 0"):
        LongstaffSchwartzEngine(0, 10, 1).price(inst, m)
