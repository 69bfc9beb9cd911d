"""Pins the CPU oracle against the reference's own known-answer tests.

The reference (Rust) cannot be built here, so the oracle (oracle/of_oracle.c)
is checked (1) against an independent pure-Python restatement of the same
reference source for the bit-level pieces (xoshiro256++, SplitMix64 seeding,
stream seeds, Acklam inverse, Hart CDF) and (2) against every statistical and
closed-form known answer the reference's tests hold for this path.
"""
import math

import numpy as np
import pytest
from scipy.special import ndtr

from conftest import load_golden
from openferric_b200._abi import (OF_AVG_ARITHMETIC, OF_AVG_GEOMETRIC, OF_CALL, OF_CV_GEOMETRIC_ASIAN, OF_CV_NONE,
                                  OF_CV_TERMINAL_SPOT, OF_CV_VANILLA_TERMINAL, OF_MODEL_GBM, OF_PAYOFF_ASIAN,
                                  OF_PAYOFF_BARRIER, OF_PAYOFF_VANILLA, OF_PUT, OfMcConfig, OfModel, OfPayoff)

M64 = (1 << 64) - 1

from openferric_b200.analytic import _fma as fma  # noqa: E402  (exact single-rounding fma)


# ---- independent pure-Python restatement (src/math/fast_rng.rs, fast_norm.rs) ----
def py_splitmix(state):
    state = (state + 0x9E3779B97F4A7C15) & M64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return state, z ^ (z >> 31)


class PyXoshiro:
    def __init__(self, seed):
        st, s = seed & M64, []
        for _ in range(4):
            st, z = py_splitmix(st)
            s.append(z)
        if not any(s):
            s[0] = 1
        self.s = s

    @staticmethod
    def rotl(x, k):
        return ((x << k) | (x >> (64 - k))) & M64

    def next_u64(self):
        s = self.s
        result = (self.rotl((s[0] + s[3]) & M64, 23) + s[0]) & M64
        t = (s[1] << 17) & M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = self.rotl(s[3], 45)
        return result

    def next_f64(self):
        return float(self.next_u64() >> 11) * (1.0 / 9007199254740992.0)


def py_acklam(p):
    A = [-3.969683028665376e1, 2.209460984245205e2, -2.759285104469687e2, 1.38357751867269e2,
         -3.066479806614716e1, 2.506628277459239]
    B = [-5.447609879822406e1, 1.615858368580409e2, -1.556989798598866e2, 6.680131188771972e1,
         -1.328068155288572e1]
    Cc = [-7.784894002430293e-3, -3.223964580411365e-1, -2.400758277161838, -2.549732539343734,
          4.374664141464968, 2.938163982698783]
    D = [7.784695709041462e-3, 3.224671290700398e-1, 2.445134137142996, 3.754408661907416]
    f = fma

    def tail(q):
        return f(f(f(f(f(Cc[0], q, Cc[1]), q, Cc[2]), q, Cc[3]), q, Cc[4]), q, Cc[5]) / \
            f(f(f(f(D[0], q, D[1]), q, D[2]), q, D[3]), q, 1.0)

    if p < 0.02425:
        return tail(math.sqrt(-2.0 * math.log(p)))
    if p <= 1.0 - 0.02425:
        q = p - 0.5
        r = q * q
        return f(f(f(f(f(A[0], r, A[1]), r, A[2]), r, A[3]), r, A[4]), r, A[5]) * q / \
            f(f(f(f(f(B[0], r, B[1]), r, B[2]), r, B[3]), r, B[4]), r, 1.0)
    return -tail(math.sqrt(-2.0 * math.log(1.0 - p)))


def py_open01(u):
    eps = 2.220446049250313e-16
    return eps if u < eps else (1.0 - eps if u > 1.0 - eps else u)


# ---- bit-level pieces ---------------------------------------------------------
@pytest.mark.parametrize("seed", [0, 1, 42, 7919, 2 ** 63 + 5, M64])
def test_xoshiro_matches_python_restatement(orc, seed):
    a, b = orc.Xoshiro(seed), PyXoshiro(seed)
    assert a.state() == b.s
    for _ in range(2000):
        assert a.next_u64() == b.next_u64()


class PyPcg64:
    """Pcg64 of fast_rng.rs:86-128 in Python integers: a second restatement
    that checks the C oracle's 128-bit arithmetic."""
    MUL = 0x2360ED051FC65DA44385DF649FCCF645
    M128 = (1 << 128) - 1

    def __init__(self, seed):
        st = seed & M64
        st, hi = py_splitmix(st)
        st, lo = py_splitmix(st)
        st, stream = py_splitmix(st)
        self.inc = ((stream << 1) | 1) & self.M128
        self.state = (hi << 64) | lo
        self.next_u64()

    def next_u64(self):
        old = self.state
        self.state = (old * self.MUL + self.inc) & self.M128
        x = ((old >> 64) ^ old) & M64
        rot = old >> 122
        return ((x >> rot) | (x << ((64 - rot) & 63))) & M64


@pytest.mark.parametrize("seed", [0, 1, 42, M64, 0x0123456789ABCDEF])
def test_pcg64_matches_python_restatement(orc, seed):
    a, b = orc.Pcg64(seed), PyPcg64(seed)
    for _ in range(2000):
        assert a.next_u64() == b.next_u64()


def test_mc_run_pcg64_draws_from_pcg_streams(orc):
    """FastRng::from_seed(Pcg64, stream_seed(seed, i)) per sample
    (simulation.rs:215-216): the oracle's MC on Pcg64 streams equals its MC on
    the same streams' normals injected, and differs from the xoshiro run."""
    import ctypes as C
    from openferric_b200 import _abi as A
    n, steps, seed = 64, 12, 9
    model = A.OfModel(kind=A.OF_MODEL_GBM, s0=100.0, mu=0.03, sigma=0.25, maturity=1.0, steps=steps)
    payoff = A.OfPayoff(kind=A.OF_PAYOFF_VANILLA, option_type=A.OF_CALL, strike=100.0)
    z = []
    for i in range(n):
        g = PyPcg64((seed + i * 7919) & M64)
        for _ in range(steps):
            u = float(g.next_u64() >> 11) * (1.0 / 9007199254740992.0)
            z.append(orc.acklam(min(max(u, 2.0 ** -52), 1.0 - 2.0 ** -52)))
    zz = np.array(z)
    pcg = orc.mc_run(model, payoff, A.OfMcConfig(num_paths=n, seed=seed, discount_factor=1.0,
                                                   rng_kind=A.OF_RNG_PCG64))
    inj = orc.mc_run(model, payoff, A.OfMcConfig(num_paths=n, seed=seed, discount_factor=1.0,
                                                   injected_normals=zz.ctypes.data_as(C.POINTER(C.c_double)),
                                                   n_injected=zz.size))
    xo = orc.mc_run(model, payoff, A.OfMcConfig(num_paths=n, seed=seed, discount_factor=1.0))
    assert pcg.price == inj.price and pcg.stderr_ == inj.stderr_
    assert pcg.price != xo.price


def test_xoshiro_reproducible_and_unit_interval(orc):
    # fast_rng.rs:250-277
    a, b = orc.Xoshiro(42), orc.Xoshiro(42)
    assert [a.next_u64() for _ in range(128)] == [b.next_u64() for _ in range(128)]
    r = orc.Xoshiro(1)
    for _ in range(1000):
        assert 0.0 <= r.next_f64() < 1.0


def test_stream_seed_wraps(orc):
    assert orc.lib().orc_stream_seed(M64, 3) == (M64 + 3 * 7919) & M64
    assert orc.lib().orc_stream_seed(42, 10) == 42 + 79190


def test_run_normals_follow_reference_draw_order(orc):
    """MonteCarloEngine::run draws z1[j], z2[j] interleaved per step, one stream per sample."""
    z = orc.run_normals(123, 3, 5, 2).reshape(3, 5, 2)
    for i in range(3):
        r = PyXoshiro((123 + i * 7919) & M64)
        for j in range(5):
            for k in range(2):
                assert z[i, j, k] == py_acklam(py_open01(r.next_f64()))


def test_acklam_bit_equal_to_python_restatement(orc):
    rng = np.random.default_rng(5)
    ps = np.concatenate([rng.random(20000), rng.random(2000) * 0.03, 1.0 - rng.random(2000) * 0.03,
                         [2.220446049250313e-16, 0.02425, 0.97575, 0.5, 1.0 - 2.220446049250313e-16]])
    for p in ps:
        assert orc.acklam(float(p)) == py_acklam(float(p))


def test_acklam_edge_values(orc):
    assert math.isnan(orc.acklam(float("nan")))
    assert math.isnan(orc.acklam(-0.1)) and math.isnan(orc.acklam(1.1))
    assert orc.acklam(0.0) == -math.inf and orc.acklam(1.0) == math.inf


# ---- fast_norm.rs:151-219 -----------------------------------------------------
def test_hart_cdf_matches_reference_table(orc):
    for x in (-8.0, -5.0, -4.0, -3.0, -2.0, -1.0, -0.5, 0.0, 0.5, 1.0, 2.0, 3.0, 4.0, 5.0, 8.0):
        assert abs(orc.hart_cdf(x) - float(ndtr(x))) < 1e-7


def test_hart_cdf_symmetry(orc):
    for i in range(81):
        x = i / 10.0
        assert abs(orc.hart_cdf(x) + orc.hart_cdf(-x) - 1.0) < 1e-12


def test_inverse_round_trips_cdf(orc):
    for i in range(1, 1000):
        p = i / 1000.0
        assert abs(orc.hart_cdf(orc.acklam(p)) - p) < 2e-7


def test_inverse_known_values(orc):
    assert abs(orc.acklam(0.5)) < 1e-10
    assert abs(orc.acklam(0.841344746068543) - 1.0) < 1e-6
    assert abs(orc.acklam(0.9772498680518208) - 2.0) < 1e-6


# ---- stochastic.rs:103-146, simulation.rs:352-463 ------------------------------
def test_gbm_path_generator_lengths_and_positivity(orc):
    m = OfModel(kind=OF_MODEL_GBM, s0=100.0, mu=0.05, sigma=0.2, maturity=1.0, steps=50)
    path = orc.generate_path(m, np.zeros(50))
    assert len(path) == 51 and np.all(path > 0)
    # zero-noise path grows by exp((mu - sigma^2/2) dt) per step
    assert abs(path[-1] - 100.0 * math.exp(0.03)) < 1e-10


def test_heston_path_generator(orc):
    m = OfModel(kind=1, s0=100.0, mu=0.03, maturity=1.0, steps=40, kappa=1.5, theta=0.04, xi=0.5, rho=-0.7, v0=0.04)
    path = orc.generate_path(m, np.full(40, 0.1), np.full(40, -0.2))
    assert len(path) == 41 and np.all(path > 0)


def _gbm(steps, s0=100.0, mu=0.05, sigma=0.2, T=1.0):
    return OfModel(kind=OF_MODEL_GBM, s0=s0, mu=mu, sigma=sigma, maturity=T, steps=steps)


def test_mc_call_within_two_stderr_of_bs(orc):
    # simulation.rs:397-421: 60k antithetic x 252, seed 42
    r = orc.mc_run(_gbm(252), OfPayoff(kind=OF_PAYOFF_VANILLA, option_type=OF_CALL, strike=100.0),
                   OfMcConfig(num_paths=60000, seed=42, antithetic=1, discount_factor=math.exp(-0.05)), threads=8)
    bs = orc.bs_price(OF_CALL, 100, 100, 0.05, 0, 0.2, 1.0)
    assert abs(r.price - bs) <= 2.0 * r.stderr_ + 2e-2


def test_dividend_paths_reproduce_the_schedule_forward(orc):
    """DiscreteDividendGbmPathGenerator (mc_engine.rs:123-175): the mean
    terminal spot is DividendSchedule::forward_price (dividends.rs:145-184)."""
    from openferric_b200 import DividendEvent, DividendSchedule
    from openferric_b200.engines import Gbm, GbmPathGenerator
    sched = DividendSchedule.new([DividendEvent.cash(0.25, 1.5), DividendEvent.proportional(0.5, 0.02),
                                  DividendEvent.cash(0.75, 2.0), DividendEvent.cash(1.5, 9.0)])
    gen = GbmPathGenerator(Gbm(0.04, 0.25), 100.0, 1.0, 64, sched)
    r = orc.mc_run(gen.to_abi(), OfPayoff(kind=OF_PAYOFF_VANILLA, option_type=OF_CALL, strike=1e-9),
                   OfMcConfig(num_paths=200000, seed=3, discount_factor=1.0), threads=8)
    fwd = sched.forward_price(100.0, 0.04, 0.0, 1.0)
    assert abs(r.price - fwd) <= 4.0 * r.stderr_
    # a path with a tiny vol lands on the deterministic jump sequence
    gen0 = GbmPathGenerator(Gbm(0.0, 1e-9), 100.0, 1.0, 8, sched)
    path = orc.generate_path(gen0.to_abi(), np.zeros(8))
    assert path[2] == pytest.approx(98.5, abs=1e-6)            # cash 1.5 after t = 0.25
    assert path[4] == pytest.approx(98.5 * 0.98, abs=1e-6)     # 2 % at t = 0.5
    assert path[6] == pytest.approx(98.5 * 0.98 - 2.0, abs=1e-6)
    assert path[8] == path[6]                                    # the t = 1.5 event is past maturity


def test_dividend_barrier_knock_in(orc):
    """dividend_modelling_issue58.rs:57-112 on the oracle: ~10 with the jump, ~0 without."""
    from openferric_b200 import DividendEvent, DividendSchedule
    from openferric_b200.engines import Gbm, GbmPathGenerator
    pay = OfPayoff(kind=OF_PAYOFF_BARRIER, option_type=OF_PUT, strike=100.0, barrier_direction=1, barrier_style=0,
                   barrier_level=95.0, rebate=0.0, expiry=1.0)
    cfg = OfMcConfig(num_paths=20000, seed=42, antithetic=1, discount_factor=1.0)
    with_div = GbmPathGenerator(Gbm(0.0, 1e-8), 100.0, 1.0, 252, DividendSchedule.new([DividendEvent.cash(0.5, 10.0)]))
    no_div = GbmPathGenerator(Gbm(0.0, 1e-8), 100.0, 1.0, 252)
    assert orc.mc_run(no_div.to_abi(), pay, cfg, threads=4).price <= 1e-3
    assert abs(orc.mc_run(with_div.to_abi(), pay, cfg, threads=4).price - 10.0) <= 1e-3


def test_control_variate_not_worse(orc):
    # simulation.rs:424-462
    m = _gbm(126)
    p = OfPayoff(kind=OF_PAYOFF_VANILLA, option_type=OF_CALL, strike=100.0)
    df = math.exp(-0.05)
    bs = orc.bs_price(OF_CALL, 100, 100, 0.05, 0, 0.2, 1.0)
    r0 = orc.mc_run(m, p, OfMcConfig(num_paths=20000, seed=123, discount_factor=df), threads=8)
    r1 = orc.mc_run(m, p, OfMcConfig(num_paths=20000, seed=123, discount_factor=df,
                                     control_variate=OF_CV_TERMINAL_SPOT, cv_expected=100.0 * math.exp(0.05)),
                    threads=8)
    assert abs(r1.price - bs) <= abs(r0.price - bs) + 0.15


# ---- mc_engine.rs:991-1167 ------------------------------------------------------
def test_mc_european_within_one_percent_of_bs(orc):
    r = orc.mc_run(_gbm(252), OfPayoff(kind=OF_PAYOFF_VANILLA, option_type=OF_CALL, strike=100.0),
                   OfMcConfig(num_paths=100000, seed=42, discount_factor=math.exp(-0.05)), threads=8)
    bs = orc.bs_price(OF_CALL, 100, 100, 0.05, 0, 0.2, 1.0)
    assert abs(r.price - bs) / bs <= 0.01


def test_antithetic_lower_stderr(orc):
    p = OfPayoff(kind=OF_PAYOFF_VANILLA, option_type=OF_CALL, strike=100.0)
    plain = orc.mc_run(_gbm(252), p, OfMcConfig(num_paths=100000, seed=42, discount_factor=math.exp(-0.05)), 8)
    anti = orc.mc_run(_gbm(252), p, OfMcConfig(num_paths=100000, seed=42, antithetic=1,
                                               discount_factor=math.exp(-0.05)), 8)
    assert anti.stderr_ < plain.stderr_


def test_control_variate_within_half_percent(orc):
    df = math.exp(-0.05)
    bs = orc.bs_price(OF_CALL, 100, 100, 0.05, 0, 0.2, 1.0)
    r = orc.mc_run(_gbm(252), OfPayoff(kind=OF_PAYOFF_VANILLA, option_type=OF_CALL, strike=100.0),
                   OfMcConfig(num_paths=100000, seed=42, discount_factor=df, control_variate=OF_CV_VANILLA_TERMINAL,
                              cv_expected=bs / df), 8)
    assert abs(r.price - bs) / bs <= 0.005


def test_geometric_asian_closed_form_about_5_31(orc):
    obs = [m / 11.0 for m in range(12)]
    assert abs(orc.geometric_asian(OF_CALL, 100, 100, 0.05, 0.0, 0.2, obs) - 5.31) <= 0.15


def _asian_payoff(obs, option_type=OF_CALL, strike=100.0, averaging=OF_AVG_ARITHMETIC, expiry=1.0):
    import ctypes as C
    arr = np.ascontiguousarray(obs, dtype=np.float64)
    p = OfPayoff(kind=OF_PAYOFF_ASIAN, option_type=option_type, strike=strike, averaging=averaging,
                 observation_times=arr.ctypes.data_as(C.POINTER(C.c_double)), n_observations=len(arr), expiry=expiry)
    return p, arr


def test_arithmetic_asian_within_two_percent_of_5_73(orc):
    obs = [m / 11.0 for m in range(12)]
    p, keep = _asian_payoff(obs)
    geo = orc.geometric_asian(OF_CALL, 100, 100, 0.05, 0.0, 0.2, obs)
    df = math.exp(-0.05)
    r = orc.mc_run(_gbm(252), p, OfMcConfig(num_paths=100000, seed=42, antithetic=1, discount_factor=df,
                                            control_variate=OF_CV_GEOMETRIC_ASIAN, cv_expected=geo / df), 8)
    assert abs(r.price - 5.73) / 5.73 <= 0.02


def test_seeded_runs_reproduce(orc):
    p = OfPayoff(kind=OF_PAYOFF_VANILLA, option_type=OF_CALL, strike=100.0)
    c = OfMcConfig(num_paths=20000, seed=123, discount_factor=math.exp(-0.05))
    a, b = orc.mc_run(_gbm(64), p, c), orc.mc_run(_gbm(64), p, c)
    assert a.price == b.price and a.stderr_ == b.stderr_


def test_parallel_fold_matches_sequential(orc):
    p = OfPayoff(kind=OF_PAYOFF_VANILLA, option_type=OF_PUT, strike=95.0)
    c = OfMcConfig(num_paths=9999, seed=9, antithetic=1, discount_factor=0.97)
    a, b = orc.mc_run(_gbm(33), p, c, 1), orc.mc_run(_gbm(33), p, c, 8)
    assert abs(a.price - b.price) <= 1e-12 * abs(a.price)


def test_asian_quantlib_cases4_within_two_stderr(orc):
    """tests/asian_quantlib.rs:185-256 on the 12-fixing case (MonteCarloPricingEngine 80k x 128, seed 42)."""
    cases = load_golden("asian_cases4.json")["cases"]
    case = next(c for c in cases if abs(c["first"] - 1.0 / 12.0) <= 1e-15 and c["fixings"] == 12)
    n = case["fixings"]
    dt = case["length"] / (n - 1)
    obs = [case["first"] + i * dt for i in range(n)]
    expiry = obs[-1]
    ot = OF_PUT if case["option_type"] == "Put" else OF_CALL
    p, keep = _asian_payoff(obs, ot, case["strike"], expiry=expiry)
    mu = case["risk_free_rate"] - case["dividend_yield"]
    m = OfModel(kind=OF_MODEL_GBM, s0=case["underlying"], mu=mu, sigma=case["volatility"], maturity=expiry, steps=128)
    df = math.exp(-case["risk_free_rate"] * expiry)
    fine = orc.mc_run(m, p, OfMcConfig(num_paths=80000, seed=42, discount_factor=df), 8)
    coarse = orc.mc_run(m, p, OfMcConfig(num_paths=20000, seed=42, discount_factor=df), 8)
    assert abs(fine.price - case["expected"]) <= 2.0 * fine.stderr_
    assert abs(fine.price - case["expected"]) <= abs(coarse.price - case["expected"]) + 5e-3


# ---- analytic oracles ---------------------------------------------------------
def test_heston_semi_analytic_matches_quantlib_lewis_table(orc):
    g = load_golden("heston_lewis.json")
    p = g["params"]
    rows = g["rows"]
    # First row: exact (the Lewis table's parameters); the reference checks the
    # first three rows with tolerance 1.0 (tests/heston_quantlib.rs:117-151).
    r0 = rows[0]
    c0 = orc.heston_call(p["spot"], r0["strike"], p["risk_free_rate"], p["dividend_rate"], p["maturity"], p["v0"],
                         p["kappa"], p["theta"], p["sigma_v"], p["rho"])
    assert abs(c0 - r0["call"]) < 1e-8
    for r in rows[:3]:
        c = orc.heston_call(p["spot"], r["strike"], p["risk_free_rate"], p["dividend_rate"], p["maturity"], p["v0"],
                            p["kappa"], p["theta"], p["sigma_v"], p["rho"])
        assert abs(c - r["call"]) <= 1.0


def test_heston_semi_analytic_matches_fang_oosterlee(orc):
    g = load_golden("fang_oosterlee.json")
    p = g["params"]
    for v in g["values"]:
        c = orc.heston_call(p["SPOT"], v["strike"], p["RATE"], p["DIVIDEND"], v["maturity"], p["V0"], p["KAPPA"],
                            p["THETA"], p["SIGMA_V"], p["RHO"])
        assert abs(c - v["reference"]) < min(v["tolerance"], 1e-6)


def test_heston_put_call_parity(orc):
    args = (100.0, 90.0, 0.03, 0.01, 1.5, 0.04, 2.0, 0.04, 0.5, -0.7)
    c, p = orc.heston_call(*args), orc.heston_put(*args)
    assert abs(c - p - (100 * math.exp(-0.015) - 90 * math.exp(-0.045))) < 1e-10


def test_heston_degenerates_to_black_scholes(orc):
    # xi -> 0 with v0 = theta: constant variance
    c = orc.heston_call(100, 105, 0.03, 0.0, 1.0, 0.04, 2.0, 0.04, 1e-4, 0.0)
    bs = 100 * ndtr((math.log(100 / 105) + (0.03 + 0.02)) / 0.2) - 105 * math.exp(-0.03) * ndtr(
        (math.log(100 / 105) + (0.03 - 0.02)) / 0.2)
    assert abs(c - bs) < 1e-5


def test_crr_american_put_converges(orc):
    a = orc.crr_american(OF_PUT, 36, 40, 0.06, 0.0, 0.2, 1.0, 2000)
    assert abs(a - 4.478) < 0.02  # Longstaff-Schwartz (2001) finite-difference value
    assert orc.crr_american(OF_CALL, 100, 100, 0.05, 0.0, 0.2, 1.0, 2000) == pytest.approx(
        orc.bs_price(OF_CALL, 100, 100, 0.05, 0, 0.2, 1.0), abs=5e-3)


# ---- LSM (tests/lsm_reference.rs:29-223, pricing/american.rs:141-173) -----------
def test_lsm_longstaff_schwartz_table1(orc):
    g = load_golden("lsm_table1.json")
    e = g["engine"]
    for c in g["cases"]:
        price, se = orc.lsm_price(OF_PUT, g["strike"], c["expiry"], 1, c["spot"], g["rate"], 0.0, c["sigma"],
                                  e["num_paths"], e["num_steps"], e["seed"])
        assert abs(price - c["expected"]) <= c["tolerance"], (c, price)


def test_lsm_degree3_agrees_with_degree2_and_crr(orc):
    crr = orc.crr_american(OF_PUT, 40, 40, 0.06, 0.0, 0.4, 1.0, 2000)
    p2, s2 = orc.lsm_price(OF_PUT, 40, 1.0, 1, 40, 0.06, 0.0, 0.4, 50000, 50, 7, degree=2)
    p3, s3 = orc.lsm_price(OF_PUT, 40, 1.0, 1, 40, 0.06, 0.0, 0.4, 50000, 50, 7, degree=3)
    assert abs(p2 - crr) < 0.1 and abs(p3 - crr) < 0.1
    assert abs(p3 - p2) < 4 * s2


def test_lsm_barrier_in_plus_out_is_the_european_on_the_same_stream(orc):
    """LongstaffSchwartzEngine::price(BarrierOption) (longstaff_schwartz.rs:632-736)
    draws the engine's single stream in the same path-major order as its
    vanilla pricing (:467-509): on one seed, knock-in + knock-out (no rebate)
    equals the European-exercise LSM price path by path, up to the discount
    exp(-rT) against disc^steps."""
    args = dict(spot=100.0, rate=0.05, q=0.0, vol=0.25, num_paths=20000, num_steps=50, seed=42)
    ko, _ = orc.lsm_barrier(OF_PUT, 105.0, 0.5, False, False, 90.0, 0.0, **args)
    ki, _ = orc.lsm_barrier(OF_PUT, 105.0, 0.5, False, True, 90.0, 0.0, **args)
    plain, _ = orc.lsm_price(OF_PUT, 105.0, 0.5, 0, **args)
    assert abs((ki + ko) - plain) <= 1e-12 * plain
    assert 0.0 < ko < plain and 0.0 < ki < plain
    # a rebate is paid on the inactive paths: in + out with rebate R = plain + R e^(-rT)
    kor, _ = orc.lsm_barrier(OF_PUT, 105.0, 0.5, False, False, 90.0, 2.0, **args)
    kir, _ = orc.lsm_barrier(OF_PUT, 105.0, 0.5, False, True, 90.0, 2.0, **args)
    assert abs((kir + kor) - (plain + 2.0 * math.exp(-0.05 * 0.5))) <= 1e-12 * plain


def test_lsm_european_exercise_is_discounted_payoff(orc):
    p, s = orc.lsm_price(OF_PUT, 40, 1.0, 0, 40, 0.06, 0.0, 0.2, 100000, 50, 3)
    bs = orc.bs_price(OF_PUT, 40, 40, 0.06, 0, 0.2, 1.0)
    assert abs(p - bs) < 3 * s + 1e-3


# ---- Sobol QMC (src/math/sobol.rs:128-188, mc_qmc.rs:152-199) --------------------
def test_sobol_points_unit_interval_and_reproducible(orc):
    p = orc.sobol_points(8, 42, 1000)
    assert p.min() >= 0.0 and p.max() < 1.0
    assert np.array_equal(orc.sobol_points(5, 99, 100), orc.sobol_points(5, 99, 100))


def test_sobol_first_dimension_is_van_der_corput_and_beats_prng_mean(orc):
    n = 1000
    p = orc.sobol_points(1, 7, n)[:, 0]
    sobol_mean = p.mean()
    rng = orc.Xoshiro(7)
    prng_mean = sum(rng.next_f64() for _ in range(n)) / n
    assert abs(sobol_mean - 0.5) <= abs(prng_mean - 0.5)
    v, scr = orc.sobol_dimension(0, 7)
    assert v == [1 << (63 - j) for j in range(64)]
    # point n of dimension 0 = gray(n) bit-reversed, XOR the scrambler
    for n in (1, 2, 3, 17, 1000):
        g = n ^ (n >> 1)
        x = 0
        for j in range(64):
            if (g >> j) & 1:
                x ^= v[j]
        assert p[n - 1] == fma(float(x ^ scr), 2.0 ** -64, 2.0 ** -65)


def test_sobol_direction_numbers_are_odd_and_bounded(orc):
    for dim in (1, 5, 200):
        v, _ = orc.sobol_dimension(dim, 123)
        for j, vj in enumerate(v):
            m = vj >> (63 - j)
            assert m & 1 and m < (1 << (j + 1))


def test_qmc_known_answers(orc):
    """mc_qmc.rs:178-198: 10k points (1 step, seed 11) within 0.1 % of BS;
    :160-176: at 50k the QMC stderr is no worse than 1.2 x the PRNG one."""
    bs = orc.bs_price(OF_CALL, 100, 100, 0.05, 0, 0.2, 1.0)
    p, _ = orc.mc_european_qmc(OF_CALL, 100.0, 100.0, 0.05, 0.0, 0.2, 1.0, 10000, 1, 11)
    assert abs(p - bs) / bs <= 0.001
    _, qse = orc.mc_european_qmc(OF_CALL, 100.0, 100.0, 0.05, 0.0, 0.2, 1.0, 50000, 1, 7)
    r = orc.mc_run(_gbm(1), OfPayoff(kind=OF_PAYOFF_VANILLA, option_type=OF_CALL, strike=100.0),
                   OfMcConfig(num_paths=50000, seed=7, discount_factor=math.exp(-0.05)), threads=8)
    assert qse < 1.2 * r.stderr_


def test_qmc_reference_edge_results(orc):
    assert all(math.isnan(x) for x in orc.mc_european_qmc(OF_CALL, 100, 100, 0.05, 0, 0.2, 1.0, 0, 10, 1))
    assert orc.mc_european_qmc(OF_PUT, 90, 100, 0.05, 0, 0.2, 0.0, 100, 10, 1) == (10.0, 0.0)
    assert all(math.isnan(x) for x in orc.mc_european_qmc(OF_CALL, 100, 100, 0.05, 0, -0.2, 1.0, 100, 10, 1))


# ---- Bermudan LSM (tests/bermudan_quantlib.rs:73-389) ----------------------------
def _schedule(c):
    s = [(t, c["strike"]) for t in c["dates"]]
    if c["expiry"] - s[-1][0] > 1e-12:
        s.append((c["expiry"], c["strike"]))
    return s


def test_bermudan_oracle_matches_quantlib_fd_puts(orc):
    """The reference's own check: LSM(450000 paths, 120 steps, seed 7) within
    0.5 % of the QuantLib FD price on every put case, with a populated boundary."""
    g = load_golden("bermudan_quantlib.json")
    e = g["lsm_engine"]
    puts = [c for c in g["cases"] if c["option_type"] == "Put"]
    assert len(puts) == 5
    for c in puts:
        p, se, recs = orc.lsm_bermudan(OF_PUT, c["expiry"], _schedule(c), c["spot"], c["rate"], c["dividend"],
                                       e["num_paths"], e["num_steps"], e["seed"], dynamics=0, vol=c["vol"])
        assert abs(p - c["quantlib_fd_price"]) / c["quantlib_fd_price"] <= g["rel_tolerance"], (c, p, se)
        assert any(r[2] is not None for r in recs)
        # chronological, terminal last: (expiry, K, K, itm, itm)
        assert [r[0] for r in recs] == sorted(r[0] for r in recs)
        assert recs[-1][0] == c["expiry"] and recs[-1][2] == c["strike"] and recs[-1][3] == recs[-1][4]
        for t, k, b, itm, ex in recs[:-1]:
            assert ex <= itm
            if b is not None:
                assert b < k  # a put is exercised below the strike


def test_bermudan_oracle_step_down_strike_is_cheaper(orc):
    dates = [0.25, 0.5, 0.75, 1.0]
    step = orc.lsm_bermudan(OF_PUT, 1.0, list(zip(dates, [100.0, 97.5, 95.0, 92.5])), 100.0, 0.03, 0.0, 60000, 100,
                            42, vol=0.25)
    const = orc.lsm_bermudan(OF_PUT, 1.0, [(t, 100.0) for t in dates], 100.0, 0.03, 0.0, 60000, 100, 42, vol=0.25)
    assert step[0] < const[0]
    assert [r[1] for r in step[2]] == [100.0, 97.5, 95.0, 92.5]


def test_bermudan_oracle_local_vol_and_heston_dynamics(orc):
    """bermudan_quantlib.rs:268-335 at reduced path counts: finite positive
    prices and a populated boundary under both dynamics; a flat local-vol grid
    and a zero vol-of-vol Heston reproduce the GBM price on the same draws'
    distribution within a few SE."""
    from openferric_b200.market import Market
    sched = [(t, 100.0) for t in (0.2, 0.4, 0.6, 0.8, 1.0)]

    def smile(k, t):
        return max(0.18 + 0.08 * abs(k / 100.0 - 1.0) + 0.03 * math.sqrt(max(t, 1e-6)), 0.05)

    m = Market.builder().spot(100).rate(0.02).dividend_yield(0.01).vol_surface(smile).build()
    lv = m.vol.grid()
    p, se, recs = orc.lsm_bermudan(OF_PUT, 1.0, sched, 100.0, 0.02, 0.01, 20000, 90, 123, dynamics=1, lv=lv)
    assert math.isfinite(p) and p > 0 and any(r[2] is not None for r in recs)
    p, se, recs = orc.lsm_bermudan(OF_PUT, 1.0, sched, 100.0, 0.02, 0.01, 20000, 100, 321, dynamics=2,
                                   heston=(2.0, 0.04, 0.6, -0.5, 0.04))
    assert math.isfinite(p) and p > 0 and any(r[2] is not None for r in recs)
    flat = (np.ones(1), np.ones(1), np.full((1, 1), 0.2))
    g = orc.lsm_bermudan(OF_PUT, 1.0, sched, 100.0, 0.02, 0.01, 40000, 50, 5, dynamics=0, vol=0.2)
    l = orc.lsm_bermudan(OF_PUT, 1.0, sched, 100.0, 0.02, 0.01, 40000, 50, 5, dynamics=1, lv=flat)
    h = orc.lsm_bermudan(OF_PUT, 1.0, sched, 100.0, 0.02, 0.01, 40000, 50, 6, dynamics=2,
                         heston=(1.0, 0.04, 0.0, 0.0, 0.04))
    assert abs(g[0] - l[0]) < 1e-9  # same single stream, same GBM arithmetic up to the 1e-12 floor
    assert abs(g[0] - h[0]) < 4 * math.hypot(g[1], h[1])


def test_sampled_vol_matches_python_mirror(orc):
    from openferric_b200.market import Market

    def smile(k, t):
        return 0.2 + 0.1 * (k / 100.0 - 1.0) ** 2 + 0.02 * t

    m = Market.builder().spot(100).vol_surface(smile).build()
    K, T, V = m.vol.grid()
    rng = np.random.default_rng(3)
    for k, t in zip(rng.uniform(10, 300, 500), rng.uniform(0, 15, 500)):
        assert orc.sampled_vol(K, T, V, k, t) == m.vol_for(k, t)
    for k in K:  # grid points take the lower interval with weight 1, as the linear scan does
        for t in T:
            assert orc.sampled_vol(K, T, V, k, t) == m.vol_for(k, t)


# ---- mc_aad.rs:344-480, mc_greeks.rs:344-419 ------------------------------------
def test_pathwise_aad_recovers_bs_greeks(orc):
    g = orc.gbm_pathwise_aad(OF_CALL, 100.0, 100.0, 0.03, 0.01, 0.2, 1.0, 120000, 64, 42, True)
    ref = orc.bs_greeks(OF_CALL, 100.0, 100.0, 0.03, 0.01, 0.2, 1.0)
    assert abs(g["delta"] - ref["delta"]) < 6e-3
    assert abs(g["vega"] - ref["vega"]) < 8e-2
    assert abs(g["rho"] - ref["rho"]) < 7e-2
    assert abs(g["theta"] - ref["theta"]) < 9e-2


def test_heston_delta_matches_crn_bump(orc):
    kw = dict(mu=0.03, kappa=1.8, theta=0.04, xi=0.6, rho=-0.5, v0=0.04, num_paths=60000, num_steps=64, seed=7)
    _, d = orc.heston_price_delta(OF_CALL, 70.0, 1.0, 100.0, 0.03, **kw)
    up, _ = orc.heston_price_delta(OF_CALL, 70.0, 1.0, 100.0 + 1e-3, 0.03, **kw)
    dn, _ = orc.heston_price_delta(OF_CALL, 70.0, 1.0, 100.0 - 1e-3, 0.03, **kw)
    assert abs(d - (up - dn) / 2e-3) < 1e-4


def test_mc_greek_estimators_reference_values(orc):
    g = orc.mc_greek_estimators(OF_CALL, 100.0, 100.0, 0.05, 0.0, 0.2, 1.0, 100000, 42)
    d1 = (0.05 + 0.02) / 0.2
    assert abs(g["pathwise_delta"] - ndtr(d1)) / ndtr(d1) <= 0.02
    vega = 100 * math.exp(-0.5 * d1 * d1) / math.sqrt(2 * math.pi)
    assert abs(g["lr_vega"] - vega) / vega <= 0.05
    assert abs(g["pathwise_delta"] - 0.6368) / 0.6368 < 0.02
    assert abs(g["pathwise_gamma"] - 0.01876) / 0.01876 < 0.20
    assert abs(g["lr_vega"] - 37.524) / 37.524 < 0.05


def test_philox_known_answer(orc):
    # Random123 known-answer vector for Philox4x32-10, counter 0 / key 0.
    assert orc.philox4x32_10([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]


def test_wgsl_restatement_prices_near_bs(orc):
    p, s = orc.wgsl_european(100.0, 100.0, 0.05, 0.2, 1.0, 200000, 64, 7, True)
    bs = orc.bs_price(OF_CALL, 100, 100, 0.05, 0, 0.2, 1.0)
    assert abs(p - bs) < 4 * s + 0.02
