"""Host closed forms the control variates need (no GPU)."""
import random

from openferric_b200.analytic import geometric_asian_cov_sum_sorted, min_sum_in_order


def _double_loop(obs):
    # sum_i sum_j min(t_i, t_j), i outer, j inner (src/pricing/asian.rs:86-136)
    total = 0.0
    for ti in obs:
        for tj in obs:
            total += min(ti, tj)
    return total


def test_min_sum_in_order_is_bit_identical_to_the_double_loop():
    rng = random.Random(11)
    for n in (0, 1, 2, 3, 255, 256, 257, 600):
        for sort in (True, False):
            obs = [rng.uniform(0.0, 5.0) for _ in range(n)]
            if sort:
                obs.sort()
            assert min_sum_in_order(obs) == _double_loop(obs), (n, sort)
    daily = [2.0 * j / 504 for j in range(1, 505)]
    assert min_sum_in_order(daily) == _double_loop(daily)
    # the sorted O(n log n) form agrees up to summation order
    assert abs(geometric_asian_cov_sum_sorted(daily) - _double_loop(daily)) <= 1e-12 * _double_loop(daily)


def test_exact_fma_is_correctly_rounded():
    """_fma_exact (the reference's f64::mul_add on Pythons without math.fma)
    against exact rational arithmetic: cancellations, signed zeros,
    subnormal results and wide exponent ranges."""
    import math
    from fractions import Fraction

    from openferric_b200.analytic import _fma_exact
    rng = random.Random(3)

    def rnd(e):
        return rng.uniform(-1.0, 1.0) * 10.0 ** rng.randint(-e, e) if e else rng.uniform(-2.0, 2.0)

    checked = 0
    for _ in range(20000):
        e = rng.choice([0, 1, 5, 30, 150])
        a, b = rnd(e), rnd(e)
        c = rng.choice([-a * b, a * b * (1.0 + 1e-15), rnd(e), 0.0, -0.0, 5e-324, math.ldexp(3.0, -1074)])
        exact = float(Fraction(a) * Fraction(b) + Fraction(c))
        got = _fma_exact(a, b, c)
        assert got == exact and math.copysign(1.0, got) == math.copysign(1.0, exact), (a, b, c, got, exact)
        checked += 1
    assert checked == 20000
    assert _fma_exact(0.1, 10.0, -1.0) == 5.551115123125783e-17  # the product's rounding error, kept
    assert math.isnan(_fma_exact(math.inf, 0.0, 1.0))
