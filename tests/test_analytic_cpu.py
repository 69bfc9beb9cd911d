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
