"""The CPU restatement of the book's Greeks mode (oracle/book_oracle.py), checked
on its own before it checks the GPU: its Philox draws against the C oracle's
Philox4x32-10 (pinned to the Random123 known-answer vector in test_oracle.py),
and its pathwise Greeks against central differences of its own prices on the
same draws."""
import numpy as np
import pytest

from oracle.book_oracle import GreekOption, book_greeks, philox4x32_10


def test_vectorised_philox_matches_the_c_oracle(orc):
    rng = np.random.default_rng(5)
    for _ in range(20):
        ctr = [int(x) for x in rng.integers(0, 2 ** 32, 4)]
        seed = int(rng.integers(0, 2 ** 63))
        got = [int(v) for v in philox4x32_10(*ctr, seed)]
        ref = orc.philox4x32_10(ctr, [seed & 0xFFFFFFFF, seed >> 32])
        assert got == list(ref)


def _opts():
    daily = [0.0] + [1.0] * 24
    monthly = [0.0] * 25
    for k in range(0, 25, 4):
        monthly[k] += 1.0
    base = dict(s0=100.0, r=0.03, q=0.01, sigma=0.3, T=1.25, steps=24, stream=3)
    return [
        GreekOption("vanilla", True, strike=105.0, **base),
        GreekOption("vanilla", False, strike=95.0, antithetic=True, **base),
        GreekOption("asian", True, strike=100.0, weights=daily, **base),
        GreekOption("asian", False, strike=102.0, weights=monthly, antithetic=True, **base),
        GreekOption("asian", True, strike=98.0, weights=daily, geometric=True, **base),
        GreekOption("asian", True, strike=1.0, weights=monthly, floating=True, **base),
        GreekOption("barrier", True, strike=100.0, up=True, barrier=135.0, **base),
        GreekOption("barrier", False, strike=100.0, up=False, barrier=75.0, rebate=1.5, antithetic=True, **base),
        GreekOption("barrier", True, strike=100.0, up=True, knock_in=True, barrier=125.0, rebate=0.5, **base),
        GreekOption("barrier", False, strike=100.0, up=False, knock_in=True, barrier=85.0, **base),
    ]


@pytest.mark.parametrize("k", range(10))
def test_oracle_greeks_are_the_derivatives_of_its_prices(k):
    o = _opts()[k]
    n, seed, h = 4096, 11, 1e-5
    price, g = book_greeks(o, n, seed)
    for t, name in enumerate(("s0", "sigma", "r", "T")):
        up, dn = GreekOption(**o.__dict__), GreekOption(**o.__dict__)
        setattr(up, name, getattr(o, name) * (1 + h))
        setattr(dn, name, getattr(o, name) * (1 - h))
        fd = (book_greeks(up, n, seed)[0] - book_greeks(dn, n, seed)[0]) / (2 * h * getattr(o, name))
        if name == "T":
            fd = -fd
        assert abs(g[t] - fd) <= max(2e-4 * abs(fd), 2e-5), (o.kind, name, g[t], fd)
    assert np.isfinite(price)
