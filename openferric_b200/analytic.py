"""Host-side closed forms the Monte Carlo engines need for their control
variates (the expected value E[Y] the engine passes to the device).

They restate the reference's host code: the Hart normal CDF
(src/math/fast_norm.rs:28-50), bs_price (src/engines/analytic/black_scholes.rs:62-108)
and geometric_asian_discrete_fixed_closed_form (src/pricing/asian.rs:86-136).
"""
from __future__ import annotations

import math
from typing import Sequence

import numpy as np

from .core import OptionType

_INV_SQRT_2PI = 0.3989422804014327


def _fma_exact(a: float, b: float, c: float) -> float:
    # a*b + c rounded once: exact integer arithmetic over the operands' ratios
    # (their denominators are powers of two), then one int/int true division,
    # which Python rounds correctly.
    if not (math.isfinite(a) and math.isfinite(b) and math.isfinite(c)):
        return a * b + c
    na, da = a.as_integer_ratio()
    nb, db = b.as_integer_ratio()
    nc, dc = c.as_integer_ratio()
    d = da * db
    if dc >= d:
        return (na * nb * (dc // d) + nc) / dc
    return (na * nb + nc * (d // dc)) / d


_fma = getattr(math, "fma", _fma_exact)


def fast_norm_pdf(x: float) -> float:
    return _INV_SQRT_2PI * math.exp((-0.5 * x) * x)


def hart_norm_cdf(x: float) -> float:
    p, a1, a2, a3, a4, a5 = 0.2316419, 0.319381530, -0.356563782, 1.781477937, -1.821255978, 1.330274429
    z = abs(x)
    t = 1.0 / _fma(p, z, 1.0)
    poly = _fma(_fma(_fma(_fma(a5, t, a4), t, a3), t, a2), t, a1) * t
    cdf_pos = _fma(fast_norm_pdf(z), -poly, 1.0)
    sign = 1.0 if math.copysign(1.0, x) < 0 else 0.0
    return _fma(sign, 1.0 - 2.0 * cdf_pos, cdf_pos)


def _vanilla(option_type: OptionType, spot: float, strike: float) -> float:
    v = spot - strike if option_type is OptionType.Call else strike - spot
    return v if v > 0.0 else 0.0


def bs_price(option_type: OptionType, spot: float, strike: float, rate: float, q: float, vol: float,
             expiry: float) -> float:
    if expiry <= 0.0:
        return _vanilla(option_type, spot, strike)
    df_r = math.exp(-rate * expiry)
    df_q = math.exp(-q * expiry)
    if vol <= 0.0:
        v = spot * df_q - strike * df_r if option_type is OptionType.Call else strike * df_r - spot * df_q
        return max(v, 0.0)
    sig_sqrt_t = vol * math.sqrt(expiry)
    d1 = (math.log(spot / strike) + _fma(0.5 * vol, vol, rate - q) * expiry) / sig_sqrt_t
    d2 = d1 - sig_sqrt_t
    nd1, nd2 = hart_norm_cdf(d1), hart_norm_cdf(d2)
    s_df_q, k_df_r = spot * df_q, strike * df_r
    call = _fma(s_df_q, nd1, -(k_df_r * nd2))
    return call if option_type is OptionType.Call else call - s_df_q + k_df_r


def bs_greeks(option_type: OptionType, spot: float, strike: float, rate: float, q: float, vol: float,
              expiry: float):
    """bs_delta/bs_gamma/bs_vega/bs_theta/bs_rho (black_scholes.rs:110-214)."""
    if expiry <= 0.0 or vol <= 0.0 or spot <= 0.0:
        return dict(delta=0.0, gamma=0.0, vega=0.0, theta=0.0, rho=0.0)
    sqrt_t = math.sqrt(expiry)
    sig_sqrt_t = vol * sqrt_t
    d1 = (math.log(spot / strike) + _fma(0.5 * vol, vol, rate - q) * expiry) / sig_sqrt_t
    d2 = d1 - sig_sqrt_t
    df_q, df_r = math.exp(-q * expiry), math.exp(-rate * expiry)
    nd1, nd2, pdf = hart_norm_cdf(d1), hart_norm_cdf(d2), fast_norm_pdf(d1)
    call = option_type is OptionType.Call
    delta = df_q * nd1 if call else df_q * (nd1 - 1.0)
    gamma = df_q * pdf / (spot * vol * sqrt_t)
    vega = spot * df_q * pdf * sqrt_t
    common = -spot * df_q * pdf * vol / (2.0 * sqrt_t)
    if call:
        theta = common + q * spot * df_q * nd1 - rate * strike * df_r * nd2
        rho = strike * expiry * df_r * nd2
    else:
        theta = common - q * spot * df_q * (1.0 - nd1) + rate * strike * df_r * (1.0 - nd2)
        rho = -strike * expiry * df_r * (1.0 - nd2)
    return dict(delta=delta, gamma=gamma, vega=vega, theta=theta, rho=rho)


def min_sum_in_order(times: Sequence[float], rows_per_block: int = 256) -> float:
    """sum_i sum_j min(t_i, t_j) added in the reference's order (i outer, j
    inner, one FP64 add at a time: src/pricing/asian.rs:86-136), so the
    result is bit-identical to its double loop.  np.cumsum adds strictly left
    to right; blocks of rows bound the temporary to rows_per_block x n."""
    t = np.asarray(times, dtype=np.float64)
    total = 0.0
    for a in range(0, t.size, rows_per_block):
        block = np.minimum.outer(t[a:a + rows_per_block], t).ravel()
        total = float(np.cumsum(np.concatenate(([total], block)))[-1])
    return total


def geometric_asian_discrete_fixed(option_type: OptionType, s0: float, k: float, r: float, q: float, sigma: float,
                                   observation_times: Sequence[float], exact_order: bool = True) -> float:
    """exact_order=True adds the covariance sum in the reference's order
    (bit-identical to its double loop, O(n^2)); False uses the sorted O(n log n)
    form for callers that need no bit-level parity with the reference (the
    FP32 batched book).  The sorted form is within about 1e-15 of the exact
    sum; the double loop's own rounding reaches about 1e-12 relative at 900
    fixings, so the two differ by up to that much."""
    obs = list(observation_times)
    if not obs:
        return _vanilla(option_type, s0, k)
    maturity = max(max(obs), 0.0)
    if maturity <= 0.0 or sigma <= 0.0:
        return math.exp(-r * maturity) * _vanilla(option_type, s0, k)
    n = float(len(obs))
    mean_t = sum(obs) / n
    cov_sum = min_sum_in_order(obs) if exact_order else geometric_asian_cov_sum_sorted(obs)
    var = sigma * sigma * cov_sum / (n * n)
    m = math.log(s0) + _fma(-0.5 * sigma, sigma, r - q) * mean_t
    df = math.exp(-r * maturity)
    if var <= 0.0:
        return df * _vanilla(option_type, math.exp(m), k)
    sqrt_v = math.sqrt(var)
    d1 = (m - math.log(k) + var) / sqrt_v
    d2 = d1 - sqrt_v
    eg = math.exp(m + 0.5 * var)
    if option_type is OptionType.Call:
        return df * (eg * hart_norm_cdf(d1) - k * hart_norm_cdf(d2))
    return df * (k * hart_norm_cdf(-d2) - eg * hart_norm_cdf(-d1))


def geometric_asian_cov_sum_sorted(observation_times: Sequence[float]) -> float:
    """sum_{i,j} min(t_i, t_j) in O(n log n): with the times sorted, t_(i)
    is the minimum of 2(n - i) - 1 ordered pairs, so the sum is one dot
    product (within about 1e-15 relative of the exact sum), used for long
    fixing schedules."""
    ts = np.sort(np.asarray(observation_times, dtype=np.float64))
    n = ts.size
    return float(np.dot(ts, (2 * (n - np.arange(n)) - 1).astype(np.float64)))
