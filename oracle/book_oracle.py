"""CPU restatement of the batched book's Greeks mode (numpy, FP64).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU kernel
(openferric_b200/csrc/book_greeks.cuh); the product package never imports it.

It draws the kernel's own Philox4x32-10 blocks (counter {block, sample lo,
sample hi, option index}, key = the 64-bit seed; the Random123 algorithm,
restated here vectorised over samples) and evaluates, per sample, in FP64:
- the price of MonteCarloPricingEngine's payoffs (vanilla, Asian, barrier by
  one-step survival) on GBM log-Euler paths with the kernel's Box-Muller
  normals, y_i = sum_j (alpha + beta z_j);
- the pathwise delta, vega, rho and theta of the discounted payoff, by the
  closed forms of the reference's tape (src/engines/monte_carlo/mc_aad.rs:15-72)
  for vanillas and Asians, and by forward tangents through the survival steps
  for barriers (Glasserman & Staum, Oper. Res. 49, 2001).
So the GPU's FP64 mode must equal it to rounding, and the GPU's FP32 Greeks to
FP32 path precision.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
from scipy.special import ndtr, ndtri

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = 0x9E3779B9, 0xBB67AE85
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, seed: int):
    """Philox4x32-10 on uint32 arrays (broadcast), key = (seed lo, seed hi)."""
    c0, c1, c2, c3 = (np.asarray(c, dtype=np.uint64) & _MASK for c in (c0, c1, c2, c3))
    k0, k1 = seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF
    for _ in range(10):
        p0 = _M0 * c0
        p1 = _M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK
        c0, c1, c2, c3 = hi1 ^ c1 ^ np.uint64(k0), lo1, hi0 ^ c3 ^ np.uint64(k1), lo0
        k0 = (k0 + _W0) & 0xFFFFFFFF
        k1 = (k1 + _W1) & 0xFFFFFFFF
    return c0, c1, c2, c3


def _unif(r):
    """(k + 0.5) 2^-23 with k the top 23 bits (uniform_from_u32's grid)."""
    return ((r >> np.uint64(9)).astype(np.float64) + 0.5) * 2.0 ** -23


def _pair(a, b):
    """Box-Muller: radius sqrt(-2 ln u1), angle pi (2 f - 3), f = 1 + k 2^-23."""
    rad = np.sqrt(-2.0 * np.log(_unif(a)))
    f = 1.0 + (b >> np.uint64(9)).astype(np.float64) * 2.0 ** -23
    ang = math.pi * (2.0 * f - 3.0)
    return rad * np.cos(ang), rad * np.sin(ang)


@dataclass
class GreekOption:
    """One GBM book option as the Greeks mode sees it."""
    kind: str                 # "vanilla", "asian", "barrier"
    call: bool
    s0: float
    strike: float
    r: float
    q: float
    sigma: float
    T: float
    steps: int
    stream: int               # the option's index in its book
    weights: Optional[Sequence[float]] = None  # Asian: observation count per step index 0..steps
    geometric: bool = False
    floating: bool = False
    up: bool = True
    knock_in: bool = False
    barrier: float = 0.0
    rebate: float = 0.0
    antithetic: bool = False


def _normals(o: GreekOption, idx, seed):
    """z[sample, step]: the kernel's Box-Muller normals, 4 steps per block."""
    lo, hi = idx & 0xFFFFFFFF, idx >> 32
    nb = (o.steps + 3) // 4
    z = np.empty((len(idx), nb * 4))
    for qb in range(nb):
        r0, r1, r2, r3 = philox4x32_10(np.full_like(lo, qb), lo, hi, np.full_like(lo, o.stream), seed)
        z[:, 4 * qb], z[:, 4 * qb + 1] = _pair(r0, r1)
        z[:, 4 * qb + 2], z[:, 4 * qb + 3] = _pair(r2, r3)
    return z[:, :o.steps]


def _uniforms(o: GreekOption, idx, seed):
    lo, hi = idx & 0xFFFFFFFF, idx >> 32
    nb = (o.steps + 3) // 4
    u = np.empty((len(idx), nb * 4))
    for qb in range(nb):
        r = philox4x32_10(np.full_like(lo, qb), lo, hi, np.full_like(lo, o.stream), seed)
        for k in range(4):
            u[:, 4 * qb + k] = _unif(r[k])
    return u[:, :o.steps]


def _vanilla(call, u, v, du, dv):
    d = u - v if call else v - u
    m = np.where(d > 0.0, 1.0 if call else -1.0, 0.0)
    return np.maximum(d, 0.0), m * (du - dv)


def _leg(o: GreekOption, z):
    """Undiscounted payoff x and dx along (ln S0, sigma, r, T) of the
    unconditioned paths with normals z[sample, step]."""
    dt = o.T / o.steps
    a = o.r - o.q - 0.5 * o.sigma ** 2
    alpha, beta = a * dt, o.sigma * math.sqrt(dt)
    y = np.cumsum(alpha + beta * z, axis=1)
    yT = y[:, -1]
    sT = o.s0 * np.exp(yT)
    ds = np.stack([sT, sT * ((yT - a * o.T) / o.sigma - o.sigma * o.T), sT * o.T, sT * (yT + a * o.T) / (2 * o.T)])
    zero = np.zeros_like(ds)
    if o.kind == "vanilla" or o.weights is None:
        if o.floating:
            return np.zeros_like(sT), zero
        return _vanilla(o.call, sT, o.strike, ds, zero)
    w = np.asarray(o.weights, dtype=np.float64)
    n = w.sum()
    idx = np.arange(o.steps + 1, dtype=np.float64)
    yall = np.concatenate([np.zeros((len(yT), 1)), y], axis=1)
    if o.geometric:
        q = (yall * w).sum(axis=1)
        w1 = (w * idx).sum()
        g = o.s0 * np.exp(q / n)
        da = np.stack([g, g / n * (q / o.sigma - (a / o.sigma + o.sigma) * dt * w1), g / n * dt * w1,
                       g / n * (q + a * dt * w1) / (2 * o.T)])
        avg = g
    else:
        e = w * np.exp(yall)
        p0, p1, p2 = e.sum(axis=1), (e * yall).sum(axis=1), (e * idx).sum(axis=1)
        sn = o.s0 / n
        avg = sn * p0
        da = np.stack([avg, sn * (p1 / o.sigma - (a / o.sigma + o.sigma) * dt * p2), sn * dt * p2,
                       sn * (p1 + a * dt * p2) / (2 * o.T)])
    if o.floating:
        return _vanilla(o.call, sT, avg, ds, da)
    return _vanilla(o.call, avg, o.strike, da, zero)


def _survival(o: GreekOption, u):
    """Barrier leg by one-step survival from uniforms u[sample, step]."""
    dt = o.T / o.steps
    a = o.r - o.q - 0.5 * o.sigma ** 2
    alpha, beta = a * dt, o.sigma * math.sqrt(dt)
    sgn = 1.0 if o.up else -1.0
    bar = math.log(o.barrier / o.s0)
    sib = sgn / beta
    ns = u.shape[0]
    y, ypl = np.zeros(ns), np.zeros(ns)
    L = np.full(ns, 1.0 if sgn * bar > 0.0 else 0.0)
    yd, ld = np.zeros((4, ns)), np.zeros((4, ns))
    c_b = np.array([-1.0, o.sigma * dt, -dt, -alpha / o.T])        # b' - alpha'
    c_e = np.array([0.0, 1.0 / o.sigma, 0.0, 1.0 / (2 * o.T)])    # beta' / beta
    c_a = np.array([0.0, -o.sigma * dt, dt, alpha / o.T])          # alpha'
    c_s = np.array([0.0, math.sqrt(dt), 0.0, beta / (2 * o.T)])   # beta'
    for j in range(o.steps):
        uj = u[:, j]
        h = np.maximum(sib * (bar - y - alpha), -37.0)
        p = ndtr(h)
        v = np.maximum(uj * p, 1e-300)
        qv = np.maximum(1.0 - uj * p, 1e-300)
        zeta = np.where(v <= 0.5, ndtri(v), -ndtri(qv))
        z = sgn * zeta
        g = np.exp(-0.5 * h * h) / math.sqrt(2 * math.pi) / p
        k = beta * sgn * (v / (np.exp(-0.5 * zeta * zeta) / math.sqrt(2 * math.pi))) * g
        for t in range(4):
            hd = sib * (c_b[t] - yd[t]) - h * c_e[t]
            ld[t] += g * hd
            yd[t] += c_a[t] + c_s[t] * z + k * hd
        y = y + alpha + beta * z
        L = L * p
        ypl = ypl + alpha + beta * ndtri(uj)
    so = o.s0 * np.exp(y)
    ds = np.stack([so * (1.0 + yd[0]), so * yd[1], so * yd[2], so * yd[3]])
    fo, dfo = _vanilla(o.call, so, o.strike, ds, np.zeros_like(ds))
    if not o.knock_in:
        return L * fo + (1.0 - L) * o.rebate, L * (ld * (fo - o.rebate) + dfo)
    spl = o.s0 * np.exp(ypl)
    dsp = np.stack([spl, spl * ((ypl - a * o.T) / o.sigma - o.sigma * o.T), spl * o.T,
                    spl * (ypl + a * o.T) / (2 * o.T)])
    fp, dfp = _vanilla(o.call, spl, o.strike, dsp, np.zeros_like(dsp))
    return fp - L * (fo - o.rebate), dfp - L * (ld * (fo - o.rebate) + dfo)


def book_greeks(o: GreekOption, num_paths: int, seed: int):
    """(price, [delta, vega, rho, theta]) of one option over samples
    0..samples-1 (antithetic pairs count as one sample), FP64."""
    samples = (num_paths + 1) // 2 if o.antithetic else num_paths
    idx = np.arange(samples, dtype=np.uint64)
    df = math.exp(-o.r * o.T)
    if o.kind == "barrier":
        u = _uniforms(o, idx, seed)
        x, dx = _survival(o, u)
        if o.antithetic:
            xb, dxb = _survival(o, 1.0 - u)
            x, dx = 0.5 * (x + xb), 0.5 * (dx + dxb)
    else:
        z = _normals(o, idx, seed)
        x, dx = _leg(o, z)
        if o.antithetic:
            xb, dxb = _leg(o, -z)
            x, dx = 0.5 * (x + xb), 0.5 * (dx + dxb)
    pv = df * x
    g = np.stack([df * dx[0] / o.s0, df * dx[1], df * dx[2] - o.T * pv, o.r * pv - df * dx[3]])
    return float(pv.mean()), [float(v) for v in g.mean(axis=1)]
