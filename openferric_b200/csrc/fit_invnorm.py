"""Fits the FP32 inverse-normal polynomials used by the Philox kernels.

Method (the structure of M. Giles, "Approximating the erfinv function", GPU
Computing Gems Jade, 2011; the coefficients here are fitted by this script):
for u in (0,1) let x = 2u-1 and w = -log2(4u(1-u)) = -log2(1-x^2).  Then
    Phi^-1(u) = sqrt(2) erfinv(x) = x * P(w)
with one polynomial for w < W_SPLIT (the central 99.66 % of draws) and a second
one in s = sqrt(w) for the tails.  Each polynomial is a weighted least-squares
fit (relative error) on Chebyshev nodes in float64, then rounded to float32;
the script reports the float32 relative error over the domain reached by the
uniforms the kernels produce, u = (k + 0.5) 2^-23 for k < 2^23.

Run:  python openferric_b200/csrc/fit_invnorm.py > openferric_b200/csrc/invnorm_coeffs.h
"""
import numpy as np
from scipy.special import erfinv

W_SPLIT = 7.25  # in log2 units; tail probability 2*P(u < ~1.6e-3)
DEG_C = 8
DEG_T = 8
S_LO, S_HI = np.sqrt(W_SPLIT), np.sqrt(26.0)


def target_from_w(w):
    x2 = 1.0 - np.exp2(-w)
    x = np.sqrt(x2)
    return np.sqrt(2.0) * erfinv(x) / x


def cheb_nodes(lo, hi, n):
    k = np.arange(n)
    return 0.5 * (lo + hi) + 0.5 * (hi - lo) * np.cos(np.pi * (k + 0.5) / n)


def fit(var_lo, var_hi, deg, to_w, center):
    v = cheb_nodes(var_lo, var_hi, 4000)
    w = to_w(v)
    f = np.where(w < 1e-12, np.sqrt(np.pi / 2.0) * 1.0, 0.0)
    mask = w >= 1e-12
    f[mask] = target_from_w(w[mask])
    t = v - center
    A = np.vander(t, deg + 1, increasing=True) / f[:, None]
    coef, *_ = np.linalg.lstsq(A, np.ones_like(f), rcond=None)
    return coef


def horner32(coef32, t):
    acc = np.float32(coef32[-1]) * np.ones_like(t, dtype=np.float32)
    for c in coef32[-2::-1]:
        acc = (acc * t + np.float32(c)).astype(np.float32)
    return acc


def main():
    c_center = W_SPLIT / 2.0
    cc = fit(0.0, W_SPLIT, DEG_C, lambda v: v, c_center).astype(np.float32)
    t_center = 0.5 * (S_LO + S_HI)
    tc = fit(S_LO, S_HI, DEG_T, lambda s: s * s, t_center).astype(np.float32)

    # float32 check over the uniforms the kernels emit: u = (k + 0.5) * 2^-23, k < 2^23
    k = np.unique(np.concatenate([np.arange(0, 2 ** 16), np.linspace(0, 2 ** 23 - 1, 2 ** 20).astype(np.int64),
                                  2 ** 23 - 1 - np.arange(0, 2 ** 16)]))
    u = ((k.astype(np.float64) + 0.5) * 2.0 ** -23).astype(np.float32)
    x = (np.float32(2.0) * u - np.float32(1.0)).astype(np.float32)
    # the kernel forms t = fmaf(-x, x, 1): 1 - x^2 rounded once from the exact value
    tt = (1.0 - x.astype(np.float64) ** 2).astype(np.float32)
    w = (-np.log2(tt.astype(np.float64))).astype(np.float32)
    p = np.where(w < W_SPLIT, horner32(cc, (w - np.float32(c_center)).astype(np.float32)),
                 horner32(tc, (np.sqrt(w) - np.float32(t_center)).astype(np.float32)))
    z = (x * p).astype(np.float64)
    exact = np.sqrt(2.0) * erfinv(x.astype(np.float64))
    rel = np.abs(z - exact) / np.maximum(np.abs(exact), 1e-30)
    worst = float(np.max(rel[np.abs(exact) > 1e-6]))

    def arr(name, c):
        body = ", ".join(f"{float(v):.9e}f" for v in c)
        return f"static __device__ __constant__ const float {name}[{len(c)}] = {{{body}}};"

    print("/* Generated by openferric_b200/csrc/fit_invnorm.py; do not edit by hand.")
    print(f" * Phi^-1(u) = x * P(w), x = 2u-1, w = -log2(4u(1-u)); central P in (w - {c_center}) for w < {W_SPLIT},")
    print(f" * tail P in (sqrt(w) - {t_center:.9f}).  Max float32 relative error on u = (k+0.5) 2^-23: {worst:.3e} */")
    print("#pragma once")
    print(f"#define OF_INVN_W_SPLIT {W_SPLIT:.9e}f")
    print(f"#define OF_INVN_C_CENTER {c_center:.9e}f")
    print(f"#define OF_INVN_T_CENTER {t_center:.9e}f")
    print(f"#define OF_INVN_DEG_C {DEG_C}")
    print(f"#define OF_INVN_DEG_T {DEG_T}")
    print(arr("kInvnCentral", cc))
    print(arr("kInvnTail", tc))


if __name__ == "__main__":
    main()
