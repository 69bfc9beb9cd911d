"""Fits the FP32 Mills-ratio polynomial used by the one-step-survival steps.

Method (the form of Hastings' approximation of the normal tail, as in
Abramowitz & Stegun 26.2.17, with coefficients fitted here): for x >= 0 the
Mills ratio M(x) = (1 - Phi(x)) / phi(x) is written as
    M(x) = t P(t),   t = 1 / (1 + C x),
with P a polynomial in t.  M(x) ~ 1/x for large x, so M(x) / t tends to C as
t -> 0 and P is smooth on t in (0, 1].  P is a weighted least-squares fit of
M(x) / t (relative error) on Chebyshev nodes in t, in float64, rounded to
float32; the script reports the float32 relative error of t P(t) over
x in [0, 13], evaluated the way the kernel evaluates it.  The normal tail is
then Phi(-x) = phi(x) M(x) with phi computed from an exact split of x^2.

Run:  python openferric_b200/csrc/fit_mills.py > openferric_b200/csrc/mills_coeffs.h
"""
import numpy as np
from scipy.special import erfcx

C = 0.4
DEG = 9


def mills(x):
    # M(x) = sqrt(pi/2) erfcx(x / sqrt(2))
    return np.sqrt(np.pi / 2.0) * erfcx(x / np.sqrt(2.0))


def main():
    k = np.arange(6000)
    t = 0.5 + 0.5 * np.cos(np.pi * (k + 0.5) / len(k))  # Chebyshev nodes on (0, 1)
    t = t[t > 1e-6]
    x = (1.0 / t - 1.0) / C
    f = mills(x) / t
    A = np.vander(t, DEG + 1, increasing=True) / f[:, None]
    coef, *_ = np.linalg.lstsq(A, np.ones_like(f), rcond=None)
    c32 = coef.astype(np.float32)
    # float32 check, evaluated as the kernel does: t = 1 / (1 + C x), Horner in t, times t
    xs = np.linspace(0.0, 13.0, 400001).astype(np.float32)
    t32 = (np.float32(1.0) / (np.float32(1.0) + np.float32(C) * xs)).astype(np.float32)
    p = np.float32(c32[-1]) * np.ones_like(t32)
    for c in c32[-2::-1]:
        p = (p * t32 + np.float32(c)).astype(np.float32)
    m32 = (t32 * p).astype(np.float32)
    err = np.max(np.abs(m32.astype(np.float64) / mills(xs.astype(np.float64)) - 1.0))
    print("/* Generated by openferric_b200/csrc/fit_mills.py; do not edit by hand.")
    print(f" * Mills ratio M(x) = (1 - Phi(x)) / phi(x) = t P(t), t = 1 / (1 + {C} x), x >= 0.")
    print(f" * Max float32 relative error over x in [0, 13]: {err:.3e} */")
    print("#pragma once")
    print(f"#define OF_MILLS_C {C:.9e}f")
    print(f"#define OF_MILLS_DEG {DEG}")
    print("static __device__ __constant__ const float kMills[%d] = {%s};" %
          (DEG + 1, ", ".join(f"{float(c):.9e}f" for c in c32)))


if __name__ == "__main__":
    main()
