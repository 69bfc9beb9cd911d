"""The fitted FP32 approximations of the kernels, checked on the CPU in float32
emulation: the Mills-ratio normal CDF of the survival steps (mills_coeffs.h,
written by csrc/fit_mills.py) against scipy's ndtr."""
import os
import re
import subprocess
import sys

import numpy as np
from scipy.special import ndtr

from conftest import ROOT

CSRC = os.path.join(ROOT, "openferric_b200", "csrc")


def _mills():
    src = open(os.path.join(CSRC, "mills_coeffs.h")).read()
    c = np.float32(float(re.search(r"OF_MILLS_C ([0-9.e+-]+)f", src).group(1)))
    co = [np.float32(float(x.rstrip("f"))) for x in re.search(r"kMills\[\d+\] = \{(.*)\}", src).group(1).split(", ")]
    return c, co


def test_mills_header_is_the_fit_scripts_output():
    out = subprocess.run([sys.executable, os.path.join(CSRC, "fit_mills.py")], capture_output=True, text=True,
                         check=True).stdout
    assert out == open(os.path.join(CSRC, "mills_coeffs.h")).read()


def test_mills_normal_cdf_and_ratio_in_float32():
    c, co = _mills()
    h = np.linspace(-12.0, 12.0, 100001).astype(np.float32)
    a = np.abs(h)
    t = (np.float32(1) / (c * a + np.float32(1))).astype(np.float32)
    m = co[-1] * np.ones_like(t)
    for k in co[-2::-1]:
        m = (m * t + k).astype(np.float32)
    m = (m * t).astype(np.float32)
    a2 = (a * a).astype(np.float32)
    a2lo = (a.astype(np.float64) ** 2 - a2.astype(np.float64)).astype(np.float32)
    phi = (np.float32(0.3989422804014327) * np.exp(np.float32(-0.5) * a2) *
           (np.float32(1) - np.float32(0.5) * a2lo)).astype(np.float32)
    tail = (phi * m).astype(np.float32)
    p = np.where(h < 0, tail, np.float32(1) - tail)
    g = np.where(h < 0, np.float32(1) / m, phi / p)
    pe = ndtr(h.astype(np.float64))
    ge = np.exp(-0.5 * h.astype(np.float64) ** 2) / np.sqrt(2 * np.pi) / pe
    assert np.max(np.abs(p / pe - 1)) < 1e-6
    assert np.max(np.abs(g / ge - 1)) < 1e-6
