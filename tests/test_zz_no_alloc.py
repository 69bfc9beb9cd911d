"""The no-allocation strike strip (of_mc_strip_noalloc), called through the C ABI.

Some callers cannot allocate device memory when they price: their HBM is
already reserved in full by another allocator, or they cannot take the
device-wide synchronisation of cudaFree.  This entry point serves them from a
static device array instead.  The test checks its output against the existing
entry point (of_mc_strip, which draws its scratch from the context's pool) on
two calls in a row, so that the second call also sees the array the first one
left behind.  It runs last (file name) and passes alone or after the rest of
the suite.
"""
import ctypes as C
import math
import warnings

import pytest

from openferric_b200 import Gbm, GbmPathGenerator, Heston, HestonPathGenerator, OptionType, price_strike_strip
from openferric_b200 import _abi as A
from openferric_b200 import _lib

pytestmark = pytest.mark.gpu

STRIKES = [80.0 + 2.0 * k for k in range(21)]


def noalloc_strip(model, option_type, strikes, num_paths, seed, df, antithetic=False, tile_ilp=0, stream=None):
    L = _lib.load()
    ks = (C.c_double * len(strikes))(*strikes)
    cfg = A.OfMcConfig(num_paths=num_paths, seed=seed, precision=A.OF_PREC_FP32_PHILOX, discount_factor=df,
                       antithetic=int(antithetic), tile_ilp=tile_ilp)
    out = (A.OfMcResult * len(strikes))()
    err = C.create_string_buffer(256)
    st = L.of_mc_strip_noalloc(stream, C.byref(model), option_type, ks, len(strikes), C.byref(cfg), out, err,
                               len(err))
    return st, err.value.decode(), [(r.price, r.stderr_) for r in out]


def test_noalloc_strip_matches_existing_entry_point_on_two_calls():
    gen = HestonPathGenerator(Heston(0.03, 2.0, 0.04, 0.5, -0.7, 0.04), 100.0, 1.0, 64)
    df = math.exp(-0.03)
    ref = price_strike_strip(gen, OptionType.Call, STRIKES, 1 << 18, 7, df)
    for _ in range(2):
        st, msg, got = noalloc_strip(gen.to_abi(), A.OF_CALL, STRIKES, 1 << 18, 7, df)
        assert st == A.OF_OK, msg
        for (p, s), (rp, rs) in zip(got, ref):
            # same kernel, same draws: equal up to the FP32 partial-sum grouping
            assert abs(p - rp) <= 1e-9 * abs(rp) + 1e-12, (p, rp)
            assert abs(s - rs) <= 1e-9 * abs(rs) + 1e-12


def test_noalloc_strip_full_strike_layout_gbm_antithetic_two_samples_per_thread():
    """64 strikes fill the static scratch's strike and sum rows (two strikes
    per lane), with GBM antithetic pairs and two samples in flight per thread:
    the same kernel of_mc_strip picks for that request."""
    gen = GbmPathGenerator(Gbm(0.05, 0.25), 100.0, 1.0, 52)
    df = math.exp(-0.05)
    strikes = [70.0 + k for k in range(64)]
    ref = price_strike_strip(gen, OptionType.Put, strikes, 1 << 17, 11, df, antithetic=True, tile_ilp=2)
    for _ in range(2):
        st, msg, got = noalloc_strip(gen.to_abi(), A.OF_PUT, strikes, 1 << 17, 11, df, antithetic=True, tile_ilp=2)
        assert st == A.OF_OK, msg
        for (p, s), (rp, rs) in zip(got, ref):
            assert abs(p - rp) <= 1e-9 * abs(rp) + 1e-12, (p, rp)
            assert abs(s - rs) <= 1e-9 * abs(rs) + 1e-12


def test_noalloc_strip_warp_specialised_shape():
    """tile_ilp=3 runs the warp-specialised kernel from the static array (its
    ring status word included) and matches of_mc_strip with the same shape."""
    gen = HestonPathGenerator(Heston(0.03, 2.0, 0.04, 0.5, -0.7, 0.04), 100.0, 1.0, 63)
    df = math.exp(-0.03)
    ref = price_strike_strip(gen, OptionType.Call, STRIKES, 100_003, 3, df, tile_ilp=3)
    for _ in range(2):
        st, msg, got = noalloc_strip(gen.to_abi(), A.OF_CALL, STRIKES, 100_003, 3, df, tile_ilp=3)
        assert st == A.OF_OK, msg
        for (p, s), (rp, rs) in zip(got, ref):
            assert abs(p - rp) <= 1e-9 * abs(rp) + 1e-12, (p, rp)
            assert abs(s - rs) <= 1e-9 * abs(rs) + 1e-12


def test_noalloc_strip_rejects_sizes_beyond_its_static_scratch():
    gen = HestonPathGenerator(Heston(0.03, 2.0, 0.04, 0.5, -0.7, 0.04), 100.0, 1.0, 8)
    too_many = [90.0 + 0.1 * k for k in range(65)]
    st, msg, _ = noalloc_strip(gen.to_abi(), A.OF_CALL, too_many, 1 << 10, 1, 1.0)
    assert st == A.OF_ERR_INVALID_INPUT
    assert "64" in msg


def test_noalloc_strip_refuses_a_capturing_stream():
    """The entry point synchronises its stream, which a capture forbids: on a
    capturing stream it returns OF_ERR_UNSUPPORTED before issuing any work,
    and the capture ends cleanly."""
    import torch
    gen = GbmPathGenerator(Gbm(0.03, 0.2), 100.0, 1.0, 16)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            st, msg, _ = noalloc_strip(gen.to_abi(), A.OF_CALL, STRIKES, 4096, 3, 1.0,
                                       stream=C.c_void_p(s.cuda_stream))
        finally:
            with warnings.catch_warnings():  # the refused call leaves the graph empty, which torch reports
                warnings.simplefilter("ignore", UserWarning)
                g.capture_end()
    assert st == A.OF_ERR_UNSUPPORTED and "capturing" in msg, (st, msg)
    st, msg, res = noalloc_strip(gen.to_abi(), A.OF_CALL, STRIKES, 4096, 3, 1.0,
                                 stream=C.c_void_p(s.cuda_stream))
    assert st == A.OF_OK, msg
    assert all(math.isfinite(p) for p, _ in res)
