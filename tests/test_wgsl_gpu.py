"""engines::gpu::mc_european_gpu.  stream="xoshiro128" (the reference's WGSL
kernel semantics on CUDA) against the oracle's C float restatement of the
shader math: both run f32 arithmetic with different libm implementations of
exp/log/sin/cos, so they agree at f32 rounding level, not bit level.  The
default stream, this engine's own FP32 Philox GBM path, against Black-Scholes
and the shader's kernel."""
import pytest

from openferric_b200.analytic import bs_price
from openferric_b200.core import OptionType
from openferric_b200.gpu_mc import mc_european_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("steps", [1, 2, 63, 64])
@pytest.mark.parametrize("is_call", [True, False])
def test_wgsl_port_matches_c_restatement(orc, steps, is_call):
    g = mc_european_gpu(100.0, 105.0, 0.03, 0.25, 1.0, 50_000, steps, 17, is_call, stream="xoshiro128")
    p, s = orc.wgsl_european(100.0, 105.0, 0.03, 0.25, 1.0, 50_000, steps, 17, is_call)
    assert abs(g.price - p) <= 2e-5 * abs(p) + 1e-6, (g.price, p)
    assert abs(g.stderr - s) <= 2e-4 * abs(s)


def test_wgsl_port_prices_near_black_scholes():
    r = mc_european_gpu(100.0, 100.0, 0.05, 0.2, 1.0, 1 << 20, 64, 3, True, stream="xoshiro128")
    bs = bs_price(OptionType.Call, 100.0, 100.0, 0.05, 0.0, 0.2, 1.0)
    assert abs(r.price - bs) <= 4 * r.stderr + 0.01


@pytest.mark.parametrize("is_call", [True, False])
def test_native_path_behind_the_reference_entry_point(is_call):
    """The default stream is this engine's own FP32 Philox GBM path: within
    4 standard errors of Black-Scholes and of the reference shader's kernel."""
    nat = mc_european_gpu(100.0, 105.0, 0.03, 0.25, 1.0, 1 << 20, 64, 17, is_call)
    wg = mc_european_gpu(100.0, 105.0, 0.03, 0.25, 1.0, 1 << 20, 64, 17, is_call, stream="xoshiro128")
    bs = bs_price(OptionType.Call if is_call else OptionType.Put, 100.0, 105.0, 0.03, 0.0, 0.25, 1.0)
    assert abs(nat.price - bs) <= 4 * nat.stderr + 0.01
    assert abs(nat.price - wg.price) <= 4 * (nat.stderr ** 2 + wg.stderr ** 2) ** 0.5 + 0.01
