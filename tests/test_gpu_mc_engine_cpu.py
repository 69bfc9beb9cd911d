"""GpuMcEngine, the reference Python module's McEngine surface
(python/src/engines.rs:1230-1438): argument parsing and error behaviour,
which run on the host before any device work."""
import pytest

from openferric_b200 import GpuMcEngine

BASE = dict(option_type="call", spot=100.0, strike=100.0, expiry=1.0, rate=0.05, dividend_yield=0.0, vol=0.2,
            num_paths=1000, num_steps=10, seed=1)


def _vanilla(**kw):
    args = dict(BASE)
    args.update(kw)
    return GpuMcEngine.vanilla_price(**args)


@pytest.mark.parametrize("kw, message", [
    (dict(option_type="straddle"), "option_type must be 'call' or 'put'"),
    (dict(spot=-1.0), "invalid market inputs"),
    (dict(variance_reduction="Sobol"), "unsupported variance reduction 'sobol'"),
    (dict(rng_kind="MT19937"), "unsupported rng kind 'mt19937'"),
    (dict(accuracy_tier="Ultra"), "unsupported accuracy tier 'ultra'"),
    (dict(exercise_style="Asian"), "unsupported exercise style 'asian'"),
    (dict(precision="fp16"), "unsupported precision 'fp16'"),
    (dict(num_paths=0), 'InvalidInput("num_paths must be > 0")'),
    (dict(num_steps=0), 'InvalidInput("num_steps must be > 0")'),
    (dict(strike=-5.0), 'InvalidInput("vanilla strike must be > 0")'),
    (dict(exercise_style="bermudan"), 'InvalidInput("bermudan exercise dates cannot be empty")'),
])
def test_vanilla_price_errors_match_the_reference_binding(kw, message):
    with pytest.raises(ValueError) as e:
        _vanilla(**kw)
    assert str(e.value) == message


def test_stream_options_the_gpu_does_not_have_are_value_errors():
    msg = 'InvalidInput("the GPU engine supports the reproducible Xoshiro256PlusPlus stream only")'
    with pytest.raises(ValueError) as e:
        GpuMcEngine.greeks_pathwise("put", 100, 100, 1, 0.05, 0, 0.2, 1000, 1, rng_kind="pcg64")
    assert str(e.value) == msg
    with pytest.raises(ValueError) as e:
        GpuMcEngine.arithmetic_asian_price("call", 100, 100, 1, 0.05, 0, 0.2, [0.5, 1.0], 1000, 10, 1,
                                           reproducible=False)
    assert str(e.value) == msg
    with pytest.raises(ValueError, match="spread options"):
        GpuMcEngine.spread_price(100, 95, 5, 0.2, 0.25, 0.5, 0, 0, 0.05, 1.0, 1000, 1)


def test_expiry_zero_is_intrinsic_without_device_work():
    r = _vanilla(option_type="PUT", strike=110.0, expiry=0.0)
    assert r.price == 10.0 and r.stderr == 0.0
