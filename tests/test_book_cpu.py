"""Host logic of the book's standard-error targeting (no GPU)."""
from openferric_b200.book import paths_for_stderr


def test_paths_for_stderr_scales_with_the_square_of_the_ratio():
    assert paths_for_stderr(1024, 0.02, 0.01, margin=1.0) == 4096
    assert paths_for_stderr(1024, 0.02, 0.01) == 4352  # 5 % margin (the driver's default), up to a multiple of 256
    assert paths_for_stderr(1024, 0.02, 0.01, margin=1.1) == 4608
    assert paths_for_stderr(1000, 0.01, 0.01) == 1000  # already at the target
    assert paths_for_stderr(1000, 0.001, 0.01) == 1000  # never fewer paths
    assert paths_for_stderr(256, 0.0101, 0.01, margin=1.0, granule=256) == 512


def test_asian_validation_matches_the_reference_check():
    """AsianOption.validate: observation times outside [0, expiry] are
    rejected with the reference's message (src/instruments/asian.rs:55-64);
    a NaN time compares false there and passes, as in the reference."""
    import math

    import pytest

    from openferric_b200.core import AsianSpec, Averaging, OptionType, PricingError, StrikeType
    from openferric_b200.instruments import AsianOption

    def opt(times):
        return AsianOption.new(OptionType.Call, 100.0, 1.0, AsianSpec(Averaging.Arithmetic, StrikeType.Fixed, times))

    opt([0.0, 0.5, 1.0]).validate()
    opt([0.25, math.nan]).validate()
    for bad in ([-1e-12, 0.5], [0.5, 1.0 + 1e-12]):
        with pytest.raises(PricingError, match="observation_times must lie"):
            opt(bad).validate()
    with pytest.raises(PricingError, match="cannot be empty"):
        opt([]).validate()
