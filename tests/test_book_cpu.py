"""Host logic of the book's standard-error targeting (no GPU)."""
from openferric_b200.book import paths_for_stderr


def test_paths_for_stderr_scales_with_the_square_of_the_ratio():
    assert paths_for_stderr(1024, 0.02, 0.01, margin=1.0) == 4096
    assert paths_for_stderr(1024, 0.02, 0.01) == 4608  # 10 % margin, rounded up to a multiple of 256
    assert paths_for_stderr(1000, 0.01, 0.01) == 1000  # already at the target
    assert paths_for_stderr(1000, 0.001, 0.01) == 1000  # never fewer paths
    assert paths_for_stderr(256, 0.0101, 0.01, margin=1.0, granule=256) == 512
