"""Autotuner: candidates are timed with CUDA events, the winner is cached in
the JSON table and read back without re-timing; the tuned tile prices the
same as the default."""
import json
import math

import pytest

from openferric_b200 import Heston, HestonPathGenerator, OptionType, price_strike_strip
from openferric_b200 import autotune
from openferric_b200.book import BookPlan, synthetic_book

pytestmark = pytest.mark.gpu

HESTON = Heston(mu=0.03, kappa=2.0, theta=0.04, xi=0.5, rho=-0.7, v0=0.04)


def test_tune_strip_caches_winner(tmp_path, monkeypatch):
    monkeypatch.setenv("OF_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    gen = HestonPathGenerator(HESTON, 100.0, 1.0, 64)
    strikes = [80.0 + k for k in range(41)]
    assert autotune.best_strip_ilp(gen, len(strikes)) == 0
    best, times = autotune.tune_strip(gen, strikes, 1 << 17, reps=3, candidates=(1, 2, 3))
    assert best in (1, 2, 3) and set(times) == {1, 2, 3} and all(t > 0 for t in times.values())
    assert autotune.best_strip_ilp(gen, len(strikes)) == best
    table = json.loads((tmp_path / "tune.json").read_text())
    assert len(table) == 1 and next(iter(table.values()))["ilp"] == best
    tuned = price_strike_strip(gen, OptionType.Call, strikes, 1 << 16, 5, math.exp(-0.03), tile_ilp=best)
    default = price_strike_strip(gen, OptionType.Call, strikes, 1 << 16, 5, math.exp(-0.03))
    for (a, _), (b, _) in zip(tuned, default):
        assert abs(a - b) <= 2e-6 * max(1.0, abs(a))


def test_tune_book_caches_winner(tmp_path, monkeypatch):
    monkeypatch.setenv("OF_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    book = synthetic_book(64, seed=3, min_log2_paths=12, max_log2_paths=13)
    cands = ((256, 4), (128, 8))
    best, times = autotune.tune_book(book, seed=1, candidates=cands, reps=2)
    assert best in cands and len(times) == 2
    assert autotune.best_book_tile(len(book)) == best
    plan = BookPlan(book, 1, block=best[0], paths_per_thread=best[1])
    plan.launch()
    res = plan.results()
    plan.close()
    assert all(math.isfinite(r.price) for r in res)


def test_native_autotune_rejects_bad_candidates(tmp_path, monkeypatch):
    monkeypatch.setenv("OF_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    from openferric_b200 import PricingError
    gen = HestonPathGenerator(HESTON, 100.0, 1.0, 8)
    with pytest.raises(PricingError, match="1 or 2"):
        autotune.tune_strip(gen, [100.0], 1 << 12, candidates=(1, 4))
    with pytest.raises(PricingError, match="reps"):
        autotune.tune_strip(gen, [100.0], 1 << 12, reps=0)
    book = synthetic_book(4, seed=3, min_log2_paths=10, max_log2_paths=11)
    with pytest.raises(PricingError, match="multiple of 32"):
        autotune.tune_book(book, candidates=((512, 4),))
    assert not (tmp_path / "tune.json").exists()  # nothing cached from a refused call
