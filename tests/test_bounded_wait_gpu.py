"""The bounded mbarrier wait of the bulk-copy pipelines (of_test_bounded_wait):
a phase that completes is seen at once; a phase that nothing completes makes
the wait give up after its limit, the kernel return, and the context stay
usable.  No GPU fault or hang is involved: the failing wait is a loop on the
global timer that ends by itself."""
import ctypes as C

import pytest

from openferric_b200._lib import context

pytestmark = pytest.mark.gpu


def _wait(ctx, arrive, limit_us):
    ok, us = C.c_int32(-1), C.c_double(-1.0)
    ctx.check(ctx._L.of_test_bounded_wait(ctx.handle, arrive, limit_us, C.byref(ok), C.byref(us)))
    return ok.value, us.value


def test_completed_phase_is_seen_at_once():
    ctx = context(0)
    ok, us = _wait(ctx, 1, 100000)
    assert ok == 1 and 0.0 <= us < 1000.0


def test_wait_with_no_arrival_gives_up_and_the_context_survives():
    ctx = context(0)
    ok, us = _wait(ctx, 0, 2000)
    assert ok == 0
    assert 2000.0 <= us < 200000.0
    ok, _ = _wait(ctx, 1, 100000)  # the context still runs kernels
    assert ok == 1


def test_bounded_wait_rejects_bad_limits():
    from openferric_b200 import PricingError
    ctx = context(0)
    with pytest.raises(PricingError, match="limit_us"):
        _wait(ctx, 1, 0)
