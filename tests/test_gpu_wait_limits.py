"""Failure detection without a GPU fault: every wait in the kernels is
bounded in time and ends in an error flag the host reads.  The library's
self-test runs the two waits to their limit on purpose, with a short limit
in place of the kernels' own (1 s for a tile's staging wait, 2 s for the
ensemble's lane barrier):

* a tile's staging wait (mbar_wait, cb_tma.cuh) on an mbarrier that needs two
  arrivals and gets one, with no copy in flight: it gives up, sets the error
  flag the host reports as a staging failure, and returns false;
* the ensemble's lane barrier (lane_sync, cb_sync.cuh) of a two-CTA lane
  whose second CTA exits without arriving: the first gives up, sets the
  abort flag that ends every lane, and returns false.

Afterwards the device is still usable: a small run goes through and its
summaries match the reference's (the bm32x87 golden deck)."""
import ctypes

import pytest

from cloverleaf_b200 import Chunk, HydroRun, library
from cloverleaf_b200 import deck as D
from golden_util import deck_text, rel, summaries

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("limit_ms", [20.0, 100.0])
def test_waits_give_up_at_their_limit(limit_ms):
    sf, sr, lf, lr = (ctypes.c_int(-1) for _ in range(4))
    sms, lms = ctypes.c_double(-1.0), ctypes.c_double(-1.0)
    rc = library().cb_selftest_wait_limits(limit_ms, ctypes.byref(sf), ctypes.byref(sr), ctypes.byref(sms), ctypes.byref(lf),
                                           ctypes.byref(lr), ctypes.byref(lms))
    assert rc == 0
    assert (sf.value, sr.value) == (1, 0)  # the staging wait gave up and flagged it
    assert (lf.value, lr.value) == (1, 0)  # the lane barrier gave up and set the abort flag
    for ms in (sms.value, lms.value):
        assert limit_ms <= ms < limit_ms + 500.0, (ms, limit_ms)


def test_device_usable_after_the_waits_gave_up():
    sf, sr, lf, lr = (ctypes.c_int(-1) for _ in range(4))
    sms, lms = ctypes.c_double(-1.0), ctypes.c_double(-1.0)
    assert library().cb_selftest_wait_limits(10.0, ctypes.byref(sf), ctypes.byref(sr), ctypes.byref(sms), ctypes.byref(lf),
                                             ctypes.byref(lr), ctypes.byref(lms)) == 0
    dk = D.parse_deck(deck_text("bm32x87"))
    c = Chunk(dk.x_cells, dk.y_cells, gamma=dk.gamma)
    r = HydroRun(c, dk)
    r.run()
    gold = summaries("bm32x87")
    assert len(r.summaries) == len(gold)
    for s, g in zip(r.summaries, gold):
        for a, b in zip((s.vol, s.mass, s.ie, s.ke, s.press), g[2:]):
            assert rel(a, b) <= 1e-12, (s.step, a, b)
    c.close()
