"""The Lagrangian pass run ahead of its calls (cb_set_dt_ahead, with call
fusion): cb_calc_dt, given the driver's dt clamp, also enqueues the
Lagrangian pass with the clamped dt formed on the device; the four calls
that follow (predictor, accelerate, corrector, flux_calc) find it done when
their dt and halo depths match.  Checked against the same calls without it
(HydroRun's host loop, call fusion off):

* FP64: dt of every step, every summary and every state field (halos
  included) bit-identical, on meshes with and without interior tiles and a
  moving circle; every pass run ahead consumed (stats: one per step);
* a clamp that differs from the driver's (a wrong dtmax given to the
  library): the predictor's dt does not match, the pass run ahead is
  dropped and the calls run as made -- still bit-identical, none consumed;
* a field read after the predictor and again after accelerate: the calls
  matched so far run as made before the read -- bit-identical;
* FP32 within the FP32 form's rounding.
"""
import numpy as np
import pytest

from cloverleaf_b200 import FP32, FP64, Chunk, HydroRun
from test_gpu_fused_calls import STATE_FIELDS, assert_same, deck_a, deck_b, run

pytestmark = pytest.mark.gpu


def run_ahead(dk, precision=FP64, probe=None, chunk_hook=None):
    c = Chunk(dk.x_cells, dk.y_cells, precision=precision, gamma=dk.gamma)
    if chunk_hook:
        chunk_hook(c)
    r = HydroRun(c, dk, fuse_calls=True, dt_ahead=True, probe=probe)
    r.run()
    return c, r


@pytest.mark.parametrize("dk", [deck_a(), deck_b(), deck_a(200, 150, 25)], ids=["bm64x48", "circle40x56", "bm200x150"])
def test_dt_ahead_fp64_bit_identical(dk):
    c1, r1 = run(dk)
    c2, r2 = run_ahead(dk)
    assert_same(c1, r1, c2, r2)
    assert c2.dt_ahead_stats() == (r2.step, r2.step)
    c1.close()
    c2.close()


def test_wrong_clamp_is_dropped():
    dk = deck_b()
    c1, r1 = run(dk)

    def hook(c):
        real = c.set_dt_ahead
        c.set_dt_ahead = lambda dtold, dtrise, dtmax: real(dtold, dtrise, 0.5 * dtmax)

    c2, r2 = run_ahead(dk, chunk_hook=hook)
    assert_same(c1, r1, c2, r2)
    launched, used = c2.dt_ahead_stats()
    assert launched == r2.step and used < launched


def test_interrupted_pass_runs_its_calls():
    dk = deck_b()
    c1, r1 = run(dk)
    holder = {}

    def probe(name):
        # after the predictor matched (before accelerate) on odd steps, after
        # accelerate matched (before the corrector) on even steps
        r = holder["r"]
        if (name == "accelerate" and r.step % 2 == 1) or (name == "pdv_correct" and r.step % 2 == 0):
            holder["c"].read("density1")

    c2 = Chunk(dk.x_cells, dk.y_cells, gamma=dk.gamma)
    holder["c"] = c2
    r2 = HydroRun(c2, dk, fuse_calls=True, dt_ahead=True, probe=probe)
    holder["r"] = r2
    r2.run()
    assert_same(c1, r1, c2, r2)
    launched, used = c2.dt_ahead_stats()
    assert launched == r2.step and used == 0


def test_dt_ahead_fp32_close():
    dk = deck_a()
    c1, r1 = run(dk, FP32)
    c2, r2 = run_ahead(dk, FP32)
    assert r2.step == r1.step
    assert np.allclose(r2.dt_trace, r1.dt_trace, rtol=1e-5, atol=0)
    for f in STATE_FIELDS:
        x, y = c1.read(f), c2.read(f)
        scale = max(np.abs(x).max(), 1e-30)
        assert np.abs(x - y).max() <= 1e-5 * scale, f
