"""cb_lagrangian (the PdV predictor, accelerate, the PdV corrector and
flux_calc as one pass) against the four C-ABI calls it replaces, inside whole
runs of the driver's call sequence (HydroRun with lagrangian=True).

FP64: the dt of every step, every summary and every state field (halos
included) are bit-identical.  FP32 is compared within 1e-5 of each field's
largest magnitude: the fused kernel may contract single-precision products
and sums differently.  Without folding (fold off, or a mesh under 8 cells)
the call runs the four phases as their own passes.  A run that switches to
the device-resident loop after fused host steps stays identical too (the
pressure's two buffers are swapped by both).
"""
import numpy as np
import pytest

from cloverleaf_b200 import FP32, FP64, Chunk, HydroRun
from cloverleaf_b200.deck import GEOM_CIRC, GEOM_RECT, Deck, State, benchmark_deck, nudged

pytestmark = pytest.mark.gpu

STATE_FIELDS = ("density0", "density1", "energy0", "energy1", "pressure", "viscosity", "soundspeed", "xvel0", "xvel1",
                "yvel0", "yvel1", "vol_flux_x", "vol_flux_y", "mass_flux_x", "mass_flux_y")


def deck_a(nx=64, ny=48, end_step=30):
    d = benchmark_deck(nx, end_step, end_time=10.0, ny=ny)
    d.summary_frequency = 7
    return nudged(d)


def deck_b(nx=40, ny=56):
    """Moving circle, gamma != 1.4, ends on its time."""
    d = Deck(x_cells=nx, y_cells=ny, xmin=0.0, ymin=0.0, xmax=10.0, ymax=14.0, end_time=0.9, dtinit=0.04,
             dtmax=0.04, dtrise=1.5, summary_frequency=4, gamma=1.55)
    d.states = [State(density=0.2, energy=1.0, defined=True),
                State(density=1.0, energy=2.5, geometry=GEOM_RECT, xmin=0.0, xmax=5.0, ymin=0.0, ymax=3.0, defined=True),
                State(density=1.5, energy=3.0, xvel=0.3, yvel=-0.2, geometry=GEOM_CIRC, xmin=6.0, ymin=8.0, radius=2.0,
                      defined=True)]
    return nudged(d)


def run(dk, precision, lagrangian, fold=True, steps=None):
    c = Chunk(dk.x_cells, dk.y_cells, precision=precision, gamma=dk.gamma)
    r = HydroRun(c, dk, fold=fold, lagrangian=lagrangian)
    r.run(max_steps=steps)
    return c, r


def assert_same(c1, r1, c2, r2):
    assert (r2.step, r2.time, r2.dtold, r2.advect_x) == (r1.step, r1.time, r1.dtold, r1.advect_x)
    assert r2.dt_trace == r1.dt_trace
    assert r2.summaries == r1.summaries
    for f in STATE_FIELDS:
        x, y = c1.read(f), c2.read(f)
        assert np.array_equal(x.view(np.int64), y.view(np.int64)), f


@pytest.mark.parametrize("deck", ["a", "b"])
@pytest.mark.parametrize("fold", [True, False])
def test_lagrangian_fp64_bit_identical(deck, fold):
    dk = deck_a() if deck == "a" else deck_b()
    c1, r1 = run(dk, FP64, False, fold)
    c2, r2 = run(dk, FP64, True, fold)
    assert r1.step > 10
    assert_same(c1, r1, c2, r2)


@pytest.mark.parametrize("nx,ny", [(6, 5), (7, 12), (8, 8), (65, 9)])
def test_lagrangian_small_and_ragged_meshes(nx, ny):
    """Below 8 cells nothing folds (the four passes); 8 x 8 is the smallest fused mesh; 65 x 9 leaves
    one-column and one-row tiles at the high edges."""
    dk = deck_a(nx, ny, end_step=12)
    c1, r1 = run(dk, FP64, False)
    c2, r2 = run(dk, FP64, True)
    assert_same(c1, r1, c2, r2)


def test_lagrangian_fp32_close():
    dk = deck_a()
    c1, r1 = run(dk, FP32, False)
    c2, r2 = run(dk, FP32, True)
    assert r2.step == r1.step == 30
    assert np.allclose(r2.dt_trace, r1.dt_trace, rtol=1e-5, atol=0)
    for f in STATE_FIELDS:
        x, y = c1.read(f), c2.read(f)
        scale = max(np.abs(x).max(), 1e-30)
        assert np.abs(x - y).max() <= 1e-5 * scale, f


def test_lagrangian_launches():
    """Folded, one kernel and the pressure's outer-ring copy replace the four phase kernels."""
    dk = deck_a(48, 48, end_step=6)
    counts = []
    for lag in (False, True):
        c = Chunk(48, 48)
        r = HydroRun(c, dk, lagrangian=lag)
        r.start()
        n0 = c.launch_count()
        for _ in range(6):
            r.hydro_step()
        counts.append(c.launch_count() - n0)
    assert counts[1] == counts[0] - 2 * 6


@pytest.mark.parametrize("fuse", [False, True])
def test_lagrangian_then_device_loop(fuse):
    """Fused host steps leave the pressure in its second buffer; the device-resident loop takes over from there."""
    dk = deck_b()
    c1, r1 = run(dk, FP64, False)
    c2 = Chunk(dk.x_cells, dk.y_cells, gamma=dk.gamma)
    r2 = HydroRun(c2, dk, lagrangian=True)
    r2.start()
    for _ in range(5):
        r2.hydro_step()
    assert r2.run_steps_on_device(fuse=fuse)
    assert_same(c1, r1, c2, r2)


def test_lagrangian_alternating_with_the_four_calls():
    """Steps alternate between cb_lagrangian and the four calls: the pressure's buffer changes every other step."""
    dk = deck_b()
    c1, r1 = run(dk, FP64, False)
    c2 = Chunk(dk.x_cells, dk.y_cells, gamma=dk.gamma)
    r2 = HydroRun(c2, dk)
    r2.start()
    while True:
        r2.lagrangian = r2.step % 2 == 0
        if r2.hydro_step():
            break
    assert_same(c1, r1, c2, r2)


@pytest.mark.parametrize("precision", [FP64, FP32])
def test_lagrangian_depth_one(precision):
    """halo_depth 1: every output folded to depth 1, as the four calls at depth 1 leave them."""
    dk = deck_a(48, 40, end_step=5)
    chunks = []
    for lag in (False, True):
        c = Chunk(dk.x_cells, dk.y_cells, precision=precision, gamma=dk.gamma)
        r = HydroRun(c, dk)
        r.start()
        for _ in range(4):
            r.hydro_step()
        r.timestep()
        if lag:
            c.lagrangian(r.dt, 1)
        else:
            c.pdv(True, r.dt, full=True, halo_depth=1)
            c.accelerate(r.dt, 1)
            c.pdv(False, r.dt, halo_depth=1)
            c.flux_calc(r.dt, 1)
        chunks.append(c)
    for f in STATE_FIELDS:
        x, y = chunks[0].read(f), chunks[1].read(f)
        if precision == FP64:
            assert np.array_equal(x.view(np.int64), y.view(np.int64)), f
        else:
            assert np.abs(x - y).max() <= 1e-5 * max(np.abs(x).max(), 1e-30), f


def test_lagrangian_arguments_rejected():
    from cloverleaf_b200.chunk import CloverError
    c = Chunk(16, 16)
    with pytest.raises(CloverError, match="halo depth"):
        c.lagrangian(0.01, 3)
