"""Call fusion (CB_OPT_FUSE_CALLS): the reference driver's phase calls, made
one by one, run as the library's fused passes -- ideal_gas + viscosity held
back until calc_dt (one pass), the PdV predictor + accelerate + the PdV
corrector until flux_calc (the Lagrangian pass), the second sweeps until
reset_field (which they then do).  Checked against the same calls with the
option off (HydroRun's host loop):

* FP64: the dt of every step, every summary and every state field (halos
  included) bit-identical, on meshes with and without interior tiles, with
  the x or the y sweep first, for runs that end on their step count or time;
* any other call in the middle of a held-back group (a field read, a halo
  pass with work to do, a summary) first runs the group's calls as they were
  made: still bit-identical;
* meshes too small to fold, and folding off, hold nothing back;
* a step launches the fused passes' kernels only (six fewer than unfused);
* FP32 within the FP32 form's rounding (the fused kernels may contract
  single-precision products differently).
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


def run(dk, precision=FP64, fuse_calls=False, fold=True, probe=None):
    c = Chunk(dk.x_cells, dk.y_cells, precision=precision, gamma=dk.gamma)
    r = HydroRun(c, dk, fold=fold, fuse_calls=fuse_calls, probe=probe)
    r.run()
    return c, r


def assert_same(c1, r1, c2, r2):
    assert (r2.step, r2.time, r2.dtold, r2.advect_x) == (r1.step, r1.time, r1.dtold, r1.advect_x)
    assert r2.dt_trace == r1.dt_trace
    assert r2.summaries == r1.summaries
    for f in STATE_FIELDS:
        x, y = c1.read(f), c2.read(f)
        assert np.array_equal(x.view(np.int64), y.view(np.int64)), f


@pytest.mark.parametrize("dk", [deck_a(), deck_b(), deck_a(200, 150, 25)], ids=["bm64x48", "circle40x56", "bm200x150"])
def test_fused_calls_fp64_bit_identical(dk):
    c1, r1 = run(dk)
    c2, r2 = run(dk, fuse_calls=True)
    assert_same(c1, r1, c2, r2)
    c1.close()
    c2.close()


def test_interrupted_groups_run_as_called():
    """A probe reads a field before the calls that complete each group: the
    held-back calls run one by one first, and the result is unchanged."""
    dk = deck_b()
    c1, r1 = run(dk)
    holder = {}

    def probe(name):
        # before viscosity (ideal_gas held), before the corrector (predictor and
        # accelerate held), before the second momentum sweep (cell sweep held)
        if name in ("viscosity", "pdv_correct", "advec_mom_s2"):
            holder["c"].read("pressure")

    c2 = Chunk(dk.x_cells, dk.y_cells, gamma=dk.gamma)
    holder["c"] = c2
    r2 = HydroRun(c2, dk, fuse_calls=True, probe=probe)
    r2.run()
    assert_same(c1, r1, c2, r2)


def test_nothing_held_without_folding():
    for dk, fold in ((deck_a(6, 5, 12), True), (deck_a(), False)):
        c1, r1 = run(dk, fold=fold)
        n1 = c1.launch_count()
        c2, r2 = run(dk, fuse_calls=True, fold=fold)
        assert c2.launch_count() == n1
        assert_same(c1, r1, c2, r2)


def test_fused_calls_launch_count():
    """Per step, unfused: ideal_gas, viscosity, calc_dt, the predictor,
    accelerate, the corrector, flux_calc, four sweeps (the last with its halo
    ring copy) and reset_field = 13 kernels.  Fused: the ideal_gas +
    viscosity + calc_dt pass, the pressure ring copy and the Lagrangian pass,
    four sweeps (+ the ring copy) = 8: five fewer."""
    dk = deck_a(48, 48, 12)
    c1, r1 = run(dk)
    c2, r2 = run(dk, fuse_calls=True)
    assert r1.step == r2.step == 12
    assert c1.launch_count() - c2.launch_count() == 5 * 12


def test_fused_calls_fp32_close():
    dk = deck_a()
    c1, r1 = run(dk, FP32)
    c2, r2 = run(dk, FP32, fuse_calls=True)
    assert r2.step == r1.step
    assert np.allclose(r2.dt_trace, r1.dt_trace, rtol=1e-5, atol=0)
    for f in STATE_FIELDS:
        x, y = c1.read(f), c2.read(f)
        scale = max(np.abs(x).max(), 1e-30)
        assert np.abs(x - y).max() <= 1e-5 * scale, f
