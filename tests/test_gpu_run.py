"""cb_run (the whole hydro loop as one device-resident CUDA graph) against the
host-driven loop of the same chunk (HydroRun.hydro_step through the C ABI).

The graph launches the same phase kernels with dt read from the device, so
the check is exact: the dt of every step, the step count, every summary
record and every state field (halos included) are bit-identical, in both
precisions, with and without halo folding, on meshes too small to fold, when
the run ends on its time or on its step count, when the loop is split into
several graphs, and when the graph takes over a run the host started.

With fuse = 1 the graph runs ideal_gas and viscosity with calc_dt, the PdV
predictor, accelerate, the PdV corrector and flux_calc as one pass and
reset_field inside the second sweeps: FP64 stays bit-identical;
FP32 is compared within 1e-5 (relative to each field's largest magnitude),
because the fused kernels may contract single-precision products and sums
differently.
"""
import numpy as np
import pytest

from cloverleaf_b200 import FP32, FP64, Chunk, HydroRun
from cloverleaf_b200.chunk import CloverError, RunParams, RunState
from cloverleaf_b200.deck import GEOM_CIRC, GEOM_RECT, Deck, State, benchmark_deck, nudged

pytestmark = pytest.mark.gpu

STATE_FIELDS = ("density0", "density1", "energy0", "energy1", "pressure", "viscosity", "soundspeed", "xvel0", "xvel1",
                "yvel0", "yvel1", "vol_flux_x", "vol_flux_y", "mass_flux_x", "mass_flux_y")


def deck_a(nx=64, ny=48, end_step=40, end_time=10.0, freq=7):
    d = benchmark_deck(nx, end_step, end_time=end_time, ny=ny)
    d.summary_frequency = freq
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


def host_run(dk, precision, fold=True, steps=None):
    c = Chunk(dk.x_cells, dk.y_cells, precision=precision, gamma=dk.gamma)
    r = HydroRun(c, dk, fold=fold)
    r.run(max_steps=steps)
    return c, r


def device_run(dk, precision, fold=True, host_steps=0, chunk_steps=4096, steps=None, fuse=False):
    c = Chunk(dk.x_cells, dk.y_cells, precision=precision, gamma=dk.gamma)
    r = HydroRun(c, dk, fold=fold)
    r.start()
    for _ in range(host_steps):
        r.hydro_step()
    done = r.run_steps_on_device(max_steps=steps, chunk_steps=chunk_steps, fuse=fuse)
    return c, r, done


def assert_same(c1, r1, c2, r2):
    assert r2.step == r1.step
    assert r2.time == r1.time
    assert r2.advect_x == r1.advect_x
    assert r2.dtold == r1.dtold
    assert r2.dt_trace == r1.dt_trace
    assert len(r2.summaries) == len(r1.summaries)
    for a, b in zip(r1.summaries, r2.summaries):
        assert a == b, (a, b)
    for f in STATE_FIELDS:
        x, y = c1.read(f), c2.read(f)
        assert np.array_equal(x.view(np.int64), y.view(np.int64)), f


@pytest.mark.parametrize("precision", [FP64, FP32])
@pytest.mark.parametrize("fold", [True, False])
def test_run_matches_host_loop(precision, fold):
    dk = deck_a()
    c1, r1 = host_run(dk, precision, fold)
    c2, r2, done = device_run(dk, precision, fold)
    assert done and r1.step == 40
    assert_same(c1, r1, c2, r2)


@pytest.mark.parametrize("precision", [FP64, FP32])
def test_run_ends_on_time(precision):
    dk = deck_b()
    c1, r1 = host_run(dk, precision)
    c2, r2, done = device_run(dk, precision)
    assert done and r1.time + 1e-16 > dk.end_time and r1.step < dk.end_step
    assert_same(c1, r1, c2, r2)


def test_run_split_into_graphs_and_taken_over():
    dk = deck_b()
    c1, r1 = host_run(dk, FP64)
    c2, r2, _ = device_run(dk, FP64, host_steps=5, chunk_steps=6)
    assert_same(c1, r1, c2, r2)
    # a max_steps bound stops the device loop where the host loop's bound stops
    c3, r3 = host_run(dk, FP64, steps=11)
    c4, r4, done = device_run(dk, FP64, steps=11)
    assert not done and r4.step == 11
    assert_same(c3, r3, c4, r4)


@pytest.mark.parametrize("nx,ny", [(6, 5), (7, 12)])
def test_run_small_mesh_unfolded(nx, ny):
    """Meshes below 8 cells do not fold: every update_halo is its own pass inside the graph."""
    dk = deck_a(nx, ny, end_step=15, freq=4)
    c1, r1 = host_run(dk, FP64)
    c2, r2, _ = device_run(dk, FP64)
    assert_same(c1, r1, c2, r2)


def test_run_small_timestep_reports():
    dk = deck_a(32, 32, end_step=10)
    dk.dtmin = 1.0  # every dt is below it
    c = Chunk(32, 32)
    r = HydroRun(c, dk)
    r.start()
    with pytest.raises(CloverError, match="small timestep"):
        r.run_steps_on_device()
    assert r.step == 1


def test_run_arguments_rejected():
    c = Chunk(16, 16)
    p = RunParams(1e-7, 0.04, 1.5, 0.7, 0.5, 0.5, 0.7, 1.0, 10, 0, 1, 0)
    st = RunState(0, 1, 0.0, 0.04, 0.04, 0)
    with pytest.raises(CloverError, match="max_steps"):
        c.run(p, st, 0)
    bad = RunState(0, 1, 0.0, 0.0, 0.04, 0)
    with pytest.raises(CloverError, match="dtold"):
        c.run(p, bad, 3)


def test_run_launch_count():
    """The graph counts its kernels: the host loop's phase launches (the first
    step's mass-flux halo pass runs before the loop) plus the loop's own
    scalar kernels: 1 to start, 3 per step, 1 per summary."""
    dk = deck_a(48, 48, end_step=12, freq=5)  # summaries at steps 5, 10 and 12
    counts = []
    for device in (False, True):
        c = Chunk(48, 48)
        r = HydroRun(c, dk)
        r.start()
        n0 = c.launch_count()
        if device:
            r.run_steps_on_device()
        else:
            while not r.hydro_step():
                pass
        counts.append(c.launch_count() - n0)
        assert r.step == 12 and len(r.summaries) == 4
    assert counts[1] == counts[0] + 1 + 3 * 12 + 3


@pytest.mark.parametrize("deck", ["a", "b"])
def test_run_fused_fp64_bit_identical(deck):
    dk = deck_a() if deck == "a" else deck_b()
    c1, r1 = host_run(dk, FP64)
    c2, r2, done = device_run(dk, FP64, fuse=True)
    assert done
    assert_same(c1, r1, c2, r2)


def test_run_fused_fp64_split_and_taken_over():
    dk = deck_b()
    c1, r1 = host_run(dk, FP64)
    c2, r2, _ = device_run(dk, FP64, host_steps=3, chunk_steps=5, fuse=True)
    assert_same(c1, r1, c2, r2)


def test_run_fused_fp32_close():
    dk = deck_a()  # ends on its step count
    c1, r1 = host_run(dk, FP32)
    c2, r2, done = device_run(dk, FP32, fuse=True)
    assert done and r2.step == r1.step == 40
    assert np.allclose(r2.dt_trace, r1.dt_trace, rtol=1e-5, atol=0)
    for a, b in zip(r1.summaries, r2.summaries):
        assert a.step == b.step
        for q in ("vol", "mass", "ie", "ke", "press"):
            assert abs(getattr(a, q) - getattr(b, q)) <= 1e-5 * abs(getattr(a, q)), (q, a, b)
    for f in STATE_FIELDS:
        x, y = c1.read(f), c2.read(f)
        scale = max(np.abs(x).max(), 1e-30)
        assert np.abs(x - y).max() <= 1e-5 * scale, f


@pytest.mark.parametrize("nx,ny,fold", [(6, 5, True), (64, 48, False)])
def test_run_fused_falls_back(nx, ny, fold):
    """Without folding producers (small meshes, or fold off) fuse = 1 runs the unfused step."""
    dk = deck_a(nx, ny, end_step=12, freq=4)
    c1, r1 = host_run(dk, FP64, fold=fold)
    c2, r2, _ = device_run(dk, FP64, fold=fold, fuse=True)
    assert_same(c1, r1, c2, r2)


def test_run_fused_launch_count():
    """Fused, a step launches seven kernels fewer: ideal_gas, viscosity, accelerate, the PdV corrector, flux_calc and
    reset_field run inside others, and the second momentum sweep, writing level 0 only, copies no halo ring; once per
    run, four launches restore energy1, xvel1 and yvel1 (the level-1 values the fused second sweeps skip)."""
    dk = deck_a(48, 48, end_step=12, freq=5)
    counts = []
    for fuse in (False, True):
        c = Chunk(48, 48)
        r = HydroRun(c, dk)
        r.start()
        n0 = c.launch_count()
        r.run_steps_on_device(fuse=fuse)
        counts.append(c.launch_count() - n0)
    assert counts[1] == counts[0] - 7 * 12 + 4


@pytest.mark.parametrize("fuse", [False, True], ids=["unfused", "fused"])
def test_kept_graph_follows_the_chunk(fuse):
    """cb_run keeps its instantiated graph for the next run on the chunk and
    launches it again only when the chunk is as the graph was captured for:
    runs of a few steps each, with gamma changed between two of them (the
    pressure's factor is baked into the launches) and a phase-by-phase step
    in between (which moves the double-buffered fields to other buffers),
    end bit-identical to the host-driven loop making the same changes."""
    dk = deck_b()

    def host_then(r, c, steps):
        for _ in range(steps):
            r.hydro_step()

    c1 = Chunk(dk.x_cells, dk.y_cells, gamma=dk.gamma)
    r1 = HydroRun(c1, dk)
    r1.start()
    host_then(r1, c1, 6)
    c1.set_gamma(1.62)
    host_then(r1, c1, 7)

    c2 = Chunk(dk.x_cells, dk.y_cells, gamma=dk.gamma)
    r2 = HydroRun(c2, dk)
    r2.start()
    r2.hydro_step()  # a settled halo state for the graph
    r2.run_steps_on_device(max_steps=3, fuse=fuse)
    r2.run_steps_on_device(max_steps=6, fuse=fuse)  # the kept graph again
    c2.set_gamma(1.62)
    r2.run_steps_on_device(max_steps=9, fuse=fuse)  # captured anew: gamma changed
    r2.hydro_step()  # the double-buffered fields now live in other buffers
    r2.run_steps_on_device(max_steps=13, fuse=fuse)  # captured anew: another buffer map
    assert_same(c1, r1, c2, r2)
    c1.close()
    c2.close()
