"""The fused paths on meshes with interior tiles, against the oracle.

The fused kernels (the ideal_gas + viscosity + calc_dt pass, the Lagrangian
pass, the advection sweeps) compile a second form of their tile for tiles
that lie away from the mesh edge: no extent checks, no upwind clamp, no halo
fold.  A tile is interior when x0 >= 12 and x0 + 64 <= nx - 8 (and likewise
in y), so only meshes of about 140 cells and more have any; the small decks
of the other run tests never reach that form.  Here:

* config 1 (the reference's clover_bm_short deck: 960^2, 87 steps,
  test_problem 2) through the fused device-resident graph (cb_run, fuse = 1),
  through the host loop with the fused Lagrangian pass (cb_lagrangian),
  through the host loop with call fusion (every fused pass, the x sweeps as
  one pass each), the same with the Lagrangian pass run ahead from calc_dt
  (cb_set_dt_ahead: every pass consumed by its four calls) and through the
  unfused graph: the dt of every step equal to the oracle's, every
  final per-cell field bit-identical to the oracle's, every state field
  (halos included) bit-identical to the phase-by-phase host loop, the
  driver's PASS check, and the summaries within 5e-11 of the reference's
  printed sums (its sequential sum over 921,600 cells carries up to 2.5e-11
  rounding) and within 1e-13 of the exactly rounded sums of the oracle's
  per-cell terms;
* the FP32 form's fused graph on the same deck against the FP64 run: density
  L1 relative error <= 1e-5 (the FP32 form's bound), mass drift <= 1e-6;
* a 200 x 170 deck with a moving circle and gamma 1.55 (interior tiles in
  both directions, ragged edge tiles on the high sides): fused graph and
  cb_lagrangian against the oracle, cell for cell, and against the host loop
  on every state field.
"""
import numpy as np
import pytest

import oracle
from cloverleaf_b200 import FP32, FP64, Chunk, HydroRun
from cloverleaf_b200 import deck as D
from cloverleaf_b200.deck import GEOM_CIRC, GEOM_RECT, Deck, State, nudged
from golden_util import CAPTURED, deck_text, interior, rel, summaries

pytestmark = pytest.mark.gpu

STATE_FIELDS = ("density0", "density1", "energy0", "energy1", "pressure", "viscosity", "soundspeed", "xvel0", "xvel1",
                "yvel0", "yvel1", "vol_flux_x", "vol_flux_y", "mass_flux_x", "mass_flux_y")
KE_TEST_PROBLEM_2 = 1.19316898756307  # driver/report.cpp:79-80


class OracleRun:
    """One whole oracle run of a deck: final per-cell fields, dt sequence,
    summaries and the exact sums of the final state."""

    def __init__(self, dk):
        o = oracle.OracleChunk(dk.x_cells, dk.y_cells, dk.gamma)
        self.recs, self.steps, trace = o.run(dk, dt_trace_len=dk.end_step + 1)
        self.dt = trace[:self.steps]
        self.fields = {fid: np.array(interior(o.field(fid), dk.x_cells, dk.y_cells, kind)) for fid, kind in CAPTURED}
        self.exact = o.field_summary(exact=True)
        o.close()


def run_path(dk, path, precision=FP64):
    c = Chunk(dk.x_cells, dk.y_cells, precision=precision, gamma=dk.gamma)
    r = HydroRun(c, dk, lagrangian=(path == "lagrangian"), fuse_calls=(path in ("fuse_calls", "ahead")), dt_ahead=(path == "ahead"))
    if path in ("host", "lagrangian", "fuse_calls", "ahead"):
        r.run()
        if path == "ahead":  # every step's Lagrangian pass ran ahead and was consumed
            assert c.dt_ahead_stats() == (r.step, r.step)
    else:
        r.start()
        assert r.run_steps_on_device(fuse=(path == "fused"))
    return c, r


def check_against_oracle(dk, ref, c, r, label):
    assert r.step == ref.steps, label
    assert r.dt_trace == ref.dt, label
    for fid, kind in CAPTURED:
        got = interior(c.read(fid), dk.x_cells, dk.y_cells, kind)
        if not np.array_equal(got, ref.fields[fid]):
            bad = np.argwhere(got != ref.fields[fid])
            raise AssertionError(f"{label}: field {fid} differs from the oracle at {len(bad)} points, first {bad[0]}")
    assert len(r.summaries) == len(ref.recs), label
    for s, g in zip(r.summaries, ref.recs):
        assert (s.step, s.time) == (g[0], g[1]), label
    last = r.summaries[-1]
    for a, b in zip((last.vol, last.mass, last.ie, last.ke, last.press), ref.exact):
        assert rel(a, b) <= 1e-13, (label, a, b)


def check_same_state(c1, c2, label):
    for f in STATE_FIELDS:
        x, y = c1.read(f), c2.read(f)
        if not np.array_equal(x.view(np.int64), y.view(np.int64)):
            bad = np.argwhere(x.view(np.int64) != y.view(np.int64))
            raise AssertionError(f"{label}: {f} differs from the host loop at {len(bad)} points, first {bad[0]}")


@pytest.fixture(scope="module")
def config1():
    dk = D.parse_deck(deck_text("bm960x87"))
    ref = OracleRun(dk)
    host = run_path(dk, "host")
    yield dk, ref, host
    host[0].close()


@pytest.mark.slow
@pytest.mark.parametrize("path", ["fused", "lagrangian", "fuse_calls", "ahead", "graph"])
def test_config1_fused_paths_match_oracle(config1, path):
    dk, ref, (ch, rh) = config1
    c, r = run_path(dk, path)
    check_against_oracle(dk, ref, c, r, path)
    check_same_state(ch, c, path)
    ke = r.summaries[-1].ke
    assert abs(100.0 * (ke / KE_TEST_PROBLEM_2) - 100.0) < 0.001  # the driver's PASS check
    gold = summaries("bm960x87")
    assert len(gold) == len(r.summaries)
    for s, g in zip(r.summaries, gold):
        for a, b in zip((s.vol, s.mass, s.ie, s.ke, s.press), g[2:]):
            assert rel(a, b) <= 5e-11, (path, s.step, a, b)
    for a, b in zip(r.summaries, rh.summaries):
        assert a == b, (path, a, b)
    c.close()


def l1_rel(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


@pytest.mark.slow
def test_config1_fp32_fused_within_bound(config1):
    dk, _, (ch, rh) = config1
    c32, r32 = run_path(dk, "fused", FP32)
    assert r32.step == rh.step == 87
    for name, bound in (("density0", 1e-5), ("energy0", 1e-5), ("pressure", 1e-5), ("xvel0", 1e-4), ("yvel0", 1e-4)):
        a64 = ch.read(name)[2:-2, 2:-2]
        a32 = c32.read(name)[2:-2, 2:-2]
        assert np.isfinite(a32).all(), name
        assert l1_rel(a32, a64) <= bound, (name, l1_rel(a32, a64))
    m0 = r32.summaries[0].mass
    for s32 in r32.summaries:
        assert abs(s32.mass - m0) / m0 <= 1e-6, (s32.step, s32.mass, m0)
    assert abs(r32.summaries[-1].ke - KE_TEST_PROBLEM_2) / KE_TEST_PROBLEM_2 <= 1e-4
    c32.close()


def circle_deck():
    """200 x 170 cells, a rectangle and a moving circle, gamma 1.55, 60 steps."""
    dk = Deck(x_cells=200, y_cells=170, xmin=0.0, ymin=0.0, xmax=10.0, ymax=8.5, end_step=60, end_time=10.0, dtinit=0.04,
              dtmax=0.04, dtrise=1.5, summary_frequency=9, gamma=1.55)
    dk.states = [State(density=0.2, energy=1.0, defined=True),
                 State(density=1.0, energy=2.5, geometry=GEOM_RECT, xmin=0.0, xmax=5.0, ymin=0.0, ymax=2.0, defined=True),
                 State(density=1.6, energy=3.2, xvel=0.4, yvel=-0.3, geometry=GEOM_CIRC, xmin=6.0, ymin=5.0, radius=1.7,
                       defined=True)]
    return nudged(dk)


@pytest.fixture(scope="module")
def circle():
    dk = circle_deck()
    ref = OracleRun(dk)
    host = run_path(dk, "host")
    check_against_oracle(dk, ref, *host, "host loop")
    yield dk, ref, host
    host[0].close()


@pytest.mark.parametrize("path", ["fused", "lagrangian", "fuse_calls", "ahead"])
def test_circle_200x170_fused_paths(circle, path):
    dk, ref, (ch, _) = circle
    c, r = run_path(dk, path)
    check_against_oracle(dk, ref, c, r, path)
    check_same_state(ch, c, path)
    c.close()
