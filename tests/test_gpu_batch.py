"""The batched ensemble on the GPU against sequential single-deck runs.

Every deck of a batch is advanced by one persistent launch; the check is the
same deck run on its own through the C ABI in the driver's call order
(HydroRun on a Chunk of the same precision and gamma):
* the dt of every step and the step count are identical;
* every final cell and node field is bit-identical (xvel1/yvel1 on their
  interior: the batch does not copy the untouched halo ring of the last
  momentum sweep, which no later phase reads);
* summaries: identical steps and times, sums within 1e-13 relative (the
  batch's reduction groups the same per-cell terms differently).
For gamma != 1.4 the batch is also checked against the CPU oracle, which
takes gamma as a parameter.
"""
import numpy as np
import pytest

import oracle
from cloverleaf_b200 import FP32, FP64, Batch, Chunk, HydroRun
from cloverleaf_b200 import batch as B
from cloverleaf_b200.deck import GEOM_CIRC, GEOM_POINT, GEOM_RECT, Deck, State, nudged

pytestmark = pytest.mark.gpu

CELL_FIELDS = ("density0", "energy0", "pressure", "soundspeed", "viscosity", "density1", "energy1", "mass_flux_x",
               "mass_flux_y", "vol_flux_x", "vol_flux_y", "xvel0", "yvel0")


def vertex(dk, i, j):
    """The coordinates of vertex (i, j) (0-based array index, halo included)
    as the mesh set-up forms them: a point state paints the cell whose
    low-left vertex equals its point exactly (src/serial/generate_chunk.cpp:116-126)."""
    o = oracle.OracleChunk(dk.x_cells, dk.y_cells)
    o.build_field()
    o.initialise_chunk(dk.xmin, dk.ymin, dk.xmax, dk.ymax)
    x, y = float(o.geom("vertexx")[i]), float(o.geom("vertexy")[j])
    o.close()
    return x, y


def with_point(dk, density, energy, xvel, yvel, i, j):
    """Appends a point state at vertex (i, j); the deck is already nudged, so
    the point is set after the nudge (the reader would move it off the vertex)."""
    x, y = vertex(dk, i, j)
    dk.states.append(State(density=density, energy=energy, xvel=xvel, yvel=yvel, geometry=GEOM_POINT, xmin=x, ymin=y,
                           defined=True))
    return dk


def mixed_decks():
    """Uneven meshes (8 cells up to 130), gamma, rectangles, circles and
    points, moving states; three-state decks."""
    rng = np.random.default_rng(7)
    sizes = [(8, 8), (13, 9), (40, 24), (64, 64), (96, 40), (130, 70), (17, 33), (70, 130), (24, 24), (9, 57)]
    out = []
    for k, (nx, ny) in enumerate(sizes):
        dk = Deck(x_cells=nx, y_cells=ny, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0 * ny / nx, end_time=0.6,
                  dtinit=0.04, dtmax=0.04, dtrise=1.5, summary_frequency=3 + k % 4, gamma=float(rng.uniform(1.3, 1.67)))
        dk.states = [State(density=0.2, energy=1.0, defined=True),
                     State(density=float(rng.uniform(0.5, 2.0)), energy=float(rng.uniform(1.0, 4.0)), geometry=GEOM_RECT,
                           xmin=0.0, xmax=float(rng.uniform(2, 8)), ymin=0.0, ymax=float(rng.uniform(1, 5)) * ny / nx,
                           defined=True)]
        if k % 3 == 1:
            dk.states.append(State(density=1.5, energy=3.0, xvel=0.3, yvel=-0.2, geometry=GEOM_CIRC, xmin=6.0,
                                   ymin=3.0 * ny / nx, radius=1.5, defined=True))
        if k == 4:
            dk.end_step, dk.end_time = 9, 10.0  # ends on its step count
        dk = nudged(dk)
        if k % 3 == 2:  # background, rectangle and a moving point: three states
            with_point(dk, 3.0, 2.0, 0.2 * (k % 2) - 0.1, 0.15, 2 + nx // 2, 2 + (2 * ny) // 3)
        out.append(dk)
    return out


def sequential(dk, precision):
    c = Chunk(dk.x_cells, dk.y_cells, precision=precision, gamma=dk.gamma)
    r = HydroRun(c, dk)
    r.run()
    return c, r


def check_deck(b, k, c, r):
    res = b.result(k)
    assert res.status == B.DECK_DONE, (k, res)
    assert res.steps == r.step, (k, res.steps, r.step)
    assert b.dt_trace(k) == r.dt_trace, k
    assert abs(res.time - r.time) == 0.0, k
    bs = b.summaries(k)
    assert [(s.step, s.time) for s in bs] == [(s.step, s.time) for s in r.summaries], k
    for s, t in zip(bs, r.summaries):
        for x, y in ((s.vol, t.vol), (s.mass, t.mass), (s.ie, t.ie), (s.ke, t.ke), (s.press, t.press)):
            assert abs(x - y) <= 1e-13 * max(abs(y), 1e-300), (k, s.step, x, y)
    for name in CELL_FIELDS:
        x, y = b.read(k, name), c.read(name)
        assert np.array_equal(x, y), (k, name, np.argwhere(x != y)[:3])
    for name in ("xvel1", "yvel1"):
        x, y = b.read(k, name), c.read(name)
        assert np.array_equal(x[2:-2, 2:-2], y[2:-2, 2:-2]), (k, name)


def large_decks():
    """The ensemble's largest sides, 256 and 384 cells (tiles away from the
    mesh edge, which smaller decks do not have), one of them with four states
    (rectangle, circle, point), plus a 192 x 320 deck."""
    out = []
    for k, (nx, ny) in enumerate([(256, 256), (384, 384), (192, 320)]):
        dk = Deck(x_cells=nx, y_cells=ny, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0 * ny / nx, end_time=0.5,
                  dtinit=0.04, dtmax=0.04, dtrise=1.5, summary_frequency=5, gamma=1.4 + 0.1 * k)
        dk.states = [State(density=0.2, energy=1.0, defined=True),
                     State(density=1.2 + 0.3 * k, energy=2.0 + k, geometry=GEOM_RECT, xmin=0.0, xmax=4.0 + k,
                           ymin=0.0, ymax=2.5, defined=True)]
        if k != 1:
            dk.states.append(State(density=1.5, energy=3.0, xvel=0.3, yvel=-0.2, geometry=GEOM_CIRC, xmin=6.5,
                                   ymin=6.0 * ny / nx, radius=1.4, defined=True))
        dk = nudged(dk)
        if k == 0:
            with_point(dk, 4.0, 3.5, -0.2, 0.25, 2 + 3 * nx // 4, 2 + nx // 3)
        out.append(dk)
    return out


def test_batch_large_decks_match_sequential_fp64():
    decks = large_decks()
    seq = [sequential(dk, FP64) for dk in decks]
    with Batch(decks, FP64) as b:
        b.set_schedule(cells_per_cta=4096, variant=1)
        sched, lanes, ctas = b.schedule()
        assert ctas > lanes  # the large decks run on lanes of several CTAs
        b.run()
        b.synchronize()
        for k, (c, r) in enumerate(seq):
            check_deck(b, k, c, r)
    for c, _ in seq:
        c.close()


@pytest.fixture(scope="module")
def decks():
    return mixed_decks()


@pytest.fixture(scope="module")
def seq64(decks):
    out = [sequential(dk, FP64) for dk in decks]
    yield out
    for c, _ in out:
        c.close()


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("cells_per_cta", [1 << 30, 2048, 512])
def test_batch_matches_sequential_fp64(decks, seq64, variant, cells_per_cta):
    with Batch(decks, FP64) as b:
        b.set_schedule(cells_per_cta=cells_per_cta, variant=variant)
        sched, lanes, ctas = b.schedule()
        # lanes: grid / W summed over the widths W the decks use
        if cells_per_cta == 1 << 30:
            assert lanes == ctas  # every deck on a lane of one CTA
        if cells_per_cta == 512:
            assert lanes > ctas  # lanes of one CTA and lanes of several
        b.run()
        ms = b.synchronize()
        assert ms > 0.0
        for k, (c, r) in enumerate(seq64):
            check_deck(b, k, c, r)


def test_batch_matches_sequential_fp32(decks):
    """The FP32 form is built with multiply-add contraction, which the
    compiler applies per inlined context: the batch kernel and the one-launch
    kernels may round a few products differently.  So the FP32 batch is held
    to the FP32 form's own error scale against the FP32 sequential run: the
    same step count, dt within 1e-5, fields within 1e-6 L1 relative."""
    with Batch(decks, FP32) as b:
        b.set_schedule(cells_per_cta=1024, variant=1)
        b.run()
        b.synchronize()
        for k, dk in enumerate(decks):
            c, r = sequential(dk, FP32)
            res = b.result(k)
            assert res.status == B.DECK_DONE and res.steps == r.step, (k, res, r.step)
            assert np.allclose(b.dt_trace(k), r.dt_trace, rtol=1e-5, atol=0.0), k
            bs = b.summaries(k)
            assert [s.step for s in bs] == [s.step for s in r.summaries], k
            for s, t in zip(bs, r.summaries):
                for x, y in ((s.mass, t.mass), (s.ie, t.ie), (s.ke + s.ie, t.ke + t.ie)):
                    assert abs(x - y) <= 1e-6 * abs(y), (k, s.step, x, y)
            for name in ("density0", "energy0", "pressure", "xvel0", "yvel0"):
                x, y = b.read(k, name)[2:-2, 2:-2], c.read(name)[2:-2, 2:-2]
                assert np.abs(x - y).sum() <= 1e-6 * np.abs(y).sum(), (k, name)
            c.close()


def test_batch_runs_again_from_the_start(decks, seq64):
    """A second launch of the captured run starts every deck from t = 0 again."""
    with Batch(decks[:4], FP64) as b:
        b.run()
        b.synchronize()
        b.run()
        b.synchronize()
        for k in range(4):
            check_deck(b, k, *seq64[k])
        assert b.launch_count() == 2


@pytest.mark.parametrize("gamma", [1.3, 1.5, 1.67])
def test_batch_gamma_against_oracle(gamma):
    dk = nudged(Deck(x_cells=20, y_cells=14, xmin=0.0, ymin=0.0, xmax=10.0, ymax=7.0, end_step=25, dtinit=0.04,
                     dtmax=0.04, dtrise=1.5, summary_frequency=5, gamma=gamma,
                     states=[State(density=0.2, energy=1.0, defined=True),
                             State(density=1.3, energy=3.1, geometry=GEOM_RECT, xmin=0.0, xmax=4.2, ymin=0.0, ymax=2.3,
                                   defined=True)]))
    with Batch([dk], FP64) as b:
        b.run()
        b.synchronize()
        o = oracle.OracleChunk(dk.x_cells, dk.y_cells, gamma)
        recs, steps, trace = o.run(dk, dt_trace_len=dk.end_step)
        assert b.result(0).steps == steps
        assert b.dt_trace(0) == trace[:steps]
        for s, g in zip(b.summaries(0), recs):
            assert (s.step, s.time) == (g[0], g[1])
            for x, y in zip((s.vol, s.mass, s.ie, s.ke, s.press), g[2:]):
                assert abs(x - y) <= 1e-13 * abs(y), (s.step, x, y)
        for name in ("density0", "energy0", "pressure", "xvel0", "yvel0"):
            got = b.read(0, name)
            ref = np.asarray(o.field(name))[:got.shape[0], :got.shape[1]]
            assert np.array_equal(got[2:-2, 2:-2], ref[2:-2, 2:-2]), name


def test_small_timestep_stops_only_that_deck(decks):
    bad = nudged(decks[3])
    bad.dtmin = 1.0  # every dt is below it: the deck stops at its first step
    ds = [decks[0], bad, decks[2]]
    with Batch(ds, FP64) as b:
        b.run()
        b.synchronize()
        assert b.result(1).status == B.DECK_SMALL_DT
        assert b.result(1).steps == 1
        assert b.result(0).status == B.DECK_DONE and b.result(2).status == B.DECK_DONE


def test_autotune_picks_the_fastest(decks):
    with Batch(decks, FP64) as b:
        best, log = b.autotune(repeats=1)
        assert len(log) == 14  # cells per CTA 1024 .. 65536 (7 values) x two tile variants
        fastest = min(log, key=lambda t: t["ms"])
        assert best == fastest["schedule"]
        b.run()
        b.synchronize()
        assert all(b.result(k).status == B.DECK_DONE for k in range(len(decks)))


def test_batch_runs_the_golden_decks_as_the_reference_does():
    """One batch of the golden decks the reference build ran (the reference's
    own Sod decks InputDecks/clover_sodxy.in, 10 x 10, and clover_sodbig.in,
    200^2 over 1,330 steps, with the benchmark and moving-circle decks):
    every final field the fixtures hold bit for bit the reference's, every
    summary at the reference's steps and times with sums within 1e-12 of
    its printed ones (its sums are sequential, the batch's a reduction)."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from cloverleaf_b200 import deck as D
    from golden_util import CAPTURED, GOLDEN, deck_text, fields, interior, rel, summaries
    names = ["sodxy10x10", "bm32x87", "bm40x24x120", "circ24x20x70", "sodbig200"]
    decks = [D.parse_deck(deck_text(n)) for n in names]
    with Batch(decks, FP64) as b:
        b.run()
        b.synchronize()
        for k, (name, dk) in enumerate(zip(names, decks)):
            gold = summaries(name)
            got = b.summaries(k)
            assert [(s.step, s.time) for s in got] == [(g[0], g[1]) for g in gold], name
            for s, g in zip(got, gold):
                for x, y in zip((s.vol, s.mass, s.ie, s.ke, s.press), g[2:]):
                    assert rel(x, y) <= 1e-12, (name, s.step, x, y)
            if os.path.exists(os.path.join(GOLDEN, name + ".fields.bin")):
                gf = fields(name)
                for fid, kind in CAPTURED:
                    assert np.array_equal(interior(b.read(k, fid), dk.x_cells, dk.y_cells, kind), gf[fid]), (name, fid)
