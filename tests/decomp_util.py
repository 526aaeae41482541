"""Test infrastructure for decomposed runs: one rank's chunk held by the CPU
oracle, with the chunk calls a HydroRun makes (the counterpart of
cloverleaf_b200.decomp.DecomposedChunk, which holds it on a GPU), and the
rank body both the CPU and the GPU tests spawn.

A decomposed run is not the whole mesh's run in every deck: each chunk's
advec_cell clamps the upwind cell at its own right / top edge face
(src/serial/advec_cell.cpp:77, :169), which a single chunk does only at the
mesh's edges, and the two chunks of a shared face each compute that face's
flux (and the shared vertices' velocities) for themselves.  Where the flow
crosses a chunk edge against the clamp the two runs part; the decomposed
run on oracle chunks is then the reference for the library's.

The oracle chunk's geometry is the reference's for a chunk of a decomposed
grid (src/serial/initialise_chunk.cpp:30-85 with t_left / t_bottom the
chunk's first global cell): the same operations in the same order as the
library's cb_initialise_chunk_in.  The PdV predictor is taken apart as
src/serial/PdV.cpp:92-133 does it (kernel, ideal_gas on level 1, the
pressure halo, revert), so that its pressure halo is an exchange too.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)

from cloverleaf_b200 import decomp as DC  # noqa: E402

VOLUME, XAREA, YAREA = 22, 23, 24


class OracleDecomposedChunk:
    def __init__(self, info, deck, group=None):
        import oracle
        self.info, self.deck, self.group = info, deck, group
        self.o = oracle.OracleChunk(info.nx, info.ny, deck.gamma)
        self.faces = 0
        for side, bit in ((DC.LEFT, 1), (DC.RIGHT, 2), (DC.BOTTOM, 4), (DC.TOP, 8)):
            if info.neighbours[side] < 0:
                self.faces |= bit

    def set_option(self, *_):
        pass

    def build_field(self):
        self.o.build_field()

    def initialise_chunk(self, xmin, ymin, xmax, ymax):
        o, d, i = self.o, self.deck, self.info
        o.initialise_chunk(xmin, ymin, xmax, ymax)  # array shapes; the values are replaced below
        dx = (xmax - xmin) / float(d.x_cells)
        dy = (ymax - ymin) / float(d.y_cells)
        x0 = xmin + dx * float(i.left - 1)
        y0 = ymin + dy * float(i.bottom - 1)
        vx, vy = o.geom("vertexx"), o.geom("vertexy")
        nvx, nvy = i.nx + 6, i.ny + 6  # (x_max + 3) - (x_min - 2) + 1 with x_min = 1
        for j in range(nvx):
            vx[j] = x0 + dx * float(j - 1 - 1)
        for k in range(nvy):
            vy[k] = y0 + dy * float(k - 1 - 1)
        o.geom("vertexdx")[:nvx] = dx
        o.geom("vertexdy")[:nvy] = dy
        cx, cy = o.geom("cellx"), o.geom("celly")
        for j in range(nvx - 1):
            cx[j] = 0.5 * (vx[j] + vx[j + 1])
        for k in range(nvy - 1):
            cy[k] = 0.5 * (vy[k] + vy[k + 1])
        o.geom("celldx")[:nvx - 1] = dx
        o.geom("celldy")[:nvy - 1] = dy
        o.field(VOLUME)[...] = dx * dy
        o.field(XAREA)[...] = dy
        o.field(YAREA)[...] = dx

    def generate_chunk(self, _states):
        self.o.generate_chunk(self.deck)

    def ideal_gas(self, predict, halo_depth=0):
        self.o.ideal_gas(predict)

    def viscosity(self, halo_depth=0):
        self.o.viscosity()

    def calc_dt(self, *args):
        dt, control, jldt, kldt, small = self.o.calc_dt(*args)
        return DC.dt_min(dt, self.group), control, jldt, kldt, small

    def pdv(self, predict, dt, full=False, halo_depth=0):
        if full:  # src/serial/PdV.cpp:92-133
            self.o.pdv_kernel(True, dt)
            self.o.ideal_gas(True)
            self.update_halo([4], 1)  # pressure
            self.o.revert()
        else:
            self.o.pdv_kernel(predict, dt)

    def accelerate(self, dt, halo_depth=0):
        self.o.accelerate(dt)

    def flux_calc(self, dt, halo_depth=0):
        self.o.flux_calc(dt)

    def advec_cell(self, sweep, direction, halo_depth=0):
        self.o.advec_cell(sweep, direction)

    def advec_mom(self, vel_mask, sweep, direction, halo_depth=0):
        # the reference's two calls, x velocity then y (driver/advection.cpp:56-57, :85-86)
        if vel_mask & 1:
            self.o.advec_mom(1, sweep, direction)
        if vel_mask & 2:
            self.o.advec_mom(2, sweep, direction)

    def reset_field(self, halo_depth=0):
        self.o.reset_field()

    def update_halo(self, fields, depth):
        fids = sorted(set(int(f) for f in fields))
        if any(n >= 0 for n in self.info.neighbours):
            arrays = {f: self.o.field(f) for f in fids}  # views of the oracle's arrays
            DC.exchange(self.info, arrays, fids, depth, self.group)
        self.o.update_halo([1 if f in fids else 0 for f in range(15)], depth, self.faces)

    def field_summary(self):
        return tuple(DC.summary_sum(self.o.field_summary(), self.group))

    def read(self, f):
        return np.array(self.o.field(f))

    def close(self):
        self.o.close()


CAPTURED = (0, 2, 4, 5, 6, 7, 9, 11, 12, 13, 14)  # density0, energy0, pressure, viscosity, soundspeed, xvel0, yvel0, fluxes


def window(info, a, fid):
    """The interior of chunk `info` in a whole-mesh array of field fid (halo 2)."""
    xe, ye = DC.EXTRA[fid]
    return a[2 + info.bottom - 1:2 + info.bottom - 1 + info.ny + ye, 2 + info.left - 1:2 + info.left - 1 + info.nx + xe]


def own(info, a, fid):
    xe, ye = DC.EXTRA[fid]
    return a[2:2 + info.ny + ye, 2:2 + info.nx + xe]


def deck_for(name):
    from cloverleaf_b200.deck import GEOM_CIRC, GEOM_RECT, State, benchmark_deck, nudged, parse_deck
    if name.startswith("sod"):  # the reference's own Sod decks (golden fixtures); the 200^2 one cut to 200 steps
        from golden_util import deck_text
        dk = parse_deck(deck_text(name))
        if name == "sodbig200":
            dk.end_step = 200
        return dk
    if name == "bm":
        dk = benchmark_deck(64, 24, end_time=10.0, ny=48)
    else:
        dk = benchmark_deck(56, 40, end_time=10.0, ny=40)
        dk.summary_frequency = 7
        dk.gamma = 1.55
        dk.states = [State(density=0.2, energy=1.0, defined=True),
                     State(density=1.0, energy=2.5, geometry=GEOM_RECT, xmin=0.0, xmax=4.1, ymin=0.0, ymax=3.1, defined=True),
                     State(density=1.6, energy=3.0, xvel=0.3, yvel=-0.2, geometry=GEOM_CIRC, xmin=6.3, ymin=5.2, radius=2.1,
                           defined=True)]
    return nudged(dk)


def compare(info, mine, ref, ref_is_whole):
    """Captured fields of this chunk that differ from the reference run's: as
    (field id, cells) pairs; with ref_is_whole the reference is the whole
    mesh and this chunk's window of it is compared."""
    bad = []
    for f in CAPTURED:
        a = own(info, mine.read(f), f)
        b = window(info, np.array(ref.field(f)), f) if ref_is_whole else own(info, ref.read(f), f)
        if not np.array_equal(a, b):
            bad.append((f, int((a != b).sum())))
    return bad


def rank_body(rank, world, port, out, deck_name, on_gpu, mode="plain"):
    """One rank of a decomposed run of deck `deck_name` ("bm" or "circle").

    on_gpu False: the chunk is held by the oracle and the run is compared with
    the whole mesh's oracle run.  on_gpu True: the chunk is held by the
    library (DecomposedChunk on cuda:0) and the run is compared with the same
    decomposed run on oracle chunks; mode "fold" passes HydroRun's halo depths
    to the calls and "fuse" turns the chunk's call fusion on as well (a chunk
    with an internal face folds no halo, so both must give the same run).  Every captured field of the chunk, the
    step count and the dt of every step must agree to the bit; the final
    summary's sums within 1e-13 (relative) of the exactly rounded sums of the
    reference run's per-cell terms (the whole mesh's, or the oracle chunks'
    reduced over the ranks)."""
    import datetime

    import torch.distributed as dist
    import oracle
    from cloverleaf_b200 import HydroRun

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    dk = deck_for(deck_name)
    info = DC.decompose(dk.x_cells, dk.y_cells, world)[rank]
    c = OracleDecomposedChunk(info, dk)
    r = HydroRun(c, dk, fold=False)
    r.run()
    if on_gpu:
        ref, ref_r = c, r
        c = DC.DecomposedChunk(info, dk)
        r = HydroRun(c, dk, fold=mode != "plain", fuse_calls=mode == "fuse")
        r.run()
        res = {"steps": (r.step, ref_r.step), "dt": r.dt_trace == ref_r.dt_trace,
               "bad": compare(info, c, ref, False),
               "summary_steps": [(s.step, s.time) for s in r.summaries] == [(s.step, s.time) for s in ref_r.summaries]}
        # the oracle chunks' exactly rounded sums, reduced over the ranks (their
        # sequential sums carry their own rounding, which grows with the chunk)
        got, want = r.summaries[-1], DC.summary_sum(ref.o.field_summary(exact=True), None)
    else:
        g = oracle.OracleChunk(dk.x_cells, dk.y_cells, dk.gamma)
        recs, steps, trace = g.run(dk, dt_trace_len=dk.end_step + 1)
        res = {"steps": (r.step, steps), "dt": r.dt_trace == list(trace[:steps]), "bad": compare(info, c, g, True),
               "summary_steps": [(s.step, s.time) for s in r.summaries] == [(q[0], q[1]) for q in recs]}
        got, want = r.summaries[-1], g.field_summary(exact=True)
        g.close()
        ref = None
    res["sums"] = [abs(a - b) / abs(b) for a, b in zip((got.vol, got.mass, got.ie, got.ke, got.press), want)]
    c.close()
    if ref is not None:
        ref.close()
    out[rank] = res
    dist.barrier()
    dist.destroy_process_group()
