"""The hydro time loop over a `Chunk`, in the call order of the reference's
unchanged driver: driver/start.cpp:43-138, driver/hydro.cpp:46-223,
driver/timestep.cpp:37-109, driver/advection.cpp:29-105 and the model's
PdV driver src/serial/PdV.cpp:92-133.

It makes the same sequence of C-ABI calls as the C++ model glue under
cloverleaf_b200/model/ (which serves the reference's own C++ driver), so
Python tests and the benchmark exercise the same path.  With ``fold=True``
each producer writes the halo the next update_halo needs and those
update_halo calls become no-ops; with ``fold=False`` every update_halo runs
as its own pass, exactly like the reference.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, List, Optional

from .chunk import OPT_FUSE_CALLS, Chunk, RunParams, RunState
from .deck import G_SMALL, G_BIG, Deck

D0, D1, E0, E1, P, Q, C, U0, U1, V0, V1, VFX, VFY, MFX, MFY = range(15)


@dataclasses.dataclass
class Summary:
    step: int
    time: float
    vol: float
    mass: float
    ie: float
    ke: float
    press: float


class HydroRun:
    """State of one run: globals.step, time, dt, dtold, advect_x (driver/definitions.h:258-280)."""

    def __init__(self, chunk: Chunk, deck: Deck, fold: bool = True, forced_dt: Optional[List[float]] = None,
                 probe: Optional[Callable[[str], None]] = None, lagrangian: bool = False, fuse_calls: bool = False,
                 dt_ahead: bool = False):
        self.c = chunk
        self.deck = deck
        self.fold = fold
        # fuse_calls: the same calls, with the chunk's call fusion on (the
        # library runs ideal_gas + viscosity + calc_dt, the four Lagrangian
        # calls, and the second sweeps + reset_field as its fused passes)
        chunk.set_option(OPT_FUSE_CALLS, int(fuse_calls))
        # lagrangian: the PdV / accelerate / PdV / flux_calc calls as one cb_lagrangian call
        self.lagrangian = lagrangian
        # dt_ahead: each calc_dt also runs the Lagrangian pass ahead with this
        # loop's dt clamp (cb_set_dt_ahead; with fuse_calls), and the four
        # Lagrangian calls find it done
        self.dt_ahead = dt_ahead
        # forced_dt replays a recorded dt sequence (calc_dt still runs); probe(name)
        # is called as each phase is about to be enqueued ("end" closes a step)
        self.forced_dt = forced_dt
        self.probe = probe
        self.step = 0
        self.time = 0.0
        self.dt = deck.dtinit
        self.dtold = deck.dtinit
        self.advect_x = True
        self.summaries: List[Summary] = []
        self.dt_trace: List[float] = []

    def _depth(self, d: int) -> int:
        return d if self.fold else 0

    def _mark(self, name: str):
        if self.probe is not None:
            self.probe(name)

    # driver/start.cpp:43-138
    def start(self):
        c, d = self.c, self.deck
        c.build_field()
        c.initialise_chunk(d.xmin, d.ymin, d.xmax, d.ymax)
        c.generate_chunk(d.states)
        c.ideal_gas(False)
        c.update_halo([D0, E0, P, Q, D1, E1, U0, V0, U1, V1], 2)
        self.field_summary()

    def field_summary(self):
        s = self.c.field_summary()
        self.summaries.append(Summary(self.step, self.time, *s))

    # driver/timestep.cpp:37-109
    def timestep(self):
        c, d = self.c, self.deck
        self.dt = G_BIG
        self._mark("ideal_gas")
        c.ideal_gas(False, self._depth(1))
        c.update_halo([P, E0, D0, U0, V0], 1)
        self._mark("viscosity")
        c.viscosity(self._depth(1))
        c.update_halo([Q], 1)
        self._mark("calc_dt")
        if self.dt_ahead and self.forced_dt is None:
            c.set_dt_ahead(self.dtold, d.dtrise, d.dtmax)
        dtlp, control, jldt, kldt, small = c.calc_dt(d.dtmin, d.dtc_safe, d.dtu_safe, d.dtv_safe, d.dtdiv_safe)
        if self.forced_dt is not None:
            dtlp = self.forced_dt[self.step - 1]
        if dtlp <= self.dt:
            self.dt = dtlp
        m = self.dtold * d.dtrise
        m = m if m < self.dt else self.dt
        self.dt = d.dtmax if d.dtmax < m else m
        if self.dt < d.dtmin:
            raise RuntimeError(f"timestep: small timestep {self.dt} at step {self.step}")
        self.dtold = self.dt

    # driver/advection.cpp:29-105; the two advec_mom calls of a sweep run as one pass
    def advection(self):
        c = self.c
        direction = 1 if self.advect_x else 2
        self._mark("advec_cell_s1")
        c.update_halo([E1, D1, VFX, VFY], 2)
        c.advec_cell(1, direction, self._depth(2))
        c.update_halo([D1, E1, U1, V1, MFX, MFY], 2)
        self._mark("advec_mom_s1")
        c.advec_mom(3, 1, direction, self._depth(2))
        direction = 2 if self.advect_x else 1
        self._mark("advec_cell_s2")
        c.advec_cell(2, direction, self._depth(2))
        c.update_halo([D1, E1, U1, V1, MFX, MFY], 2)
        self._mark("advec_mom_s2")
        c.advec_mom(3, 2, direction, 0)

    # driver/hydro.cpp:53-108 (one pass of the while loop); returns True when complete
    def hydro_step(self) -> bool:
        c, d = self.c, self.deck
        self.step += 1
        self.timestep()
        self.dt_trace.append(self.dt)
        if self.lagrangian:
            self._mark("lagrangian")
            c.lagrangian(self.dt, self._depth(2))
        else:
            self._mark("pdv_predict")
            c.pdv(True, self.dt, full=True, halo_depth=1)  # the predictor's own pressure halo
            self._mark("accelerate")
            c.accelerate(self.dt, self._depth(2))
            self._mark("pdv_correct")
            c.pdv(False, self.dt, halo_depth=self._depth(2))
            self._mark("flux_calc")
            c.flux_calc(self.dt, self._depth(2))
        self.advection()
        self._mark("reset_field")
        c.reset_field(self._depth(1))
        self.advect_x = not self.advect_x
        self.time += self.dt
        done = self.time + G_SMALL > d.end_time or self.step >= d.end_step
        if d.summary_frequency != 0 and self.step % d.summary_frequency == 0:
            self._mark("field_summary")
            self.field_summary()
        if done:
            self._mark("field_summary")
            self.field_summary()
        self._mark("end")
        return done

    # driver/hydro.cpp:53-111, the whole loop on the device (cb_run)
    def run_steps_on_device(self, max_steps: Optional[int] = None, chunk_steps: int = 4096, fuse: bool = False) -> bool:
        """Makes the steps `hydro_step` would make, up to the end of the run or
        up to step `max_steps`, as device-resident CUDA graphs of at most
        `chunk_steps` steps each (the host waits once per graph).  Fields, dt
        sequence and summaries are those of the `hydro_step` loop.  With
        `fuse`, phases that share inputs run as one pass (FP64 results
        unchanged to the bit, FP32 within its rounding).  Returns True when
        the run is complete."""
        if self.forced_dt is not None or self.probe is not None:
            raise ValueError("run_steps_on_device: forced_dt and probe need the host-driven loop")
        d = self.deck
        p = RunParams(d.dtmin, d.dtmax, d.dtrise, d.dtc_safe, d.dtu_safe, d.dtv_safe, d.dtdiv_safe, d.end_time,
                      d.end_step, d.summary_frequency, int(self.fold), int(fuse))
        st = RunState(self.step, int(self.advect_x), self.time, self.dtold, self.dt, 0)
        last = d.end_step if max_steps is None else min(d.end_step, max_steps)
        while self.step < last:
            n = min(chunk_steps, last - self.step)
            cap = n // d.summary_frequency + 2 if d.summary_frequency > 0 else 2
            try:
                trace, recs, _ = self.c.run(p, st, n, cap)
            finally:
                self.step, self.time, self.dt, self.dtold = st.step, st.time, st.dt, st.dtold
                self.advect_x = bool(st.advect_x)
            self.dt_trace.extend(float(x) for x in trace)
            self.summaries.extend(Summary(int(r[0]), *(float(x) for x in r[1:])) for r in recs)
            if st.done:
                return True
        return False

    def run(self, max_steps: Optional[int] = None, on_step: Optional[Callable[["HydroRun"], None]] = None):
        self.start()
        while True:
            done = self.hydro_step()
            if on_step:
                on_step(self)
            if done or (max_steps is not None and self.step >= max_steps):
                break
        return self.summaries
