"""Batched ensemble: many independent decks advanced by one persistent kernel
launch (the cb_batch_* part of include/cloverb200.h).

Each deck follows the reference driver's per-chunk call sequence
(driver/start.cpp:43-138, driver/hydro.cpp:46-223) with its own gamma,
states, dt controls and end time; its final fields are bit-identical to a
`HydroRun` of the same deck on a `Chunk` of the same precision.

`ensemble_decks` draws the seeded ensemble of the batched benchmark: square
meshes of side {64, 96, 128, 192, 256, 384} on [0, 10]^2, background
rho = 0.2, e = 1.0, a rectangle [0, x1] x [0, y1] with rho ~ U[0.5, 2],
e ~ U[1, 4], x1 ~ U[2, 8], y1 ~ U[1, 5], gamma ~ U[1.3, 1.67], each run to
t = 0.5.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .chunk import FIELD_ID, FP64, LAYOUT_XFAST, CloverError, State, _check, _dptr, library
from .deck import GEOM_RECT, Deck, State as DeckState, nudged
from .hydro import Summary

MAX_STATES = 8
DECK_PENDING, DECK_DONE, DECK_SMALL_DT, DECK_STAGE_FAIL, DECK_SYNC_FAIL = range(5)
ENSEMBLE_SIDES = (64, 96, 128, 192, 256, 384)
ENSEMBLE_SEED = 0xC10E


class CDeck(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("xmin", ctypes.c_double), ("ymin", ctypes.c_double),
                ("xmax", ctypes.c_double), ("ymax", ctypes.c_double), ("gamma", ctypes.c_double), ("nstates", ctypes.c_int),
                ("states", State * MAX_STATES), ("dtinit", ctypes.c_double), ("dtmin", ctypes.c_double),
                ("dtmax", ctypes.c_double), ("dtrise", ctypes.c_double), ("dtc_safe", ctypes.c_double),
                ("dtu_safe", ctypes.c_double), ("dtv_safe", ctypes.c_double), ("dtdiv_safe", ctypes.c_double),
                ("end_time", ctypes.c_double), ("end_step", ctypes.c_int), ("summary_frequency", ctypes.c_int)]


class Schedule(ctypes.Structure):
    _fields_ = [("cells_per_cta", ctypes.c_int), ("max_lane_width", ctypes.c_int), ("ctas_per_sm", ctypes.c_int),
                ("variant", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Trial(ctypes.Structure):
    _fields_ = [("schedule", Schedule), ("lanes", ctypes.c_int), ("ctas", ctypes.c_int), ("ms", ctypes.c_float)]


EXPORTS = ["cb_batch_create", "cb_batch_destroy", "cb_batch_set_schedule", "cb_batch_get_schedule", "cb_batch_autotune",
           "cb_batch_run", "cb_batch_synchronize", "cb_batch_deck_result", "cb_batch_read_summaries", "cb_batch_read_dt",
           "cb_batch_read_field", "cb_batch_get_stream", "cb_batch_launch_count"]

_bound = False


def _lib():
    global _bound
    L = library()
    if not _bound:
        P, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        ip, dp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        sig = {
            "cb_batch_create": ([i, ctypes.POINTER(CDeck), i, i, ctypes.POINTER(P)], i),
            "cb_batch_destroy": ([P], i),
            "cb_batch_set_schedule": ([P, ctypes.POINTER(Schedule)], i),
            "cb_batch_get_schedule": ([P, ctypes.POINTER(Schedule), ip, ip], i),
            "cb_batch_autotune": ([P, i, ctypes.POINTER(Trial), i, ip, ctypes.POINTER(Schedule)], i),
            "cb_batch_run": ([P], i),
            "cb_batch_synchronize": ([P, ctypes.POINTER(ctypes.c_float)], i),
            "cb_batch_deck_result": ([P, i, ip, ip, dp, ip], i),
            "cb_batch_read_summaries": ([P, i, dp, i, ip], i),
            "cb_batch_read_dt": ([P, i, dp, i, ip], i),
            "cb_batch_read_field": ([P, i, i, dp, ctypes.c_size_t, i], i),
            "cb_batch_get_stream": ([P, ctypes.POINTER(P)], i),
            "cb_batch_launch_count": ([P, ctypes.POINTER(ctypes.c_longlong)], i),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _bound = True
    return L


def to_cdeck(dk: Deck) -> CDeck:
    """A (nudged) :class:`Deck` as the C ABI's cb_deck."""
    if len(dk.states) > MAX_STATES:
        raise CloverError(f"a batch deck holds at most {MAX_STATES} states")
    c = CDeck()
    c.nx, c.ny = dk.x_cells, dk.y_cells
    c.xmin, c.ymin, c.xmax, c.ymax = dk.xmin, dk.ymin, dk.xmax, dk.ymax
    c.gamma = dk.gamma
    c.nstates = len(dk.states)
    for k, s in enumerate(dk.states):
        c.states[k] = State(s.density, s.energy, s.xvel, s.yvel, s.geometry, s.xmin, s.ymin, s.xmax, s.ymax, s.radius)
    c.dtinit, c.dtmin, c.dtmax, c.dtrise = dk.dtinit, dk.dtmin, dk.dtmax, dk.dtrise
    c.dtc_safe, c.dtu_safe, c.dtv_safe, c.dtdiv_safe = dk.dtc_safe, dk.dtu_safe, dk.dtv_safe, dk.dtdiv_safe
    c.end_time, c.end_step, c.summary_frequency = dk.end_time, dk.end_step, dk.summary_frequency
    return c


def ensemble_deck(side: int, rho: float, e: float, x1: float, y1: float, gamma: float, end_time: float = 0.5) -> Deck:
    """One deck of the benchmark ensemble (nudged, as the driver reads it)."""
    dk = Deck(x_cells=side, y_cells=side, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0, end_time=end_time,
              dtinit=0.04, dtmax=0.04, dtrise=1.5, summary_frequency=10, gamma=gamma)
    dk.states = [DeckState(density=0.2, energy=1.0, defined=True),
                 DeckState(density=rho, energy=e, geometry=GEOM_RECT, xmin=0.0, xmax=x1, ymin=0.0, ymax=y1, defined=True)]
    return nudged(dk)


def ensemble_decks(n: int = 512, seed: int = ENSEMBLE_SEED, sides: Sequence[int] = ENSEMBLE_SIDES,
                   end_time: float = 0.5) -> List[Deck]:
    """The seeded ensemble (numpy PCG64 generator, draws in the order side, rho, e, x1, y1, gamma per deck)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        side = int(sides[rng.integers(len(sides))])
        rho, e = rng.uniform(0.5, 2.0), rng.uniform(1.0, 4.0)
        x1, y1 = rng.uniform(2.0, 8.0), rng.uniform(1.0, 5.0)
        gamma = rng.uniform(1.3, 1.67)
        out.append(ensemble_deck(side, float(rho), float(e), float(x1), float(y1), float(gamma), end_time))
    return out


@dataclasses.dataclass
class DeckResult:
    status: int
    steps: int
    time: float
    nsummaries: int


class Batch:
    """Many decks resident on one B200, advanced by one persistent launch (cb_batch)."""

    def __init__(self, decks: Sequence[Deck], precision: int = FP64, device: int = 0):
        self._L = _lib()
        self._h = ctypes.c_void_p()
        self.decks = list(decks)
        arr = (CDeck * len(self.decks))(*[to_cdeck(d) for d in self.decks])
        _check(self._L.cb_batch_create(len(self.decks), arr, precision, device, ctypes.byref(self._h)))
        self.precision = precision

    def close(self):
        if self._h:
            self._L.cb_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_schedule(self, cells_per_cta: int = 16384, max_lane_width: int = 0, ctas_per_sm: int = 0, variant: int = 0):
        s = Schedule(cells_per_cta, max_lane_width, ctas_per_sm, variant)
        _check(self._L.cb_batch_set_schedule(self._h, ctypes.byref(s)))

    def schedule(self) -> Tuple[dict, int, int]:
        s, lanes, ctas = Schedule(), ctypes.c_int(), ctypes.c_int()
        _check(self._L.cb_batch_get_schedule(self._h, ctypes.byref(s), ctypes.byref(lanes), ctypes.byref(ctas)))
        return s.as_dict(), lanes.value, ctas.value

    def autotune(self, repeats: int = 1):
        trials = (Trial * 64)()
        nt, best = ctypes.c_int(), Schedule()
        _check(self._L.cb_batch_autotune(self._h, repeats, trials, 64, ctypes.byref(nt), ctypes.byref(best)))
        log = [{"schedule": trials[k].schedule.as_dict(), "lanes": trials[k].lanes, "ctas": trials[k].ctas,
                "ms": float(trials[k].ms)} for k in range(min(nt.value, 64))]
        return best.as_dict(), log

    def run(self):
        _check(self._L.cb_batch_run(self._h))

    def synchronize(self) -> float:
        ms = ctypes.c_float()
        _check(self._L.cb_batch_synchronize(self._h, ctypes.byref(ms)))
        return float(ms.value)

    def result(self, k: int) -> DeckResult:
        st, steps, nsum, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _check(self._L.cb_batch_deck_result(self._h, k, ctypes.byref(st), ctypes.byref(steps), ctypes.byref(t),
                                            ctypes.byref(nsum)))
        return DeckResult(st.value, steps.value, t.value, nsum.value)

    def summaries(self, k: int) -> List[Summary]:
        r = self.result(k)
        n = max(r.nsummaries, 0)
        buf = np.zeros((max(n, 1), 7), dtype=np.float64)
        cnt = ctypes.c_int()
        _check(self._L.cb_batch_read_summaries(self._h, k, _dptr(buf), n, ctypes.byref(cnt)))
        return [Summary(int(row[0]), *map(float, row[1:])) for row in buf[:cnt.value]]

    def dt_trace(self, k: int) -> List[float]:
        r = self.result(k)
        buf = np.zeros(max(r.steps, 1), dtype=np.float64)
        cnt = ctypes.c_int()
        _check(self._L.cb_batch_read_dt(self._h, k, _dptr(buf), r.steps, ctypes.byref(cnt)))
        return [float(x) for x in buf[:cnt.value]]

    def read(self, k: int, field) -> np.ndarray:
        """Final field of deck k as an (sy, sx) array indexed [j, i] (as Chunk.read)."""
        fid = FIELD_ID[field] if isinstance(field, str) else int(field)
        dk = self.decks[k]
        nx, ny = dk.x_cells, dk.y_cells
        sx = nx + 5 if fid in (7, 8, 9, 10, 11, 13) else nx + 4
        sy = ny + 5 if fid in (7, 8, 9, 10, 12, 14) else ny + 4
        out = np.empty((sy, sx), dtype=np.float64)
        _check(self._L.cb_batch_read_field(self._h, k, fid, _dptr(out), out.size, LAYOUT_XFAST))
        return out

    def launch_count(self) -> int:
        n = ctypes.c_longlong()
        _check(self._L.cb_batch_launch_count(self._h, ctypes.byref(n)))
        return n.value
