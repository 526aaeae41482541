"""clover.in deck reader.

Restates the reference's input reader, driver/read_input.cpp:37-277: the same
defaults (:37-69), the same keywords (:142-254), ``key=value`` and
``key value`` forms (the line is split on spaces and '=' like strtok, :138-141),
and the same nudge of every non-background state's extents by a hundredth of
a cell (:268-276).  Unknown keywords are ignored, as in the reference.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional

import numpy as np

G_SMALL = 1.0e-16  # driver/definitions.h:34
G_BIG = 1.0e21  # driver/definitions.h:35
G_IBIG = 640000  # driver/definitions.h:33

GEOM_RECT, GEOM_CIRC, GEOM_POINT = 1, 2, 3


@dataclasses.dataclass
class State:
    """One ``state N ...`` line (driver/definitions.h:79-95)."""

    density: float = 0.0
    energy: float = 0.0
    xvel: float = 0.0
    yvel: float = 0.0
    geometry: int = 0
    xmin: float = 0.0
    ymin: float = 0.0
    xmax: float = 0.0
    ymax: float = 0.0
    radius: float = 0.0
    defined: bool = False


@dataclasses.dataclass
class Deck:
    """The subset of ``global_config`` a deck sets (driver/definitions.h:227-256)."""

    x_cells: int = 10
    y_cells: int = 10
    xmin: float = 0.0
    ymin: float = 0.0
    xmax: float = 0.0
    ymax: float = 0.0
    end_time: float = 10.0
    end_step: int = G_IBIG
    visit_frequency: int = 0
    summary_frequency: int = 10
    tiles_per_chunk: int = 1
    dtinit: float = 0.1
    dtmax: float = 1.0
    dtmin: float = 0.0000001
    dtrise: float = 1.5
    dtc_safe: float = 0.7
    dtu_safe: float = 0.5
    dtv_safe: float = 0.5
    dtdiv_safe: float = 0.7
    profiler_on: bool = False
    test_problem: int = 0
    states: List[State] = dataclasses.field(default_factory=list)
    gamma: float = 1.4  # not a deck keyword; the reference hard-codes 1.4

    @property
    def cells(self) -> int:
        return self.x_cells * self.y_cells


def _words(line: str) -> List[str]:
    out, cur = [], []
    for ch in line:
        if ch in " =":
            if cur:
                out.append("".join(cur))
                cur = []
        else:
            cur.append(ch)
    if cur:
        out.append("".join(cur))
    return out


def _stoi(s: str) -> int:
    s = s.strip()
    n = 0
    while n < len(s) and (s[n].isdigit() or (n == 0 and s[n] in "+-")):
        n += 1
    return int(s[:n])


def parse_deck(text: str, nudge: bool = True) -> Deck:
    """Parse deck text into a :class:`Deck` (states nudged unless ``nudge=False``)."""
    d = Deck()
    lines = text.splitlines()
    state_max = 0
    for line in lines:
        if not line:
            continue
        w = line.split()
        if w and w[0] == "state":
            state_max = max(state_max, _stoi(w[1]))
    if state_max < 1:
        raise ValueError("read_input: No states defined.")
    d.states = [State() for _ in range(state_max)]
    for line in lines:
        if not line:
            continue
        w = _words(line)
        if not w:
            continue
        k = w[0]
        if k == "initial_timestep":
            d.dtinit = float(w[1])
        elif k == "max_timestep":
            d.dtmax = float(w[1])
        elif k == "timestep_rise":
            d.dtrise = float(w[1])
        elif k == "end_time":
            d.end_time = float(w[1])
        elif k == "end_step":
            d.end_step = _stoi(w[1])
        elif k == "xmin":
            d.xmin = float(w[1])
        elif k == "xmax":
            d.xmax = float(w[1])
        elif k == "ymin":
            d.ymin = float(w[1])
        elif k == "ymax":
            d.ymax = float(w[1])
        elif k == "x_cells":
            d.x_cells = _stoi(w[1])
        elif k == "y_cells":
            d.y_cells = _stoi(w[1])
        elif k == "visit_frequency":
            d.visit_frequency = _stoi(w[1])
        elif k == "summary_frequency":
            d.summary_frequency = _stoi(w[1])
        elif k == "tiles_per_chunk":
            d.tiles_per_chunk = _stoi(w[1])
        elif k == "tiles_per_problem":
            d.tiles_per_chunk = _stoi(w[1])  # one rank: tiles_per_problem / 1
        elif k == "profiler_on":
            d.profiler_on = True
        elif k == "test_problem":
            d.test_problem = _stoi(w[1])
        elif k == "state":
            s = d.states[_stoi(w[1]) - 1]
            if s.defined:
                raise ValueError("read_input: State defined twice.")
            s.defined = True
            i = 2
            while i < len(w):
                key = w[i]
                if key in ("xvel", "yvel", "xmin", "ymin", "xmax", "ymax", "radius", "density", "energy"):
                    i += 1
                    setattr(s, key, float(w[i]))
                elif key == "geometry":
                    i += 1
                    s.geometry = {"rectangle": GEOM_RECT, "circle": GEOM_CIRC, "point": GEOM_POINT}.get(w[i], s.geometry)
                i += 1
    if nudge:
        # driver/read_input.cpp:268-276; (float)x_cells is exact for any sane mesh
        dx = (d.xmax - d.xmin) / float(np.float32(d.x_cells))
        dy = (d.ymax - d.ymin) / float(np.float32(d.y_cells))
        for s in d.states[1:]:
            s.xmin += dx / 100.0
            s.ymin += dy / 100.0
            s.xmax -= dx / 100.0
            s.ymax -= dy / 100.0
    return d


def read_deck(path: str, nudge: bool = True) -> Deck:
    with open(path, "r") as f:
        return parse_deck(f.read(), nudge=nudge)


def format_deck(d: Deck) -> str:
    """Write a deck the reference reader accepts (states written un-nudged).

    ``d`` must hold the states as they appear in the file (``nudge=False``).
    """
    geo = {GEOM_RECT: "rectangle", GEOM_CIRC: "circle", GEOM_POINT: "point"}
    out = ["*clover"]
    for n, s in enumerate(d.states, start=1):
        parts = [f" state {n} density={s.density!r} energy={s.energy!r}"]
        if s.xvel != 0.0:
            parts.append(f"xvel={s.xvel!r}")
        if s.yvel != 0.0:
            parts.append(f"yvel={s.yvel!r}")
        if n > 1:
            parts.append(f"geometry={geo[s.geometry]}")
            if s.geometry == GEOM_RECT:
                parts.append(f"xmin={s.xmin!r} xmax={s.xmax!r} ymin={s.ymin!r} ymax={s.ymax!r}")
            elif s.geometry == GEOM_CIRC:
                parts.append(f"xmin={s.xmin!r} ymin={s.ymin!r} radius={s.radius!r}")
            else:
                parts.append(f"xmin={s.xmin!r} ymin={s.ymin!r}")
        out.append(" ".join(parts))
    out += [
        f" x_cells={d.x_cells}",
        f" y_cells={d.y_cells}",
        f" xmin={d.xmin!r}",
        f" ymin={d.ymin!r}",
        f" xmax={d.xmax!r}",
        f" ymax={d.ymax!r}",
        f" initial_timestep={d.dtinit!r}",
        f" timestep_rise={d.dtrise!r}",
        f" max_timestep={d.dtmax!r}",
        f" end_time={d.end_time!r}",
        f" end_step={d.end_step}",
        f" summary_frequency={d.summary_frequency}",
    ]
    if d.visit_frequency:
        out.append(f" visit_frequency={d.visit_frequency}")
    if d.test_problem:
        out.append(f" test_problem {d.test_problem}")
    out.append("*endclover")
    return "\n".join(out) + "\n"


def benchmark_deck(cells: int, end_step: int, end_time: float = 10.0, test_problem: int = 0,
                   ny: Optional[int] = None) -> Deck:
    """The reference benchmark problem (InputDecks/clover_bm*.in) at any size:
    background rho=0.2 e=1.0, rectangle [0,5]x[0,2] with rho=1.0 e=2.5 on
    [0,10]^2, dtinit=dtmax=0.04, dtrise=1.5.  States are un-nudged; pass the
    result through :func:`nudged` before handing it to a solver."""
    d = Deck()
    d.x_cells = cells
    d.y_cells = cells if ny is None else ny
    d.xmin, d.ymin, d.xmax, d.ymax = 0.0, 0.0, 10.0, 10.0
    d.dtinit, d.dtrise, d.dtmax = 0.04, 1.5, 0.04
    d.end_time, d.end_step, d.test_problem = end_time, end_step, test_problem
    d.states = [State(density=0.2, energy=1.0, defined=True),
                State(density=1.0, energy=2.5, geometry=GEOM_RECT, xmin=0.0, xmax=5.0, ymin=0.0, ymax=2.0, defined=True)]
    return d


def nudged(d: Deck) -> Deck:
    """A copy of ``d`` with the reader's state nudge applied."""
    return _with_gamma(parse_deck(format_deck(d), nudge=True), d.gamma)


def _with_gamma(d: Deck, gamma: float) -> Deck:
    d.gamma = gamma
    return d
