"""The deck reader (cloverleaf_b200/deck.py) against driver/read_input.cpp semantics."""
import numpy as np

from cloverleaf_b200 import deck as D
from golden_util import SMALL_DECKS, deck_text


def test_defaults_and_keywords():
    d = D.parse_deck(deck_text("default10x2"))
    assert (d.x_cells, d.y_cells) == (10, 2)
    assert (d.xmin, d.ymin, d.xmax, d.ymax) == (0.0, 0.0, 10.0, 2.0)
    assert d.dtinit == 0.04 and d.dtmax == 0.04 and d.dtrise == 1.5
    assert d.end_time == 3.0 and d.end_step == D.G_IBIG
    assert d.summary_frequency == 10 and d.test_problem == 1
    assert d.dtmin == 0.0000001 and d.dtc_safe == 0.7 and d.dtu_safe == 0.5 and d.dtdiv_safe == 0.7
    assert len(d.states) == 2 and d.states[1].geometry == D.GEOM_RECT


def test_state_nudge():
    raw = D.parse_deck(deck_text("default10x2"), nudge=False)
    d = D.parse_deck(deck_text("default10x2"))
    dx = (10.0 - 0.0) / float(np.float32(10))
    dy = (2.0 - 0.0) / float(np.float32(2))
    assert d.states[1].xmin == raw.states[1].xmin + dx / 100.0
    assert d.states[1].ymax == raw.states[1].ymax - dy / 100.0
    assert d.states[0].xmin == raw.states[0].xmin  # the background is not nudged


def test_space_separated_values_and_unknown_keywords():
    text = "*clover\n state 1 density=0.2 energy 1.0\n state 2 density 1.0 energy=2.5 geometry=circle xmin=1 ymin=2 radius=0.5\n" \
           " x_cells 16\n y_cells=8\n xmax=4\n ymax=2\n use_c_kernels\n end_step 5\n profiler_on\n*endclover\n"
    d = D.parse_deck(text)
    assert d.states[0].energy == 1.0 and d.states[1].geometry == D.GEOM_CIRC and d.states[1].radius == 0.5
    assert d.x_cells == 16 and d.end_step == 5 and d.profiler_on


def test_format_round_trip():
    for name in SMALL_DECKS + ["circ16x12x3v"]:
        raw = D.parse_deck(deck_text(name), nudge=False)
        again = D.parse_deck(D.format_deck(raw), nudge=False)
        for a, b in zip(raw.states, again.states):
            assert a == b
        assert (raw.x_cells, raw.y_cells, raw.end_step, raw.visit_frequency) == \
            (again.x_cells, again.y_cells, again.end_step, again.visit_frequency)
    assert D.parse_deck(deck_text("circ16x12x3v")).visit_frequency == 2
