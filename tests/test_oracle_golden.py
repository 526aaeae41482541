"""The CPU oracle (oracle/clover_oracle.c) against the reference's own outputs.

The golden fixtures were produced by the reference driver + serial model
compiled from the reference sources (tests/golden/make_golden.py).  The
oracle must reproduce them bit for bit: every summary value and every final
per-cell field; the decks include the reference's own Sod shock tubes
(InputDecks/clover_sod*.in: 10 x 2, 2 x 10, 10 x 10 and 200 x 200) and its
QA deck (clover_qa.in, 1024^2).  The 960^2 deck also checks the reference's hard-coded
expected kinetic energy (driver/report.cpp:79-80, test_problem 2).
"""
import numpy as np
import pytest

import oracle
from cloverleaf_b200 import deck as D
from golden_util import CAPTURED, SMALL_DECKS, SUMMARY_DECKS, deck_text, fields, interior, summaries


@pytest.mark.parametrize("name", SMALL_DECKS)
def test_oracle_matches_reference_bitwise(name):
    dk = D.parse_deck(deck_text(name))
    c = oracle.OracleChunk(dk.x_cells, dk.y_cells)
    recs, steps, _ = c.run(dk)
    gold = summaries(name)
    assert len(recs) == len(gold)
    for a, b in zip(recs, gold):
        assert a == b, (a, b)
    gf = fields(name)
    for fid, kind in CAPTURED:
        assert np.array_equal(interior(c.field(fid), dk.x_cells, dk.y_cells, kind), gf[fid]), fid


def test_oracle_config1_960_pass():
    """Config 1 (960^2, 87 steps): bit-exact summaries and the reference's PASS check."""
    dk = D.parse_deck(deck_text("bm960x87"))
    c = oracle.OracleChunk(dk.x_cells, dk.y_cells)
    recs, steps, _ = c.run(dk)
    assert steps == 87
    assert recs == summaries("bm960x87")
    ke = recs[-1][5]
    qa_diff = abs(100.0 * (ke / 1.19316898756307) - 100.0)  # driver/report.cpp:79-80, :102
    assert qa_diff < 0.001


@pytest.mark.parametrize("name", SUMMARY_DECKS)
def test_oracle_reference_decks_summaries(name):
    """The reference's Sod deck on 200^2 to t = 30 (1,330 steps) and its QA deck
    on 1024^2 over a domain centred on the origin: every summary bit for bit."""
    dk = D.parse_deck(deck_text(name))
    c = oracle.OracleChunk(dk.x_cells, dk.y_cells)
    recs, steps, _ = c.run(dk, max_summaries=4096)
    assert recs == summaries(name)


def test_default_deck_test_problem_1():
    dk = D.parse_deck(deck_text("default10x2"))
    c = oracle.OracleChunk(dk.x_cells, dk.y_cells)
    recs, _, _ = c.run(dk)
    ke = recs[-1][5]
    assert abs(100.0 * (ke / 1.82280367310258) - 100.0) < 0.001  # driver/report.cpp:76-78


def test_exact_summary_is_order_free():
    """The double-double summary equals the sequential one to rounding, and the
    sequential (reference) order carries its own rounding error of up to ~1e-11
    on a 960^2 mesh -- which is why GPU sums are compared to the exact sum."""
    dk = D.parse_deck(deck_text("bm32x87"))
    c = oracle.OracleChunk(dk.x_cells, dk.y_cells)
    c.run(dk)
    seq = c.field_summary()
    ex = c.field_summary(exact=True)
    for a, b in zip(seq, ex):
        assert abs(a - b) <= 1e-13 * abs(b)
