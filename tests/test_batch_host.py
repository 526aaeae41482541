"""Host side of the batched ensemble, without a GPU.

* The ctypes structures of cloverleaf_b200.batch match include/cloverb200.h
  (sizes and field offsets, measured by compiling the header with gcc).
* The seeded ensemble generator is deterministic and draws from the stated
  ranges.
* cb_batch_create rejects bad decks before touching a device.
"""
import ctypes
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from cloverleaf_b200 import batch as B
from cloverleaf_b200 import library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_layout_matches_header():
    fields = {"cb_deck": [n for n, _ in B.CDeck._fields_], "cb_batch_schedule": [n for n, _ in B.Schedule._fields_],
              "cb_batch_trial": [n for n, _ in B.Trial._fields_]}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cloverb200.h"', "int main(void) {"]
    for t, names in fields.items():
        lines.append(f'  printf("{t} size %zu\\n", sizeof({t}));')
        for n in names:
            lines.append(f'  printf("{t} {n} %zu\\n", offsetof({t}, {n}));')
    lines.append("  return 0; }")
    with tempfile.TemporaryDirectory() as tmp:
        src, exe = os.path.join(tmp, "l.c"), os.path.join(tmp, "l")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for line in out:
        w = line.split()
        if len(w) == 3:
            got[(w[0], w[1])] = int(w[2])
    for t, cls in (("cb_deck", B.CDeck), ("cb_batch_schedule", B.Schedule), ("cb_batch_trial", B.Trial)):
        assert got[(t, "size")] == ctypes.sizeof(cls), t
        for n, _ in cls._fields_:
            assert got[(t, n)] == getattr(cls, n).offset, (t, n)


def test_ensemble_is_seeded_and_in_range():
    a = B.ensemble_decks(64)
    b = B.ensemble_decks(64)
    assert [(d.x_cells, d.gamma, d.states[1].density) for d in a] == [(d.x_cells, d.gamma, d.states[1].density) for d in b]
    c = B.ensemble_decks(64, seed=1)
    assert [d.gamma for d in a] != [d.gamma for d in c]
    for d in a:
        assert d.x_cells == d.y_cells and d.x_cells in B.ENSEMBLE_SIDES
        assert 1.3 <= d.gamma <= 1.67
        bg, rect = d.states
        assert (bg.density, bg.energy) == (0.2, 1.0)
        assert 0.5 <= rect.density <= 2.0 and 1.0 <= rect.energy <= 4.0
        dx = 10.0 / d.x_cells
        # nudged extents (driver/read_input.cpp:268-276)
        assert abs(rect.xmin - dx / 100.0) < 1e-15 and 2.0 - dx / 100 <= rect.xmax <= 8.0
        assert d.end_time == 0.5 and d.xmax == 10.0 and d.ymax == 10.0
    sides = {d.x_cells for d in B.ensemble_decks(512)}
    assert sides == set(B.ENSEMBLE_SIDES)


def test_create_rejects_bad_decks_before_device():
    lib = B._lib()
    h = ctypes.c_void_p()
    dk = B.to_cdeck(B.ensemble_deck(64, 1.0, 2.0, 4.0, 3.0, 1.4))
    bad = B.CDeck.from_buffer_copy(dk)
    bad.nx = 7
    assert lib.cb_batch_create(1, (B.CDeck * 1)(bad), 0, 0, ctypes.byref(h)) == 1
    assert b"at least 8 cells" in library().cb_last_error()
    bad = B.CDeck.from_buffer_copy(dk)
    bad.gamma = 1.0
    assert lib.cb_batch_create(1, (B.CDeck * 1)(bad), 0, 0, ctypes.byref(h)) == 1
    assert b"gamma" in library().cb_last_error()
    bad = B.CDeck.from_buffer_copy(dk)
    bad.nstates = 9
    assert lib.cb_batch_create(1, (B.CDeck * 1)(bad), 0, 0, ctypes.byref(h)) == 1
    assert lib.cb_batch_create(1, (B.CDeck * 1)(dk), 5, 0, ctypes.byref(h)) == 1
    assert lib.cb_batch_create(0, None, 0, 0, ctypes.byref(h)) == 1
    assert lib.cb_batch_destroy(None) == 0
    assert lib.cb_batch_run(None) == 1


def test_too_many_states_rejected_in_python():
    dk = B.ensemble_deck(64, 1.0, 2.0, 4.0, 3.0, 1.4)
    dk.states = dk.states * 5
    with pytest.raises(Exception):
        B.to_cdeck(dk)
