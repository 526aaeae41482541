"""Loading the committed golden fixtures (tests/golden/, made by make_golden.py)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SMALL_DECKS = ["default10x2", "bm32x87", "bm40x24x120", "circ24x20x70", "sodx10x2", "sody2x10", "sodxy10x10"]
# the reference's own larger decks (InputDecks/clover_sodbig.in, clover_qa.in): summaries only
SUMMARY_DECKS = ["sodbig200", "qa1024"]
# (field id, kind) of the arrays a fields.bin holds
CAPTURED = [(0, "cell"), (2, "cell"), (4, "cell"), (5, "cell"), (6, "cell"), (7, "node"), (9, "node"),
            (11, "xface"), (12, "yface")]


def deck_text(name):
    with open(os.path.join(GOLDEN, name + ".in")) as f:
        return f.read()


def summaries(name):
    out = []
    with open(os.path.join(GOLDEN, name + ".summary.txt")) as f:
        for line in f:
            w = line.split()
            out.append((int(w[0]),) + tuple(float(x) for x in w[1:]))
    return out


def fields(name):
    import oracle
    return oracle.read_fields(os.path.join(GOLDEN, name + ".fields.bin"))


def interior(arr, nx, ny, kind):
    w = nx + (1 if kind in ("node", "xface") else 0)
    h = ny + (1 if kind in ("node", "yface") else 0)
    return np.asarray(arr)[2:2 + h, 2:2 + w]


def rel(a, b):
    return abs(a - b) / abs(b) if b != 0 else abs(a - b)
