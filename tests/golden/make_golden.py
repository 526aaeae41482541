"""Regenerates the golden fixtures in this directory from the reference itself.

Runs the reference driver + serial model (built from the reference sources by
`make -C oracle ref`, with the capture hooks of oracle/ref_hooks/) on a set
of decks and stores, per deck:
  <name>.in            the deck
  <name>.summary.txt   every field_summary at full precision (step time vol mass ie ke press)
  <name>.fields.bin    the final interior fields (CLVF format, small decks only)
  <name>.stdout.txt    the lines of the reference's stdout that carry the verdict
and, for the dump deck, the reference's --dump output of driver/shared.cpp:96-189 as
  <name>.dump.sha256   one line per dump file: its name and the sha256 of its
                       text with the work_array blocks removed (dump_filter.py)
and, for the reference's decks that carry a test_problem, the deck alone (the
driver checks their final kinetic energy against its own table), and, for the
visit deck, the files driver/visit.cpp:31-192 writes as
  <name>.visit.sha256  one line per file (clover.visit and each .vtk): its name
                       and the sha256 of its bytes

Usage: python tests/golden/make_golden.py [deck names]   (needs oracle/_ref/serial-capture and
oracle/_ref/serial, and the reference checkout for the InputDecks decks)
"""
import hashlib
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from cloverleaf_b200 import deck as D  # noqa: E402

# The built-in deck of driver/clover_leaf.cpp:156-171 (test_problem 1).
DEFAULT_DECK = """*clover
 state 1 density=0.2 energy=1.0
 state 2 density=1.0 energy=2.5 geometry=rectangle xmin=0.0 xmax=5.0 ymin=0.0 ymax=2.0
 x_cells=10
 y_cells=2
 xmin=0.0
 ymin=0.0
 xmax=10.0
 ymax=2.0
 initial_timestep=0.04
 timestep_rise=1.5
 max_timestep=0.04
 end_time=3.0
 test_problem 1
*endclover
"""


# The reference checkout: CLOVER_REFERENCE, else the directory beside this repository.
REFERENCE = os.environ.get("CLOVER_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))

# The reference's own shock-tube and QA decks (InputDecks/), read from the
# reference checkout and written back in this package's deck format: name ->
# (file, keep the final fields).  The two larger runs keep summaries only.
REFERENCE_DECKS = {"sodx10x2": ("clover_sodx.in", True), "sody2x10": ("clover_sody.in", True),
                   "sodxy10x10": ("clover_sodxy.in", True), "sodbig200": ("clover_sodbig.in", False),
                   "qa1024": ("clover_qa.in", False)}


# The reference's decks that carry a test_problem, whose final kinetic
# energy the driver checks against its table (driver/report.cpp:75-97): only
# the decks are written (no reference run), the table is the known answer.
KNOWN_ANSWER_DECKS = {"bm960x2955": "clover_bm.in", "bm3840x87": "clover_bm16_short.in", "bm3840x2955": "clover_bm16.in",
                      "bm3840x8": "clover_bm16_very_short.in", "bm1920x960x87": "clover_bm2_short.in",
                      "bm1920x87": "clover_bm4_short.in"}


# Known-answer decks whose outcome the reference build itself reports is kept
# too (<name>.stdout.txt): its test_problem 3 deck ends 0.0206% from the
# table's kinetic energy, not within the 0.001% the driver accepts.
KNOWN_ANSWER_RUNS = ["bm960x2955"]


def write_known_answer_decks():
    for name, fn in KNOWN_ANSWER_DECKS.items():
        with open(os.path.join(REFERENCE, "InputDecks", fn)) as f:
            raw = D.parse_deck(f.read(), nudge=False)
        text = D.format_deck(raw)
        with open(os.path.join(HERE, name + ".in"), "w") as f:
            f.write(text)
        if name in KNOWN_ANSWER_RUNS:  # the reference OpenMP build on every core
            res = oracle.run_reference(text, exe="omp", threads=os.cpu_count())
            keep = [l for l in res["stdout"].splitlines() if "within" in l or "PASSED" in l or "Outcome" in l]
            with open(os.path.join(HERE, name + ".stdout.txt"), "w") as f:
                f.write("\n".join(keep) + "\n")
        print(name, "deck", "and the reference's outcome" if name in KNOWN_ANSWER_RUNS else "")


def reference_decks():
    out = {}
    for name, (fn, keep) in REFERENCE_DECKS.items():
        with open(os.path.join(REFERENCE, "InputDecks", fn)) as f:
            raw = D.parse_deck(f.read(), nudge=False)
        out[name] = (D.format_deck(raw), keep)
    return out


def decks():
    out = {"default10x2": (DEFAULT_DECK, True)}
    out["bm32x87"] = (D.format_deck(D.benchmark_deck(32, 87)), True)
    out["bm40x24x120"] = (D.format_deck(D.benchmark_deck(40, 120, ny=24)), True)
    c = D.benchmark_deck(24, 70, ny=20)
    c.states.append(D.State(density=2.0, energy=3.0, xvel=0.5, yvel=-0.25, geometry=D.GEOM_CIRC, xmin=6.0, ymin=6.0,
                            radius=2.0, defined=True))
    c.states.append(D.State(density=0.5, energy=1.5, xvel=-0.3, yvel=0.2, geometry=D.GEOM_RECT, xmin=6.0, xmax=9.0,
                            ymin=1.0, ymax=3.0, defined=True))
    out["circ24x20x70"] = (D.format_deck(c), True)
    # the reference benchmark at 960^2, 87 steps (test_problem 2): summaries only
    out["bm960x87"] = (D.format_deck(D.benchmark_deck(960, 87, test_problem=2)), False)
    out.update(reference_decks())
    return out


def dump_deck():
    """16 x 12 cells, a rectangle and a moving circle, 3 steps."""
    c = D.benchmark_deck(16, 3, ny=12)
    c.states.append(D.State(density=2.0, energy=3.0, xvel=0.5, yvel=-0.25, geometry=D.GEOM_CIRC, xmin=6.0, ymin=6.0,
                            radius=2.5, defined=True))
    return "circ16x12x3", D.format_deck(c)


def write_dump_fixture():
    from dump_filter import filtered
    name, text = dump_deck()
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "clover.in"), "w") as f:
            f.write(text)
        p = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "serial"), "--file", "clover.in", "--dump", "dumps"], cwd=tmp,
                           capture_output=True, text=True, timeout=600)
        if p.returncode != 0:
            raise SystemExit(f"{name}: reference exited {p.returncode}")
        files = sorted(os.listdir(os.path.join(tmp, "dumps")))
        with open(os.path.join(HERE, name + ".in"), "w") as f:
            f.write(text)
        with open(os.path.join(HERE, name + ".dump.sha256"), "w") as f:
            for fn in files:
                body = filtered(open(os.path.join(tmp, "dumps", fn)).read())
                f.write(f"{fn} {hashlib.sha256(body.encode()).hexdigest()}\n")
    print(name, len(files), "dump files")


def visit_deck():
    """The dump deck with visit output every second step (driver/hydro.cpp:95-96,
    :112; driver/start.cpp:131): files at steps 0, 2 and 3."""
    c = D.benchmark_deck(16, 3, ny=12)
    c.states.append(D.State(density=2.0, energy=3.0, xvel=0.5, yvel=-0.25, geometry=D.GEOM_CIRC, xmin=6.0, ymin=6.0,
                            radius=2.5, defined=True))
    c.visit_frequency = 2
    return "circ16x12x3v", D.format_deck(c)


def write_visit_fixture():
    name, text = visit_deck()
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "clover.in"), "w") as f:
            f.write(text)
        p = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "serial"), "--file", "clover.in"], cwd=tmp,
                           capture_output=True, text=True, timeout=600)
        if p.returncode != 0:
            raise SystemExit(f"{name}: reference exited {p.returncode}")
        files = sorted(fn for fn in os.listdir(tmp) if fn.endswith((".vtk", ".visit")))
        with open(os.path.join(HERE, name + ".in"), "w") as f:
            f.write(text)
        with open(os.path.join(HERE, name + ".visit.sha256"), "w") as f:
            for fn in files:
                body = open(os.path.join(tmp, fn), "rb").read()
                f.write(f"{fn} {hashlib.sha256(body).hexdigest()}\n")
    print(name, len(files), "visit files")


def main(only=None):
    if only is None:
        write_dump_fixture()
        write_visit_fixture()
        write_known_answer_decks()
    for name, (text, keep_fields) in decks().items():
        if only is not None and name not in only:
            continue
        res = oracle.run_reference(text)
        if res["returncode"] != 0:
            raise SystemExit(f"{name}: reference exited {res['returncode']}")
        with open(os.path.join(HERE, name + ".in"), "w") as f:
            f.write(text)
        with open(os.path.join(HERE, name + ".summary.txt"), "w") as f:
            for r in res["summaries"]:
                f.write("%d %.17e %.17e %.17e %.17e %.17e %.17e\n" % r)
        keep = [l for l in res["stdout"].splitlines() if "within" in l or "PASSED" in l or "Outcome" in l]
        with open(os.path.join(HERE, name + ".stdout.txt"), "w") as f:
            f.write("\n".join(keep) + "\n")
        if keep_fields:
            fl = res["fields"]
            d = D.parse_deck(text)
            oracle.write_fields(os.path.join(HERE, name + ".fields.bin"), d.x_cells, d.y_cells, fl)
        print(name, len(res["summaries"]), "summaries", "fields" if keep_fields else "")


if __name__ == "__main__":
    main(sys.argv[1:] or None)  # names: only those decks
