"""The tile primitives against the oracle's restatement of the reference's
kernels, on seeded random states (every element, halos included, bit for bit):

* cb_copy_tile_halo: each of update_tile_halo_{l,r,b,t}_kernel
  (src/serial/update_tile_halo_kernel.cpp), depth 1 and 2, all 15 fields,
  tiles of different widths along the shared face's normal;
* cb_set_external_faces + cb_update_halo: update_halo_kernel's reflective
  fill on the external faces only (src/serial/update_halo.cpp:41-71), and no
  producer folds its halo while a face is internal.

The reference driver's own tiles_per_chunk > 1 path cannot be run: its
serial and OpenMP builds end in a segmentation fault on every such deck
(its neighbour indices, driver/comms.cpp:212-215, point one tile off and
tile_bottom equals tile_top, driver/definitions.h:58).  The b200 model
rejects such a deck with the driver's error report instead.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from cloverleaf_b200 import chunk as C
from golden_util import deck_text
from gpu_util import Pair

pytestmark = pytest.mark.gpu

ALL = list(range(15))
SIDES = [C.FACE_LEFT, C.FACE_RIGHT, C.FACE_BOTTOM, C.FACE_TOP]


def tile_pair(side, seed):
    """dst and src tiles sharing the face's extent: 13 x 9 and (8 or 13) x (9 or 5)."""
    dst = Pair(13, 9, seed=seed)
    src = Pair(8, 9, seed=seed + 1) if side in (C.FACE_LEFT, C.FACE_RIGHT) else Pair(13, 5, seed=seed + 1)
    return dst, src


@pytest.mark.parametrize("side", SIDES)
@pytest.mark.parametrize("depth", [1, 2])
def test_copy_tile_halo_matches_reference_kernel(side, depth):
    dst, src = tile_pair(side, 40 + side + depth)
    fields = [f for f in ALL if (f + side) % 3 != 0]  # a subset: the others stay untouched
    dst.g.copy_tile_halo(src.g, side, fields, depth)
    dst.o.tile_halo(src.o, side, [1 if f in fields else 0 for f in ALL], depth)
    dst.assert_equal(ALL, f"tile halo side {side} depth {depth}")
    src.assert_equal(ALL, "source tile unchanged")


@pytest.mark.parametrize("faces", [0, 1, 2, 4, 8, 5, 10, 14])
@pytest.mark.parametrize("depth", [1, 2])
def test_update_halo_external_faces_only(faces, depth):
    p = Pair(11, 9, seed=60 + faces)
    p.g.set_external_faces(faces)
    p.g.update_halo(ALL, depth)
    p.o.update_halo([1] * 15, depth, faces)
    p.assert_equal(ALL, f"update_halo faces {faces} depth {depth}")


def test_no_fold_with_an_internal_face():
    """A producer asked for a halo depth folds nothing when a face is internal:
    the halo is then written by update_halo on the external faces only."""
    p = Pair(40, 24, seed=70)
    p.g.set_external_faces(C.FACE_LEFT | C.FACE_BOTTOM | C.FACE_TOP)
    p.g.ideal_gas(False, 1)
    p.g.update_halo(["pressure"], 1)
    p.o.ideal_gas(False)
    flags = [0] * 15
    flags[C.FIELD_ID["pressure"]] = 1
    p.o.update_halo(flags, 1, C.FACE_LEFT | C.FACE_BOTTOM | C.FACE_TOP)
    p.assert_equal(ALL, "ideal_gas + update_halo with an internal right face")


def test_driver_rejects_tiles_per_chunk():
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cloverleaf_b200", "bin", "clover_leaf")
    text = deck_text("bm32x87").replace("*endclover", "tiles_per_chunk 2\n*endclover")
    with tempfile.TemporaryDirectory() as tmp:
        deck = os.path.join(tmp, "clover.in")
        open(deck, "w").write(text)
        p = subprocess.run([exe, "--file", deck], cwd=tmp, capture_output=True, text=True, timeout=120)
    assert p.returncode != 0 and p.returncode != -11  # an error report, not a crash
    assert "tiles_per_chunk" in p.stdout + p.stderr
