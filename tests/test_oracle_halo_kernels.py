"""The oracle's restatements of the reference's halo kernels against the
reference code itself: oracle/_ref/halo_kernels (oracle/ref_checks/
halo_kernels.cpp, built by `make -C oracle refchecks` from the reference
sources) calls update_tile_halo_{l,r,b,t}_kernel and update_halo_kernel on
seeded fields; the oracle's oc_tile_halo and oc_update_halo_faces must
produce every element of every field bit for bit.  (The reference driver
never reaches the tile kernels: it crashes in its tile decomposition.)

update_halo_kernel reads tile_neighbours[tile_bottom] and [tile_top], and
the reference declares both names as 3 (driver/definitions.h:58), so it can
only mark the bottom and top faces external together: the face masks here
keep those two bits equal."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "halo_kernels")

pytestmark = pytest.mark.skipif(not os.path.exists(EXE), reason="oracle/_ref/halo_kernels not built (needs the reference sources)")

# extent over the cells' (nx+4, ny+4) of each field (driver/definitions.cpp:4-41)
EXTRA = {0: (0, 0), 1: (0, 0), 2: (0, 0), 3: (0, 0), 4: (0, 0), 5: (0, 0), 6: (0, 0), 7: (1, 1), 8: (1, 1), 9: (1, 1),
         10: (1, 1), 11: (1, 0), 12: (0, 1), 13: (1, 0), 14: (0, 1)}


def seeded(nx, ny, tile):
    o = oracle.OracleChunk(nx, ny)
    for f in range(15):
        sx, sy = nx + 4 + EXTRA[f][0], ny + 4 + EXTRA[f][1]
        j, i = np.mgrid[0:sy, 0:sx]
        o.field(f)[:sy, :sx] = f * 1e6 + tile * 1e5 + j * 300.0 + i + 0.25
    return o


def reference(args, nx, ny):
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "out.bin")
        subprocess.run([EXE, *map(str, args), out], check=True, timeout=60)
        data = np.fromfile(out, dtype=np.float64)
    res, pos = {}, 0
    for f in range(15):
        sx, sy = nx + 4 + EXTRA[f][0], ny + 4 + EXTRA[f][1]
        res[f] = data[pos:pos + sx * sy].reshape(sy, sx)
        pos += sx * sy
    assert pos == data.size
    return res


def check(o, ref, nx, ny, what):
    for f in range(15):
        sx, sy = nx + 4 + EXTRA[f][0], ny + 4 + EXTRA[f][1]
        got = np.asarray(o.field(f))[:sy, :sx]
        assert np.array_equal(got, ref[f]), (what, f, np.argwhere(got != ref[f])[:4])


@pytest.mark.parametrize("side", [1, 2, 4, 8])
@pytest.mark.parametrize("depth", [1, 2])
def test_tile_halo_matches_reference(side, depth):
    nx, ny = 11, 7
    nx2, ny2 = (6, ny) if side in (1, 2) else (nx, 5)
    dst, src = seeded(nx, ny, 0), seeded(nx2, ny2, 1)
    dst.tile_halo(src, side, [1] * 15, depth)
    check(dst, reference(["tile", side, depth, nx, ny, nx2, ny2], nx, ny), nx, ny, f"tile side {side} depth {depth}")


@pytest.mark.parametrize("faces", [0, 1, 2, 3, 12, 13, 14, 15])
@pytest.mark.parametrize("depth", [1, 2])
def test_masked_update_halo_matches_reference(faces, depth):
    nx, ny = 9, 8
    o = seeded(nx, ny, 0)
    o.update_halo([1] * 15, depth, faces)
    check(o, reference(["halo", faces, depth, nx, ny], nx, ny), nx, ny, f"update_halo faces {faces} depth {depth}")
