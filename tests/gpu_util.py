"""Shared helpers of the GPU parity tests: one seeded random mesh state loaded
identically into the CPU oracle and a GPU chunk, and field comparison."""
import numpy as np

import oracle
from cloverleaf_b200 import Chunk
from cloverleaf_b200.chunk import FP64

KIND = {0: "cell", 1: "cell", 2: "cell", 3: "cell", 4: "cell", 5: "cell", 6: "cell", 7: "node", 8: "node",
        9: "node", 10: "node", 11: "xface", 12: "yface", 13: "xface", 14: "yface"}


def extent(nx, ny, fid):
    k = KIND[fid]
    return (nx + (5 if k in ("node", "xface") else 4), ny + (5 if k in ("node", "yface") else 4))


def random_state(nx, ny, seed):
    """Plausible hydro fields over the whole extent (halos too): positive
    density/energy/pressure, small velocities and fluxes so every volume in
    the advection stays positive."""
    rng = np.random.default_rng(seed)
    dx, dy = 3.7 / nx, 1.9 / ny
    vol = dx * dy
    out = {}
    for fid in range(15):
        sx, sy = extent(nx, ny, fid)
        shape = (sy, sx)
        if fid in (0, 1):
            a = rng.uniform(0.5, 2.0, shape)
        elif fid in (2, 3):
            a = rng.uniform(1.0, 3.0, shape)
        elif fid == 4:
            a = rng.uniform(0.1, 1.0, shape)
        elif fid == 5:
            a = rng.uniform(0.0, 0.05, shape) * (rng.uniform(size=shape) < 0.3)
        elif fid == 6:
            a = rng.uniform(0.5, 1.5, shape)
        elif fid in (7, 8, 9, 10):
            a = rng.uniform(-0.3, 0.3, shape)
            a[rng.uniform(size=shape) < 0.1] = 0.0
        elif fid in (11, 12):
            a = rng.uniform(-0.08, 0.08, shape) * vol
        else:
            a = rng.uniform(-0.08, 0.08, shape) * vol * 1.5
        out[fid] = a
    return out, (0.0, 0.0, 3.7, 1.9)


class Pair:
    """The same state on the oracle and on a GPU chunk."""

    def __init__(self, nx, ny, seed=0, precision=FP64, gamma=1.4):
        self.nx, self.ny = nx, ny
        self.o = oracle.OracleChunk(nx, ny, gamma)
        self.g = Chunk(nx, ny, precision=precision, gamma=gamma)
        state, dom = random_state(nx, ny, seed)
        self.o.build_field()
        self.o.initialise_chunk(*dom)
        self.g.build_field()
        self.g.initialise_chunk(*dom)
        for fid, a in state.items():
            sy, sx = a.shape
            self.o.field(fid)[:sy, :sx] = a
            self.g.write(fid, a)

    def gpu(self, fid):
        return self.g.read(fid)

    def cpu(self, fid):
        sx, sy = extent(self.nx, self.ny, fid)
        return np.array(self.o.field(fid)[:sy, :sx])

    def assert_equal(self, fids, what=""):
        for fid in fids:
            a, b = self.gpu(fid), self.cpu(fid)
            if not np.array_equal(a, b):
                bad = np.argwhere(a != b)
                j, i = bad[0]
                raise AssertionError(f"{what}: field {fid} differs at {len(bad)} points, first (i={i}, j={j}): "
                                     f"gpu {a[j, i]!r} oracle {b[j, i]!r}")
