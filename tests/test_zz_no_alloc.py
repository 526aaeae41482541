"""cb_field_summary_noalloc: the field summary for callers that must not
allocate device memory where they need it (their memory comes from their own
pool, or they sit in a loop that must stay allocation-free).  It works on
device arrays the caller owns and keeps its reduction scratch in a fixed
array inside the library.

Checked against cb_field_summary (the chunk's own summary, which allocates
its scratch with the chunk) on the same state: the five sums within 1e-13
relative (same per-cell terms, different grouping of the sums), the
ideal-gas pressure and sound speed bit for bit, and two calls in a row give
the same result (the shared scratch is reset between calls).  This file is
collected last, and passes alone or after the other tests."""
import ctypes

import numpy as np
import pytest

from cloverleaf_b200 import Chunk, HydroRun, benchmark_deck, library, nudged

pytestmark = pytest.mark.gpu

CB_EINVAL = 1


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _padded(torch, a, rows, pitch):
    buf = np.zeros((rows, pitch))
    buf[:a.shape[0], :a.shape[1]] = a
    return torch.from_numpy(buf).cuda()


def _call(lib, torch, nx, ny, pitch, arrays, out, stream):
    d0, e0, u0, v0, cdx, cdy = arrays
    p, c, sums = out
    return lib.cb_field_summary_noalloc(nx, ny, pitch, _ptr(d0), _ptr(e0), _ptr(u0), _ptr(v0), _ptr(cdx), _ptr(cdy), _ptr(p), _ptr(c),
                                        1.4, _ptr(sums), ctypes.c_void_p(stream))


@pytest.mark.parametrize("nx,ny,steps", [(300, 200, 25), (2048, 2048, 6)])
def test_noalloc_summary_matches_chunk_summary_twice(nx, ny, steps):
    """300 x 200, and 2048 x 2048: the largest square mesh the fixed scratch
    takes (exactly 16384 blocks of 32 x 8 cells)."""
    torch = pytest.importorskip("torch")
    chunk = Chunk(nx, ny)
    HydroRun(chunk, nudged(benchmark_deck(nx, steps, ny=ny))).run()  # a state with motion in it
    lib = library()
    pitch, rows = nx + 5, ny + 5
    arrays = [_padded(torch, chunk.read(n), rows, pitch) for n in ("density0", "energy0", "xvel0", "yvel0")]
    arrays += [torch.from_numpy(chunk.read_geom(g)).cuda() for g in ("celldx", "celldy")]
    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for _ in range(2):
        out = [torch.zeros((rows, pitch), dtype=torch.float64, device="cuda"),
               torch.zeros((rows, pitch), dtype=torch.float64, device="cuda"),
               torch.full((5,), float("nan"), dtype=torch.float64, device="cuda")]
        assert _call(lib, torch, nx, ny, pitch, arrays, out, stream) == 0, lib.cb_last_error()
        torch.cuda.synchronize()
        results.append([o.cpu().numpy() for o in out])
    ref = chunk.field_summary()  # the chunk's own summary (recomputes pressure and sound speed)
    for p, c, sums in results:
        for a, b in zip(sums, ref):
            assert abs(a - b) <= 1e-13 * abs(b), (a, b)
        assert np.array_equal(p[2:ny + 2, 2:nx + 2], chunk.read("pressure")[2:ny + 2, 2:nx + 2])
        assert np.array_equal(c[2:ny + 2, 2:nx + 2], chunk.read("soundspeed")[2:ny + 2, 2:nx + 2])
    assert np.array_equal(results[0][2], results[1][2])


@pytest.mark.parametrize("nx,ny,blocks", [(2100, 2100, 17358), (2049, 2048, 16640), (2050, 2040, 16575)])
def test_noalloc_rejects_mesh_beyond_scratch(nx, ny, blocks):
    """A mesh is accepted when ceil(nx/32) * ceil(ny/8) <= 16384: one column
    past 2048 x 2048 is rejected, and so is 2050 x 2040 although it has fewer
    than 4,194,304 cells.  Nothing is launched, so the arrays are never read."""
    torch = pytest.importorskip("torch")
    lib = library()
    small = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = lib.cb_field_summary_noalloc(nx, ny, nx + 5, *([_ptr(small)] * 8), 1.4, _ptr(small), ctypes.c_void_p(0))
    assert rc == CB_EINVAL
    msg = lib.cb_last_error()
    assert str(blocks).encode() in msg and b"16384" in msg and b"ceil(nx/32) * ceil(ny/8)" in msg, msg
