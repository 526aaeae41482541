"""A decomposed run on the GPU: each gloo rank holds one chunk of the mesh in
the library (DecomposedChunk on cuda:0: the chunk's geometry from
cb_initialise_chunk_in, the reflective halo on its physical faces only, the
internal faces filled by the exchange of driver/comms.cpp:clover_exchange,
dt and the summary's sums reduced over the ranks), driven by HydroRun's call
sequence.  Checked, rank by rank, against the same decomposed run on oracle
chunks (tests/decomp_util.py): every captured field of every chunk, the step
count and the dt of every step bit-identical in FP64; the final summary's
sums within 1e-13 of the oracle chunks' exactly rounded sums.

Decks: the benchmark deck (64 x 48) and a deck whose flow crosses the
chunk edges both ways (a moving circle, gamma 1.55; 56 x 40), so that
each chunk's own upwind clamp at its right / top edge face
(src/serial/advec_cell.cpp:77, :169) is exercised; over two (2 x 1), three (3 x 1, ragged
columns), four (2 x 2) and six (2 x 3, ragged rows in the circle deck) ranks.  The ranks' kernels never wait on one another: the
exchange is a host-side gloo step between the calls.

The face strips on their own (cb_pack_face / cb_unpack_face): a strip packed
by one chunk and unpacked into its neighbour moves exactly the elements the
host exchange (decomp.exchange, checked against the whole mesh on CPU)
moves, for every field, both depths, all four faces and both precisions,
and nothing else.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from cloverleaf_b200 import FP32, FP64, Chunk  # noqa: E402
from cloverleaf_b200 import decomp as DC  # noqa: E402

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.timeout(600)
@pytest.mark.parametrize("world", [2, 3, 4, 6])
@pytest.mark.parametrize("deck_name", ["bm", "circle"])
def test_decomposed_gpu_run_is_the_decomposed_oracle_run(deck_name, world):
    from decomp_util import rank_body
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(rank_body, args=(world, port, out, deck_name, True), nprocs=world, join=True)
        res = dict(out)
    _check(res, world)


def _check(res, world):
    for r in range(world):
        assert res[r]["steps"][0] == res[r]["steps"][1], (r, res[r]["steps"])
        assert res[r]["dt"], r
        assert res[r]["summary_steps"], r
        assert res[r]["bad"] == [], (r, res[r]["bad"])
        assert max(res[r]["sums"]) <= 1e-13, (r, res[r]["sums"])


@pytest.mark.timeout(600)
@pytest.mark.parametrize("mode", ["fold", "fuse"])
def test_decomposed_run_with_folds_and_call_fusion(mode):
    """The circle deck on four ranks with HydroRun's halo depths passed to the
    calls, and with the chunk's call fusion on: with internal faces the
    chunks fold no halo and run the held-back calls as made, so the run is
    the decomposed oracle run, bit for bit."""
    from decomp_util import rank_body
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(rank_body, args=(4, port, out, "circle", True, mode), nprocs=4, join=True)
        res = dict(out)
    _check(res, 4)


@pytest.mark.timeout(600)
@pytest.mark.parametrize("deck_name", ["sodxy10x10", "sodbig200"])
def test_decomposed_run_of_the_reference_sod_decks(deck_name):
    """The reference's own Sod decks decomposed over four ranks (2 x 2:
    chunks of 5 x 5 cells, below the size at which the library folds halos,
    and of 100 x 100 over 200 steps): the GPU run is the decomposed oracle
    run, bit for bit."""
    from decomp_util import rank_body
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(rank_body, args=(4, port, out, deck_name, True), nprocs=4, join=True)
        res = dict(out)
    _check(res, 4)


def _info(nx, ny):
    return DC.ChunkInfo(rank=0, left=1, right=nx, bottom=1, top=ny, neighbours=(-1, -1, -1, -1))


@pytest.mark.parametrize("precision", [FP64, FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("depth", [1, 2])
@pytest.mark.parametrize("pair", ["left_right", "bottom_top"])
def test_face_strip_moves_what_the_host_exchange_moves(pair, depth, precision):
    rng = np.random.default_rng(17 + depth + 3 * precision)
    # a and b share the face's extent: a is left of (below) b
    (anx, any_), (bnx, bny) = ((13, 9), (8, 9)) if pair == "left_right" else ((11, 7), (11, 10))
    a, b = Chunk(anx, any_, precision=precision), Chunk(bnx, bny, precision=precision)
    for c in (a, b):
        for f in range(15):
            sx, sy = c.extent(f)
            c.write(f, rng.standard_normal((sy, sx)))
    before_a = {f: a.read(f) for f in range(15)}
    before_b = {f: b.read(f) for f in range(15)}
    lo, hi = (DC.LEFT, DC.RIGHT) if pair == "left_right" else (DC.BOTTOM, DC.TOP)
    fids = list(range(15))
    dtype = torch.float64 if precision == FP64 else torch.float32
    # a's strip for its neighbour on the high side into b's low halo, and b's for a
    n_ab = a.face_strip_size(DC._FACE_BIT[hi], fids, depth)
    n_ba = b.face_strip_size(DC._FACE_BIT[lo], fids, depth)
    assert n_ab == n_ba
    buf_ab = torch.empty(n_ab, dtype=dtype, device="cuda")
    buf_ba = torch.empty(n_ba, dtype=dtype, device="cuda")
    a.pack_face(DC._FACE_BIT[hi], fids, depth, buf_ab.data_ptr(), n_ab)
    b.pack_face(DC._FACE_BIT[lo], fids, depth, buf_ba.data_ptr(), n_ba)
    a.synchronize()
    b.synchronize()
    b.unpack_face(DC._FACE_BIT[lo], fids, depth, buf_ab.data_ptr(), n_ab)
    a.unpack_face(DC._FACE_BIT[hi], fids, depth, buf_ba.data_ptr(), n_ba)
    a.synchronize()
    b.synchronize()
    ia, ib = _info(anx, any_), _info(bnx, bny)
    for f in fids:
        want_b, want_a = before_b[f].copy(), before_a[f].copy()
        want_b[DC._recv_slice(ib, f, lo, depth)] = before_a[f][DC._send_slice(ia, f, hi, depth)]
        want_a[DC._recv_slice(ia, f, hi, depth)] = before_b[f][DC._send_slice(ib, f, lo, depth)]
        assert np.array_equal(b.read(f), want_b), f
        assert np.array_equal(a.read(f), want_a), f
    with pytest.raises(Exception):
        a.pack_face(DC._FACE_BIT[hi], fids, depth, buf_ab.data_ptr(), n_ab - 1)  # too small a buffer is refused
    a.close()
    b.close()
