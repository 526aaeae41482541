"""A decomposed run on the GPU: each gloo rank holds one chunk of the mesh in
the library (DecomposedChunk on cuda:0: the chunk's geometry from
cb_initialise_chunk_in, the reflective halo on its physical faces only, the
internal faces filled by the exchange of driver/comms.cpp:clover_exchange,
dt and the summary's sums reduced over the ranks), driven by HydroRun's call
sequence.  Checked, rank by rank, against the same decomposed run on oracle
chunks (tests/decomp_util.py): every captured field of every chunk, the step
count and the dt of every step bit-identical in FP64; the final summary's
sums within 1e-13.

Decks: the benchmark deck (64 x 48) and a deck whose flow crosses the
chunk edges both ways (a moving circle, gamma 1.55; 56 x 40), so that
each chunk's own upwind clamp at its right / top edge face
(src/serial/advec_cell.cpp:77, :169) is exercised; over two (2 x 1), three (3 x 1, ragged
columns), four (2 x 2) and six (2 x 3, ragged rows in the circle deck) ranks.  The ranks' kernels never wait on one another: the
exchange is a host-side gloo step between the calls.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

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
    for r in range(world):
        assert res[r]["steps"][0] == res[r]["steps"][1], (r, res[r]["steps"])
        assert res[r]["dt"], r
        assert res[r]["summary_steps"], r
        assert res[r]["bad"] == [], (r, res[r]["bad"])
        assert max(res[r]["sums"]) <= 1e-13, (r, res[r]["sums"])
