"""The host side of a decomposed run (cloverleaf_b200/decomp.py) on gloo
ranks on the CPU (127.0.0.1), against one undivided mesh held by the oracle:

* decompose() splits meshes as driver/comms.cpp:64-156 does (extents,
  remainders on the first columns / rows, neighbours);
* on a 2 x 2 split of a 13 x 10 mesh (4 ranks, uneven chunks), a seeded
  state is cut into the four chunks with their internal-face halos cleared;
  exchange() at depth 2 restores every element of every state field, halos
  and corners included, to the undivided mesh's values (depth 1 fills only
  the first halo layer);
* dt_min() over the chunks' own calc_dt (the oracle on each chunk) is the
  undivided mesh's calc_dt, to the bit; summary_sum() of the chunks' exactly
  rounded summaries is the undivided mesh's to 1e-15.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)

from cloverleaf_b200 import decomp as DC  # noqa: E402

NX, NY = 13, 10


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_decompose_as_the_reference():
    c = DC.decompose(13, 10, 4)  # mesh ratio 1.3: 2 x 2; 13 = 7 + 6, 10 = 5 + 5
    assert [(k.left, k.right, k.bottom, k.top) for k in c] == [(1, 7, 1, 5), (8, 13, 1, 5), (1, 7, 6, 10), (8, 13, 6, 10)]
    assert [k.neighbours for k in c] == [(-1, 1, -1, 2), (0, -1, -1, 3), (-1, 3, 0, -1), (2, -1, 1, -1)]
    c = DC.decompose(100, 10, 3)  # prime: 1-D along the longer axis
    assert [(k.left, k.right) for k in c] == [(1, 34), (35, 67), (68, 100)] and all(k.bottom == 1 and k.top == 10 for k in c)
    c = DC.decompose(10, 100, 6)  # mesh ratio 0.1: 1 x 6
    assert [(k.bottom, k.top) for k in c] == [(1, 17), (18, 34), (35, 51), (52, 68), (69, 84), (85, 100)]
    c = DC.decompose(64, 32, 8)  # mesh ratio 2: 8 / 1 > 2, 4 / 2 <= 2 -> 4 x 2
    assert len({k.left for k in c}) == 4 and len({k.bottom for k in c}) == 2


def _global_state():
    from gpu_util import random_state
    import oracle
    state, dom = random_state(NX, NY, seed=91)
    o = oracle.OracleChunk(NX, NY)
    o.build_field()
    o.initialise_chunk(*dom)
    for fid, a in state.items():
        o.field(fid)[:a.shape[0], :a.shape[1]] = a
    return o, state


def _local(info, g):
    """The chunk's window of a global array."""
    return lambda a, xe, ye: np.array(a[info.bottom - 1:info.bottom - 1 + info.ny + 4 + ye,
                                        info.left - 1:info.left - 1 + info.nx + 4 + xe])


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.dirname(os.path.abspath(__file__))):
        if p not in sys.path:
            sys.path.insert(0, p)
    import oracle
    from cloverleaf_b200 import decomp as dc
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    info = dc.decompose(NX, NY, world)[rank]
    og, state = _global_state()
    win = _local(info, og)
    want = {f: win(state[f], *dc.EXTRA[f]) for f in range(15)}
    res = {}
    for depth in (1, 2):
        fields = {f: want[f].copy() for f in range(15)}
        for f in range(15):  # clear the internal faces' halos, two deep
            for side in range(4):
                if info.neighbours[side] >= 0:
                    rs, cs = dc._recv_slice(info, f, side, 2)
                    fields[f][rs, cs] = 0.0
        dc.exchange(info, fields, range(15), depth)
        if depth == 2:
            res["exact"] = all(np.array_equal(fields[f], want[f]) for f in range(15))
        else:  # the first halo layer only
            ok = True
            for f in range(15):
                for side in range(4):
                    if info.neighbours[side] < 0:
                        continue
                    r1, c1 = dc._recv_slice(info, f, side, 1)
                    ok &= np.array_equal(fields[f][r1, c1], want[f][r1, c1])
            res["depth1"] = bool(ok)
    # calc_dt and the summary on the chunk, reduced over the chunks
    ol = oracle.OracleChunk(info.nx, info.ny)
    for f in range(15):
        a = want[f]
        ol.field(f)[:a.shape[0], :a.shape[1]] = a
    for f in (22, 23, 24):  # volume, xarea, yarea: the chunk's window of the mesh's
        xe, ye = (0, 0) if f == 22 else ((1, 0) if f == 23 else (0, 1))
        a = win(np.asarray(og.field(f)), xe, ye)
        ol.field(f)[:a.shape[0], :a.shape[1]] = a
    for g in ("cellx", "celly", "celldx", "celldy", "vertexx", "vertexy", "vertexdx", "vertexdy"):
        along_x = g in ("cellx", "celldx", "vertexx", "vertexdx")
        o0, n = (info.left - 1, info.nx) if along_x else (info.bottom - 1, info.ny)
        n += 5 if g.startswith("vertex") else 4
        ol.geom(g)[:n] = og.geom(g)[o0:o0 + n]
    res["dt"] = dc.dt_min(ol.calc_dt()[0])
    res["dt_global"] = og.calc_dt()[0]
    res["sums"] = dc.summary_sum(ol.field_summary(exact=True))
    res["sums_global"] = list(og.field_summary(exact=True))
    out[rank] = res
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_four_chunks_exchange_and_reduce_as_one_mesh():
    world, port = 4, _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        assert res[r]["exact"], r
        assert res[r]["depth1"], r
        assert res[r]["dt"] == res[r]["dt_global"], (r, res[r]["dt"], res[r]["dt_global"])
        for a, b in zip(res[r]["sums"], res[r]["sums_global"]):
            assert abs(a - b) <= 1e-15 * abs(b), (r, a, b)


@pytest.mark.timeout(300)
@pytest.mark.parametrize("world", [2, 4])
def test_decomposed_oracle_run_is_the_whole_mesh_run(world):
    """The benchmark deck (64 x 48) decomposed over two (2 x 1) and four
    (2 x 2) gloo ranks, each chunk held by the CPU oracle and driven by
    HydroRun's call sequence (update_halo = exchange of the internal faces,
    then the reflective fill of the physical ones): the dt of every step and
    every captured field of each chunk equal, bit for bit, the whole mesh's
    run; the summaries (sums reduced over the ranks) within 1e-13 of the
    whole mesh's exactly rounded sums.  (In this deck, split at column 32
    and row 24, the flow never crosses a chunk edge against advec_cell's
    upwind clamp, so the decomposed run is the whole mesh's run; split 3 x 1,
    at columns 22 and 43, it does, and the runs part.)"""
    from decomp_util import rank_body
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(rank_body, args=(world, port, out, "bm", False), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        assert res[r]["steps"][0] == res[r]["steps"][1], r
        assert res[r]["dt"], r
        assert res[r]["summary_steps"], r
        assert res[r]["bad"] == [], (r, res[r]["bad"])
        assert max(res[r]["sums"]) <= 1e-13, (r, res[r]["sums"])
