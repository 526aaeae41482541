"""The host side of a decomposed (multi-process) run: chunk extents and
neighbours, the halo exchange between neighbouring chunks, and the two
reductions of the step, over torch.distributed (NCCL on GPUs, gloo on CPUs).

* decompose(): the 2-D split of driver/comms.cpp:64-156 (clover_decompose):
  chunk_x x chunk_y chunks, the first columns / rows one cell wider when the
  cells do not divide evenly, neighbours as 0-based ranks (-1: the mesh
  edge, where the reflective fill applies instead).
* exchange(): the update_halo exchange of src/serial/comms_kernel.cpp:54-...
  (clover_exchange): the left / right strips first, then the bottom / top
  ones, so that corner elements arrive from the diagonal chunk in two hops.
  Each strip is the sender's interior rows / columns next to the face and
  lands in the receiver's halo at the same global position -- the index
  rules of the reference's pack / unpack kernels (src/serial/pack_kernel.cpp),
  which are those of its tile halo kernels (one element further out for the
  arrays that extend one past the cells across the face).
* dt_min() / summary_sum(): calc_dt's minimum over chunks (one all_reduce
  MIN of a double) and field_summary's five sums (one all_reduce SUM).
* DecomposedChunk: one rank's chunk on its GPU with the calls a HydroRun
  makes, so that HydroRun(DecomposedChunk(...), deck, fold=False) is the
  reference driver's decomposed run: geometry as the reference forms a
  chunk's (cb_initialise_chunk_in), the reflective fill on the physical faces
  only (cb_set_external_faces), every update_halo an exchange of the internal
  faces followed by that fill (driver/update_halo.cpp), the PdV predictor's
  pressure halo likewise, calc_dt's minimum and the summary reduced over the
  ranks.  The strips stay on the device: the library packs each face's
  strip into a linear device buffer (cb_pack_face), the buffers go to the
  neighbours -- NCCL send/recv of the device buffers when the process group
  is NCCL's, through host memory for gloo -- and the library unpacks what
  arrives into the halo (cb_unpack_face).  exchange() is the same exchange
  on host arrays (the oracle's chunks in the tests).

Fields are 2-D arrays in the reference's index convention (x fastest, a
2-deep halo: cells (ny+4, nx+4), nodes (ny+5, nx+5), x faces (ny+4, nx+5),
y faces (ny+5, nx+4)), keyed by field id (driver/definitions.h:61-77).
"""
from __future__ import annotations

import dataclasses
from typing import Dict, Iterable, List, Tuple

import numpy as np

# extent beyond the cells' along x and y of each field id (driver/definitions.cpp:4-41)
EXTRA = {0: (0, 0), 1: (0, 0), 2: (0, 0), 3: (0, 0), 4: (0, 0), 5: (0, 0), 6: (0, 0), 7: (1, 1), 8: (1, 1), 9: (1, 1),
         10: (1, 1), 11: (1, 0), 12: (0, 1), 13: (1, 0), 14: (0, 1)}
LEFT, RIGHT, BOTTOM, TOP = 0, 1, 2, 3  # driver/definitions.h:57 (chunk_left .. chunk_top)
_FACE_BIT = {LEFT: 1, RIGHT: 2, BOTTOM: 4, TOP: 8}  # the library's CB_FACE_* bits


@dataclasses.dataclass
class ChunkInfo:
    rank: int
    left: int    # first and last interior cell, 1-based global indices (driver/comms.cpp:122-125)
    right: int
    bottom: int
    top: int
    neighbours: Tuple[int, int, int, int]  # LEFT, RIGHT, BOTTOM, TOP: ranks, -1 at the mesh edge

    @property
    def nx(self) -> int:
        return self.right - self.left + 1

    @property
    def ny(self) -> int:
        return self.top - self.bottom + 1


def decompose(x_cells: int, y_cells: int, nchunks: int) -> List[ChunkInfo]:
    """The chunks of driver/comms.cpp:64-156, in rank order."""
    mesh_ratio = x_cells / y_cells
    chunk_x, chunk_y, found = nchunks, 1, False
    for c in range(1, nchunks + 1):
        if nchunks % c == 0:
            factor_x, factor_y = nchunks / c, c
            if factor_x / factor_y <= mesh_ratio:
                chunk_y, chunk_x, found = c, nchunks // c, True
                break
    if not found or chunk_y == nchunks:  # a prime count or a 1-D split
        chunk_x, chunk_y = (nchunks, 1) if mesh_ratio >= 1.0 else (1, nchunks)
    delta_x, delta_y = x_cells // chunk_x, y_cells // chunk_y
    mod_x, mod_y = x_cells % chunk_x, y_cells % chunk_y
    out = []
    add_y_prev = 0
    for cy in range(1, chunk_y + 1):
        add_x_prev = 0
        for cx in range(1, chunk_x + 1):
            add_x = 1 if cx <= mod_x else 0
            add_y = 1 if cy <= mod_y else 0
            left = (cx - 1) * delta_x + 1 + add_x_prev
            bottom = (cy - 1) * delta_y + 1 + add_y_prev
            rank = chunk_x * (cy - 1) + cx - 1
            nb = (rank - 1 if cx > 1 else -1, rank + 1 if cx < chunk_x else -1,
                  rank - chunk_x if cy > 1 else -1, rank + chunk_x if cy < chunk_y else -1)
            out.append(ChunkInfo(rank, left, left + delta_x - 1 + add_x, bottom, bottom + delta_y - 1 + add_y, nb))
            if cx <= mod_x:
                add_x_prev += 1
        if cy <= mod_y:
            add_y_prev += 1
    return out


def _send_slice(info: ChunkInfo, fid: int, side: int, depth: int) -> Tuple[slice, slice]:
    """(rows, columns) of the strip this chunk sends to its neighbour on `side`."""
    xe, ye = EXTRA[fid]
    nx, ny = info.nx, info.ny
    rows_lr = slice(2 - depth, ny + ye + depth + 2)
    cols_bt = slice(2 - depth, nx + xe + depth + 2)
    if side == LEFT:  # clover_pack_message_left: field(x_min + x_inc - 1 + j + 2, k)
        return rows_lr, slice(2 + xe, 2 + xe + depth)
    if side == RIGHT:  # clover_pack_message_right: field(x_max + 1 - j, k)
        return rows_lr, slice(nx + 2 - depth, nx + 2)
    if side == BOTTOM:
        return slice(2 + ye, 2 + ye + depth), cols_bt
    return slice(ny + 2 - depth, ny + 2), cols_bt


def _recv_slice(info: ChunkInfo, fid: int, side: int, depth: int) -> Tuple[slice, slice]:
    """(rows, columns) of this chunk's halo that the neighbour on `side` fills."""
    xe, ye = EXTRA[fid]
    nx, ny = info.nx, info.ny
    rows_lr = slice(2 - depth, ny + ye + depth + 2)
    cols_bt = slice(2 - depth, nx + xe + depth + 2)
    if side == LEFT:  # clover_unpack_message_left: field(x_min - j, k)
        return rows_lr, slice(2 - depth, 2)
    if side == RIGHT:
        return rows_lr, slice(nx + 2 + xe, nx + 2 + xe + depth)
    if side == BOTTOM:
        return slice(2 - depth, 2), cols_bt
    return slice(ny + 2 + ye, ny + 2 + ye + depth), cols_bt


def exchange(info: ChunkInfo, fields: Dict[int, np.ndarray], fids: Iterable[int], depth: int, group=None):
    """Fills this chunk's halos on its internal faces, `depth` deep, for the
    listed fields, from its neighbours (collective: every rank calls it with
    the same fids and depth)."""
    import torch
    import torch.distributed as dist
    fids = sorted(set(int(f) for f in fids))
    if depth not in (1, 2):
        raise ValueError("exchange: depth must be 1 or 2")
    for pair in ((LEFT, RIGHT), (BOTTOM, TOP)):
        reqs, recv = [], []
        for side in pair:
            nb = info.neighbours[side]
            if nb < 0:
                continue
            send = np.concatenate([np.ascontiguousarray(fields[f][_send_slice(info, f, side, depth)]).ravel() for f in fids])
            buf = torch.empty(send.size, dtype=torch.float64)
            reqs.append(dist.isend(torch.from_numpy(send), nb, group=group))
            reqs.append(dist.irecv(buf, nb, group=group))
            recv.append((side, buf))
        for r in reqs:
            r.wait()
        for side, buf in recv:
            flat, pos = buf.numpy(), 0
            for f in fids:
                rs, cs = _recv_slice(info, f, side, depth)
                dst = fields[f][rs, cs]
                dst[...] = flat[pos:pos + dst.size].reshape(dst.shape)
                pos += dst.size


def dt_min(local_dt: float, group=None) -> float:
    """calc_dt's minimum over every chunk (driver/comms.cpp: clover_min)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(local_dt)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    return float(t.item())


def summary_sum(local: Iterable[float], group=None) -> List[float]:
    """field_summary's five sums over every chunk (driver/comms.cpp: clover_sum)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x) for x in local], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return [float(x) for x in t.tolist()]


class DecomposedChunk:
    """One rank's chunk of a decomposed run (see the module docstring); the
    other chunk calls go to the chunk as they are."""

    def __init__(self, info: ChunkInfo, deck, precision: int = 0, device: int = 0, group=None):
        from .chunk import FACE_BOTTOM, FACE_LEFT, FACE_RIGHT, FACE_TOP, Chunk
        self.info, self.deck, self.group, self.device = info, deck, group, device
        self._bufs = {}
        self.c = Chunk(info.nx, info.ny, precision=precision, gamma=deck.gamma, device=device)
        faces = 0
        for side, bit in ((LEFT, FACE_LEFT), (RIGHT, FACE_RIGHT), (BOTTOM, FACE_BOTTOM), (TOP, FACE_TOP)):
            if info.neighbours[side] < 0:
                faces |= bit
        self.c.set_external_faces(faces)

    def __getattr__(self, name):
        return getattr(self.c, name)

    def initialise_chunk(self, xmin, ymin, xmax, ymax):
        d, i = self.deck, self.info
        self.c.initialise_chunk_in(xmin, ymin, xmax, ymax, d.x_cells, d.y_cells, i.left, i.bottom)

    def update_halo(self, fields, depth: int):
        fids = sorted(set(int(f) for f in fields))
        if any(n >= 0 for n in self.info.neighbours):
            self._exchange_strips(fids, depth)
        self.c.update_halo(fids, depth)

    def _strip_buffers(self, side: int, fids: List[int], depth: int):
        """The send and receive device buffers of one face strip, kept for the
        chunk's life (the library's stream uses them after this call returns)."""
        import torch
        key = (side, tuple(fids), depth)
        if key not in self._bufs:
            from .chunk import FP64
            n = self.c.face_strip_size(_FACE_BIT[side], fids, depth)
            dtype = torch.float64 if self.c.precision == FP64 else torch.float32
            dev = torch.device("cuda", self.device)
            self._bufs[key] = (torch.empty(n, dtype=dtype, device=dev), torch.empty(n, dtype=dtype, device=dev), n)
        return self._bufs[key]

    def _exchange_strips(self, fids: List[int], depth: int):
        """clover_exchange on the device: left / right strips, then bottom / top."""
        import torch
        import torch.distributed as dist
        stream = torch.cuda.ExternalStream(self.c.stream(), device=torch.device("cuda", self.device))
        nccl = dist.get_backend(self.group) == "nccl"
        if nccl:
            torch.cuda.set_device(self.device)  # NCCL's point-to-point calls run on the current device
        for pair in ((LEFT, RIGHT), (BOTTOM, TOP)):
            sides = [s for s in pair if self.info.neighbours[s] >= 0]
            if not sides:
                continue
            bufs = {s: self._strip_buffers(s, fids, depth) for s in sides}
            for s in sides:
                snd, _, n = bufs[s]
                self.c.pack_face(_FACE_BIT[s], fids, depth, snd.data_ptr(), n)
            if nccl:  # device buffers straight to the neighbours, ordered on the chunk's stream
                with torch.cuda.stream(stream):
                    ops = []
                    for s in sides:
                        snd, rcv, _ = bufs[s]
                        ops.append(dist.P2POp(dist.isend, snd, self.info.neighbours[s], group=self.group))
                        ops.append(dist.P2POp(dist.irecv, rcv, self.info.neighbours[s], group=self.group))
                    for w in dist.batch_isend_irecv(ops):
                        w.wait()
            else:  # gloo: the strips through host memory
                self.c.synchronize()
                reqs, host = [], {}
                for s in sides:
                    snd, _, n = bufs[s]
                    host[s] = torch.empty(n, dtype=snd.dtype)
                    reqs.append(dist.isend(snd.cpu(), self.info.neighbours[s], group=self.group))
                    reqs.append(dist.irecv(host[s], self.info.neighbours[s], group=self.group))
                for r in reqs:
                    r.wait()
                with torch.cuda.stream(stream):
                    for s in sides:
                        bufs[s][1].copy_(host[s])
            for s in sides:
                _, rcv, n = bufs[s]
                self.c.unpack_face(_FACE_BIT[s], fids, depth, rcv.data_ptr(), n)

    def pdv(self, predict: bool, dt: float, full: bool = False, halo_depth: int = 0):
        # the predictor's own pressure halo (src/serial/PdV.cpp:118-124) is an exchange too
        self.c.pdv(predict, dt, full=full, halo_depth=0)
        if full and halo_depth > 0:
            self.update_halo([4], halo_depth)  # pressure

    def calc_dt(self, *args, **kw):
        dt, control, jldt, kldt, small = self.c.calc_dt(*args, **kw)
        return dt_min(dt, self.group), control, jldt, kldt, small

    def field_summary(self):
        return tuple(summary_sum(self.c.field_summary(), self.group))

    def close(self):
        self.c.close()
