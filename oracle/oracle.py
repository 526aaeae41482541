"""ctypes front end of the CPU oracle (oracle/clover_oracle.c) and a runner for
the reference build under oracle/_ref/.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, always as the checker, never as the thing that is
measured or shipped.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
import tempfile
from typing import Dict, List, Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

NUM_2D = 25
FIELD_NAMES = ["density0", "density1", "energy0", "energy1", "pressure", "viscosity", "soundspeed",
               "xvel0", "xvel1", "yvel0", "yvel1", "vol_flux_x", "vol_flux_y", "mass_flux_x", "mass_flux_y",
               "work1", "work2", "work3", "work4", "work5", "work6", "work7", "volume", "xarea", "yarea"]
FIELD_ID = {n: i for i, n in enumerate(FIELD_NAMES)}
GEOM_NAMES = ["cellx", "celly", "celldx", "celldy", "vertexx", "vertexy", "vertexdx", "vertexdy"]
GEOM_ID = {n: i for i, n in enumerate(GEOM_NAMES)}


class _State(ctypes.Structure):
    _fields_ = [("density", ctypes.c_double), ("energy", ctypes.c_double), ("xvel", ctypes.c_double),
                ("yvel", ctypes.c_double), ("geometry", ctypes.c_int), ("xmin", ctypes.c_double),
                ("ymin", ctypes.c_double), ("xmax", ctypes.c_double), ("ymax", ctypes.c_double),
                ("radius", ctypes.c_double)]


class _Config(ctypes.Structure):
    _fields_ = [("x_cells", ctypes.c_int), ("y_cells", ctypes.c_int), ("xmin", ctypes.c_double),
                ("ymin", ctypes.c_double), ("xmax", ctypes.c_double), ("ymax", ctypes.c_double),
                ("dtinit", ctypes.c_double), ("dtmin", ctypes.c_double), ("dtmax", ctypes.c_double),
                ("dtrise", ctypes.c_double), ("dtu_safe", ctypes.c_double), ("dtv_safe", ctypes.c_double),
                ("dtc_safe", ctypes.c_double), ("dtdiv_safe", ctypes.c_double), ("end_time", ctypes.c_double),
                ("end_step", ctypes.c_int), ("summary_frequency", ctypes.c_int), ("number_of_states", ctypes.c_int),
                ("states", ctypes.POINTER(_State)), ("gamma", ctypes.c_double)]


class _Summary(ctypes.Structure):
    _fields_ = [("step", ctypes.c_int), ("time", ctypes.c_double), ("vol", ctypes.c_double),
                ("mass", ctypes.c_double), ("ie", ctypes.c_double), ("ke", ctypes.c_double),
                ("press", ctypes.c_double)]


class _Chunk(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("sx", ctypes.c_int), ("sy", ctypes.c_int),
                ("gamma", ctypes.c_double), ("f", ctypes.POINTER(ctypes.c_double) * NUM_2D),
                ("g", ctypes.POINTER(ctypes.c_double) * 8)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run `make -C oracle`)")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(_Chunk)
        d = ctypes.c_double
        i = ctypes.c_int
        L.oc_create.restype = P
        L.oc_create.argtypes = [i, i, d]
        L.oc_destroy.argtypes = [P]
        for name, args in [("oc_build_field", []), ("oc_ideal_gas", [i]), ("oc_viscosity", []),
                           ("oc_pdv_kernel", [i, d]), ("oc_pdv", [i, d]), ("oc_revert", []), ("oc_accelerate", [d]),
                           ("oc_flux_calc", [d]), ("oc_advec_cell", [i, i]), ("oc_advec_mom", [i, i, i]),
                           ("oc_reset_field", []), ("oc_advection", [i]),
                           ("oc_initialise_chunk", [d, d, d, d])]:
            fn = getattr(L, name)
            fn.argtypes = [P] + args
            fn.restype = None
        L.oc_generate_chunk.argtypes = [P, i, ctypes.POINTER(_State)]
        L.oc_update_halo.argtypes = [P, ctypes.POINTER(ctypes.c_int), i]
        L.oc_update_halo_faces.argtypes = [P, ctypes.POINTER(ctypes.c_int), i, i]
        L.oc_tile_halo.argtypes = [P, P, i, ctypes.POINTER(ctypes.c_int), i]
        L.oc_field_summary.argtypes = [P, ctypes.POINTER(d)]
        L.oc_field_summary_exact.argtypes = [P, ctypes.POINTER(d)]
        ip = ctypes.POINTER(i)
        L.oc_calc_dt.argtypes = [P, d, d, d, d, d, ip, ip, ip, ip]
        L.oc_calc_dt.restype = d
        L.oc_run.argtypes = [P, ctypes.POINTER(_Config), ctypes.POINTER(_Summary), i, ip, ctypes.POINTER(d), i]
        L.oc_run.restype = i
        _lib = L
    return _lib


def _states(deck) -> ctypes.Array:
    arr = (_State * len(deck.states))()
    for k, s in enumerate(deck.states):
        arr[k] = _State(s.density, s.energy, s.xvel, s.yvel, s.geometry, s.xmin, s.ymin, s.xmax, s.ymax, s.radius)
    return arr


class OracleChunk:
    """One mesh chunk held by the C oracle; field views are (ny+5, nx+5) numpy arrays indexed [j, i]."""

    def __init__(self, nx: int, ny: int, gamma: float = 1.4):
        self._L = lib()
        self._c = self._L.oc_create(nx, ny, gamma)
        if not self._c:
            raise MemoryError("oc_create failed")
        self.nx, self.ny = nx, ny

    def close(self):
        if self._c:
            self._L.oc_destroy(self._c)
            self._c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field(self, name) -> np.ndarray:
        fid = FIELD_ID[name] if isinstance(name, str) else int(name)
        ptr = self._c.contents.f[fid]
        return np.ctypeslib.as_array(ptr, shape=(self.ny + 5, self.nx + 5))

    def geom(self, name) -> np.ndarray:
        gid = GEOM_ID[name] if isinstance(name, str) else int(name)
        ptr = self._c.contents.g[gid]
        return np.ctypeslib.as_array(ptr, shape=(max(self.nx, self.ny) + 6,))

    # per-phase restatements
    def build_field(self): self._L.oc_build_field(self._c)
    def initialise_chunk(self, xmin, ymin, xmax, ymax): self._L.oc_initialise_chunk(self._c, xmin, ymin, xmax, ymax)
    def generate_chunk(self, deck):
        st = _states(deck)
        self._L.oc_generate_chunk(self._c, len(deck.states), st)
    def ideal_gas(self, predict): self._L.oc_ideal_gas(self._c, int(predict))
    def viscosity(self): self._L.oc_viscosity(self._c)
    def pdv_kernel(self, predict, dt): self._L.oc_pdv_kernel(self._c, int(predict), dt)
    def pdv(self, predict, dt): self._L.oc_pdv(self._c, int(predict), dt)
    def revert(self): self._L.oc_revert(self._c)
    def accelerate(self, dt): self._L.oc_accelerate(self._c, dt)
    def flux_calc(self, dt): self._L.oc_flux_calc(self._c, dt)
    def advec_cell(self, sweep, direction): self._L.oc_advec_cell(self._c, sweep, direction)
    def advec_mom(self, which_vel, sweep, direction): self._L.oc_advec_mom(self._c, which_vel, sweep, direction)
    def reset_field(self): self._L.oc_reset_field(self._c)
    def advection(self, advect_x): self._L.oc_advection(self._c, int(advect_x))

    def update_halo(self, fields, depth, faces=15):
        """fields: 15 flags; faces: the external faces filled (1 left, 2 right, 4 bottom, 8 top)."""
        arr = (ctypes.c_int * 15)(*[1 if f else 0 for f in fields])
        if faces == 15:
            self._L.oc_update_halo(self._c, arr, depth)
        else:
            self._L.oc_update_halo_faces(self._c, arr, depth, faces)

    def tile_halo(self, src, side, fields, depth):
        """This tile's halo on `side` from `src` (update_tile_halo_kernel.cpp); fields: 15 flags."""
        arr = (ctypes.c_int * 15)(*[1 if f else 0 for f in fields])
        self._L.oc_tile_halo(self._c, src._c, side, arr, depth)

    def calc_dt(self, dtmin=0.0000001, dtc_safe=0.7, dtu_safe=0.5, dtv_safe=0.5, dtdiv_safe=0.7):
        a, b, c_, s = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        dt = self._L.oc_calc_dt(self._c, dtmin, dtc_safe, dtu_safe, dtv_safe, dtdiv_safe,
                                ctypes.byref(a), ctypes.byref(b), ctypes.byref(c_), ctypes.byref(s))
        return dt, a.value, b.value, c_.value, s.value

    def field_summary(self, exact=False) -> Tuple[float, ...]:
        out = (ctypes.c_double * 5)()
        (self._L.oc_field_summary_exact if exact else self._L.oc_field_summary)(self._c, out)
        return tuple(out)

    def run(self, deck, max_summaries=4096, dt_trace_len=0):
        """Whole run of a (nudged) deck; returns (summaries, steps, dt_trace)."""
        st = _states(deck)
        cfg = _Config(deck.x_cells, deck.y_cells, deck.xmin, deck.ymin, deck.xmax, deck.ymax, deck.dtinit,
                      deck.dtmin, deck.dtmax, deck.dtrise, deck.dtu_safe, deck.dtv_safe, deck.dtc_safe,
                      deck.dtdiv_safe, deck.end_time, deck.end_step, deck.summary_frequency,
                      len(deck.states), st, deck.gamma)
        out = (_Summary * max_summaries)()
        steps = ctypes.c_int()
        trace = (ctypes.c_double * max(dt_trace_len, 1))()
        n = self._L.oc_run(self._c, ctypes.byref(cfg), out, max_summaries, ctypes.byref(steps), trace, dt_trace_len)
        if n < 0:
            raise RuntimeError(f"oracle run stopped: small timestep at step {steps.value}")
        recs = [(r.step, r.time, r.vol, r.mass, r.ie, r.ke, r.press) for r in out[:min(n, max_summaries)]]
        return recs, steps.value, list(trace[:dt_trace_len])


def run_reference(deck_text: str, exe: str = "serial-capture", threads: Optional[int] = None,
                  timeout: float = 3600.0) -> Dict:
    """Run a reference build from oracle/_ref on a deck; returns the captured
    summaries, the final interior fields (capture build only), the stdout
    and the PASS/FAIL outcome."""
    path = os.path.join(REF_DIR, exe)
    if not os.path.exists(path):
        raise RuntimeError(f"reference build missing: {path} (run `make -C oracle ref`)")
    with tempfile.TemporaryDirectory() as tmp:
        deck = os.path.join(tmp, "clover.in")
        with open(deck, "w") as f:
            f.write(deck_text)
        env = dict(os.environ)
        env["CLOVER_CAPTURE_SUMMARY"] = os.path.join(tmp, "summary.txt")
        env["CLOVER_CAPTURE_FIELDS"] = os.path.join(tmp, "fields.bin")
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        p = subprocess.run([path, "--file", deck, "--out", os.path.join(tmp, "clover.out")], cwd=tmp, env=env,
                           capture_output=True, text=True, timeout=timeout)
        res = {"returncode": p.returncode, "stdout": p.stdout, "summaries": [], "fields": {}}
        sp = env["CLOVER_CAPTURE_SUMMARY"]
        if os.path.exists(sp):
            for line in open(sp):
                w = line.split()
                res["summaries"].append((int(w[0]),) + tuple(float(x) for x in w[1:]))
        fp = env["CLOVER_CAPTURE_FIELDS"]
        if os.path.exists(fp):
            res["fields"] = read_fields(fp)
        return res


def read_fields(path: str) -> Dict[int, np.ndarray]:
    """Read a CLVF file (oracle/ref_hooks/finalise.cpp) into {field id: (h, w) array}."""
    with open(path, "rb") as f:
        data = f.read()
    if data[:4] != b"CLVF":
        raise ValueError("not a CLVF file")
    nx, ny, nf = struct.unpack_from("<iii", data, 4)
    off = 16
    out = {}
    for _ in range(nf):
        fid, w, h = struct.unpack_from("<iii", data, off)
        off += 12
        a = np.frombuffer(data, dtype="<f8", count=w * h, offset=off).reshape(h, w).copy()
        off += 8 * w * h
        out[fid] = a
    return out


def write_fields(path: str, nx: int, ny: int, fields: Dict[int, np.ndarray]):
    with open(path, "wb") as f:
        f.write(b"CLVF")
        f.write(struct.pack("<iii", nx, ny, len(fields)))
        for fid, a in fields.items():
            h, w = a.shape
            f.write(struct.pack("<iii", fid, w, h))
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())


CAPTURED = [(0, "cell"), (2, "cell"), (4, "cell"), (5, "cell"), (6, "cell"), (7, "node"), (9, "node"),
            (11, "xface"), (12, "yface")]


def interior(arr: np.ndarray, nx: int, ny: int, kind: str) -> np.ndarray:
    """The interior block a CLVF file stores for a field of the given kind."""
    w = nx + (1 if kind in ("node", "xface") else 0)
    h = ny + (1 if kind in ("node", "yface") else 0)
    return arr[2:2 + h, 2:2 + w].copy()
