"""ctypes binding of libcloverb200.so (include/cloverb200.h).

`Chunk` mirrors the reference's per-model interface (driver/NAME.h): one
method per entry point, same names, same argument meaning.  There is no CPU
fallback: if the library or a CUDA device is missing, construction raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Iterable, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcloverb200.so")

FIELD_NAMES = ["density0", "density1", "energy0", "energy1", "pressure", "viscosity", "soundspeed",
               "xvel0", "xvel1", "yvel0", "yvel1", "vol_flux_x", "vol_flux_y", "mass_flux_x", "mass_flux_y",
               "work_array1", "work_array2", "work_array3", "work_array4", "work_array5", "work_array6",
               "work_array7", "volume", "xarea", "yarea"]
FIELD_ID = {n: i for i, n in enumerate(FIELD_NAMES)}
GEOM_NAMES = ["cellx", "celly", "celldx", "celldy", "vertexx", "vertexy", "vertexdx", "vertexdy"]
GEOM_ID = {n: i for i, n in enumerate(GEOM_NAMES)}
FP64, FP32 = 0, 1
LAYOUT_XFAST, LAYOUT_YFAST = 0, 1
OPT_FOLD_HALO, OPT_FUSE_CALLS = 1, 3
FACE_LEFT, FACE_RIGHT, FACE_BOTTOM, FACE_TOP = 1, 2, 4, 8

# Every symbol include/cloverb200.h declares.
EXPORTS = ["cb_version", "cb_last_error", "cb_device_count", "cb_device_name", "cb_create", "cb_destroy", "cb_set_gamma", "cb_set_option", "cb_get_extent",
           "cb_read_field", "cb_write_field", "cb_read_geom", "cb_write_geom", "cb_build_field", "cb_initialise_chunk", "cb_initialise_chunk_in",
           "cb_generate_chunk", "cb_ideal_gas", "cb_viscosity", "cb_calc_dt", "cb_set_dt_ahead", "cb_dt_ahead_stats", "cb_pdv", "cb_revert", "cb_accelerate",
           "cb_flux_calc", "cb_lagrangian", "cb_advec_cell", "cb_advec_mom", "cb_reset_field", "cb_update_halo", "cb_field_summary",
           "cb_synchronize", "cb_get_stream", "cb_launch_count", "cb_run", "cb_field_summary_noalloc",
           "cb_set_external_faces", "cb_copy_tile_halo", "cb_face_strip_size", "cb_pack_face", "cb_unpack_face",
           "cb_batch_create", "cb_batch_destroy", "cb_batch_set_schedule", "cb_batch_get_schedule", "cb_batch_autotune",
           "cb_batch_run", "cb_batch_synchronize", "cb_batch_deck_result", "cb_batch_read_summaries", "cb_batch_read_dt",
           "cb_batch_read_field", "cb_batch_get_stream", "cb_batch_launch_count",
           "cb_adjoint_create", "cb_adjoint_destroy", "cb_adjoint_set_initial", "cb_adjoint_set_checkpoint_interval",
           "cb_adjoint_forward", "cb_adjoint_dt", "cb_adjoint_gradient", "cb_adjoint_tangent", "cb_adjoint_read_tangent",
           "cb_adjoint_read_field", "cb_adjoint_stats", "cb_selftest_width_ratio", "cb_selftest_wait_limits"]


class CloverError(RuntimeError):
    pass


class State(ctypes.Structure):
    _fields_ = [("density", ctypes.c_double), ("energy", ctypes.c_double), ("xvel", ctypes.c_double),
                ("yvel", ctypes.c_double), ("geometry", ctypes.c_int), ("xmin", ctypes.c_double),
                ("ymin", ctypes.c_double), ("xmax", ctypes.c_double), ("ymax", ctypes.c_double),
                ("radius", ctypes.c_double)]


class DtParams(ctypes.Structure):
    _fields_ = [("dtmin", ctypes.c_double), ("dtc_safe", ctypes.c_double), ("dtu_safe", ctypes.c_double),
                ("dtv_safe", ctypes.c_double), ("dtdiv_safe", ctypes.c_double)]


class RunParams(ctypes.Structure):
    _fields_ = [("dtmin", ctypes.c_double), ("dtmax", ctypes.c_double), ("dtrise", ctypes.c_double),
                ("dtc_safe", ctypes.c_double), ("dtu_safe", ctypes.c_double), ("dtv_safe", ctypes.c_double),
                ("dtdiv_safe", ctypes.c_double), ("end_time", ctypes.c_double), ("end_step", ctypes.c_int),
                ("summary_frequency", ctypes.c_int), ("fold", ctypes.c_int), ("fuse", ctypes.c_int)]


class RunState(ctypes.Structure):
    _fields_ = [("step", ctypes.c_int), ("advect_x", ctypes.c_int), ("time", ctypes.c_double),
                ("dtold", ctypes.c_double), ("dt", ctypes.c_double), ("done", ctypes.c_int)]


_lib = None


def library() -> ctypes.CDLL:
    """Load libcloverb200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CloverError(f"libcloverb200.so not built at {LIB_PATH}; run `make -C cloverleaf_b200` "
                          "(or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    i, d, sz = ctypes.c_int, ctypes.c_double, ctypes.c_size_t
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    sig = {
        "cb_version": ([], i), "cb_last_error": ([], ctypes.c_char_p),
        "cb_device_count": ([ip], i), "cb_device_name": ([i, ctypes.c_char_p, sz], i),
        "cb_create": ([i, i, i, i, ctypes.POINTER(P)], i), "cb_destroy": ([P], i),
        "cb_set_gamma": ([P, d], i), "cb_set_option": ([P, i, i], i), "cb_get_extent": ([P, i, ip, ip], i),
        "cb_read_field": ([P, i, dp, sz, i], i), "cb_write_field": ([P, i, dp, sz, i], i),
        "cb_read_geom": ([P, i, dp, sz], i), "cb_write_geom": ([P, i, dp, sz], i),
        "cb_build_field": ([P], i), "cb_initialise_chunk": ([P, d, d, d, d], i),
        "cb_initialise_chunk_in": ([P, d, d, d, d, i, i, i, i], i),
        "cb_generate_chunk": ([P, i, ctypes.POINTER(State)], i),
        "cb_ideal_gas": ([P, i, i], i), "cb_viscosity": ([P, i], i),
        "cb_calc_dt": ([P, ctypes.POINTER(DtParams), dp, ip, ip, ip, ip], i),
        "cb_set_dt_ahead": ([P, d, d, d], i),
        "cb_dt_ahead_stats": ([P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)], i),
        "cb_pdv": ([P, i, d, i, i], i), "cb_revert": ([P], i), "cb_accelerate": ([P, d, i], i),
        "cb_flux_calc": ([P, d, i], i), "cb_lagrangian": ([P, d, i], i), "cb_advec_cell": ([P, i, i, i], i), "cb_advec_mom": ([P, i, i, i, i], i),
        "cb_reset_field": ([P, i], i), "cb_update_halo": ([P, ip, i], i), "cb_field_summary": ([P, dp], i),
        "cb_synchronize": ([P], i), "cb_get_stream": ([P, ctypes.POINTER(P)], i),
        "cb_launch_count": ([P, ctypes.POINTER(ctypes.c_longlong)], i),
        "cb_run": ([P, ctypes.POINTER(RunParams), ctypes.POINTER(RunState), i, dp, dp, i, ip], i),
        "cb_field_summary_noalloc": ([i, i, ctypes.c_longlong] + [P] * 8 + [d, P, P], i),
        "cb_selftest_width_ratio": ([ctypes.c_longlong, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_longlong)], i),
        "cb_selftest_wait_limits": ([d, ip, ip, dp, ip, ip, dp], i),
        "cb_set_external_faces": ([P, i], i), "cb_copy_tile_halo": ([P, P, i, ip, i], i),
        "cb_face_strip_size": ([P, i, ip, i, ctypes.POINTER(sz)], i),
        "cb_pack_face": ([P, i, ip, i, P, sz], i), "cb_unpack_face": ([P, i, ip, i, P, sz], i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def _field_flags(fields: Iterable):
    flags = [0] * 15
    for f in fields:
        flags[FIELD_ID[f] if isinstance(f, str) else int(f)] = 1
    return (ctypes.c_int * 15)(*flags)


def _check(rc: int):
    if rc != 0:
        msg = library().cb_last_error().decode(errors="replace")
        raise CloverError(f"libcloverb200 error {rc}: {msg}")


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Chunk:
    """One mesh chunk resident on a B200 (cb_chunk)."""

    def __init__(self, nx: int, ny: int, precision: int = FP64, device: int = 0, gamma: float = 1.4):
        self._L = library()
        self._h = ctypes.c_void_p()
        _check(self._L.cb_create(nx, ny, precision, device, ctypes.byref(self._h)))
        self.nx, self.ny, self.precision = nx, ny, precision
        if gamma != 1.4:
            _check(self._L.cb_set_gamma(self._h, gamma))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            self._L.cb_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- configuration / data movement
    def set_gamma(self, g: float): _check(self._L.cb_set_gamma(self._h, g))
    def set_option(self, opt: int, value: int): _check(self._L.cb_set_option(self._h, opt, int(value)))

    def extent(self, field) -> Tuple[int, int]:
        fid = FIELD_ID[field] if isinstance(field, str) else int(field)
        sx, sy = ctypes.c_int(), ctypes.c_int()
        _check(self._L.cb_get_extent(self._h, fid, ctypes.byref(sx), ctypes.byref(sy)))
        return sx.value, sy.value

    def read(self, field) -> np.ndarray:
        """Whole field as an (sy, sx) array indexed [j, i]."""
        fid = FIELD_ID[field] if isinstance(field, str) else int(field)
        sx, sy = self.extent(fid)
        out = np.empty((sy, sx), dtype=np.float64)
        _check(self._L.cb_read_field(self._h, fid, _dptr(out), out.size, LAYOUT_XFAST))
        return out

    def read_into(self, field, out: np.ndarray) -> np.ndarray:
        """Whole field into `out` ((sy, sx) float64, C-contiguous), e.g. a pinned
        host buffer, with no intermediate copy."""
        fid = FIELD_ID[field] if isinstance(field, str) else int(field)
        sx, sy = self.extent(fid)
        if out.shape != (sy, sx) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise CloverError(f"read_into {field}: expected a C-contiguous float64 array of shape {(sy, sx)}")
        _check(self._L.cb_read_field(self._h, fid, _dptr(out), out.size, LAYOUT_XFAST))
        return out

    def write(self, field, arr: np.ndarray):
        fid = FIELD_ID[field] if isinstance(field, str) else int(field)
        sx, sy = self.extent(fid)
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != (sy, sx):
            raise CloverError(f"write {field}: expected shape {(sy, sx)}, got {a.shape}")
        _check(self._L.cb_write_field(self._h, fid, _dptr(a), a.size, LAYOUT_XFAST))

    def read_geom(self, g) -> np.ndarray:
        gid = GEOM_ID[g] if isinstance(g, str) else int(g)
        n = (self.nx if gid in (0, 2) else self.ny) + 4 if gid < 4 else (self.nx if gid in (4, 6) else self.ny) + 5
        out = np.empty(n, dtype=np.float64)
        _check(self._L.cb_read_geom(self._h, gid, _dptr(out), n))
        return out

    def write_geom(self, g, arr):
        gid = GEOM_ID[g] if isinstance(g, str) else int(g)
        a = np.ascontiguousarray(arr, dtype=np.float64)
        _check(self._L.cb_write_geom(self._h, gid, _dptr(a), a.size))

    # ---- setup (driver/build_field.h, initialise_chunk.h, generate_chunk.h)
    def build_field(self): _check(self._L.cb_build_field(self._h))
    def initialise_chunk(self, xmin, ymin, xmax, ymax): _check(self._L.cb_initialise_chunk(self._h, xmin, ymin, xmax, ymax))

    def initialise_chunk_in(self, xmin, ymin, xmax, ymax, x_cells: int, y_cells: int, left: int, bottom: int):
        """The geometry of this chunk as cell (left, bottom) onward of an x_cells x y_cells grid."""
        _check(self._L.cb_initialise_chunk_in(self._h, xmin, ymin, xmax, ymax, x_cells, y_cells, left, bottom))

    def generate_chunk(self, states: Sequence):
        arr = (State * len(states))()
        for k, s in enumerate(states):
            arr[k] = State(s.density, s.energy, s.xvel, s.yvel, s.geometry, s.xmin, s.ymin, s.xmax, s.ymax, s.radius)
        _check(self._L.cb_generate_chunk(self._h, len(states), arr))

    # ---- hydro phases (driver/NAME.h)
    def ideal_gas(self, predict: bool, halo_depth: int = 0): _check(self._L.cb_ideal_gas(self._h, int(predict), halo_depth))
    def viscosity(self, halo_depth: int = 0): _check(self._L.cb_viscosity(self._h, halo_depth))

    def calc_dt(self, dtmin=0.0000001, dtc_safe=0.7, dtu_safe=0.5, dtv_safe=0.5, dtdiv_safe=0.7):
        p = DtParams(dtmin, dtc_safe, dtu_safe, dtv_safe, dtdiv_safe)
        dt = ctypes.c_double()
        ctl, jl, kl, sm = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(self._L.cb_calc_dt(self._h, ctypes.byref(p), ctypes.byref(dt), ctypes.byref(ctl), ctypes.byref(jl),
                                  ctypes.byref(kl), ctypes.byref(sm)))
        return dt.value, ctl.value, jl.value, kl.value, sm.value

    def set_dt_ahead(self, dtold: float, dtrise: float, dtmax: float):
        """Arms the next calc_dt to run the Lagrangian pass ahead with the
        driver's clamp of its minimum (with call fusion; cb_set_dt_ahead)."""
        _check(self._L.cb_set_dt_ahead(self._h, dtold, dtrise, dtmax))

    def dt_ahead_stats(self):
        """(passes run ahead, passes the four Lagrangian calls consumed)."""
        a, u = ctypes.c_longlong(), ctypes.c_longlong()
        _check(self._L.cb_dt_ahead_stats(self._h, ctypes.byref(a), ctypes.byref(u)))
        return a.value, u.value

    def pdv(self, predict: bool, dt: float, full: bool = False, halo_depth: int = 0):
        _check(self._L.cb_pdv(self._h, int(predict), dt, int(full), halo_depth))

    def revert(self): _check(self._L.cb_revert(self._h))
    def accelerate(self, dt: float, halo_depth: int = 0): _check(self._L.cb_accelerate(self._h, dt, halo_depth))
    def flux_calc(self, dt: float, halo_depth: int = 0): _check(self._L.cb_flux_calc(self._h, dt, halo_depth))

    def lagrangian(self, dt: float, halo_depth: int = 0):
        """pdv(True, dt, full=True, halo_depth=1), accelerate, pdv(False) and flux_calc (all at halo_depth) in one pass."""
        _check(self._L.cb_lagrangian(self._h, dt, halo_depth))

    def advec_cell(self, sweep_number: int, direction: int, halo_depth: int = 0):
        _check(self._L.cb_advec_cell(self._h, sweep_number, direction, halo_depth))

    def advec_mom(self, which_vel: int, sweep_number: int, direction: int, halo_depth: int = 0):
        _check(self._L.cb_advec_mom(self._h, which_vel, sweep_number, direction, halo_depth))

    def reset_field(self, halo_depth: int = 0): _check(self._L.cb_reset_field(self._h, halo_depth))

    def update_halo(self, fields: Iterable, depth: int):
        _check(self._L.cb_update_halo(self._h, _field_flags(fields), depth))

    # ---- tiles (driver/update_tile_halo.cpp)
    def set_external_faces(self, faces: int):
        """Faces on the physical boundary (FACE_* bits); the others border tiles."""
        _check(self._L.cb_set_external_faces(self._h, int(faces)))

    def copy_tile_halo(self, src: "Chunk", side: int, fields: Iterable, depth: int):
        """This chunk's halo on `side` (one FACE_* value) from `src`, the tile on that side."""
        _check(self._L.cb_copy_tile_halo(self._h, src._h, int(side), _field_flags(fields), depth))

    # ---- decomposed runs (driver/comms.cpp:clover_exchange, src/serial/pack_kernel.cpp)
    def face_strip_size(self, side: int, fields: Iterable, depth: int) -> int:
        """Elements (of the chunk's precision) of the face strip on `side` (one FACE_* value)."""
        n = ctypes.c_size_t(0)
        _check(self._L.cb_face_strip_size(self._h, int(side), _field_flags(fields), depth, ctypes.byref(n)))
        return int(n.value)

    def pack_face(self, side: int, fields: Iterable, depth: int, dev_ptr: int, capacity: int):
        """The strip the neighbour on `side` needs, into the device buffer at dev_ptr (on the chunk's stream)."""
        _check(self._L.cb_pack_face(self._h, int(side), _field_flags(fields), depth, ctypes.c_void_p(dev_ptr), capacity))

    def unpack_face(self, side: int, fields: Iterable, depth: int, dev_ptr: int, capacity: int):
        """This chunk's halo on `side` from the strip its neighbour there packed (on the chunk's stream)."""
        _check(self._L.cb_unpack_face(self._h, int(side), _field_flags(fields), depth, ctypes.c_void_p(dev_ptr), capacity))

    def field_summary(self) -> Tuple[float, float, float, float, float]:
        out = (ctypes.c_double * 5)()
        _check(self._L.cb_field_summary(self._h, out))
        return tuple(out)

    def run(self, params: RunParams, state: RunState, max_steps: int, max_summaries: int = 0):
        """cb_run: hydro steps on the device until the run completes or
        max_steps steps were made; `state` is updated in place.  Returns
        (dt of each step, summary records (n, 7), total summaries)."""
        trace = np.zeros(max_steps, dtype=np.float64)
        recs = np.zeros((max(max_summaries, 1), 7), dtype=np.float64)
        n = ctypes.c_int()
        step0 = state.step
        rc = self._L.cb_run(self._h, ctypes.byref(params), ctypes.byref(state), max_steps, _dptr(trace), _dptr(recs),
                            max_summaries, ctypes.byref(n))
        _check(rc)
        return trace[:state.step - step0], recs[:min(n.value, max_summaries)], n.value

    def synchronize(self): _check(self._L.cb_synchronize(self._h))

    def stream(self) -> int:
        """The chunk's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        s = ctypes.c_void_p()
        _check(self._L.cb_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def launch_count(self) -> int:
        n = ctypes.c_longlong()
        _check(self._L.cb_launch_count(self._h, ctypes.byref(n)))
        return n.value
