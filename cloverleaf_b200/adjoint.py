"""Gradient of the final kinetic energy with respect to the initial state
(the cb_adjoint_* part of include/cloverb200.h), and a torch.autograd
harness around it.

The map differentiated is the FP64 plain path run for a number of steps
with the dt sequence of a forward run held fixed: initial interior density
and energy (nx * ny each) and gamma -> final kinetic energy (field_summary's
ke).  `Adjoint.gradient` is the reverse sweep of hand-written adjoint kernels
over sqrt(N)-step checkpoints; `Adjoint.tangent` is the tangent-linear run
that checks it; `KineticEnergy` wraps both in a torch.autograd.Function.

Arrays are (ny, nx) numpy arrays indexed [j, i] over the interior.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence, Tuple

import numpy as np

from .batch import CDeck, to_cdeck
from .chunk import FIELD_ID, CloverError, _check, _dptr, library
from .deck import Deck

EXPORTS = ["cb_adjoint_create", "cb_adjoint_destroy", "cb_adjoint_set_initial", "cb_adjoint_set_checkpoint_interval",
           "cb_adjoint_forward", "cb_adjoint_dt", "cb_adjoint_gradient", "cb_adjoint_tangent", "cb_adjoint_read_tangent",
           "cb_adjoint_read_field", "cb_adjoint_stats"]

_bound = False


def _lib():
    global _bound
    L = library()
    if not _bound:
        P, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        ip, dp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        sig = {
            "cb_adjoint_create": ([ctypes.POINTER(CDeck), i, ctypes.POINTER(P)], i),
            "cb_adjoint_destroy": ([P], i),
            "cb_adjoint_set_initial": ([P, dp, dp, d], i),
            "cb_adjoint_set_checkpoint_interval": ([P, i], i),
            "cb_adjoint_forward": ([P, i, dp, dp], i),
            "cb_adjoint_dt": ([P, dp, i, ip], i),
            "cb_adjoint_gradient": ([P, dp, dp, dp], i),
            "cb_adjoint_tangent": ([P, dp, dp, d, dp, dp], i),
            "cb_adjoint_read_tangent": ([P, i, i, dp, ctypes.c_size_t], i),
            "cb_adjoint_read_field": ([P, i, dp, ctypes.c_size_t], i),
            "cb_adjoint_stats": ([P, ip, ip, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_size_t)], i),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _bound = True
    return L


def _interior(a, nx, ny, what) -> np.ndarray:
    x = np.ascontiguousarray(a, dtype=np.float64)
    if x.shape != (ny, nx):
        raise CloverError(f"{what}: expected shape {(ny, nx)}, got {x.shape}")
    return x


class Adjoint:
    """One FP64 problem on a B200 with its forward, adjoint and tangent runs (cb_adjoint)."""

    def __init__(self, deck: Deck, device: int = 0):
        self._L = _lib()
        self._h = ctypes.c_void_p()
        self.deck = deck
        self.nx, self.ny = deck.x_cells, deck.y_cells
        c = to_cdeck(deck)
        _check(self._L.cb_adjoint_create(ctypes.byref(c), device, ctypes.byref(self._h)))
        self.steps = 0

    def close(self):
        if self._h:
            self._L.cb_adjoint_destroy(self._h)
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

    def set_initial(self, density0, energy0, gamma: float):
        r = _interior(density0, self.nx, self.ny, "density0")
        e = _interior(energy0, self.nx, self.ny, "energy0")
        _check(self._L.cb_adjoint_set_initial(self._h, _dptr(r), _dptr(e), float(gamma)))

    def set_checkpoint_interval(self, k: int):
        _check(self._L.cb_adjoint_set_checkpoint_interval(self._h, int(k)))

    def forward(self, steps: int, dt: Optional[Sequence[float]] = None) -> float:
        ke = ctypes.c_double()
        if dt is None:
            _check(self._L.cb_adjoint_forward(self._h, steps, None, ctypes.byref(ke)))
        else:
            arr = np.ascontiguousarray(dt, dtype=np.float64)
            if arr.size < steps:
                raise CloverError("forward: fewer dt values than steps")
            _check(self._L.cb_adjoint_forward(self._h, steps, _dptr(arr), ctypes.byref(ke)))
        self.steps = steps
        return ke.value

    def dt(self) -> np.ndarray:
        out = np.zeros(max(self.steps, 1))
        n = ctypes.c_int()
        _check(self._L.cb_adjoint_dt(self._h, _dptr(out), self.steps, ctypes.byref(n)))
        return out[:n.value]

    def gradient(self) -> Tuple[np.ndarray, np.ndarray, float]:
        gr = np.zeros((self.ny, self.nx))
        ge = np.zeros((self.ny, self.nx))
        gg = ctypes.c_double()
        _check(self._L.cb_adjoint_gradient(self._h, _dptr(gr), _dptr(ge), ctypes.byref(gg)))
        return gr, ge, gg.value

    def tangent(self, d_density0, d_energy0, d_gamma: float = 0.0) -> Tuple[float, float]:
        r = _interior(d_density0, self.nx, self.ny, "d_density0")
        e = _interior(d_energy0, self.nx, self.ny, "d_energy0")
        ke, dke = ctypes.c_double(), ctypes.c_double()
        _check(self._L.cb_adjoint_tangent(self._h, _dptr(r), _dptr(e), float(d_gamma), ctypes.byref(ke), ctypes.byref(dke)))
        return ke.value, dke.value

    def _extent(self, fid):
        sx = self.nx + (5 if fid in (7, 8, 9, 10, 11, 13) else 4)
        sy = self.ny + (5 if fid in (7, 8, 9, 10, 12, 14) else 4)
        return sx, sy

    def read_tangent(self, field, which: int) -> np.ndarray:
        """Final field of the last tangent run: which 0 values, 1 tangents ((sy, sx), [j, i])."""
        fid = FIELD_ID[field] if isinstance(field, str) else int(field)
        sx, sy = self._extent(fid)
        out = np.empty((sy, sx))
        _check(self._L.cb_adjoint_read_tangent(self._h, fid, which, _dptr(out), out.size))
        return out

    def read_field(self, field) -> np.ndarray:
        """A field of the primal chunk as it stands ((sy, sx), [j, i])."""
        fid = FIELD_ID[field] if isinstance(field, str) else int(field)
        sx, sy = self._extent(fid)
        out = np.empty((sy, sx))
        _check(self._L.cb_adjoint_read_field(self._h, fid, _dptr(out), out.size))
        return out

    def stats(self) -> dict:
        k, n, rec, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong(), ctypes.c_size_t()
        _check(self._L.cb_adjoint_stats(self._h, ctypes.byref(k), ctypes.byref(n), ctypes.byref(rec), ctypes.byref(b)))
        return {"checkpoint_interval": k.value, "checkpoints": n.value, "recomputed_steps": rec.value, "device_bytes": b.value}


def kinetic_energy_function():
    """The torch.autograd.Function over an `Adjoint`: forward runs the plain
    path (recording dt on the first call unless a dt sequence is given),
    backward runs the reverse sweep of that same run."""
    import torch

    class KineticEnergy(torch.autograd.Function):
        @staticmethod
        def forward(ctx, density0, energy0, gamma, adj: Adjoint, steps: int, dt=None):
            adj.set_initial(density0.detach().cpu().numpy(), energy0.detach().cpu().numpy(), float(gamma))
            ke = adj.forward(steps, dt)
            ctx.adj = adj
            ctx.dev = density0.device
            return torch.tensor(ke, dtype=torch.float64, device=density0.device)

        @staticmethod
        def backward(ctx, grad):
            gr, ge, gg = ctx.adj.gradient()
            g = grad.to(torch.float64)
            return (g * torch.from_numpy(gr).to(ctx.dev), g * torch.from_numpy(ge).to(ctx.dev),
                    g * torch.tensor(gg, dtype=torch.float64, device=ctx.dev), None, None, None)

    return KineticEnergy
