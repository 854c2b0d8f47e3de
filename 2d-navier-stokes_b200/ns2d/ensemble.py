"""Batched ensembles (ns2d_ensemble_* of include/ns2d.h): independent
trajectories of possibly different grid sizes advanced together."""
import ctypes as C

import numpy as np

from . import abi
from ._lib import NS2DError, load

_dp = C.POINTER(C.c_double)


class Shape(C.Structure):
    """struct ns2d_ensemble_shape: block size and persistent grid of the column
    and of the row passes, and (out) the item counts of those shapes."""
    _fields_ = [(n, C.c_int32) for n in ("col_threads", "col_grid", "row_threads", "row_grid", "stage_launch",
                                          "stage_grid", "col_items", "row_items")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


def _sig(L):
    H = C.c_void_p
    sig = {
        "ns2d_ensemble_create": (C.c_int, [C.POINTER(abi.Params), C.c_int32, C.POINTER(C.c_int32), C.POINTER(H)]),
        "ns2d_ensemble_destroy": (C.c_int, [H]),
        "ns2d_ensemble_last_error": (C.c_char_p, [H]),
        "ns2d_ensemble_launch_count": (C.c_int64, [H]),
        "ns2d_ensemble_set_w_hat": (C.c_int, [H, C.c_int32, _dp]),
        "ns2d_ensemble_get_w_hat": (C.c_int, [H, C.c_int32, _dp]),
        "ns2d_ensemble_step_n": (C.c_int, [H, C.c_int32, C.c_double]),
        "ns2d_ensemble_step_async": (C.c_int, [H, C.c_int32, C.c_double]),
        "ns2d_ensemble_check": (C.c_int, [H]),
        "ns2d_ensemble_measurables": (C.c_int, [H, C.c_int32, C.POINTER(abi.Measures)]),
        "ns2d_ensemble_tune": (C.c_int, [H, C.c_double, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
        "ns2d_ensemble_set_grids": (C.c_int, [H, C.c_int32, C.c_int32]),
        "ns2d_ensemble_set_shape": (C.c_int, [H, C.POINTER(Shape)]),
        "ns2d_ensemble_get_shape": (C.c_int, [H, C.POINTER(Shape)]),
        "ns2d_ensemble_set_stream": (C.c_int, [H, C.c_void_p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


class Ensemble:
    def __init__(self, params, sizes):
        self.L = load()
        _sig(self.L)
        self.p = params.copy()
        self.sizes = [int(s) for s in sizes]
        arr = (C.c_int32 * len(self.sizes))(*self.sizes)
        h = C.c_void_p()
        st = self.L.ns2d_ensemble_create(C.byref(self.p), len(self.sizes), arr, C.byref(h))
        if st != abi.OK:
            raise NS2DError(st, "ns2d_ensemble_create failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.ns2d_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, st):
        if st != abi.OK:
            raise NS2DError(st, (self.L.ns2d_ensemble_last_error(self.h) or b"").decode())

    def set_w_hat(self, m, w):
        w = np.ascontiguousarray(w, np.complex128)
        n = self.sizes[m]
        assert w.shape == (n, n // 2 + 1)
        self._ck(self.L.ns2d_ensemble_set_w_hat(self.h, m, w.view(np.float64).ctypes.data_as(_dp)))

    def get_w_hat(self, m):
        n = self.sizes[m]
        w = np.zeros((n, n // 2 + 1), np.complex128)
        self._ck(self.L.ns2d_ensemble_get_w_hat(self.h, m, w.view(np.float64).ctypes.data_as(_dp)))
        return w

    def step_n(self, nsteps, dt):
        self._ck(self.L.ns2d_ensemble_step_n(self.h, nsteps, dt))

    def step_async(self, nsteps, dt):
        self._ck(self.L.ns2d_ensemble_step_async(self.h, nsteps, dt))

    def check(self):
        self._ck(self.L.ns2d_ensemble_check(self.h))

    def measurables(self, m):
        out = abi.Measures()
        self._ck(self.L.ns2d_ensemble_measurables(self.h, m, C.byref(out)))
        return out

    def tune(self, dt):
        cg, rg = C.c_int32(), C.c_int32()
        self._ck(self.L.ns2d_ensemble_tune(self.h, dt, C.byref(cg), C.byref(rg)))
        return cg.value, rg.value

    def set_grids(self, col_grid, row_grid):
        self._ck(self.L.ns2d_ensemble_set_grids(self.h, col_grid, row_grid))

    @property
    def shape(self):
        """Launch shape of the passes (ns2d_ensemble_get_shape) as a dict."""
        sh = Shape()
        self._ck(self.L.ns2d_ensemble_get_shape(self.h, C.byref(sh)))
        return sh.as_dict()

    def set_shape(self, col_threads=256, col_grid=1184, row_threads=256, row_grid=1184, stage_launch=0,
                  stage_grid=296):
        sh = Shape(col_threads=col_threads, col_grid=col_grid, row_threads=row_threads, row_grid=row_grid,
                   stage_launch=stage_launch, stage_grid=stage_grid)
        self._ck(self.L.ns2d_ensemble_set_shape(self.h, C.byref(sh)))

    def set_stream(self, ptr):
        self._ck(self.L.ns2d_ensemble_set_stream(self.h, C.c_void_p(ptr)))

    @property
    def launch_count(self):
        return self.L.ns2d_ensemble_launch_count(self.h)
