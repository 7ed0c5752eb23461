"""Batched linear leapfrog: B independent initial conditions on one grid.

Wraps the swals_gpu_batch_* entry points of include/swals_gpu.h.  The grid
(geometry, ELV, options) comes from a ``Domain`` created with
``timestepping_method='linear'``; every instance advances exactly as that
domain would with ``evolve_one_step(dt)``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Batch:
    def __init__(self, grid, nbatch, record_max_stage=True):
        self._L = _lib.lib()
        self.grid = grid            # keeps the grid alive
        self.nbatch = int(nbatch)
        self.nx = grid.nx
        self.dtype = grid.dtype
        h = ctypes.c_void_p()
        check(self._L.swals_gpu_batch_create(grid.handle, self.nbatch, int(bool(record_max_stage)), ctypes.byref(h)))
        self._h = h
        self._n_gauges = 0
        self._capacity = 0

    def close(self):
        if getattr(self, "_h", None):
            self._L.swals_gpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_U(self, U3, first=0):
        """U3: (count, 3, ny, nx) STG/UH/VH per instance."""
        U3 = np.ascontiguousarray(U3, dtype=self.dtype)
        assert U3.ndim == 4 and U3.shape[1:] == (3, self.nx[1], self.nx[0]), U3.shape
        check(self._L.swals_gpu_batch_upload_U(self._h, int(first), int(U3.shape[0]), _p(U3)))

    def get_U(self, first=0, count=None):
        count = self.nbatch - first if count is None else count
        out = np.empty((count, 3, self.nx[1], self.nx[0]), dtype=self.dtype)
        check(self._L.swals_gpu_batch_download_U(self._h, int(first), int(count), _p(out)))
        return out

    def max_stage(self, first=0, count=None):
        count = self.nbatch - first if count is None else count
        out = np.empty((count, self.nx[1], self.nx[0]), dtype=self.dtype)
        check(self._L.swals_gpu_batch_download_max_stage(self._h, int(first), int(count), _p(out)))
        return out

    def device_state(self):
        ptr = ctypes.c_void_p()
        pitch, plane, stride = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(self._L.swals_gpu_batch_device_state(self._h, ctypes.byref(ptr), ctypes.byref(pitch),
                                                   ctypes.byref(plane), ctypes.byref(stride)))
        return ptr.value, pitch.value, plane.value, stride.value

    def gauges_setup(self, xy, capacity):
        xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1, 2)
        check(self._L.swals_gpu_batch_gauges_setup(self._h, _p(xy), int(xy.shape[0]), int(capacity)))
        self._n_gauges, self._capacity = xy.shape[0], int(capacity)

    def gauges_read(self):
        """(records, nbatch, n_gauges) stage series."""
        out = np.zeros((self._capacity, self.nbatch, self._n_gauges))
        n = ctypes.c_int32()
        check(self._L.swals_gpu_batch_gauges_read(self._h, _p(out), self._capacity, ctypes.byref(n)))
        return out[: n.value]

    def evolve(self, nsteps, dt):
        check(self._L.swals_gpu_batch_evolve(self._h, int(nsteps), float(dt)))

    def time(self):
        t, n = ctypes.c_double(), ctypes.c_int64()
        check(self._L.swals_gpu_batch_time(self._h, ctypes.byref(t), ctypes.byref(n)))
        return t.value, n.value

    def tune(self):
        cfg, ms = ctypes.c_int32(), ctypes.c_double()
        check(self._L.swals_gpu_batch_tune(self._h, ctypes.byref(cfg), ctypes.byref(ms)))
        return cfg.value, ms.value

    @staticmethod
    def tile_config_count():
        n = ctypes.c_int32()
        check(_lib.lib().swals_gpu_batch_tile_config_count(ctypes.byref(n)))
        return n.value

    def set_tile_config(self, cfg):
        check(self._L.swals_gpu_batch_set_tile_config(self._h, int(cfg)))
