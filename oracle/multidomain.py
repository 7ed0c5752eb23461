"""Test infrastructure only: the CPU restatement of SWALS's multidomain step.

Drives the C oracle (swals_oracle.c, swals_nesting_oracle.c) in the order of
``evolve_multidomain_one_step_shallow_water`` (multidomain_mod.f90:1093-1212):
for each domain, zero its nesting flux integrals, take its refinement factor
of sub-steps (the steppers accumulate the integrals), pack its send comms;
then every domain unpacks its receive comms and applies the staggered-grid
fix-ups (domain_mod.f90:3712-3893); then every domain is flux-corrected
(domain_mod.f90:2766-3610).  Only tests and the benchmark's CPU-baseline leg
may import this module.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import numpy as np

from .oracle import METHODS, OracleDomain, _load, _ptr

STAGGERED_METHODS = {"linear", "leapfrog_linear_plus_nonlinear_friction", "leapfrog_nonlinear"}


class _NestCommC(ctypes.Structure):
    _fields_ = [
        ("send_active", ctypes.c_int32), ("recv_active", ctypes.c_int32),
        ("send_inds", ctypes.c_int32 * 6), ("recv_inds", ctypes.c_int32 * 6),
        ("cell_ratios", ctypes.c_double * 2),
        ("my_domain_is_finer", ctypes.c_int32), ("equal_cell_ratios", ctypes.c_int32),
        ("my_domain_staggered_grid", ctypes.c_int32), ("neighbour_domain_staggered_grid", ctypes.c_int32),
        ("use_wetdry_limiting", ctypes.c_int32), ("pad", ctypes.c_int32),
        ("nsend", ctypes.c_int64), ("nsend_interior", ctypes.c_int64), ("send_flux_start", ctypes.c_int64),
        ("send_timeind", ctypes.c_int64),
        ("nrecv", ctypes.c_int64), ("nrecv_interior", ctypes.c_int64), ("recv_flux_start", ctypes.c_int64),
        ("recv_timeind", ctypes.c_int64),
    ]


def _integral_len(box):
    bl, bw = box[1] - box[0] + 1, box[3] - box[2] + 1
    return 4 * (2 * bl + 2 * bw)


class OracleComm:
    """One side of a two_way_nesting_comms_type (nested_grid_comms_mod.f90:257-658)."""

    def __init__(self, my_dx, neighbour_dx, send_inds=None, recv_inds=None, send_only=False, recv_only=False,
                 use_wetdry_limiting=True, my_staggered=0, neighbour_staggered=0, real32=False):
        self.real32 = real32
        self.dtype = np.float32 if real32 else np.float64
        self.lib = _load(real32)
        self.pref = "oracle32_" if real32 else "oracle64_"
        self.c = _NestCommC()
        si = (ctypes.c_int32 * 6)(*(send_inds if send_inds is not None else [-1] * 6))
        ri = (ctypes.c_int32 * 6)(*(recv_inds if recv_inds is not None else [-1] * 6))
        f = getattr(self.lib, self.pref + "nest_comm_init")
        f.restype = ctypes.c_int
        rc = f(ctypes.byref(self.c), (ctypes.c_double * 2)(*my_dx), (ctypes.c_double * 2)(*neighbour_dx), si, ri,
               int(send_only), int(recv_only), int(use_wetdry_limiting), int(my_staggered),
               int(neighbour_staggered))
        if rc != 0:
            raise ValueError("initialise_two_way_nesting_comms would stop (bad ratios or boxes)")
        self.send_integral = np.zeros(_integral_len(send_inds), np.float64) if self.c.send_active else None
        self.recv_integral = np.zeros(_integral_len(recv_inds), np.float64) if self.c.recv_active else None
        self.recv_error = np.zeros(_integral_len(recv_inds), np.float64) if self.c.recv_active else None
        self.send_buffer = np.zeros(self.c.nsend, self.dtype) if self.c.send_active else None

    def pack(self, U: np.ndarray, time: Optional[float] = None, with_flux=True):
        """process_data_to_send; U has shape (4, ny, nx)."""
        f = getattr(self.lib, self.pref + "nest_pack")
        f.restype = None
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                      ctypes.c_double, ctypes.c_int32, ctypes.c_void_p]
        f(ctypes.byref(self.c), _ptr(U), U.shape[2], U.shape[1],
          _ptr(self.send_integral) if with_flux else None, 0.0 if time is None else float(time),
          0 if time is None else 1, _ptr(self.send_buffer))
        return self.send_buffer

    def unpack(self, buf: np.ndarray, U: np.ndarray, with_flux=True) -> float:
        """process_received_data; returns the received time."""
        f = getattr(self.lib, self.pref + "nest_unpack")
        f.restype = None
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        t = ctypes.c_double()
        f(ctypes.byref(self.c), _ptr(np.ascontiguousarray(buf, self.dtype)), _ptr(U), U.shape[2], U.shape[1],
          _ptr(self.recv_integral) if with_flux else None, _ptr(self.recv_error) if with_flux else None,
          ctypes.byref(t))
        return t.value


class OracleMultidomain:
    """The oracle's multidomain: ``domains`` are OracleDomain objects with the
    setup's widened geometry, ``all_dx`` the setup's cell sizes (2 per
    domain), ``exchanges`` the receive/send box pairs (ptha_b200.nesting
    Exchange objects or any object with sender, receiver, send_box,
    recv_box)."""

    def __init__(self, domains: Sequence[OracleDomain], methods: Sequence[str], all_dx, exchanges,
                 refinement: Optional[Sequence[int]] = None, priority_index=None, use_wetdry_limiting=True,
                 flux_correction=True):
        self.domains = list(domains)
        self.methods = list(methods)
        n = len(self.domains)
        self.all_dx = np.ascontiguousarray(np.asarray(all_dx, np.float64).reshape(n, 2))
        self.nt = list(refinement) if refinement is not None else [1] * n
        self.exchanges = list(exchanges)
        self.flux_correction = flux_correction
        self.send: List[OracleComm] = []
        self.recv: List[OracleComm] = []
        for e in self.exchanges:
            sdx, rdx = self.all_dx[e.sender], self.all_dx[e.receiver]
            ss = int(self.methods[e.sender] in STAGGERED_METHODS)
            rs = int(self.methods[e.receiver] in STAGGERED_METHODS)
            real32 = self.domains[e.sender].real32
            self.send.append(OracleComm(sdx, rdx, send_inds=list(e.send_box) + [1, 4], send_only=True,
                                        use_wetdry_limiting=use_wetdry_limiting, my_staggered=ss,
                                        neighbour_staggered=rs, real32=real32))
            self.recv.append(OracleComm(rdx, sdx, recv_inds=list(e.recv_box) + [1, 4], recv_only=True,
                                        use_wetdry_limiting=use_wetdry_limiting, my_staggered=rs,
                                        neighbour_staggered=ss, real32=real32))
        # Each domain's integral boxes: its send boxes, then its receive boxes.
        self._keep = []
        for k, d in enumerate(self.domains):
            boxes, offs, arrays = [], [], []
            for q, e in enumerate(self.exchanges):
                if e.sender == k:
                    boxes.append(e.send_box); arrays.append(("send", q))
            for q, e in enumerate(self.exchanges):
                if e.receiver == k:
                    boxes.append(e.recv_box); arrays.append(("recv", q))
            total = sum(_integral_len(b) for b in boxes)
            store = np.zeros(max(total, 1), np.float64)
            o = 0
            for (kind, q), b in zip(arrays, boxes):
                ln = _integral_len(b)
                view = store[o:o + ln]
                if kind == "send":
                    self.send[q].send_integral = view
                else:
                    self.recv[q].recv_integral = view
                offs.append(o)
                o += ln
            bx = np.ascontiguousarray(np.asarray(boxes, np.int32).reshape(-1))
            of = np.ascontiguousarray(np.asarray(offs, np.int64))
            d.c.nest_nbox = len(boxes)
            d.c.nest_boxes = _ptr(bx) if len(boxes) else None
            d.c.nest_offset = _ptr(of) if len(boxes) else None
            d.c.nest_integral = _ptr(store)
            self._keep.append((bx, of, store))
        if flux_correction:
            self.pind = [np.asfortranarray(np.asarray(p, np.int32)) for p in priority_index]
        self.time = self.domains[0].time

    def _zero_integrals(self, k):
        # nesting_boundary_flux_integral_multiply(c=0)
        self._keep[k][2][:] = 0.0 * self._keep[k][2]

    def send_halos(self, k):
        for q, e in enumerate(self.exchanges):
            if e.sender == k:
                self.send[q].pack(self.domains[k].U)

    def recv_halos(self):
        for k, d in enumerate(self.domains):
            for q, e in enumerate(self.exchanges):
                if e.receiver == k:
                    self.recv[q].unpack(self.send[q].send_buffer, d.U)
            f = getattr(d.lib, d.pref + "nest_recv_fixup")
            f.restype = None
            f.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            for q, e in enumerate(self.exchanges):
                if e.receiver == k:
                    f(ctypes.addressof(d.c), (ctypes.c_int32 * 4)(*e.recv_box))

    def flux_correct(self):
        for k, d in enumerate(self.domains):
            qs = [q for q, e in enumerate(self.exchanges) if e.receiver == k]
            if not qs:
                continue
            boxes = np.ascontiguousarray(np.asarray([self.exchanges[q].recv_box for q in qs], np.int32).reshape(-1))
            my = np.full(len(qs), k + 1, np.int32)
            nb = np.asarray([self.exchanges[q].sender + 1 for q in qs], np.int32)
            errs = [self.recv[q].recv_error for q in qs]
            offs = np.cumsum([0] + [len(a) for a in errs[:-1]]).astype(np.int64)
            err = np.ascontiguousarray(np.concatenate(errs))
            meth = np.asarray([METHODS[m] for m in self.methods], np.int32)
            f = getattr(d.lib, d.pref + "nest_flux_correction")
            f.restype = None
            f.argtypes = [ctypes.c_void_p, ctypes.c_int32] + [ctypes.c_void_p] * 8 + [ctypes.c_double]
            f(ctypes.addressof(d.c), len(qs), _ptr(boxes), _ptr(my), _ptr(nb), _ptr(err), _ptr(offs),
              _ptr(self.pind[k]), _ptr(self.all_dx), _ptr(meth), 1.0)

    def evolve_one_step(self, dt: float):
        tend = self.time + dt
        for k, d in enumerate(self.domains):
            self._zero_integrals(k)
            nt = self.nt[k]
            dt_local = dt / (1.0 * nt)
            for _ in range(nt):
                d.evolve_one_step(dt_local)
            self.send_halos(k)
            d.c.time = tend
        self.recv_halos()
        if self.flux_correction:
            self.flux_correct()
        self.time = tend
