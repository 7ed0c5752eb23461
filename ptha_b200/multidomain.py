"""``multidomain_type`` on one GPU: nested domains that exchange halos.

Mirrors the parts of SWALS's ``multidomain_type`` (multidomain_mod.f90:171-276)
that the time step needs: ``setup`` (the nesting metadata,
:2663-3553, built by :mod:`ptha_b200.nesting`), ``evolve_one_step``
(:1093-1212), ``send_halos`` / ``recv_halos`` (:2449-2565) and the flux
correction (domain_mod.f90:2766-3610).  Every domain is a
:class:`ptha_b200.Domain`; the exchange runs in the CUDA library
(``swals_gpu_md_*`` in include/swals_gpu.h).
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check
from .domain import Domain
from .nesting import (EXTRA_CELLS_IN_HALO_DEFAULT, EXTRA_HALO_BUFFER_DEFAULT, HUGE, Exchange, NestDomain,
                      setup_multidomain_native)


class Multidomain:
    """Nested domains on one GPU.

    ``specs`` are :class:`NestDomain` geometries (interior extents, method,
    ``timestepping_refinement_factor``); ``domain_kwargs`` (one dict per
    domain, optional) are passed to :class:`Domain` (precision, spherical,
    boundary conditions ...).  Setup widens nesting boundaries exactly like
    the reference, so ``domains[k].nx`` may exceed ``specs[k].nx``.
    """

    def __init__(self, specs: Sequence[NestDomain], domain_kwargs: Optional[Sequence[dict]] = None,
                 extra_halo_buffer: int = EXTRA_HALO_BUFFER_DEFAULT,
                 extra_cells_in_halo: int = EXTRA_CELLS_IN_HALO_DEFAULT, use_wetdry_limiting: bool = True,
                 flux_correction: bool = True, periodic_xs=(-HUGE, HUGE), periodic_ys=(-HUGE, HUGE), device=-1):
        self.specs = list(specs)
        # the library's native metadata builder (the numpy restatement in
        # nesting.setup_multidomain gives the same tables)
        self.exchanges: List[Exchange] = setup_multidomain_native(self.specs, extra_halo_buffer, extra_cells_in_halo,
                                                                  periodic_xs, periodic_ys)
        kw = list(domain_kwargs) if domain_kwargs is not None else [{} for _ in self.specs]
        self.domains: List[Domain] = []
        for s, k in zip(self.specs, kw):
            k = dict(k)
            k.setdefault("boundary_exterior", tuple(not b for b in s.is_nesting_boundary))
            k.setdefault("device", device)
            self.domains.append(Domain(s.nx, s.lw, s.lower_left, s.timestepping_method, **k))
        self._md = None
        self._create(use_wetdry_limiting, flux_correction)

    @classmethod
    def from_tables(cls, domains: Sequence[Domain], all_dx, exchanges: Sequence[Exchange], refinement=None,
                    priority_index=None, use_wetdry_limiting=True, flux_correction=False):
        """A multidomain over existing domains and explicit exchange boxes
        (the form initialise_two_way_nesting_comms is driven with in the
        reference's nested-comms unit test)."""
        self = cls.__new__(cls)
        self.specs = None
        self.domains = list(domains)
        self.exchanges = list(exchanges)
        self._md = None
        self._create(use_wetdry_limiting, flux_correction, all_dx=all_dx, refinement=refinement,
                     priority_index=priority_index)
        return self

    def _create(self, use_wetdry_limiting, flux_correction, all_dx=None, refinement=None, priority_index=None):
        L = _lib.lib()
        self._L = L
        n = len(self.domains)
        handles = (ctypes.c_void_p * n)(*[d.handle for d in self.domains])
        if all_dx is None:
            all_dx = [v for s in self.specs for v in s.dx]
        self._dx = np.ascontiguousarray(np.asarray(all_dx, dtype=np.float64).reshape(-1))
        if refinement is None:
            refinement = [s.timestepping_refinement_factor for s in self.specs] if self.specs else [1] * n
        self._nt = np.ascontiguousarray(np.asarray(refinement, dtype=np.int32))
        ex = (_lib.NestExchange * max(1, len(self.exchanges)))()
        for q, e in enumerate(self.exchanges):
            ex[q].sender, ex[q].receiver = e.sender, e.receiver
            for t in range(4):
                ex[q].send_box[t] = e.send_box[t]
                ex[q].recv_box[t] = e.recv_box[t]
        self._ex = ex
        pptr = None
        self._pind = []
        if flux_correction:
            if priority_index is None:
                priority_index = [s.priority_domain_index for s in self.specs]
            arrs = []
            for d, p in zip(self.domains, priority_index):
                a = np.asarray(p, dtype=np.int32)
                if a.shape != (d.nx[0], d.nx[1]):
                    raise ValueError(f"priority index shape {a.shape} != {(d.nx[0], d.nx[1])}")
                arrs.append(np.asfortranarray(a))   # (nx, ny) column-major
            self._pind = arrs
            pptr = (ctypes.c_void_p * n)(*[a.ctypes.data for a in arrs])
        h = ctypes.c_void_p()
        check(L.swals_gpu_md_create(handles, n, self._dx.ctypes.data, self._nt.ctypes.data, ex, len(self.exchanges),
                                    pptr, int(bool(use_wetdry_limiting)), int(bool(flux_correction)),
                                    ctypes.byref(h)))
        self._md = h.value

    def close(self):
        if self._md is not None:
            self._L.swals_gpu_md_destroy(self._md)
            self._md = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def evolve_one_step(self, dt: float):
        check(self._L.swals_gpu_md_evolve_one_step(self._md, float(dt)))

    def send_halos(self):
        check(self._L.swals_gpu_md_send_halos(self._md))

    def recv_halos(self):
        check(self._L.swals_gpu_md_recv_halos(self._md))

    def flux_correction(self):
        check(self._L.swals_gpu_md_flux_correction(self._md))

    def synchronize(self):
        check(self._L.swals_gpu_md_synchronize(self._md))

    def capture_graph(self, nsteps: int, dt: float):
        """Capture nsteps fixed-dt md steps (a multiple of 3) as one CUDA graph."""
        check(self._L.swals_gpu_md_capture_graph(self._md, int(nsteps), float(dt)))

    def replay(self, nreplays: int = 1):
        check(self._L.swals_gpu_md_replay(self._md, int(nreplays)))

    def buffer(self, exchange: int) -> np.ndarray:
        n = ctypes.c_int64()
        check(self._L.swals_gpu_md_buffer_size(self._md, exchange, ctypes.byref(n)))
        out = np.empty(n.value, dtype=np.float64)
        check(self._L.swals_gpu_md_download_buffer(self._md, exchange, out.ctypes.data, n.value))
        return out

    def flux(self, exchange: int, which: str) -> np.ndarray:
        """Flux integrals of an exchange: 'send', 'recv' or 'error' (the
        receiver's recv_box_flux_error)."""
        e = self.exchanges[exchange]
        box = e.send_box if which == "send" else e.recv_box
        bl, bw = box[1] - box[0] + 1, box[3] - box[2] + 1
        n = 4 * (2 * bl + 2 * bw)
        out = np.empty(n, dtype=np.float64)
        check(self._L.swals_gpu_md_download_flux(self._md, exchange, {"send": 0, "recv": 1, "error": 2}[which],
                                                 out.ctypes.data, n))
        return out

    @property
    def time(self) -> float:
        t = ctypes.c_double()
        check(self._L.swals_gpu_md_time(self._md, ctypes.byref(t)))
        return t.value

    def launch_count(self) -> int:
        n = ctypes.c_int64()
        check(self._L.swals_gpu_md_launch_count(self._md, ctypes.byref(n)))
        return n.value


class MultidomainGroup:
    """Many multidomains advanced together (``swals_gpu_md_group_*``): e.g.
    B sources on the same nest.  ``nsteps`` md steps of fixed ``dt`` of every
    member are captured into one CUDA graph (one branch per member); each
    ``replay()`` advances every member by nsteps md steps in one launch, the
    members' kernels running concurrently.  Close the group before its
    members."""

    def __init__(self, members: Sequence[Multidomain], nsteps: int, dt: float):
        self._L = _lib.lib()
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m._md for m in self.members])
        h = ctypes.c_void_p()
        check(self._L.swals_gpu_md_group_create(arr, len(self.members), int(nsteps), float(dt), ctypes.byref(h)))
        self._h = h
        self.nsteps = int(nsteps)
        self.dt = float(dt)

    def replay(self, nreplays: int = 1):
        check(self._L.swals_gpu_md_group_replay(self._h, int(nreplays)))

    def stream(self) -> int:
        s = ctypes.c_void_p()
        check(self._L.swals_gpu_md_group_stream(self._h, ctypes.byref(s)))
        return s.value

    def close(self):
        if getattr(self, "_h", None):
            self._L.swals_gpu_md_group_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
