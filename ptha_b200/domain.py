"""Host-side mirror of SWALS's ``domain_type`` for the GPU path.

Names and argument meanings follow propagation/SWALS/src/shallow_water/
domain_mod.f90 (type at :137-592): ``nx``, ``lw``, ``lower_left``,
``timestepping_method``, ``cfl``, ``theta``, ``msl_linear``,
``linear_solver_is_truely_linear``, ``friction_type``,
``linear_friction_coeff``, ``boundary_exterior`` and the type-bound
procedures ``evolve_one_step``, ``linear_timestep_max``,
``nonlinear_stationary_timestep_max``, ``stationary_timestep_max`` and
``volume_interior``.  Everything runs in libswalsgpu.so through the C ABI of
include/swals_gpu.h; errors raise :class:`SwalsError`, standing in for the
reference's ``generic_stop``.

Arrays use numpy shape ``(4, ny, nx)`` for ``U`` (plane k-1, row j-1,
column i-1 == the reference's column-major ``U(i, j, k)``).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import SwalsError, check

STG, UH, VH, ELV = 1, 2, 3, 4
NEG_HUGE = -np.finfo(np.float64).max


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Domain:
    def __init__(self, nx, lw, lower_left=(0.0, 0.0), timestepping_method="rk2", *, real_bytes=8,
                 spherical=False, coriolis=None, nofriction=False, cfl=None, theta=None, msl_linear=0.0,
                 linear_solver_is_truely_linear=True, friction_type="manning", linear_friction_coeff=0.0,
                 maximum_timestep=1.0e20, boundary_exterior=(True, True, True, True),
                 boundary_kind=_lib.BC_NONE, boundary_function_kind=_lib.BF_NONE, boundary_function_params=(),
                 record_max_stage=True, xL=0, xU=0, yL=0, yU=0, exterior_cells_width=2, boundary_subroutine=None,
                 forcing_subroutine=None, device=-1, compute_fluxes_inner_method="DE1_low_fr_diffusion"):
        L = _lib.lib()
        self._L = L
        d = _lib.DomainDesc()
        check(L.swals_gpu_desc_init(ctypes.byref(d)))
        d.nx[0], d.nx[1] = int(nx[0]), int(nx[1])
        d.lw[0], d.lw[1] = float(lw[0]), float(lw[1])
        d.lower_left[0], d.lower_left[1] = float(lower_left[0]), float(lower_left[1])
        d.timestepping_method = timestepping_method.encode()
        d.cfl = NEG_HUGE if cfl is None else float(cfl)
        d.theta = NEG_HUGE if theta is None else float(theta)
        d.msl_linear = float(msl_linear)
        d.linear_friction_coeff = float(linear_friction_coeff)
        d.maximum_timestep = float(maximum_timestep)
        d.linear_solver_is_truely_linear = int(bool(linear_solver_is_truely_linear))
        d.friction_type = {"manning": _lib.FRICTION_MANNING, "chezy": _lib.FRICTION_CHEZY}[friction_type]
        d.spherical = int(bool(spherical))
        d.coriolis = int(bool(spherical) if coriolis is None else bool(coriolis))
        d.nofriction = int(bool(nofriction))
        d.real_bytes = int(real_bytes)
        d.xL, d.xU, d.yL, d.yU = int(xL), int(xU), int(yL), int(yU)
        for k in range(4):
            d.boundary_exterior[k] = int(bool(boundary_exterior[k]))
        d.boundary_kind = int(boundary_kind)
        d.exterior_cells_width = int(exterior_cells_width)
        d.compute_fluxes_inner_method = compute_fluxes_inner_method.encode()
        d.boundary_function_kind = int(boundary_function_kind)
        for k, v in enumerate(boundary_function_params):
            d.boundary_function_params[k] = float(v)
        d.record_max_stage = int(bool(record_max_stage))
        d.has_host_boundary_subroutine = int(boundary_subroutine is not None)
        d.has_host_forcing_subroutine = int(forcing_subroutine is not None)
        d.device = int(device)
        self.desc = d
        self.nx = (int(nx[0]), int(nx[1]))
        self.dtype = np.float64 if real_bytes == 8 else np.float32
        self.timestepping_method = timestepping_method
        h = ctypes.c_void_p()
        check(L.swals_gpu_domain_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h

    # ------------------------------------------------------------------ utils
    def close(self):
        if getattr(self, "_h", None):
            self._L.swals_gpu_domain_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # ------------------------------------------------------------- state I/O
    def set_U(self, U):
        U = np.ascontiguousarray(U, dtype=self.dtype)
        assert U.shape == (4, self.nx[1], self.nx[0]), U.shape
        check(self._L.swals_gpu_upload_U(self._h, _p(U)))

    def get_U(self, out=None):
        U = np.empty((4, self.nx[1], self.nx[0]), dtype=self.dtype) if out is None else out
        assert U.dtype == self.dtype and U.shape == (4, self.nx[1], self.nx[0]) and U.flags.c_contiguous
        check(self._L.swals_gpu_download_U(self._h, _p(U)))
        return U

    def set_var(self, k, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        check(self._L.swals_gpu_upload_var(self._h, int(k), _p(a)))

    def get_var(self, k):
        a = np.empty((self.nx[1], self.nx[0]), dtype=self.dtype)
        check(self._L.swals_gpu_download_var(self._h, int(k), _p(a)))
        return a

    def set_manning_squared(self, a):
        a = np.ascontiguousarray(np.broadcast_to(a, (self.nx[1], self.nx[0])), dtype=self.dtype)
        check(self._L.swals_gpu_upload_manning_squared(self._h, _p(a)))

    def max_stage(self):
        a = np.empty((self.nx[1], self.nx[0]), dtype=self.dtype)
        check(self._L.swals_gpu_download_max_stage(self._h, _p(a)))
        return a

    def metrics(self):
        nx, ny = self.nx
        arrs = dict(x=np.zeros(nx), y=np.zeros(ny), dxb=np.zeros(ny + 1), dyl=np.zeros(nx + 1),
                    area=np.zeros(ny), coriolis=np.zeros(ny), coriolis_bottom_edge=np.zeros(ny + 1),
                    tanlat_on_radius_earth=np.zeros(ny))
        check(self._L.swals_gpu_get_metrics(self._h, *[_p(arrs[k]) for k in
                                                      ("x", "y", "dxb", "dyl", "area", "coriolis",
                                                       "coriolis_bottom_edge", "tanlat_on_radius_earth")]))
        return arrs

    @property
    def x(self):
        return self.metrics()["x"]

    @property
    def y(self):
        return self.metrics()["y"]

    # ------------------------------------------------------------- stepping
    def evolve_one_step(self, timestep=None):
        check(self._L.swals_gpu_evolve_one_step(self._h, 0.0 if timestep is None else float(timestep),
                                                0 if timestep is None else 1))

    def evolve_steps(self, nsteps, timestep=None):
        check(self._L.swals_gpu_evolve_steps(self._h, int(nsteps), 0.0 if timestep is None else float(timestep),
                                             0 if timestep is None else 1))

    def synchronize(self):
        check(self._L.swals_gpu_synchronize(self._h))

    def state(self):
        st = _lib.DomainState()
        check(self._L.swals_gpu_get_state(self._h, ctypes.byref(st)))
        return st

    @property
    def time(self):
        return self.state().time

    @time.setter
    def time(self, t):
        check(self._L.swals_gpu_set_time(self._h, float(t)))

    @property
    def max_dt(self):
        return self.state().max_dt

    @property
    def nsteps_advanced(self):
        return self.state().nsteps_advanced

    @property
    def negative_depth_fix_counter(self):
        return self.state().negative_depth_fix_counter

    # ---------------------------------------------------------- diagnostics
    def _scalar(self, fn):
        v = ctypes.c_double()
        check(fn(self._h, ctypes.byref(v)))
        return v.value

    def linear_timestep_max(self):
        return self._scalar(self._L.swals_gpu_linear_timestep_max)

    def nonlinear_stationary_timestep_max(self):
        return self._scalar(self._L.swals_gpu_nonlinear_stationary_timestep_max)

    def stationary_timestep_max(self):
        return self._scalar(self._L.swals_gpu_stationary_timestep_max)

    def volume_interior(self):
        return self._scalar(self._L.swals_gpu_volume_interior)

    # --------------------------------------------------------------- gauges
    def set_priority_mask(self, mask=None):
        """The cells this domain owns in a multidomain, (ny, nx) booleans, or None."""
        if mask is None:
            check(self._L.swals_gpu_set_priority_mask(self._h, None))
            return
        m = np.ascontiguousarray(np.asarray(mask).astype(np.uint8).reshape(self.nx[1], self.nx[0]))
        check(self._L.swals_gpu_set_priority_mask(self._h, _p(m)))

    def add_forcing_patch(self, i0, i1, j0, j1, k0, k1, start_time, end_time, forcing_work):
        """forcing_patch%setup(start_time, end_time, i0, i1, j0, j1, k0, k1)
        with its forcing_work (1-based inclusive indices; forcing_work shaped
        (k1-k0+1, j1-j0+1, i1-i0+1), i.e. [k][j][i] like get_U), applied as
        the domain's forcing (apply_forcing_patch_array).  Returns the
        patch's index."""
        w = np.ascontiguousarray(np.asarray(forcing_work, dtype=np.float64)
                                 .reshape(k1 - k0 + 1, j1 - j0 + 1, i1 - i0 + 1))
        idx = ctypes.c_int32()
        check(self._L.swals_gpu_forcing_patch_add(self._h, i0, i1, j0, j1, k0, k1, float(start_time),
                                                  float(end_time), _p(w), ctypes.byref(idx)))
        return idx.value

    def forcing_clear(self):
        check(self._L.swals_gpu_forcing_clear(self._h))

    def apply_forcing(self, dt):
        """domain%apply_forcing(dt) on the current state at domain%time."""
        check(self._L.swals_gpu_apply_forcing(self._h, float(dt)))

    def set_eddy_viscosity(self, constant, shiono_knight=0.0):
        """domain%use_eddy_viscosity = .true. with eddy_visc_constants =
        [constant, shiono_knight]: the *_eddyvisc flux variants, with a
        constant (shiono_knight = 0) or constant + Shiono-Knight viscosity.
        Finite-volume methods only."""
        check(self._L.swals_gpu_set_eddy_viscosity(self._h, 1, float(constant), float(shiono_knight)))

    def set_static_before_time(self, t):
        """domain%static_before_time: steps starting before t only advance the clock."""
        check(self._L.swals_gpu_set_static_before_time(self._h, float(t)))

    def set_max_U_update_frequency(self, every):
        """domain%max_U_update_frequency: max_stage updated every `every` steps."""
        check(self._L.swals_gpu_set_max_U_update_frequency(self._h, int(every)))

    MAX_U_VARIABLES = {"time_of_max_stage": 1, "max_speed": 2, "max_flux": 4, "arrival_time": 8, "min_stage": 16}

    def set_max_U_variables(self, names=(), stage_extrema_include_dry_cells=True,
                            arrival_stage_threshold_above_msl_linear=0.01):
        """The max_U_variables recorded after max_stage (before the first step)."""
        mask = 0
        for n in names:
            mask |= self.MAX_U_VARIABLES[n]
        check(self._L.swals_gpu_set_max_U_variables(self._h, mask, int(bool(stage_extrema_include_dry_cells)),
                                                     float(arrival_stage_threshold_above_msl_linear)))

    def max_U(self, name):
        """One recorded max_U variable as an (ny, nx) array."""
        nx, ny = self.nx
        out = np.empty(nx * ny, dtype=np.float64)
        check(self._L.swals_gpu_download_max_U(self._h, self.MAX_U_VARIABLES[name], out.ctypes.data))
        return out.reshape(ny, nx)

    def clear_eddy_viscosity(self):
        check(self._L.swals_gpu_set_eddy_viscosity(self._h, 0, 0.0, 0.0))

    GRID_VARS = {"stage": 1, "uh": 2, "vh": 4, "elevation": 8, "max_stage": 16}

    def stage_grids_real4(self, variables=("stage", "uh", "vh", "elevation"), spatial_stride=1):
        """The netCDF grid payload in REAL4: {name: (cy, cx) float32}, each
        U(start:nx:stride, start:ny:stride) with start = stride/2 + 1."""
        mask = 0
        for v in variables:
            mask |= self.GRID_VARS[v]
        st = spatial_stride // 2
        cx = (self.nx[0] - 1 - st) // spatial_stride + 1
        cy = (self.nx[1] - 1 - st) // spatial_stride + 1
        order = [v for v in self.GRID_VARS if v in variables]
        out = np.empty((len(order), cy, cx), dtype=np.float32)
        cnt = (ctypes.c_int32 * 2)()
        check(self._L.swals_gpu_stage_grids_real4(self._h, mask, int(spatial_stride), _p(out), out.size, cnt))
        assert (cnt[0], cnt[1]) == (cx, cy)
        return {v: out[k] for k, v in enumerate(order)}

    def gauges_read_real4(self):
        """Recorded gauge series in REAL4: (3, n_records, n_gauges) for STG,
        UH, VH (station fastest, as the netCDF variables)."""
        n = self._n_gauges
        cap = self._gauge_capacity
        out = np.empty((3, cap, n), dtype=np.float32)
        nrec = ctypes.c_int32()
        check(self._L.swals_gpu_gauges_read_real4(self._h, _p(out), cap, ctypes.byref(nrec)))
        flat = out.reshape(-1)[:3 * nrec.value * n]
        return flat.reshape(3, nrec.value, n).copy()

    def volume_in_priority_domain(self):
        """volume_interior over the cells set_priority_mask kept."""
        return self._scalar(self._L.swals_gpu_volume_in_priority_domain)

    def compute_domain_statistics(self):
        """compute_domain_statistics_new: dict of maxstage, maxspeed, minstage,
        minspeed, energy_potential_on_rho, energy_kinetic_on_rho, energy_total_on_rho."""
        out = (ctypes.c_double * 7)()
        check(self._L.swals_gpu_domain_statistics(self._h, out))
        keys = ["maxstage", "maxspeed", "minstage", "minspeed", "energy_potential_on_rho",
                "energy_kinetic_on_rho", "energy_total_on_rho"]
        return dict(zip(keys, list(out)))

    def gauges_setup(self, xy, capacity):
        xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1, 2)
        self._n_gauges = xy.shape[0]
        check(self._L.swals_gpu_gauges_setup(self._h, _p(xy), int(xy.shape[0]), int(capacity)))
        self._gauge_capacity = int(capacity)

    def gauges_site_index(self):
        out = np.zeros((self._n_gauges, 2), dtype=np.int32)
        check(self._L.swals_gpu_gauges_site_index(self._h, _p(out)))
        return out

    def gauges_read(self):
        out = np.zeros((self._gauge_capacity, self._n_gauges, 3), dtype=np.float64)
        n = ctypes.c_int32()
        check(self._L.swals_gpu_gauges_read(self._h, _p(out), int(self._gauge_capacity), ctypes.byref(n)))
        return out[: n.value]

    def gauges_reset(self):
        check(self._L.swals_gpu_gauges_reset(self._h))

    # ------------------------------------------------------------- adjoint
    def adjoint_linear(self, nsteps, timestep, gauge_adjoint=None, lambda_seed=None):
        """dL/d(STG,UH,VH) of the initial state, shape (3, ny, nx), given
        gauge_adjoint[n, g] = dL/d(stage at gauge g after step n+1) and/or
        lambda_seed = dL/d(state after the last step), shape (3, ny, nx)."""
        out = np.empty((3, self.nx[1], self.nx[0]), dtype=self.dtype)
        ga = None if gauge_adjoint is None else np.ascontiguousarray(gauge_adjoint, dtype=np.float64)
        ls = None if lambda_seed is None else np.ascontiguousarray(lambda_seed, dtype=self.dtype)
        check(self._L.swals_gpu_adjoint_linear(self._h, int(nsteps), float(timestep),
                                               None if ga is None else _p(ga), None if ls is None else _p(ls),
                                               _p(out)))
        return out

    def misfit_gradient(self, nsteps, timestep, target, checkpoint_every=50):
        """(L, dL/d(STG,UH,VH)_0) for L = 1/2 sum (gauge stage - target)^2
        over steps 1..nsteps from the current state (left unchanged)."""
        target = np.ascontiguousarray(target, dtype=np.float64)
        out = np.empty((3, self.nx[1], self.nx[0]), dtype=self.dtype)
        loss = ctypes.c_double()
        check(self._L.swals_gpu_misfit_gradient_linear(self._h, int(nsteps), float(timestep), _p(target),
                                                       int(checkpoint_every), ctypes.byref(loss), _p(out)))
        return loss.value, out

    def device_planes(self):
        ptrs = [ctypes.c_void_p() for _ in range(4)]
        pitch = ctypes.c_int64()
        check(self._L.swals_gpu_device_planes(self._h, *[ctypes.byref(p) for p in ptrs], ctypes.byref(pitch)))
        return [p.value for p in ptrs], pitch.value

    def timers_enable(self, on=True):
        check(self._L.swals_gpu_timers_enable(self._h, int(bool(on))))

    def timers_read(self):
        """Per-kernel-category totals: {name: (milliseconds, launches)}."""
        buf = (ctypes.c_double * (2 * len(_lib.TIMER_NAMES)))()
        n = ctypes.c_int32()
        check(self._L.swals_gpu_timers_read(self._h, buf, len(buf), ctypes.byref(n)))
        return {name: (buf[2 * c], int(buf[2 * c + 1])) for c, name in enumerate(_lib.TIMER_NAMES)}

    def launch_count(self):
        v = ctypes.c_int64()
        check(self._L.swals_gpu_launch_count(self._h, ctypes.byref(v)))
        return v.value

    def stream(self):
        s = ctypes.c_void_p()
        check(self._L.swals_gpu_stream(self._h, ctypes.byref(s)))
        return s.value
