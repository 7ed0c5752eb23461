"""Test infrastructure only: ctypes wrapper around the C oracle (swals_oracle.c).

The oracle is the CPU restatement of SWALS's time-step hot path that the CUDA
implementation is checked against.  Only tests, the smoke check and the CPU
baseline leg of bench.py may import this module.

Arrays are numpy arrays in the reference's Fortran layout: ``U`` has shape
``(4, ny, nx)`` here, i.e. C-order planes ``U[k-1, j-1, i-1]`` equal to the
reference's column-major ``U(i, j, k)`` (i fastest in memory in both).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# compute_fluxes_inner_method -> flux_variant bits (1: fr2 = 1, 2: upwind transverse momentum)
FLUX_VARIANTS = {"DE1_low_fr_diffusion": 0, "DE1": 1, "DE1_upwind_transverse": 3,
                 "DE1_low_fr_diffusion_upwind_transverse": 2}
METHODS = {
    "rk2": 1, "rk2n": 2, "midpoint": 3, "euler": 4, "linear": 5,
    "leapfrog_linear_plus_nonlinear_friction": 6, "cliffs": 7, "leapfrog_nonlinear": 8,
}
BC_NONE, BC_TRANSMISSIVE, BC_STAGE_TRANSMISSIVE_NORMAL_MOMENTUM, BC_FLATHER = 0, 1, 2, 3
BF_SOLITARY_WEST_WALLS = 1
NEG_HUGE = -np.finfo(np.float64).max


def build():
    """Compile both oracle variants (idempotent)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


# Oracle builds (oracle/Makefile): the IEEE-strict checker, the same with
# libm's pow for the friction power law, and the -Ofast-style baseline build.
VARIANTS = {"strict": "liboracle64.so", "libm": "liboracle64_libm.so", "fast": "liboracle64_fast.so",
            "native": "liboracle64_native.so"}


def _load(real32: bool, variant: str = "strict"):
    name = "liboracle32.so" if real32 else VARIANTS[variant]
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        build()
    return ctypes.CDLL(path)


class _OracleDomainC(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
        ("lw", ctypes.c_double * 2), ("lower_left", ctypes.c_double * 2),
        ("method", ctypes.c_int32), ("spherical", ctypes.c_int32), ("coriolis", ctypes.c_int32),
        ("nofriction", ctypes.c_int32), ("truely_linear", ctypes.c_int32), ("friction_chezy", ctypes.c_int32),
        ("xL", ctypes.c_int32), ("xU", ctypes.c_int32), ("yL", ctypes.c_int32), ("yU", ctypes.c_int32),
        ("exterior_cells_width", ctypes.c_int32), ("boundary_exterior", ctypes.c_int32 * 4),
        ("bc_kind", ctypes.c_int32), ("bf_kind", ctypes.c_int32), ("record_max_stage", ctypes.c_int32),
        ("flux_variant", ctypes.c_int32),
        ("theta", ctypes.c_double), ("cfl", ctypes.c_double), ("msl_linear", ctypes.c_double),
        ("linear_friction_coeff", ctypes.c_double), ("maximum_timestep", ctypes.c_double),
        ("bf_params", ctypes.c_double * 8),
        ("time", ctypes.c_double), ("max_dt", ctypes.c_double), ("dt_last_update", ctypes.c_double),
        ("evolve_step_dt", ctypes.c_double),
        ("nsteps_advanced", ctypes.c_int64), ("negative_depth_fix_counter", ctypes.c_int64),
        ("boundary_flux_store", ctypes.c_double * 4),
        ("boundary_flux_evolve_integral", ctypes.c_double),
        ("boundary_flux_time_integral", ctypes.c_double),
        ("U", ctypes.c_void_p), ("max_stage", ctypes.c_void_p), ("manning_squared", ctypes.c_void_p),
        ("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("dxb", ctypes.c_void_p), ("dyl", ctypes.c_void_p),
        ("area", ctypes.c_void_p), ("coriolis_c", ctypes.c_void_p), ("coriolis_be", ctypes.c_void_p),
        ("tanlat_on_R", ctypes.c_void_p),
        ("depth", ctypes.c_void_p), ("velocity", ctypes.c_void_p), ("flux_NS", ctypes.c_void_p),
        ("flux_EW", ctypes.c_void_p), ("explicit_source", ctypes.c_void_p),
        ("explicit_source_VH_j_minus_1", ctypes.c_void_p), ("backup_U", ctypes.c_void_p),
        ("nest_nbox", ctypes.c_int32), ("friction_work_is_setup", ctypes.c_int32), ("nest_boxes", ctypes.c_void_p),
        ("nest_offset", ctypes.c_void_p), ("nest_integral", ctypes.c_void_p), ("friction_work", ctypes.c_void_p),
        ("n_forcing", ctypes.c_int32), ("pad2", ctypes.c_int32), ("forcing", ctypes.c_void_p),
        ("advection_work", ctypes.c_void_p),
        ("use_eddy_viscosity", ctypes.c_int32), ("pad3", ctypes.c_int32),
        ("eddy_visc_constants", ctypes.c_double * 2), ("eddy_visc", ctypes.c_void_p),
        ("static_before_time", ctypes.c_double), ("max_U_update_frequency", ctypes.c_int32),
        ("max_U_extra", ctypes.c_int32), ("stage_extrema_include_dry_cells", ctypes.c_int32), ("pad5", ctypes.c_int32),
        ("arrival_stage_threshold_above_msl_linear", ctypes.c_double), ("max_U_extra_planes", ctypes.c_void_p),
    ]


class _ForcingPatchC(ctypes.Structure):
    _fields_ = [("i0", ctypes.c_int32), ("i1", ctypes.c_int32), ("j0", ctypes.c_int32), ("j1", ctypes.c_int32),
                ("k0", ctypes.c_int32), ("k1", ctypes.c_int32), ("start_time", ctypes.c_double),
                ("end_time", ctypes.c_double), ("work", ctypes.c_void_p)]


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def add_forcing_work_to_U_over_time(U, work, time, dt, start_time, end_time, real32=False):
    """forcing_mod.f90:80-156 on numpy arrays (U updated in place)."""
    lib = _load(real32)
    f = getattr(lib, ("oracle32_" if real32 else "oracle64_") + "add_forcing_work_to_U_over_time")
    R = ctypes.c_float if real32 else ctypes.c_double
    f.restype = None
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, R, R, R, R]
    assert U.flags.c_contiguous and work.shape == U.shape
    f(_ptr(U), _ptr(np.ascontiguousarray(work)), U.size, time, dt, start_time, end_time)


class OracleDomain:
    """One SWALS ``domain_type`` restated on the CPU (test checker)."""

    def __init__(self, nx, ny, lw, lower_left=(0.0, 0.0), timestepping_method="linear",
                 spherical=False, coriolis=None, nofriction=False, truely_linear=True,
                 friction_type="manning", cfl=None, theta=None, msl_linear=0.0,
                 linear_friction_coeff=0.0, maximum_timestep=1.0e20,
                 boundary_exterior=(True, True, True, True), bc_kind=BC_NONE,
                 bf_kind=0, bf_params=(), record_max_stage=True, real32=False,
                 xL=0, xU=0, yL=0, yU=0, compute_fluxes_inner_method="DE1_low_fr_diffusion", variant="strict"):
        self.real32 = real32
        self.dtype = np.float32 if real32 else np.float64
        self.lib = _load(real32, variant)
        self.pref = "oracle32_" if real32 else "oracle64_"
        if coriolis is None:
            coriolis = bool(spherical)
        c = _OracleDomainC()
        c.nx, c.ny = nx, ny
        c.lw[0], c.lw[1] = lw
        c.lower_left[0], c.lower_left[1] = lower_left
        c.method = METHODS[timestepping_method]
        c.spherical, c.coriolis, c.nofriction = int(spherical), int(coriolis), int(nofriction)
        c.truely_linear = int(truely_linear)
        c.friction_chezy = int(friction_type == "chezy")
        c.xL, c.xU, c.yL, c.yU = xL, xU, yL, yU
        c.exterior_cells_width = 2
        for k in range(4):
            c.boundary_exterior[k] = int(boundary_exterior[k])
        c.bc_kind, c.bf_kind = bc_kind, bf_kind
        for k, v in enumerate(bf_params):
            c.bf_params[k] = v
        c.record_max_stage = int(record_max_stage)
        c.flux_variant = FLUX_VARIANTS[compute_fluxes_inner_method]
        c.theta = NEG_HUGE if theta is None else theta
        c.cfl = NEG_HUGE if cfl is None else cfl
        c.msl_linear = msl_linear
        c.linear_friction_coeff = linear_friction_coeff
        c.maximum_timestep = maximum_timestep
        c.static_before_time = NEG_HUGE
        c.max_U_update_frequency = 1
        c.stage_extrema_include_dry_cells = 1
        c.arrival_stage_threshold_above_msl_linear = 0.01
        self.c = c
        dt = self.dtype
        self.U = np.zeros((4, ny, nx), dtype=dt)
        # -0.99 * huge(real(1.0, output_precision)) evaluated in float32 (domain_mod.f90:1108)
        init = np.float32(-0.99) * np.finfo(np.float32).max
        self.max_stage = np.full((ny, nx), init, dtype=dt)
        self.manning_squared = np.zeros((ny, nx), dtype=dt)
        self.x = np.zeros(nx, dt); self.y = np.zeros(ny, dt)
        self.dxb = np.zeros(ny + 1, dt); self.dyl = np.zeros(nx + 1, dt)
        self.area = np.zeros(ny, dt); self.coriolis_c = np.zeros(ny, dt)
        self.coriolis_be = np.zeros(ny + 1, dt); self.tanlat_on_R = np.zeros(ny, dt)
        self.depth = np.zeros((ny, nx), dt)
        self.velocity = np.zeros((2, ny, nx), dt)
        self.flux_NS = np.zeros((3, ny + 1, nx), dt)
        self.flux_EW = np.zeros((3, ny, nx + 1), dt)
        self.explicit_source = np.zeros((2, ny, nx), np.float64)
        self.es_jm1 = np.zeros((ny + 1, nx), np.float64)
        self.backup_U = np.zeros((3, ny, nx), dt)
        self.friction_work = np.zeros((2, ny, nx), dt)
        self.advection_work = np.zeros((5, ny, nx), dt)
        self.eddy_visc = np.zeros((ny, nx), dt)
        # time_of_max_stage, max_speed, max_flux, arrival_time, min_stage
        self.max_U_extra = np.zeros((5, ny, nx), dt)
        self.max_U_extra[:] = init
        self.max_U_extra[4] = -init
        for name, arr in [("U", self.U), ("max_stage", self.max_stage), ("manning_squared", self.manning_squared),
                          ("x", self.x), ("y", self.y), ("dxb", self.dxb), ("dyl", self.dyl), ("area", self.area),
                          ("coriolis_c", self.coriolis_c), ("coriolis_be", self.coriolis_be),
                          ("tanlat_on_R", self.tanlat_on_R), ("depth", self.depth), ("velocity", self.velocity),
                          ("flux_NS", self.flux_NS), ("flux_EW", self.flux_EW),
                          ("explicit_source", self.explicit_source),
                          ("explicit_source_VH_j_minus_1", self.es_jm1), ("backup_U", self.backup_U),
                          ("friction_work", self.friction_work), ("advection_work", self.advection_work),
                          ("eddy_visc", self.eddy_visc), ("max_U_extra_planes", self.max_U_extra)]:
            setattr(c, name, _ptr(arr))
        self._fn("apply_method_defaults")(ctypes.byref(c))
        self._fn("setup_geometry")(ctypes.byref(c))

    def _fn(self, name, restype=None):
        f = getattr(self.lib, self.pref + name)
        f.restype = restype
        return f

    # --- reference-named API -------------------------------------------
    def evolve_one_step(self, timestep=None):
        f = self._fn("evolve_one_step", ctypes.c_int)
        f.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        rc = f(ctypes.addressof(self.c), 0.0 if timestep is None else float(timestep), 0 if timestep is None else 1)
        if rc != 0:
            raise RuntimeError(f"oracle evolve_one_step failed rc={rc}")

    def linear_timestep_max(self):
        f = self._fn("linear_timestep_max", ctypes.c_double)
        f.argtypes = [ctypes.c_void_p]
        return f(ctypes.addressof(self.c))

    def nonlinear_stationary_timestep_max(self):
        f = self._fn("nonlinear_stationary_timestep_max", ctypes.c_double)
        f.argtypes = [ctypes.c_void_p]
        return f(ctypes.addressof(self.c))

    def volume_interior(self):
        f = self._fn("volume_interior", ctypes.c_double)
        f.argtypes = [ctypes.c_void_p]
        return f(ctypes.addressof(self.c))

    def volume_in_priority_domain(self, mask=None):
        """volume_interior over the cells of mask (ny, nx), or all cells."""
        f = self._fn("volume_in_priority_domain", ctypes.c_double)
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
        return f(ctypes.addressof(self.c), None if m is None else _ptr(m))

    def set_eddy_viscosity(self, constant, shiono_knight=0.0):
        """domain%use_eddy_viscosity = .true. with eddy_visc_constants =
        [constant, shiono_knight] (domain_mod.f90:233-243, 890-898); only
        the finite-volume methods support it."""
        if self.c.method not in (METHODS["rk2"], METHODS["rk2n"], METHODS["midpoint"], METHODS["euler"]):
            raise ValueError("eddy viscosity is not supported for this timestepping_method")
        self.c.use_eddy_viscosity = 1
        self.c.eddy_visc_constants[0] = constant
        self.c.eddy_visc_constants[1] = shiono_knight

    def add_forcing_patch(self, i0, i1, j0, j1, k0, k1, start_time, end_time, work):
        """forcing_patch%setup + forcing_work (forcing_mod.f90:264-319),
        applied with apply_forcing_patch_array: 1-based inclusive indices,
        work shaped (k1-k0+1, j1-j0+1, i1-i0+1)."""
        w = np.ascontiguousarray(np.asarray(work, dtype=self.dtype).reshape(k1 - k0 + 1, j1 - j0 + 1, i1 - i0 + 1))
        if not hasattr(self, "_patches"):
            self._patches = []
        self._patches.append((i0, i1, j0, j1, k0, k1, float(start_time), float(end_time), w))
        arr = (_ForcingPatchC * len(self._patches))()
        for q, (a, b, c_, d_, e, f, st, en, ww) in enumerate(self._patches):
            arr[q] = _ForcingPatchC(a, b, c_, d_, e, f, st, en, ww.ctypes.data)
        self._patch_arr = arr
        self.c.n_forcing = len(self._patches)
        self.c.forcing = ctypes.addressof(arr)

    def domain_statistics(self, mask=None):
        """compute_domain_statistics_new: (maxstage, maxspeed, minstage,
        minspeed, E_potential, E_kinetic, E_total); mask (ny, nx) of the
        domain's own priority cells, or None."""
        f = self._fn("domain_statistics")
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        out = np.zeros(7)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
        f(ctypes.addressof(self.c), None if m is None else _ptr(m), _ptr(out))
        return tuple(out)

    @property
    def time(self):
        return self.c.time

    @property
    def max_dt(self):
        return self.c.max_dt

    @property
    def nsteps_advanced(self):
        return self.c.nsteps_advanced

    @property
    def negative_depth_fix_counter(self):
        return self.c.negative_depth_fix_counter

    @property
    def theta(self):
        return self.c.theta

    @property
    def cfl(self):
        return self.c.cfl


def limited_gradient_dx(U_local, U_lower, U_upper, theta, real32=False):
    """MC limiter of extrapolation_limiting_mod.f90:44-79 (vectorised form)."""
    dt = np.float32 if real32 else np.float64
    lib = _load(real32)
    f = getattr(lib, ("oracle32_" if real32 else "oracle64_") + "limited_gradient_dx_vectorized")
    f.restype = None
    arrs = [np.ascontiguousarray(a, dtype=dt) for a in (U_local, U_lower, U_upper, theta)]
    out = np.zeros_like(arrs[0])
    f(*[_ptr(a) for a in arrs], _ptr(out), ctypes.c_int32(len(out)))
    return out


def area_lonlat_rectangle(lon1, lat1, dlon, dlat, flat=False):
    lib = _load(False)
    f = lib.oracle64_area_lonlat_rectangle
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_double] * 4 + [ctypes.c_int]
    return f(lon1, lat1, dlon, dlat, int(flat))


def gauge_site_index(xy, ll, dx, nxy):
    """point_gauge_mod.f90:336-340; returns 1-based (n,2) indices."""
    lib = _load(False)
    xy = np.ascontiguousarray(xy, dtype=np.float64)
    n = xy.shape[0]
    out = np.zeros((n, 2), dtype=np.int32)
    f = lib.oracle64_gauge_site_index
    f.restype = None
    f(_ptr(xy), ctypes.c_int32(n), _ptr(np.asarray(ll, np.float64)), _ptr(np.asarray(dx, np.float64)),
      _ptr(np.asarray(nxy, np.int32)), _ptr(out))
    return out
