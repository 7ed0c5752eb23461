"""The friction power law max(depth, mad)**p (update_U_DE1_inner_include.f90:
72-75), p = fl(-7/3) for Manning and -2 for Chezy, is one IEEE operation
sequence shared by the oracle and the device library, so the two agree bit
for bit whatever libm is present.  Here: its accuracy against 300-bit
arithmetic (Chezy correctly rounded, Manning within 3 ulp), and the parity
tolerance holding against an oracle that calls libm's pow instead (the
reference's own friction power)."""
import ctypes
import random

import mpmath
import numpy as np
import pytest

from oracle import oracle as orc
from ptha_b200 import workloads
from pairs import oracle_from_kw, rel_err, water_mask


def _ulp_error(got, want):
    return float(abs(mpmath.mpf(got) - want) / mpmath.mpf(np.spacing(abs(float(want)))))


@pytest.mark.parametrize("chezy", [0, 1])
def test_pow_friction_accuracy(chezy):
    lib = orc._load(False)
    f = lib.oracle64_pow_friction
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_double, ctypes.c_int32]
    mpmath.mp.prec = 300
    p = mpmath.mpf(-2.0 if chezy else -7.0 / 3.0)
    rng = random.Random(1234 + chezy)
    worst, exact = 0.0, 0
    n = 20000
    for k in range(n):
        u = rng.random()
        x = 1e-5 * 10 ** (9 * u) if k % 2 else 1e-5 + 80 * u
        want = mpmath.power(mpmath.mpf(x), p)
        got = f(x, chezy)
        worst = max(worst, _ulp_error(got, want))
        exact += got == float(want)
    print("chezy", chezy, "max ulp error", worst, "correctly rounded fraction", exact / n)
    if chezy:
        assert exact == n
    else:
        assert worst <= 3.0
    for x in (1e-5, 1.0, 8.0, 1e4):   # powers that are exactly representable, or nearly so
        assert _ulp_error(f(x, chezy), mpmath.power(mpmath.mpf(x), p)) <= 3.0


@pytest.mark.parametrize("method,nsteps", [("rk2", 1200), ("leapfrog_linear_plus_nonlinear_friction", 1200)])
def test_parity_tolerance_holds_against_libm_pow(method, nsteps):
    """The oracle (this library's friction power) against the same oracle
    with libm's pow, on the wet/dry beach with the wave running up the slope:
    the states stay within the 1e-10 relative parity tolerance."""
    kw, U, gauges, nsq = workloads.rk2_beach(n=96, dx=10.0 * 2048 / 96, toe=17580.0 * 96 / 2048)
    kw = dict(kw, timestepping_method=method)
    a = oracle_from_kw(kw)
    b = oracle_from_kw(kw, variant="libm")
    for o in (a, b):
        o.U[:] = U
        o.manning_squared[:] = nsq
    dt = None if method == "rk2" else 0.5 * a.linear_timestep_max()
    for _ in range(nsteps):
        a.evolve_one_step(dt)
        b.evolve_one_step(dt)
    m = water_mask(a.U[3])
    errs = [rel_err(a.U[k], b.U[k], mask=m) for k in range(3)]
    moved = (np.abs(a.U[0] - U[0]) > 1e-3) & (U[3] > -5.0) & m
    print(method, "rel differences vs libm pow", errs, "differing cells",
          int(np.sum(a.U[0] != b.U[0])), "cells moved near the shore", int(moved.sum()))
    assert moved.any()
    assert max(errs) <= 1e-10, errs


def test_boundary_cosh_is_correctly_rounded():
    """cosh of the device boundary functions (solitary wave sech^2) is the
    correctly rounded value, so oracle and GPU give identical boundary stages."""
    lib = orc._load(False)
    f = lib.oracle64_cosh_cr
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_double]
    mpmath.mp.prec = 300
    rng = random.Random(77)
    for k in range(20000):
        a = rng.uniform(-120.0, 120.0) if k % 2 else rng.uniform(-3.0, 3.0)
        want = float(mpmath.cosh(mpmath.mpf(a)))
        assert f(a) == want, (a, f(a), want)
    assert f(0.0) == 1.0


def test_pow_eddy_is_correctly_rounded():
    """depth**(1 - 1/6) of the Shiono-Knight eddy viscosity
    (compute_fluxes_DE1_inner_include.f90:1000-1002), correctly rounded."""
    lib = orc._load(False)
    f = lib.oracle64_pow_eddy
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_double]
    mpmath.mp.prec = 300
    p = mpmath.mpf(1.0 - 1.0 / 6.0)
    rng = random.Random(4321)
    for k in range(20000):
        u = rng.random()
        x = 1e-8 * 10 ** (12 * u) if k % 2 else 100 * u
        want = float(mpmath.power(mpmath.mpf(x), p))
        assert f(x) == want, (x, f(x), want)
    assert f(0.0) == 0.0
