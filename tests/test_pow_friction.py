"""The friction power law max(depth, mad)**p (update_U_DE1_inner_include.f90:
72-75) is evaluated correctly rounded (p = fl(-7/3) for Manning, -2 for
Chezy) so that oracle and GPU agree bit for bit whatever libm is present.
Check the oracle's definition against 300-bit arithmetic."""
import ctypes
import random

import mpmath
import pytest

from oracle import oracle as orc


@pytest.mark.parametrize("chezy", [0, 1])
def test_pow_friction_is_correctly_rounded(chezy):
    lib = orc._load(False)
    f = lib.oracle64_pow_friction
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_double, ctypes.c_int32]
    mpmath.mp.prec = 300
    p = mpmath.mpf(-2.0 if chezy else -7.0 / 3.0)
    rng = random.Random(1234 + chezy)
    for k in range(20000):
        u = rng.random()
        x = 1e-5 * 10 ** (9 * u) if k % 2 else 1e-5 + 80 * u
        want = float(mpmath.power(mpmath.mpf(x), p))
        assert f(x, chezy) == want, (x, f(x, chezy), want)


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
