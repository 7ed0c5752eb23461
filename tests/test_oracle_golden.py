"""Pin the CPU oracle against the reference's own unit-test known answers.

Each case restates a test of SWALS's Fortran unit suite:
- MC limiter: extrapolation_limiting_mod.f90:171-291 (10 cases, tol 100*spacing(1)).
- Spherical area: spherical_mod.f90:92-150 (known areas at R=6378137).
- Point gauges: point_gauge_mod.f90:671-776 (nearest-cell site indices).
"""
import numpy as np
import pytest

from oracle import oracle as orc


N = 10


def _base():
    U = np.arange(1, N + 1, dtype=np.float64) - 5.5
    return U


def _check(desired, answer):
    tol = np.spacing(1.0) * 100
    assert np.all(np.abs(desired - answer) < tol), (desired, answer)


@pytest.mark.parametrize("real32", [False, True])
def test_mc_limiter_known_answers(real32):
    dt = np.float32 if real32 else np.float64
    U = _base().astype(dt)

    def grad(Ul, Uu, th):
        return orc.limited_gradient_dx(U, Ul, Uu, np.full(N, th, dt), real32=real32).astype(np.float64)

    Uf = U.astype(np.float64)
    tolcheck = (lambda d, a: np.testing.assert_allclose(a, d, atol=1e-5)) if real32 else _check
    # Basic extrapolation, positive side
    a = grad(U - 1, U + 1, 1.0)
    tolcheck(0.5 * (Uf + (Uf + 1)), Uf + 0.5 * a)
    # negative side
    tolcheck(0.5 * (Uf + (Uf - 1)), Uf - 0.5 * a)
    # negative side, reduced theta
    a = grad(U - 1, U + 1, 0.5)
    tolcheck(0.5 * Uf + 0.25 * (Uf + (Uf - 1)), Uf - 0.5 * a)
    # zero theta
    a = grad(U - 1, U + 1, 0.0)
    tolcheck(Uf, Uf + 0.5 * a)
    # local min
    a = grad(U + 2, U + 3, 4.0)
    tolcheck(Uf, Uf + 0.5 * a)
    # local max
    a = grad(U - 2, U - 3, 4.0)
    tolcheck(Uf, Uf - 0.5 * a)
    # limited gradients: central 2, lower 1, upper 3
    a = grad(U - 1, U + 3, 1.0)
    tolcheck(Uf + 0.5 * 1.0, Uf + 0.5 * a)
    a = grad(U - 1, U + 3, 1.5)
    tolcheck(Uf + 0.5 * 1.5, Uf + 0.5 * a)
    tolcheck(Uf - 0.5 * 1.5, Uf - 0.5 * a)


def test_spherical_area_known_answers():
    radius_earth = 6371000.0
    test_radius = 6378137.0
    adj = (test_radius / radius_earth) ** 2
    a = orc.area_lonlat_rectangle(0.0, 0.0, 1.0, 1.0, flat=False)
    assert abs(a * adj - 12391399902.0) < 1e-6 * 12391399902.0
    d2r = np.pi / 180.0
    ans = radius_earth * radius_earth * np.cos(0.5 * d2r) * 1.0 * d2r * 1.0 * d2r
    a = orc.area_lonlat_rectangle(0.0, 0.0, 1.0, 1.0, flat=True)
    assert abs(a - ans) < 1e-6 * ans
    a = orc.area_lonlat_rectangle(108.0, -11.0, 1.0 / 60.0, 1.0 / 60.0)
    assert abs(a * adj - 3379082.32316) < 1e-6 * 3379082.32316
    a = orc.area_lonlat_rectangle(108.0, -11.0, 1.0 / 60.0, 1.0 / 120.0)
    assert abs(a * adj - 1689517.29722) < 1e-6 * 1689517.29722


def test_point_gauge_site_index_known_answers():
    ll = np.array([-100.0, 250.0])
    dx = np.array([1.0, 2.0])
    nxy = np.array([104, 104], np.int32)
    eps = 1.0e-4
    offs = np.array([[0, 0], [50, 20], [20, 50], [20, 200], [90, 10], [90, 10]], np.float64)
    xy = offs + ll + eps
    site = orc.gauge_site_index(xy, ll, dx, nxy)
    np.testing.assert_array_equal(site[:, 0], np.floor((xy[:, 0] - ll[0]) / dx[0]).astype(int) + 1)
    np.testing.assert_array_equal(site[:, 1], np.floor((xy[:, 1] - ll[1]) / dx[1]).astype(int) + 1)
    assert np.all(site <= 104) and np.all(site > 0)
    # U(i,j,k) = i + j**2 + k**3 lookup, as in the reference test
    for k in (1, 2, 3, 4):
        vals = site[:, 0] + site[:, 1] ** 2 + k ** 3
        assert np.all(vals == site[:, 0] + site[:, 1] ** 2 + k ** 3)
    # corner case: coordinate exactly on the upper edge maps to nx
    site = orc.gauge_site_index(np.array([[ll[0] + 104.0, ll[1] + 208.0]]), ll, dx, nxy)
    assert tuple(site[0]) == (104, 104)


def _forcing_case(n, lw, ll):
    """setup_domain_for_test (forcing_mod.f90:341-378): U = (x+y, x, y,
    x+y-10); forcing_work 10, 5, 1, -1 on STG, UH, VH, ELV."""
    nx, ny = n
    x = ll[0] + (np.arange(1, nx + 1) - 0.5) * lw[0] / nx
    y = ll[1] + (np.arange(1, ny + 1) - 0.5) * lw[1] / ny
    X, Y = np.meshgrid(x, y)
    U = np.stack([X + Y, X, Y, X + Y - 10.0])
    W = np.stack([np.full_like(X, v) for v in (10.0, 5.0, 1.0, -1.0)])
    return U, W


@pytest.mark.parametrize("dom", [((50, 30), (50.0, 30.0), (0.0, 0.0)), ((23, 90), (10.0, 10.0), (1.0, 1.0))])
def test_forcing_known_answers(dom):
    """test_forcing_mod (forcing_mod.f90:387-562): the fraction of
    forcing_work added for a step (time - dt, time) against the forcing
    interval, to spacing(10)*10."""
    from oracle.oracle import add_forcing_work_to_U_over_time as add
    U0, W = _forcing_case(*dom)
    tol = np.spacing(10.0) * 10
    cases = [((0.0, 10.0), 1.0), ((4.0, 10.0), 1.0), ((-4.0, 10.0), 10.0 / 14.0), ((-15.0, 15.0), 10.0 / 30.0),
             ((-15.0, 5.0), 5.0 / 20.0), ((-15.0, -5.0), 0.0)]
    for (st, en), frac in cases:
        U = U0.copy()
        add(U, W, 10.0, 10.0, st, en)
        err = np.max(np.abs(U - (U0 + W * frac)))
        assert err < tol if frac else err == 0.0, (st, en, err)
    # Test 7: stepping through the whole interval adds the whole forcing.
    U = U0.copy()
    t, dt = -10.01242, 1.4444
    for _ in range(30):
        add(U, W, t, dt, -1.332, 5.15430)
        t = t + dt
    assert np.max(np.abs(U - (U0 + W))) < tol
