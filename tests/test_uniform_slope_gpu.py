"""Steady uniform flow down a planar slope: the reference's own validation
(SW/examples/uniform_slope/uniform_slope.f90) on the GPU.

A 50 x 1000 channel (dx = 1 m) on a 1 % slope with walls on every side,
Manning n = 0.03, fed with 1 m^2/s per metre of width just inside the upper
wall, run for 600 s.  The inflow is a device forcing patch on that row (a
constant rate, so each step adds Qin dt over the row's cells, as the example
adds after each step).  Acceptance, as in the example: the volume equals
the initial volume plus the inflow to 1e-6, the discharge near the centre
equals the inflow to 1e-5 (finite volume) or 1e-4 (the leapfrog with
nonlinear friction), and the depth equals the Manning normal depth
(n^2 q^2 / S)^(3/10) to 1e-4."""
import numpy as np
import pytest

from ptha_b200 import Domain

pytestmark = pytest.mark.gpu

SLOPE = 0.01
Q = 1.0                     # discharge per unit width (m^2/s)
NX, NY, LW = 50, 1000, (50.0, 1000.0)
WALL = 1.0e6


def _initial(method):
    x = (np.arange(1, NX + 1) - 0.5) * 1.0 - LW[0] * 0.5
    y = (np.arange(1, NY + 1) - 0.5) * 1.0 - LW[1] * 0.5
    U = np.zeros((4, NY, NX))
    U[3] = (y * SLOPE)[:, None] + 0.0 * x[None, :]
    U[0] = U[3]
    if method == "leapfrog_linear_plus_nonlinear_friction":
        # the example starts this solver close to the steady state
        U[0] = U[0] + 0.485
        U[2] = -0.9999
    U[3][:, 0] = WALL
    U[3][:, -1] = WALL
    U[3][-1, :] = WALL
    U[3][0, :] = WALL
    U[0] = np.maximum(U[0], U[3])
    if method == "leapfrog_linear_plus_nonlinear_friction":
        dry = U[0] < U[3] + 1.0e-3
        dry_n = np.zeros_like(dry)
        dry_n[:-1] = dry[1:]
        U[2][dry | dry_n] = 0.0
    return U


@pytest.mark.parametrize("method", ["rk2", "midpoint", "leapfrog_linear_plus_nonlinear_friction"])
def test_uniform_slope(method):
    kw = {}
    if method == "leapfrog_linear_plus_nonlinear_friction":
        kw["linear_solver_is_truely_linear"] = False
        ts, vd_tol = 0.02, 1.0e-4
    else:
        ts, vd_tol = 0.1, 1.0e-5
    d = Domain((NX, NY), LW, (0.0, 0.0), method, **kw)
    U = _initial(method)
    d.set_U(U)
    d.set_manning_squared(np.full((NY, NX), 0.03 ** 2))
    area = 1.0
    qin = Q * (LW[0] / NX)                     # inflow per cell (m^3/s)
    span = 1.0e6                               # a constant rate over [0, span]
    work = np.full((1, 1, NX - 2), qin / area * span)
    d.add_forcing_patch(2, NX - 1, NY - 1, NY - 1, 1, 1, 0.0, span, work)
    vol0 = float(np.sum(U[0] - U[3])) * area
    nsteps = int(round(600.0 / ts)) + 1
    d.evolve_steps(nsteps, ts)
    G = d.get_U()
    t = d.time
    assert t == pytest.approx(nsteps * ts, rel=1e-12)
    vol = float(np.sum(G[0] - G[3])) * area
    # the leapfrog applies forcing at the half step (over (t - dt/2, t + dt/2)),
    # so by time t it has added the inflow up to t - dt/2
    t_in = t - 0.5 * ts if method == "leapfrog_linear_plus_nonlinear_friction" else t
    vol_th = qin * t_in * (NX - 2) + vol0
    assert abs(vol_th - vol) < 1.0e-6 * vol_th, (vol, vol_th)
    i, j = NX // 2 - 1, NY // 2 - 1            # the example's cell (nx/2, ny/2), 1-based
    vd = -G[2][j, i]
    depth = G[0][j, i] - G[3][j, i]
    d_th = (0.03 ** 2 * Q ** 2 / SLOPE) ** 0.3
    assert abs(Q - vd) < vd_tol * Q, (vd, Q)
    assert abs(d_th - depth) < 1.0e-4 * d_th, (depth, d_th)
    d.close()
