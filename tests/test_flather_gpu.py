"""flather_boundary (boundary_mod.f90:502-730) on the GPU against the oracle.

* finite volume ('rk2', 'euler'): the boundary kernel applies it after each
  stage (west/east pass, then south/north pass, corners from the second);
* staggered linear leapfrog ('linear', truly and not truly linear, with and
  without Coriolis): the ring values from the swept stage and old momenta,
  then the momentum update of the outer two rings with the boundary's
  momenta -- under each step kernel (tile, stream, async);
* the 'outside' state at rest (no boundary function) and from the solitary
  wave boundary function on the west edge.

FP64 states are compared bit for bit.  A property check: a hump radiates out
of a Flather basin, but stays in a walled one."""
import numpy as np
import pytest

from ptha_b200 import _lib, workloads
from pairs import make_pair, report

pytestmark = pytest.mark.gpu


def open_basin(n=96, dx=200.0, depth=20.0, method="rk2", shelf=True):
    """Flat basin with a Gaussian hump; with `shelf`, a beach rising above
    sea level along the north edge so some ring cells are dry."""
    lw = n * dx
    x = workloads.cell_centres(n, lw, 0.0)
    X, Y = np.meshgrid(x, x)
    U = np.zeros((4, n, n))
    elv = np.full((n, n), -depth)
    if shelf:
        elv = np.minimum(-depth + np.maximum(Y - 0.7 * lw, 0.0) * (2.0 * depth / (0.3 * lw)), 3.0)
    U[3] = elv
    U[0] = np.maximum(elv, 0.5 * np.exp(-((X - 0.4 * lw) ** 2 + (Y - 0.45 * lw) ** 2) / (2 * (6 * dx) ** 2)))
    kw = dict(nx=(n, n), lw=(lw, lw), lower_left=(0.0, 0.0), timestepping_method=method,
              boundary_kind=_lib.BC_FLATHER, boundary_function_kind=0)
    return kw, U


def _exact(g, o, tag):
    _, errs = report(tag, g, o)
    for k in ("STG", "UH", "VH", "ELV"):
        assert errs[k + "_exact"] == 1.0, errs


@pytest.mark.parametrize("method", ["rk2", "euler"])
def test_fv_flather_matches_oracle(method):
    kw, U = open_basin(method=method)
    g, o = make_pair(kw, U, manning_sq=np.full(U[0].shape, 0.025 ** 2))
    for _ in range(250):
        g.evolve_one_step()
        o.evolve_one_step()
    _exact(g, o, f"{method} flather")
    assert g.state().time == pytest.approx(o.time, rel=1e-13)


def test_rk2_flather_solitary_inflow_west():
    """Flather on the west edge only, with the solitary wave as the outside
    state; walls elsewhere by elevation."""
    kw, U, _, nsq = workloads.rk2_beach(n=96, dx=10.0 * 2048 / 96, toe=17580.0 * 96 / 2048)
    kw = dict(kw)
    kw.update(boundary_kind=_lib.BC_FLATHER, boundary_exterior=(False, False, False, True))
    g, o = make_pair(kw, U, manning_sq=nsq)
    for _ in range(300):
        g.evolve_one_step()
        o.evolve_one_step()
    _exact(g, o, "rk2 flather solitary")
    assert np.max(o.U[0][1:-1, 1:20]) > 0.05   # the wave came in


@pytest.mark.parametrize("kernel", ["tile", "stream", "async"])
@pytest.mark.parametrize("truely_linear", [True, False])
def test_linear_flather_matches_oracle(kernel, truely_linear, monkeypatch):
    monkeypatch.setenv("SWALS_LINEAR_KERNEL", kernel)
    kw, U = open_basin(n=90, dx=1000.0, depth=200.0, method="linear")
    kw["linear_solver_is_truely_linear"] = truely_linear
    kw["nx"] = (90, 70)
    kw["lw"] = (90 * 1000.0, 70 * 1000.0)
    U = U[:, :70, :].copy()
    g, o = make_pair(kw, U)
    dt = 0.7 * o.linear_timestep_max()
    for _ in range(150):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _exact(g, o, f"linear flather {kernel} tl={truely_linear}")
    assert g.volume_interior() == pytest.approx(o.volume_interior(), rel=1e-13)


@pytest.mark.parametrize("kernel", ["tile", "async"])
def test_linear_flather_spherical_coriolis(kernel, monkeypatch):
    monkeypatch.setenv("SWALS_LINEAR_KERNEL", kernel)
    kw, U = workloads.spherical_patch(nx=100, ny=70)
    U = U.copy()
    # open the ring: ocean to the boundary on all sides
    for e in (U[3][:2, :], U[3][-2:, :], U[3][:, :2], U[3][:, -2:]):
        e[...] = -3000.0
    U[0] = np.where(U[3] > 0, U[3], U[0])
    kw = dict(kw)
    kw.update(timestepping_method="linear", coriolis=True, boundary_kind=_lib.BC_FLATHER)
    g, o = make_pair(kw, U)
    dt = o.linear_timestep_max()
    for _ in range(200):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _exact(g, o, f"linear flather spherical coriolis {kernel}")


@pytest.mark.parametrize("method", ["rk2", "linear"])
def test_flather_lets_the_wave_out(method):
    """Energy leaves through Flather boundaries; walls keep it in.  (The
    staggered solver runs at half its CFL limit: with Flather at the full
    limit this basin grows unstable, in the oracle exactly as on the GPU.)"""
    kept = {}
    for bc in (_lib.BC_FLATHER, _lib.BC_NONE):
        kw, U = open_basin(n=80, dx=1000.0, depth=200.0, method=method, shelf=False)
        kw["boundary_kind"] = bc
        if bc == _lib.BC_NONE:
            for e in (U[3][:1, :], U[3][-1:, :], U[3][:, :1], U[3][:, -1:]):
                e[...] = 100.0
            U[0] = np.maximum(U[0], U[3])
        g, o = make_pair(kw, U)
        dt = 0.5 * o.linear_timestep_max() if method == "linear" else None
        for _ in range(300):
            g.evolve_one_step(dt)
        s = g.compute_domain_statistics()
        kept[bc] = s["energy_kinetic_on_rho"]
    assert np.isfinite(kept[_lib.BC_FLATHER])
    assert kept[_lib.BC_FLATHER] < 0.01 * kept[_lib.BC_NONE]
