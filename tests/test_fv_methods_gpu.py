"""The other finite-volume time steppers on the GPU against the oracle:
one_midpoint_step and one_rk2n_step (timestepping_alternatives_include.f90:
149-337), on the same stage kernels as 'rk2'.

Adaptive and fixed timesteps, the solitary-wave beach (stage boundary) and an
open basin (Flather); FP64 states, max_stage, time, max_dt and the boundary
flux integrals are compared with the oracle, the states bit for bit."""
import numpy as np
import pytest

from ptha_b200 import workloads
from pairs import make_pair, report, rel_err, water_mask
from test_flather_gpu import open_basin

pytestmark = pytest.mark.gpu


def _check(g, o, tag):
    _, errs = report(tag, g, o)
    for k in ("STG", "UH", "VH", "ELV"):
        assert errs[k + "_exact"] == 1.0, errs
    m = water_mask(o.U[3])
    assert rel_err(g.max_stage(), o.max_stage, mask=m) == 0.0
    st = g.state()
    assert st.time == pytest.approx(o.time, rel=1e-13)
    assert st.max_dt == pytest.approx(o.max_dt, rel=1e-10)
    assert st.negative_depth_fix_counter == o.negative_depth_fix_counter
    assert st.nsteps_advanced == o.nsteps_advanced
    assert st.boundary_flux_time_integral == pytest.approx(o.c.boundary_flux_time_integral, rel=1e-9, abs=1e-6)


@pytest.mark.parametrize("method", ["midpoint", "rk2n"])
@pytest.mark.parametrize("adaptive", [True, False])
def test_beach(method, adaptive):
    kw, U, _, nsq = workloads.rk2_beach(n=96, dx=10.0 * 2048 / 96, toe=17580.0 * 96 / 2048)
    kw = dict(kw)
    kw["timestepping_method"] = method
    g, o = make_pair(kw, U, manning_sq=nsq)
    dt = None
    if not adaptive:
        dt = g.stationary_timestep_max() * 0.9
        assert dt == pytest.approx(o.nonlinear_stationary_timestep_max() * 0.5 * (4.0 if method == "rk2n" else 1.0)
                                   * 0.9, rel=1e-14)
    for _ in range(250):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _check(g, o, f"{method} beach adaptive={adaptive}")


@pytest.mark.parametrize("method", ["midpoint", "rk2n"])
def test_open_basin_flather(method):
    kw, U = open_basin(method=method)
    g, o = make_pair(kw, U, manning_sq=np.full(U[0].shape, 0.025 ** 2))
    for _ in range(120):
        g.evolve_one_step()
        o.evolve_one_step()
    _check(g, o, f"{method} flather")


def test_graph_replay_rk2n():
    """evolve_steps (CUDA-graph replay) gives the steps issued one by one."""
    kw, U, _, nsq = workloads.rk2_beach(n=64, dx=10.0 * 2048 / 64, toe=17580.0 * 64 / 2048)
    kw = dict(kw)
    kw["timestepping_method"] = "rk2n"
    a, _ = make_pair(kw, U, manning_sq=nsq)
    b, _ = make_pair(kw, U, manning_sq=nsq)
    for _ in range(13):
        a.evolve_one_step()
    b.evolve_steps(13)
    np.testing.assert_array_equal(a.get_U(), b.get_U())
    assert a.state().time == b.state().time


@pytest.mark.parametrize("flux", ["DE1", "DE1_upwind_transverse", "DE1_low_fr_diffusion_upwind_transverse"])
def test_compute_fluxes_inner_methods(flux):
    """The other DE1 flux variants (compute_fluxes_alternatives_include.f90:
    11-64): plain HLL momentum diffusion, and/or upwind transverse momentum."""
    kw, U, _, nsq = workloads.rk2_beach(n=96, dx=10.0 * 2048 / 96, toe=17580.0 * 96 / 2048)
    kw = dict(kw)
    kw["compute_fluxes_inner_method"] = flux
    g, o = make_pair(kw, U, manning_sq=nsq)
    for _ in range(250):
        g.evolve_one_step()
        o.evolve_one_step()
    _check(g, o, f"rk2 {flux}")


@pytest.mark.parametrize("flux", ["DE1_upwind_transverse", "DE1_low_fr_diffusion_upwind_transverse"])
def test_upwind_transverse_spherical_coriolis(flux):
    kw, U = workloads.spherical_patch(nx=100, ny=70)
    kw = dict(kw)
    kw.update(timestepping_method="rk2", coriolis=True, compute_fluxes_inner_method=flux)
    U = U.copy()
    U[0] = np.where(U[3] > 0, U[3], U[0])
    g, o = make_pair(kw, U, manning_sq=np.full(U[0].shape, 0.025 ** 2))
    for _ in range(100):
        g.evolve_one_step()
        o.evolve_one_step()
    _, errs = report(f"rk2 sph cor {flux}", g, o)
    for k in ("STG", "UH", "VH"):
        assert errs[k + "_exact"] == 1.0, errs
