"""Eddy viscosity (the *_eddyvisc flux variants, compute_fluxes_DE1_inner_
include.f90:130-156, 289-358, 551-620, and get_eddy_viscosity, :864-1017) on
the GPU against the oracle, bit for bit.

* constant viscosity (eddy_visc_constants(2) = 0) and constant +
  Shiono-Knight, on the wet/dry solitary-wave beach with Manning friction;
* every finite-volume stepper ('rk2', 'midpoint', 'rk2n', 'euler'), adaptive
  and fixed steps (the clip uses the dt of the previous update_U);
* the upwind-transverse flux variants on a spherical patch with Coriolis;
* a CUDA-graph replay equals the steps issued one by one;
* a solver without eddy viscosity support refuses it."""
import numpy as np
import pytest

from ptha_b200 import Domain, _lib, workloads
from pairs import make_pair, report, rel_err, water_mask

pytestmark = pytest.mark.gpu


def _beach(n=96, method="rk2", flux=None):
    kw, U, _, nsq = workloads.rk2_beach(n=n, dx=10.0 * 2048 / n, toe=17580.0 * n / 2048)
    kw = dict(kw, timestepping_method=method)
    if flux:
        kw["compute_fluxes_inner_method"] = flux
    return kw, U, nsq


def _check(g, o, tag):
    _, errs = report(tag, g, o)
    for k in ("STG", "UH", "VH", "ELV"):
        assert errs[k + "_exact"] == 1.0, errs
    assert rel_err(g.max_stage(), o.max_stage, mask=water_mask(o.U[3])) == 0.0
    st = g.state()
    assert st.time == pytest.approx(o.time, rel=1e-13)
    assert st.negative_depth_fix_counter == o.negative_depth_fix_counter


@pytest.mark.parametrize("consts", [(0.5, 0.0), (0.0, 2.0), (0.1, 1.0)])
def test_rk2_beach(consts):
    kw, U, nsq = _beach()
    g, o = make_pair(kw, U, manning_sq=nsq)
    g.set_eddy_viscosity(*consts)
    o.set_eddy_viscosity(*consts)
    for _ in range(250):
        g.evolve_one_step()
        o.evolve_one_step()
    _check(g, o, f"rk2 eddy {consts}")
    assert float(o.eddy_visc.max()) > 0.0


@pytest.mark.parametrize("method", ["midpoint", "rk2n", "euler"])
@pytest.mark.parametrize("adaptive", [True, False])
def test_other_steppers(method, adaptive):
    kw, U, nsq = _beach(n=80, method=method)
    g, o = make_pair(kw, U, manning_sq=nsq)
    for d in (g, o):
        d.set_eddy_viscosity(0.05, 1.5)
    dt = None
    if not adaptive:
        dt = 0.5 * o.nonlinear_stationary_timestep_max() * (4.0 if method == "rk2n" else 1.0)
    for _ in range(150):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _check(g, o, f"{method} eddy adaptive={adaptive}")


@pytest.mark.parametrize("flux", ["DE1", "DE1_upwind_transverse", "DE1_low_fr_diffusion_upwind_transverse"])
def test_flux_variants_spherical_coriolis(flux):
    kw, U = workloads.spherical_patch(nx=100, ny=70)
    kw = dict(kw, timestepping_method="rk2", coriolis=True, compute_fluxes_inner_method=flux)
    U = U.copy()
    U[0] = np.where(U[3] > 0, U[3], U[0] + 0.3 * np.exp(-np.linspace(-3, 3, 100)[None, :] ** 2))
    g, o = make_pair(kw, U, manning_sq=np.full(U[0].shape, 0.025 ** 2))
    for d in (g, o):
        d.set_eddy_viscosity(1.0, 1.0)
    for _ in range(100):
        g.evolve_one_step()
        o.evolve_one_step()
    _, errs = report(f"rk2 sph cor eddy {flux}", g, o)
    for k in ("STG", "UH", "VH"):
        assert errs[k + "_exact"] == 1.0, errs


def test_graph_replay_and_off_switch():
    kw, U, nsq = _beach(n=64)
    a, o = make_pair(kw, U, manning_sq=nsq)
    b, _ = make_pair(kw, U, manning_sq=nsq)
    for d in (a, b, o):
        d.set_eddy_viscosity(0.2, 1.0)
    for _ in range(20):
        a.evolve_one_step()
        o.evolve_one_step()
    b.evolve_steps(20)
    np.testing.assert_array_equal(a.get_U(), b.get_U())
    _check(a, o, "rk2 eddy graph")
    # switched off, the default fluxes again
    a.clear_eddy_viscosity()
    o.c.use_eddy_viscosity = 0
    for _ in range(10):
        a.evolve_one_step()
        o.evolve_one_step()
    _check(a, o, "rk2 eddy off")


def test_unsupported_method():
    d = Domain((40, 40), (40.0, 40.0), (0.0, 0.0), "linear")
    with pytest.raises(_lib.SwalsError) as e:
        d.set_eddy_viscosity(1.0)
    assert e.value.code == 3
    d.close()
