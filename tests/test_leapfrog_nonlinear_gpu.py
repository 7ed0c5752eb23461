"""'leapfrog_nonlinear' (domain_mod_leapfrog_nonlinear_include.f90) on the
GPU against the oracle, bit for bit: a walled basin (mass conserved), a
wet/dry beach with the solitary-wave stage boundary, a spherical patch with
Coriolis and land, Chezy and linear friction, a forcing patch with CUDA-graph
replay, and a nest with an rk2 child."""
import numpy as np
import pytest

from ptha_b200 import workloads
from pairs import make_pair, rel_err, report, water_mask

pytestmark = pytest.mark.gpu
M = "leapfrog_nonlinear"


def _exact(g, o, tag):
    _, errs = report(tag, g, o)
    for k in ("STG", "UH", "VH", "ELV"):
        assert errs[k + "_exact"] == 1.0, errs


def test_basin_mass_and_parity():
    kw, U, _ = workloads.linear_gaussian_basin(n=100, dx=1000.0)
    kw = dict(kw, timestepping_method=M)
    g, o = make_pair(kw, U)
    dt = 0.5 * o.linear_timestep_max()
    v0 = o.volume_interior()
    for _ in range(200):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _exact(g, o, "nl basin")
    assert rel_err(g.max_stage(), o.max_stage) == 0.0
    assert g.volume_interior() == pytest.approx(v0, rel=1e-13)
    assert g.state().time == pytest.approx(o.time, rel=1e-14)


def test_beach_wet_dry():
    kw, U, _, nsq = workloads.rk2_beach(n=96, dx=10.0 * 2048 / 96, toe=17580.0 * 96 / 2048)
    kw = dict(kw, timestepping_method=M)
    g, o = make_pair(kw, U, manning_sq=nsq)
    dt = 0.25 * o.linear_timestep_max()
    for _ in range(500):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _exact(g, o, "nl beach")
    assert rel_err(g.max_stage(), o.max_stage, mask=water_mask(o.U[3])) == 0.0
    wet = (o.U[0] - o.U[3]) > 1e-5
    assert np.any(wet & ((U[0] - U[3]) <= 1e-5)), "the front never moved"


@pytest.mark.parametrize("friction", ["manning", "chezy"])
def test_spherical_coriolis(friction):
    kw, U = workloads.spherical_patch(nx=100, ny=70)
    kw = dict(kw, timestepping_method=M, coriolis=True, friction_type=friction, linear_friction_coeff=1.0e-5)
    U = U.copy()
    U[0] = np.where(U[3] > 0, U[3], U[0])
    nsq = np.full(U[0].shape, 0.025 ** 2 if friction == "manning" else 1.0 / 60.0 ** 2)
    g, o = make_pair(kw, U, manning_sq=nsq)
    dt = 0.5 * o.linear_timestep_max()
    for _ in range(150):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _exact(g, o, f"nl spherical {friction}")


def test_forcing_and_graph():
    kw, U, _ = workloads.linear_gaussian_basin(n=90, dx=1000.0, depth=50.0)
    kw = dict(kw, timestepping_method=M)
    U = U.copy()
    U[0] = np.where(U[3] > 0, U[3], 0.0)
    g, o = make_pair(kw, U)
    b, _ = make_pair(kw, U)
    ii, jj = np.arange(30, 61), np.arange(25, 56)
    S = 0.5 * np.sin(np.pi * (jj - 29.5) / 31)[:, None] * np.sin(np.pi * (ii - 29.5) / 31)[None, :]
    for dom in (g, o, b):
        dom.add_forcing_patch(30, 60, 25, 55, 1, 1, 5.0, 120.0, S[None])
    dt = 0.5 * o.linear_timestep_max()
    for _ in range(60):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    b.evolve_steps(60, dt)
    _exact(g, o, "nl forcing")
    np.testing.assert_array_equal(b.get_U(), g.get_U())


def test_nest_with_rk2_child():
    """A 'leapfrog_nonlinear' parent (halo 3) around a ratio-3 'rk2' child:
    every domain and every flux-correction error equal the oracle's after
    each multidomain step."""
    from nest_cases import two_level_nest
    from test_nesting_gpu import _run_pair
    specs = two_level_nest(ratio=3, child_method="rk2", parent_method=M)
    md, omd = _run_pair(specs, wetdry=False, nsteps=6)
    assert md.time == pytest.approx(omd.time)
    md.close()


def test_flather_open_basin():
    """flather_boundary through update_boundary after the stage sweep
    (domain_mod_leapfrog_nonlinear_include.f90:122-140): an open basin with
    a beach on the north edge (some ring cells dry), at half the CFL limit."""
    from test_flather_gpu import open_basin
    kw, U = open_basin(n=90, dx=1000.0, depth=200.0, method=M)
    g, o = make_pair(kw, U, manning_sq=np.full(U[0].shape, 0.025 ** 2))
    dt = 0.5 * o.linear_timestep_max()
    for _ in range(150):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _exact(g, o, "nl flather")


def test_flather_solitary_west():
    """Flather on the west edge with the solitary wave as the outside state."""
    from ptha_b200 import _lib
    kw, U, _, nsq = workloads.rk2_beach(n=96, dx=10.0 * 2048 / 96, toe=17580.0 * 96 / 2048)
    kw = dict(kw, timestepping_method=M, boundary_kind=_lib.BC_FLATHER, boundary_exterior=(False, False, False, True))
    g, o = make_pair(kw, U, manning_sq=nsq)
    dt = 0.25 * o.linear_timestep_max()
    for _ in range(400):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _exact(g, o, "nl flather solitary")
    wet = o.U[3][1:-1, 1:20] < -5.0
    assert np.max(o.U[0][1:-1, 1:20][wet]) > 0.02   # the wave came in
