"""'leapfrog_linear_plus_nonlinear_friction' (the linear leapfrog with
semi-implicit Manning/Chezy friction, linear_solver_include.f90:441-505 and
the friction work :590-618) on the GPU against the oracle, bit for bit:
truely and not truely linear, Cartesian and spherical with Coriolis, with
linear friction folded in, with a Flather boundary, under each step kernel."""
import numpy as np
import pytest

from ptha_b200 import _lib, workloads
from pairs import make_pair, report
from test_flather_gpu import open_basin

pytestmark = pytest.mark.gpu
METHOD = "leapfrog_linear_plus_nonlinear_friction"


def _exact(g, o, tag):
    _, errs = report(tag, g, o)
    for k in ("STG", "UH", "VH"):
        assert errs[k + "_exact"] == 1.0, errs


def _nsq(shape, seed=1):
    rng = np.random.default_rng(seed)
    return (0.02 + 0.02 * rng.random(shape)) ** 2


@pytest.mark.parametrize("kernel", ["tile", "stream", "async"])
@pytest.mark.parametrize("truely_linear", [True, False])
def test_basin(kernel, truely_linear, monkeypatch):
    """A shallow basin (20 m) where friction matters, a beach on the north
    side (dry cells), walls by elevation on the other sides."""
    monkeypatch.setenv("SWALS_LINEAR_KERNEL", kernel)
    kw, U = open_basin(n=90, dx=500.0, depth=20.0, method=METHOD)
    kw["boundary_kind"] = _lib.BC_NONE
    kw["linear_solver_is_truely_linear"] = truely_linear
    U = U.copy()
    U[3][:, :1] = 50.0
    U[3][:, -1:] = 50.0
    U[3][:1, :] = 50.0
    U[0] = np.maximum(U[0], U[3])
    g, o = make_pair(kw, U, manning_sq=_nsq(U[0].shape))
    dt = 0.5 * o.linear_timestep_max()
    for _ in range(200):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _exact(g, o, f"nlfric {kernel} tl={truely_linear}")
    # friction takes energy out: compare with the frictionless solver
    kw2 = dict(kw, timestepping_method="linear")
    g2, _ = make_pair(kw2, U)
    for _ in range(200):
        g2.evolve_one_step(dt)
    assert g.compute_domain_statistics()["energy_kinetic_on_rho"] < \
        0.97 * g2.compute_domain_statistics()["energy_kinetic_on_rho"]


@pytest.mark.parametrize("friction", ["manning", "chezy"])
def test_spherical_coriolis_linear_friction(friction):
    kw, U = workloads.spherical_patch(nx=100, ny=70)
    kw = dict(kw)
    kw.update(timestepping_method=METHOD, coriolis=True, linear_friction_coeff=1.0e-5, friction_type=friction)
    U = U.copy()
    U[0] = np.where(U[3] > 0, U[3], U[0])
    nsq = _nsq(U[0].shape, 2) if friction == "manning" else np.full(U[0].shape, 1.0 / 60.0 ** 2)
    g, o = make_pair(kw, U, manning_sq=nsq)
    dt = o.linear_timestep_max()
    for _ in range(150):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _exact(g, o, f"nlfric sph cor {friction}")


@pytest.mark.parametrize("truely_linear", [True, False])
def test_flather_and_graph_replay(truely_linear):
    kw, U = open_basin(n=80, dx=1000.0, depth=50.0, method=METHOD)
    kw["linear_solver_is_truely_linear"] = truely_linear
    nsq = _nsq(U[0].shape, 3)
    g, o = make_pair(kw, U, manning_sq=nsq)
    b, _ = make_pair(kw, U, manning_sq=nsq)
    dt = 0.5 * o.linear_timestep_max()
    for _ in range(120):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    b.evolve_steps(120, dt)
    _exact(g, o, f"nlfric flather tl={truely_linear}")
    np.testing.assert_array_equal(b.get_U(), g.get_U())
