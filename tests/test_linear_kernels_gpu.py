"""Every kernel of the plain linear leapfrog step against the oracle, bit for bit.

SWALS_LINEAR_KERNEL selects the step kernel of a plain linear domain
(domain_mod_linear_solver_include.f90:58-571): "tile" (shared-memory tiles),
"stream" (register-streaming warp strips), "async" (30-column strips through
per-lane cp.async), "wide8" / "wide16" (aligned 32-lane strips, 8- or 16-byte
lanes) and "bulk" (wide strips whose rows, halo granules included, arrive by
cp.async.bulk on a per-slot mbarrier).  Without it the grid size decides.
Each kernel runs here on widths that cut its strips every way -- narrower than
one strip, exactly one strip (FP64 wide strips are 64 columns, FP32 128),
ragged last strips -- and heights that leave short last segments, with land
cells, a sub-region, linear friction and msl_linear, gauges at the first and
last columns, and spherical coordinates with Coriolis; FP64 against the
IEEE-strict oracle and FP32 against its FP32 build.  STG, UH, VH, max_stage
and the gauge series must be equal bit for bit.
"""
import numpy as np
import pytest

from pairs import make_pair

pytestmark = pytest.mark.gpu

KERNELS = ["tile", "stream", "async", "wide8", "wide16", "bulk"]


def _basin(nx, ny, dx=1000.0, seed=3):
    """Rough seabed (-2000 m +- 850 m) with a dry strip on the west side and
    an island, a Gaussian hump off centre, gauges at the corners, the hump
    and the last column."""
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    X, Y = np.meshgrid(x, y)
    elv = -2000.0 + 800.0 * np.sin(X / (7.3 * dx)) * np.cos(Y / (5.1 * dx)) + rng.uniform(-50.0, 50.0, (ny, nx))
    elv[:, :3] = 30.0
    elv[(X - 0.3 * nx * dx) ** 2 + (Y - 0.7 * ny * dx) ** 2 < (3.0 * dx) ** 2] = 15.0
    U = np.zeros((4, ny, nx))
    U[3] = elv
    cx, cy, sig = 0.6 * nx * dx, 0.45 * ny * dx, 4.0 * dx
    U[0] = np.maximum(np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2.0 * sig ** 2)), elv)
    kw = dict(nx=(nx, ny), lw=(nx * dx, ny * dx), lower_left=(0.0, 0.0), timestepping_method="linear")
    gauges = np.array([[0.5 * dx, 0.5 * dx], [(nx - 0.5) * dx, (ny - 0.5) * dx], [cx, cy],
                       [(nx - 0.5) * dx, 0.5 * ny * dx], [(nx - 1.5) * dx, 1.5 * dx]])
    return kw, U, gauges


def _run_exact(kw, U, gauges, nsteps, real32, tag):
    g, o = make_pair(kw, U, real32=real32, oracle_real32=real32)
    dt = 0.8 * o.linear_timestep_max()
    g.gauges_setup(gauges, capacity=nsteps)
    site = g.gauges_site_index() - 1
    og = []
    for _ in range(nsteps):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
        og.append(np.stack([o.U[k][site[:, 1], site[:, 0]] for k in range(3)], axis=1))
    g.synchronize()
    Ug = g.get_U()
    for k, name in enumerate(("STG", "UH", "VH")):
        np.testing.assert_array_equal(Ug[k], o.U[k], err_msg=f"{tag} {name}")
    np.testing.assert_array_equal(g.max_stage(), o.max_stage, err_msg=f"{tag} max_stage")
    np.testing.assert_array_equal(g.gauges_read(), np.stack(og), err_msg=f"{tag} gauges")
    assert np.any(Ug[1] != 0) and np.any(Ug[2] != 0)
    g.close()


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("real32", [False, True])
@pytest.mark.parametrize("shape", [(40, 33), (64, 50), (128, 21), (197, 83), (260, 129)])
def test_kernel_matches_oracle(kernel, real32, shape, monkeypatch):
    monkeypatch.setenv("SWALS_LINEAR_KERNEL", kernel)
    kw, U, gauges = _basin(*shape)
    _run_exact(kw, U, gauges, 60, real32, f"{kernel} {shape} real32={real32}")


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("truely_linear", [True, False])
def test_kernel_subregion_friction_msl(kernel, truely_linear, monkeypatch):
    """xL..yU restrict the update, linear friction scales the momenta and a
    nonzero msl_linear moves the truly linear depth."""
    monkeypatch.setenv("SWALS_LINEAR_KERNEL", kernel)
    kw, U, gauges = _basin(197, 83, seed=4)
    kw.update(linear_friction_coeff=1.0e-4, xL=3, xU=190, yL=5, yU=80, msl_linear=0.5,
              linear_solver_is_truely_linear=truely_linear)
    U = U.copy()
    U[0] = np.maximum(U[0] + 0.5, U[3])
    _run_exact(kw, U, gauges, 50, False, f"{kernel} subregion tl={truely_linear}")


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("real32", [False, True])
def test_kernel_spherical_coriolis(kernel, real32, monkeypatch):
    from ptha_b200 import workloads
    monkeypatch.setenv("SWALS_LINEAR_KERNEL", kernel)
    kw, U = workloads.spherical_patch(nx=130, ny=61)
    kw.update(timestepping_method="linear", linear_solver_is_truely_linear=False, coriolis=True)
    lw, ll = kw["lw"], kw.get("lower_left", (0.0, 0.0))
    gauges = np.array([[ll[0] + 0.5 * lw[0], ll[1] + 0.5 * lw[1]], [ll[0] + 0.99 * lw[0], ll[1] + 0.01 * lw[1]]])
    _run_exact(kw, U, gauges, 60, real32, f"{kernel} spherical coriolis real32={real32}")
