"""Parity of the CUDA linear leapfrog (domain_mod_linear_solver_include.f90)
with the IEEE-strict oracle on the same seeded inputs, through the C ABI.

Tolerance: 1e-12 relative for FP64 (the kernel is compiled without FMA
contraction and follows the reference's operation order, so results are
expected to be bit-identical; the tolerance leaves room for nothing more
than last-bit differences).  FP32 state: 2e-4 relative to the FP64 oracle."""
import numpy as np
import pytest

from ptha_b200 import workloads
from pairs import make_pair, rel_err, report

TOL64 = 1e-12


def _run(kw, U, nsteps, dt=None, gauges=None, real32=False):
    g, o = make_pair(kw, U, real32=real32)
    if dt is None:
        dt = o.linear_timestep_max()
        gdt = g.linear_timestep_max()
        assert gdt == pytest.approx(dt, rel=1e-6 if real32 else 1e-15)
    if gauges is not None:
        g.gauges_setup(gauges, capacity=nsteps)
    og = []
    for _ in range(nsteps):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
        if gauges is not None:
            site = g.gauges_site_index() - 1
            og.append(np.stack([o.U[k][site[:, 1], site[:, 0]] for k in range(3)], axis=1))
    return g, o, og, dt


@pytest.mark.gpu
def test_linear_config1_full_size_parity():
    """Plain linear leapfrog 400x400, dx=1 km, 4000 m, Gaussian hump, walls,
    cfl 0.7, 2000 steps, 9 gauges: FP64 parity of STG/UH/VH, max_stage and the
    gauge series."""
    kw, U, gauges = workloads.linear_gaussian_basin()
    g, o, og, dt = _run(kw, U, 2000, gauges=gauges)
    Ug, errs = report("config1", g, o)
    for k in ("STG", "UH", "VH"):
        assert errs[k] <= TOL64, errs
    assert rel_err(g.max_stage(), o.max_stage) <= TOL64
    series = g.gauges_read()
    assert series.shape == (2000, 9, 3)
    assert rel_err(series, np.stack(og)) <= TOL64
    st = g.state()
    assert st.time == pytest.approx(o.time, rel=1e-15)
    assert st.nsteps_advanced == 2000
    # mass: the closed basin conserves volume to round-off
    assert g.volume_interior() == pytest.approx(o.volume_interior(), rel=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("truely_linear", [True, False])
@pytest.mark.parametrize("coriolis", [True, False])
def test_linear_spherical(truely_linear, coriolis):
    kw, U = workloads.spherical_patch()
    kw.update(timestepping_method="linear", linear_solver_is_truely_linear=truely_linear, coriolis=coriolis)
    g, o, _, dt = _run(kw, U, 150)
    _, errs = report(f"sph tl={truely_linear} cor={coriolis}", g, o)
    for k in ("STG", "UH", "VH"):
        assert errs[k] <= TOL64, errs
    assert rel_err(g.max_stage(), o.max_stage) <= TOL64


@pytest.mark.gpu
def test_linear_friction_and_subregion_and_odd_sizes():
    # odd sizes exercise partial tiles; xL..yU restrict the update region
    kw, U, _ = workloads.linear_gaussian_basin(n=97, dx=2000.0)
    kw.update(linear_friction_coeff=1.0e-4, xL=3, xU=90, yL=5, yU=93, msl_linear=0.5)
    U = U.copy()
    U[0] += 0.5
    g, o, _, dt = _run(kw, U, 120)
    _, errs = report("friction+subregion", g, o)
    for k in ("STG", "UH", "VH"):
        assert errs[k] <= TOL64, errs


@pytest.mark.gpu
def test_linear_stage_boundary_function():
    # boundary_stage_transmissive_normal_momentum on a staggered grid: stage
    # and elevation of the ring come from the boundary function at t+dt/2
    from ptha_b200 import _lib
    n = 80
    kw, U, _ = workloads.linear_gaussian_basin(n=n, dx=500.0, depth=50.0, wall_cells=0)
    kw.update(boundary_kind=_lib.BC_STAGE_TRANSMISSIVE_NORMAL_MOMENTUM,
              boundary_function_kind=_lib.BF_SOLITARY_WEST_WALLS,
              boundary_function_params=(2.0, 50.0, -3000.0), boundary_exterior=(True, False, True, True))
    g, o, _, dt = _run(kw, U, 100)
    _, errs = report("linear stage bc", g, o)
    # the boundary function uses cosh: libm and CUDA may differ in the last bit
    for k in ("STG", "UH", "VH", "ELV"):
        assert errs[k] <= 1e-10, errs


@pytest.mark.gpu
def test_linear_fp32_against_fp64_oracle():
    kw, U, _ = workloads.linear_gaussian_basin(n=128, dx=1000.0)
    g, o = make_pair(kw, U, real32=True)
    dt = o.linear_timestep_max()
    for _ in range(300):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    Ug = g.get_U()
    # FP32 state vs FP64 oracle; stated tolerance relative to the field maximum
    assert rel_err(Ug[0], o.U[0]) <= 2e-4
    assert rel_err(Ug[1], o.U[1]) <= 2e-4
    assert rel_err(Ug[2], o.U[2]) <= 2e-4


@pytest.mark.gpu
def test_linear_requires_timestep():
    from ptha_b200 import SwalsError
    kw, U, _ = workloads.linear_gaussian_basin(n=32)
    g, _ = make_pair(kw, U)
    with pytest.raises(SwalsError) as e:
        g.evolve_one_step()
    assert e.value.code == 7
