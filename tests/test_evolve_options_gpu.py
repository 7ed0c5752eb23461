"""evolve_one_step's own options (domain_mod.f90:1679-1813) on the GPU
against the oracle: static_before_time (steps that start before it only
advance the clock) and max_U_update_frequency (max_stage updated after every
n-th step), for the finite-volume and the leapfrog solvers, stepped one by
one and through evolve_steps."""
import numpy as np
import pytest

from ptha_b200 import workloads
from pairs import make_pair, report, water_mask

pytestmark = pytest.mark.gpu


def _exact(g, o, tag):
    _, errs = report(tag, g, o)
    for k in ("STG", "UH", "VH", "ELV"):
        assert errs[k + "_exact"] == 1.0, errs


def _beach(method):
    kw, U, _, nsq = workloads.rk2_beach(n=80, dx=10.0 * 2048 / 80, toe=17580.0 * 80 / 2048)
    return dict(kw, timestepping_method=method), U, nsq


@pytest.mark.parametrize("method", ["rk2", "linear", "leapfrog_nonlinear"])
@pytest.mark.parametrize("graph", [False, True])
def test_static_before_time(method, graph):
    kw, U, nsq = _beach(method)
    g, o = make_pair(kw, U, manning_sq=nsq)
    dt = 0.25 * o.linear_timestep_max() if method != "rk2" else 0.5 * o.nonlinear_stationary_timestep_max()
    t_static = 10.5 * dt
    g.set_static_before_time(t_static)
    o.c.static_before_time = t_static
    n = 40
    if graph:
        g.evolve_steps(n, dt)
    else:
        for _ in range(n):
            g.evolve_one_step(dt)
    for _ in range(n):
        o.evolve_one_step(dt)
    _exact(g, o, f"{method} static graph={graph}")
    st = g.state()
    assert st.time == pytest.approx(o.time, rel=1e-14) and st.nsteps_advanced == o.nsteps_advanced == n
    np.testing.assert_array_equal(g.max_stage()[water_mask(o.U[3])], o.max_stage[water_mask(o.U[3])])
    # the first 11 steps were static: the state moved only after them
    assert o.time == pytest.approx(n * dt)


@pytest.mark.parametrize("method", ["rk2", "midpoint", "linear", "leapfrog_linear_plus_nonlinear_friction"])
def test_max_U_update_frequency(method):
    kw, U, nsq = _beach(method)
    g, o = make_pair(kw, U, manning_sq=nsq)
    b, _ = make_pair(kw, U, manning_sq=nsq)
    dt = 0.25 * o.linear_timestep_max() if method not in ("rk2", "midpoint") \
        else 0.5 * o.nonlinear_stationary_timestep_max()
    for d in (g, b):
        d.set_max_U_update_frequency(3)
    o.c.max_U_update_frequency = 3
    for _ in range(37):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    b.evolve_steps(37, dt)
    _exact(g, o, f"{method} max_U every 3")
    m = water_mask(o.U[3])
    np.testing.assert_array_equal(g.max_stage()[m], o.max_stage[m])
    np.testing.assert_array_equal(b.max_stage()[m], o.max_stage[m])
    np.testing.assert_array_equal(b.get_U(), g.get_U())


MAX_U = ("time_of_max_stage", "max_speed", "max_flux", "arrival_time", "min_stage")


@pytest.mark.parametrize("method,include_dry,every", [
    ("rk2", True, 1), ("rk2", False, 2), ("linear", True, 1), ("leapfrog_nonlinear", False, 1),
    ("leapfrog_linear_plus_nonlinear_friction", True, 3)])
def test_max_U_variables(method, include_dry, every):
    """The optional max_U_variables (time_of_max_stage, max_speed, max_flux,
    arrival_time, min_stage; domain_mod.f90:2243-2404) and
    stage_extrema_include_dry_cells, stepped and through evolve_steps."""
    kw, U, nsq = _beach(method)
    g, o = make_pair(kw, U, manning_sq=nsq)
    b, _ = make_pair(kw, U, manning_sq=nsq)
    dt = 0.25 * o.linear_timestep_max() if method not in ("rk2",) else 0.5 * o.nonlinear_stationary_timestep_max()
    for d in (g, b):
        d.set_max_U_variables(MAX_U, stage_extrema_include_dry_cells=include_dry,
                              arrival_stage_threshold_above_msl_linear=0.02)
        if every > 1:
            d.set_max_U_update_frequency(every)
    o.c.max_U_extra = 31
    o.c.stage_extrema_include_dry_cells = int(include_dry)
    o.c.arrival_stage_threshold_above_msl_linear = 0.02
    o.c.max_U_update_frequency = every
    for _ in range(45):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    b.evolve_steps(45, dt)
    _exact(g, o, f"{method} max_U")
    m = water_mask(o.U[3])
    for d in (g, b):
        np.testing.assert_array_equal(d.max_stage()[m], o.max_stage[m])
        for k, name in enumerate(MAX_U):
            np.testing.assert_array_equal(d.max_U(name), o.max_U_extra[k], err_msg=name)
    assert np.any(o.max_U_extra[3] > 0)        # the wave arrived somewhere
    assert np.any(o.max_U_extra[1] > 0)


@pytest.mark.parametrize("method", ["rk2", "linear"])
def test_max_U_variables_fp32(method):
    """FP32 state (real_bytes=4, the reference's -DREALFLOAT) against the FP32
    oracle: the device clock is rounded to float for time_of_max_stage and
    arrival_time, and the arrival threshold is float(msl) + float(threshold)."""
    kw, U, nsq = _beach(method)
    g, o = make_pair(kw, U, manning_sq=nsq, real32=True, oracle_real32=True)
    dt = 0.25 * o.linear_timestep_max() if method != "rk2" else 0.5 * o.nonlinear_stationary_timestep_max()
    g.set_max_U_variables(MAX_U, stage_extrema_include_dry_cells=True, arrival_stage_threshold_above_msl_linear=0.02)
    o.c.max_U_extra = 31
    o.c.arrival_stage_threshold_above_msl_linear = 0.02
    for _ in range(45):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    Ug = g.get_U()
    m = water_mask(o.U[3])
    for k in range(3):
        a, b = Ug[k][m].astype(np.float64), o.U[k][m].astype(np.float64)
        assert np.max(np.abs(a - b)) <= 1e-5 * max(np.max(np.abs(b)), 1.0), k
    for k, name in enumerate(MAX_U):
        got = np.asarray(g.max_U(name), np.float64)[m]
        ref = np.asarray(o.max_U_extra[k], np.float64)[m]
        if name in ("time_of_max_stage", "arrival_time"):
            # float32 times: equal wherever the same step set the value
            assert np.mean(got == ref) >= 0.99, name
        else:
            assert np.max(np.abs(got - ref)) <= 1e-5 * max(np.max(np.abs(ref)), 1.0), name
    assert np.any(o.max_U_extra[3] > 0)
