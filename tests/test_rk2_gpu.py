"""Parity of the fused CUDA rk2/euler finite-volume step with the oracle
(DE1_low_fr_diffusion fluxes, wet/dry theta limiter, update_U_manning,
CFL reduction), through the C ABI.

Tolerance: FP64 1e-10 relative to the field maximum.
The kernels follow the reference's operation order without FMA, so
differences come only from libm-vs-CUDA pow/cosh last bits."""
import numpy as np
import pytest

from ptha_b200 import workloads, _lib
from pairs import make_pair, rel_err, report, water_mask

TOL64 = 1e-10


def beach(n=128, **kw):
    return workloads.rk2_beach(n=n, dx=10.0 * 2048 / n, toe=17580.0 * n / 2048)


@pytest.mark.gpu
@pytest.mark.parametrize("adaptive", [True, False])
def test_rk2_beach_solitary_wave(adaptive):
    kw, U, gauges, nsq = beach(128)
    g, o = make_pair(kw, U, manning_sq=nsq)
    dt = None if adaptive else 0.5 * o.nonlinear_stationary_timestep_max()
    for _ in range(300):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _, errs = report(f"rk2 beach adaptive={adaptive}", g, o)
    for k in ("STG", "UH", "VH", "ELV"):
        assert errs[k] <= TOL64, errs
    # Same operation order, no FMA contraction, correctly rounded pow:
    # the FP64 state is expected to be bit-identical.
    for k in ("STG", "UH", "VH", "ELV"):
        assert errs[k + "_exact"] == 1.0, errs
    assert rel_err(g.max_stage(), o.max_stage, mask=water_mask(o.U[3])) <= TOL64
    st = g.state()
    assert st.time == pytest.approx(o.time, rel=1e-12)
    assert st.max_dt == pytest.approx(o.max_dt, rel=1e-10)
    assert st.negative_depth_fix_counter == o.negative_depth_fix_counter


@pytest.mark.gpu
def test_rk2_wet_dry_front_exercised():
    """The solitary wave must reach the beach so the wet/dry branches run."""
    kw, U, gauges, nsq = beach(96)
    g, o = make_pair(kw, U, manning_sq=nsq)
    for _ in range(1500):
        g.evolve_one_step()
        o.evolve_one_step()
    Ug, errs = report("rk2 beach long", g, o)
    wet0 = (U[0] - U[3]) > 1e-5
    wet1 = (o.U[0] - o.U[3]) > 1e-5
    assert np.any(wet1 & ~wet0), "front never moved"
    for k in ("STG", "UH", "VH"):
        assert errs[k] <= TOL64, errs


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["rk2", "euler"])
@pytest.mark.parametrize("coriolis", [True, False])
def test_fv_spherical(method, coriolis):
    kw, U = workloads.spherical_patch(nx=100, ny=70)
    kw.update(timestepping_method=method, coriolis=coriolis)
    U = U.copy()
    U[0] = np.where(U[3] > 0, U[3], U[0])
    g, o = make_pair(kw, U, manning_sq=np.full(U[0].shape, 0.025 ** 2))
    for _ in range(100):
        g.evolve_one_step()
        o.evolve_one_step()
    _, errs = report(f"{method} sph cor={coriolis}", g, o)
    for k in ("STG", "UH", "VH"):
        assert errs[k] <= TOL64, errs


@pytest.mark.gpu
@pytest.mark.parametrize("friction", ["chezy", "none"])
def test_rk2_friction_variants_and_transmissive(friction):
    kw, U, gauges, nsq = beach(100)
    kw = dict(kw)
    kw.update(boundary_kind=_lib.BC_TRANSMISSIVE, boundary_function_kind=0)
    if friction == "chezy":
        kw["friction_type"] = "chezy"
        nsq = 1.0 / 50.0 ** 2
    else:
        kw["nofriction"] = True
    U = U.copy()
    U[0] = np.maximum(U[3], 0.3 * np.exp(-((np.arange(100)[None, :] - 30) ** 2) / 50.0))
    U[0] = np.where(U[3] > 1e5, U[3], U[0])
    g, o = make_pair(kw, U, manning_sq=np.full(U[0].shape, nsq))
    for _ in range(200):
        g.evolve_one_step()
        o.evolve_one_step()
    _, errs = report(f"rk2 {friction}", g, o)
    for k in ("STG", "UH", "VH", "ELV"):
        assert errs[k] <= TOL64, errs


@pytest.mark.gpu
def test_rk2_fp32_against_fp64_oracle():
    kw, U, gauges, nsq = beach(128)
    g, o = make_pair(kw, U, manning_sq=nsq, real32=True)
    for _ in range(200):
        g.evolve_one_step()
        o.evolve_one_step()
    Ug = g.get_U()
    # FP32 state with FP64 pressure/source islands vs the FP64 oracle
    assert rel_err(Ug[0], o.U[0]) <= 1e-4
    assert rel_err(Ug[1], o.U[1]) <= 5e-3
    assert rel_err(Ug[2], o.U[2]) <= 5e-3


@pytest.mark.gpu
def test_rk2_diagnostics_match_oracle():
    kw, U, gauges, nsq = beach(128)
    g, o = make_pair(kw, U, manning_sq=nsq)
    assert g.nonlinear_stationary_timestep_max() == pytest.approx(o.nonlinear_stationary_timestep_max(), rel=1e-15)
    assert g.volume_interior() == pytest.approx(o.volume_interior(), rel=1e-13)
    for _ in range(50):
        g.evolve_one_step()
        o.evolve_one_step()
    assert g.volume_interior() == pytest.approx(o.volume_interior(), rel=1e-12)
    st = g.state()
    assert st.boundary_flux_time_integral == pytest.approx(o.c.boundary_flux_time_integral, rel=1e-9, abs=1e-6)


@pytest.mark.gpu
def test_rk2_config2_full_size_properties():
    """Full-size config (2048^2): lake at rest stays at rest, mass balance of
    the interior closes with the boundary-flux integral."""
    from ptha_b200 import Domain
    kw, U, gauges, nsq = workloads.rk2_beach()
    d = Domain(**kw)
    U2 = U.copy()
    d.set_U(U2)
    d.set_manning_squared(nsq)
    v0 = d.volume_interior()
    d.evolve_steps(200)
    v1 = d.volume_interior()
    st = d.state()
    # interior volume change equals minus the integrated outward boundary flux
    assert (v1 - v0) == pytest.approx(-st.boundary_flux_time_integral, rel=1e-6, abs=1e-3)
    Ug = d.get_U()
    assert np.all(np.isfinite(Ug))
    # far from the west boundary the lake is still at rest
    east = slice(1024, 2047)
    assert np.max(np.abs(Ug[1][1:-1, east])) < 1e-9
