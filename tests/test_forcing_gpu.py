"""Forcing patches (forcing_mod.f90) on the GPU against the oracle.

* the reference's own known answers for add_forcing_work_to_U_over_time
  (test_forcing_mod, forcing_mod.f90:387-562) through
  swals_gpu_apply_forcing, to spacing(10)*10 and bit for bit with the oracle;
* rise-time sources during stepping: finite-volume steppers ('euler' with
  elevation forcing, 'rk2', 'midpoint', 'rk2n'; the patch is applied after
  every update_U) and the leapfrog solvers (between the stage and the
  momentum sweep, with max_stage and the neighbouring momenta redone), bit
  for bit with the oracle, and a CUDA-graph replay equal to single steps;
* the volume added by a stage patch in a walled basin equals the patch's
  forcing_work integrated over the cell areas."""
import numpy as np
import pytest

from ptha_b200 import Domain, _lib, workloads
from pairs import make_pair, report, rel_err, water_mask
from test_oracle_golden import _forcing_case

pytestmark = pytest.mark.gpu


def _exact(g, o, tag, keys=("STG", "UH", "VH", "ELV")):
    _, errs = report(tag, g, o)
    for k in keys:
        assert errs[k + "_exact"] == 1.0, errs


@pytest.mark.parametrize("dom", [((50, 30), (50.0, 30.0), (0.0, 0.0)), ((23, 90), (10.0, 10.0), (1.0, 1.0))])
def test_apply_forcing_known_answers(dom):
    from oracle.oracle import add_forcing_work_to_U_over_time as add
    (nx, ny), lw, ll = dom
    U0, W = _forcing_case(*dom)
    d = Domain((nx, ny), lw, ll, "euler")
    tol = np.spacing(10.0) * 10
    cases = [((0.0, 10.0), 1.0), ((4.0, 10.0), 1.0), ((-4.0, 10.0), 10.0 / 14.0), ((-15.0, 15.0), 10.0 / 30.0),
             ((-15.0, 5.0), 5.0 / 20.0), ((-15.0, -5.0), 0.0)]
    for (st, en), frac in cases:
        d.forcing_clear()
        d.set_U(U0)
        d.add_forcing_patch(1, nx, 1, ny, 1, 4, st, en, W)
        d.time = 10.0
        d.apply_forcing(10.0)
        G = d.get_U()
        ref = U0.copy()
        add(ref, W, 10.0, 10.0, st, en)
        np.testing.assert_array_equal(G, ref)
        err = np.max(np.abs(G - (U0 + W * frac)))
        assert (err < tol) if frac else (err == 0.0), (st, en, err)
    # Test 7: stepping through the whole interval adds the whole forcing.
    d.forcing_clear()
    d.set_U(U0)
    d.add_forcing_patch(1, nx, 1, ny, 1, 4, -1.332, 5.15430, W)
    t, dt = -10.01242, 1.4444
    for _ in range(30):
        d.time = t
        d.apply_forcing(dt)
        t = t + dt
    assert np.max(np.abs(d.get_U() - (U0 + W))) < tol
    d.close()


def _source(n, i0, i1, j0, j1, amp=0.8):
    """A smooth uplift over the patch box (1-based inclusive)."""
    ii = np.arange(i0, i1 + 1)
    jj = np.arange(j0, j1 + 1)
    si = np.sin(np.pi * (ii - i0 + 0.5) / (i1 - i0 + 1))
    sj = np.sin(np.pi * (jj - j0 + 0.5) / (j1 - j0 + 1))
    return amp * sj[:, None] * si[None, :]


@pytest.mark.parametrize("method", ["euler", "rk2", "midpoint", "rk2n"])
@pytest.mark.parametrize("adaptive", [True, False])
def test_fv_rise_time_source(method, adaptive):
    """generic_model.f90:155-167's use: a stage (and, for 'euler', an
    elevation) source added over a rise time while stepping."""
    n = 80
    kw, U = workloads.spherical_patch(nx=n, ny=60)
    kw = dict(kw)
    kw["timestepping_method"] = method
    U = U.copy()
    U[0] = np.where(U[3] > 0, U[3], 0.0)
    g, o = make_pair(kw, U, manning_sq=np.full(U[0].shape, 0.025 ** 2))
    i0, i1, j0, j1 = 20, 45, 15, 40
    S = _source(n, i0, i1, j0, j1)
    k1 = 4 if method == "euler" else 3
    work = np.stack([S, 0.01 * S, -0.02 * S, -S][:k1])
    for dom in (g, o):
        dom.add_forcing_patch(i0, i1, j0, j1, 1, k1, 30.0, 130.0, work)
    dt = None if adaptive else 0.4 * o.nonlinear_stationary_timestep_max() * (4.0 if method == "rk2n" else 1.0)
    for _ in range(60):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _exact(g, o, f"{method} forcing adaptive={adaptive}")
    assert rel_err(g.max_stage(), o.max_stage, mask=water_mask(o.U[3])) == 0.0
    assert g.state().time == pytest.approx(o.time, rel=1e-13)
    assert g.state().time > 30.0


@pytest.mark.parametrize("method", ["euler", "rk2"])
def test_fv_forcing_with_stage_boundary(method):
    """A rise-time source on the beach whose solitary wave enters through the
    stage-from-function west boundary, adaptive dt: the step's boundary
    updates (time + dt after stage 1, time + 2 dt after rk2's second Euler
    stage, each followed by the forcing) take column 0's boundary stage from
    the values the stage-1 update evaluated; bit for bit with the oracle."""
    n = 96
    kw, U, _, nsq = workloads.rk2_beach(n=n, dx=10.0 * 2048 / n, toe=17580.0 * n / 2048)
    kw = dict(kw)
    kw["timestepping_method"] = method
    g, o = make_pair(kw, U, manning_sq=nsq)
    i0, i1, j0, j1 = 4, 11, 30, 60      # offshore of the beach toe's shoreline
    S = _source(n, i0, i1, j0, j1, amp=0.3)
    work = np.stack([S, 0.01 * S, -0.02 * S])
    for dom in (g, o):
        dom.add_forcing_patch(i0, i1, j0, j1, 1, 3, 0.0, 200.0, work)
    for _ in range(120):
        g.evolve_one_step()
        o.evolve_one_step()
    _exact(g, o, f"{method} forcing + stage boundary")
    assert g.state().time == o.time
    assert np.max(o.max_stage[1:-1, 1]) > 1.0, "the boundary wave never entered"
    g.close()


@pytest.mark.parametrize("method,truely_linear,coriolis", [
    ("linear", True, False), ("linear", False, False), ("linear", True, True),
    ("leapfrog_linear_plus_nonlinear_friction", True, True),
    ("leapfrog_linear_plus_nonlinear_friction", False, False)])
@pytest.mark.parametrize("kernel", ["tile", "async"])
def test_leapfrog_rise_time_source(method, truely_linear, coriolis, kernel, monkeypatch):
    monkeypatch.setenv("SWALS_LINEAR_KERNEL", kernel)
    n = 90
    kw, U = workloads.spherical_patch(nx=n, ny=70)
    kw = dict(kw)
    kw.update(timestepping_method=method, linear_solver_is_truely_linear=truely_linear, coriolis=coriolis)
    U = U.copy()
    U[0] = np.where(U[3] > 0, U[3], 0.0)
    g, o = make_pair(kw, U, manning_sq=np.full(U[0].shape, 0.03 ** 2))
    i0, i1, j0, j1 = 25, 60, 20, 48
    S = _source(n, i0, i1, j0, j1)
    work = np.stack([S, 0.02 * S, -0.01 * S, -S])
    for dom in (g, o):
        dom.add_forcing_patch(i0, i1, j0, j1, 1, 4, 10.0, 200.0, work)
    dt = o.linear_timestep_max()
    for _ in range(80):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _exact(g, o, f"{method} tl={truely_linear} cor={coriolis} {kernel} forcing")
    assert rel_err(g.max_stage(), o.max_stage) == 0.0


def test_leapfrog_source_volume_and_graph():
    """A stage-only source in a walled basin adds exactly its integral; the
    same steps replayed from a CUDA graph give the same state."""
    kw, U, _ = workloads.linear_gaussian_basin(n=120, dx=1000.0)
    U = U.copy()
    U[0] = np.where(U[3] > 0, U[3], 0.0)
    i0, i1, j0, j1 = 40, 80, 30, 70
    S = _source(120, i0, i1, j0, j1, amp=1.0)
    a, o = make_pair(kw, U)
    b, _ = make_pair(kw, U)
    for dom in (a, b, o):
        dom.add_forcing_patch(i0, i1, j0, j1, 1, 1, 0.0, 100.0, S[None])
    dt = o.linear_timestep_max()
    v0 = a.volume_interior()
    for _ in range(60):
        a.evolve_one_step(dt)
        o.evolve_one_step(dt)
    b.evolve_steps(60, dt)
    _exact(a, o, "linear basin forcing", keys=("STG", "UH", "VH"))
    np.testing.assert_array_equal(a.get_U(), b.get_U())
    area = o.area[0]
    assert a.volume_interior() - v0 == pytest.approx(float(S.sum()) * area, rel=1e-9)


def test_forcing_patch_checks():
    d = Domain((40, 40), (40.0, 40.0), (0.0, 0.0), "rk2")
    w = np.ones((4, 5, 5))
    with pytest.raises(_lib.SwalsError) as e:
        d.add_forcing_patch(10, 14, 10, 14, 1, 4, 0.0, 1.0, w)     # elevation forcing with rk2
    assert e.value.code == 3
    with pytest.raises(_lib.SwalsError) as e:
        d.add_forcing_patch(10, 14, 10, 14, 1, 1, 2.0, 1.0, w[:1])  # start after end
    assert e.value.code == 1
    with pytest.raises(_lib.SwalsError) as e:
        d.add_forcing_patch(38, 42, 10, 14, 1, 1, 0.0, 1.0, w[:1])  # outside the domain
    assert e.value.code == 1
    d.close()
    lin = Domain((40, 40), (40.0, 40.0), (0.0, 0.0), "linear")
    with pytest.raises(_lib.SwalsError) as e:
        lin.add_forcing_patch(1, 5, 10, 14, 1, 1, 0.0, 1.0, w[:1])  # on the boundary ring
    assert e.value.code == 3
    lin.close()
