"""Parity with the oracle at the benchmark configurations' full sizes.

The smaller parity tests cover every code path; these run the same
comparisons on the grids the benchmark times, so that the kernels' size-
dependent partitions (warp strips, row segments, tile shapes, graph steps)
are checked where they are measured:

* rk2 wet/dry beach, 2048 x 2048, FP64, adaptive dt: 30 steps from rest and
  30 steps from a state the GPU advanced 6000 steps (the wave on the slope,
  the wet/dry front moving), STG / UH / VH / max_stage / gauges bit for bit
  and within 1e-10 relative;
* the same window with FP32 state against the FP64 oracle (stated FP32
  tolerance);
* the batched linear grid, spherical 3600 x 2400 FP32: instances of a batch
  equal single-domain stepping for every tile configuration, and equal the
  FP32 oracle;
* the nested four-domain configuration (coarse band periodic over 0-360,
  one ratio-3 and two ratio-9 rk2 wet/dry domains), all FP64, two md steps
  bit for bit against the oracle's multidomain step;
* the adjoint configuration, spherical 1200 x 800 FP64, K = 50: the misfit
  equals the oracle's, and the gradient over the 300 x 200 source window
  matches central finite differences (eps = 1e-6) on 64 random cells.
"""
import math

import numpy as np
import pytest

from oracle import oracle as orc
from ptha_b200 import workloads
from pairs import make_pair, oracle_from_kw, rel_err, water_mask

pytestmark = pytest.mark.gpu

TOL64 = 1e-10


def _gauge_cells(xy, kw):
    nx, ny = kw["nx"]
    dx = (kw["lw"][0] / nx, kw["lw"][1] / ny)
    ij = orc.gauge_site_index(xy, kw.get("lower_left", (0.0, 0.0)), dx, (nx, ny))
    return ij[:, 1] - 1, ij[:, 0] - 1   # rows, columns (0-based)


def _run_rk2_window(kw, U, nsq, t0, nsteps, gauges, real32=False, oracle=None):
    """nsteps adaptive steps of the GPU from (U, t0); the oracle too unless
    one is given (then it is returned as is)."""
    from ptha_b200 import Domain
    g = Domain(**kw, real_bytes=4 if real32 else 8)
    g.set_U(U)
    g.set_manning_squared(nsq)
    g.time = t0
    g.gauges_setup(gauges, capacity=nsteps + 4)
    rows, cols = _gauge_cells(gauges, kw)
    series = []
    o = oracle
    if o is None:
        o = oracle_from_kw(kw)
        o.U[:] = U
        o.manning_squared[:] = nsq
        o.c.time = t0
    for _ in range(nsteps):
        g.evolve_one_step()
        if oracle is None:
            o.evolve_one_step()
            series.append(np.stack([o.U[k][rows, cols] for k in range(3)], axis=1))
    return g, o, (np.array(series) if series else None)


def _compare_fp64(g, o, series, tag):
    Ug = g.get_U()
    m = water_mask(o.U[3])
    for k, name in enumerate(("STG", "UH", "VH")):
        err = rel_err(Ug[k], o.U[k], mask=m)
        exact = float(np.mean(Ug[k][m] == o.U[k][m]))
        print(tag, name, "rel", err, "exact", exact)
        assert err <= TOL64, (tag, name, err)
        assert exact == 1.0, (tag, name, exact)
    np.testing.assert_array_equal(g.max_stage()[m], o.max_stage[m])
    rec = g.gauges_read()
    assert rec.shape == series.shape, (rec.shape, series.shape)
    np.testing.assert_array_equal(rec, series)
    st = g.state()
    assert st.time == o.time
    assert st.max_dt == o.max_dt
    assert st.negative_depth_fix_counter == o.negative_depth_fix_counter


@pytest.fixture(scope="module")
def rk2_warm_state():
    """The 2048^2 beach after 6000 GPU steps (the benchmark's warm-up)."""
    from ptha_b200 import Domain
    kw, U, gauges, nsq = workloads.rk2_beach()
    d = Domain(**kw)
    d.set_U(U)
    d.set_manning_squared(nsq)
    d.evolve_steps(6000)
    Uw, tw = d.get_U(), d.time
    d.close()
    return kw, U, gauges, nsq, Uw, tw


def test_rk2_2048_fp64_from_rest():
    kw, U, gauges, nsq = workloads.rk2_beach()
    g, o, series = _run_rk2_window(kw, U, nsq, 0.0, 30, gauges)
    _compare_fp64(g, o, series, "rk2 2048 from rest")
    g.close()


def test_rk2_2048_fp64_and_fp32_warm(rk2_warm_state):
    kw, U, gauges, nsq, Uw, tw = rk2_warm_state
    # the wave is on the slope: cells between the toe and the shoreline move
    assert np.max(np.abs(Uw[1][1:-1, 1700:1900])) > 1e-3
    g, o, series = _run_rk2_window(kw, Uw, nsq, tw, 30, gauges)
    wet0 = (Uw[0] - Uw[3]) > 1e-5
    wet1 = (o.U[0] - o.U[3]) > 1e-5
    print("wet/dry cells that changed state in the window:", int(np.sum(wet0 != wet1)))
    _compare_fp64(g, o, series, "rk2 2048 warm")
    g.close()
    # FP32 state from the same start against the FP64 oracle's result
    g32, _, _ = _run_rk2_window(kw, Uw, nsq, tw, 30, gauges, real32=True, oracle=o)
    U32 = g32.get_U().astype(np.float64)
    m = water_mask(o.U[3])
    errs = [rel_err(U32[k], o.U[k], mask=m) for k in range(3)]
    print("rk2 2048 warm FP32 vs FP64 oracle", errs, "time", g32.time, o.time)
    assert errs[0] <= 1e-4 and errs[1] <= 5e-3 and errs[2] <= 5e-3, errs
    g32.close()


def test_batched_3600x2400_fp32_instances():
    from ptha_b200 import Domain
    from ptha_b200.batch import Batch
    gkw, U0, lon, lat = workloads.batched_grid()
    grid = Domain(**gkw)
    grid.set_U(U0)
    dt = grid.linear_timestep_max()
    wet = U0[3] < 0
    B, nsteps, pick = 4, 20, 2
    ics = np.zeros((B, 3) + U0.shape[1:], np.float32)
    for q in range(B):
        ics[q, 0] = workloads.batched_instance_stage(lon, lat, wet, q, 256)
    # one instance alone, as a plain FP32 domain
    single = Domain(**gkw)
    Us = U0.copy()
    Us[:3] = ics[pick]
    single.set_U(Us)
    single.evolve_steps(nsteps, dt)
    ref = single.get_U()[:3]
    ref_max = single.max_stage()
    single.close()
    for cfg in range(Batch.tile_config_count()):
        bt = Batch(grid, B)
        bt.set_U(ics)
        bt.set_tile_config(cfg)
        bt.evolve(nsteps, dt)
        got = bt.get_U(pick, 1)[0]
        assert np.array_equal(got, ref), cfg
        assert np.array_equal(bt.max_stage(pick, 1)[0], ref_max), cfg
        bt.close()
    # the FP32 oracle, and the FP64 oracle at the FP32 tolerance
    for real32 in (True, False):
        o = oracle_from_kw(dict(gkw), real32=real32)
        o.U[:] = U0
        o.U[:3] = ics[pick]
        for _ in range(nsteps):
            o.evolve_one_step(dt)
        err = rel_err(ref[0], o.U[0], mask=wet)
        exact = float(np.mean(ref[0][wet] == o.U[0][wet]))
        print("batched instance vs oracle real32", real32, "rel", err, "exact", exact)
        if real32:
            assert exact == 1.0 and err == 0.0
        else:
            assert err <= 2e-4
    grid.close()


def _nest(nts, kws):
    """The nest with its initial states set (the timestep limits depend on
    the elevation)."""
    from ptha_b200 import Multidomain
    specs, coasts = workloads.nested_specs(nts)
    md = Multidomain(specs, domain_kwargs=kws, use_wetdry_limiting=True, flux_correction=True,
                     periodic_xs=(0.0, 360.0))
    for k, (s, d) in enumerate(zip(specs, md.domains)):
        d.set_U(workloads.nested_initial_state(s, k, coasts))
        if s.timestepping_method == "rk2":
            d.set_manning_squared(0.025 ** 2)
    return specs, coasts, md


def test_nested_four_domain_fp64_two_md_steps():
    from oracle.multidomain import OracleMultidomain
    from oracle.oracle import OracleDomain
    kws = [dict(spherical=True) for _ in range(4)]
    specs, coasts, md = _nest((1, 1, 1, 1), kws)
    dt = md.domains[0].linear_timestep_max()
    lims = [d.stationary_timestep_max() if d.timestepping_method == "rk2" else dt for d in md.domains]
    nts = [max(1, int(math.ceil(dt / lim))) for lim in lims]
    md.close()
    specs, coasts, md = _nest(nts, kws)
    odoms = [OracleDomain(s.nx[0], s.nx[1], s.lw, s.lower_left, timestepping_method=s.timestepping_method,
                          spherical=True, boundary_exterior=tuple(not b for b in s.is_nesting_boundary))
             for s in specs]
    omd = OracleMultidomain(odoms, [s.timestepping_method for s in specs], [s.dx for s in specs], md.exchanges,
                            refinement=nts, priority_index=[s.priority_domain_index for s in specs],
                            use_wetdry_limiting=True, flux_correction=True)
    for k, (s, d, od) in enumerate(zip(specs, md.domains, odoms)):
        od.U[:] = d.get_U()
        if s.timestepping_method == "rk2":
            od.manning_squared[:] = 0.025 ** 2
    print("nest nts", nts, "dt", dt, "exchanges", len(md.exchanges))
    assert 5.0 < dt < 60.0 and nts[1:] == [3, 9, 8], (dt, nts)
    for step in range(2):
        md.evolve_one_step(dt)
        omd.evolve_one_step(dt)
        for k, (d, od) in enumerate(zip(md.domains, odoms)):
            np.testing.assert_array_equal(d.get_U(), od.U, err_msg=f"domain {k} md step {step}")
        for q in range(len(md.exchanges)):
            np.testing.assert_array_equal(md.flux(q, "error"), omd.recv[q].recv_error, err_msg=f"exchange {q}")
    for d in md.domains:
        U = d.get_U()
        assert np.all(np.isfinite(U)) and np.max(np.abs(U[0][U[3] < 0])) < 10.0
    md.close()


def test_adjoint_1200x800_fd_64_cells():
    from ptha_b200 import Domain
    gkw, U0, gauges, eta_t, gcells = workloads.adjoint_case()
    d = Domain(**gkw)
    d.set_U(U0)
    dt = d.linear_timestep_max()
    nsteps = int(round(2 * 3600.0 / dt))
    Ut = U0.copy()
    Ut[0] = eta_t
    d.set_U(Ut)
    d.gauges_setup(gauges, capacity=nsteps + 8)
    d.evolve_steps(nsteps, dt)
    target = d.gauges_read()[:nsteps, :, 0].copy()
    Ui = U0.copy()
    Ui[0] = 0.0

    def gpu_loss(Ustart):
        d.set_U(Ustart)
        d.time = 0.0
        d.gauges_reset()
        d.evolve_steps(nsteps, dt)
        y = d.gauges_read()[:nsteps, :, 0]
        return 0.5 * float(np.sum((y - target) ** 2))

    d.set_U(Ui)
    d.time = 0.0
    loss, grad = d.misfit_gradient(nsteps, dt, target, checkpoint_every=50)
    # the misfit itself equals the oracle's forward run
    o = oracle_from_kw(dict(gkw))
    o.U[:] = Ui
    rows, cols = gcells[:, 0], gcells[:, 1]
    L = 0.0
    for n in range(nsteps):
        o.evolve_one_step(dt)
        L += 0.5 * float(np.sum((o.U[0][rows, cols] - target[n]) ** 2))
    assert loss == pytest.approx(L, rel=1e-12), (loss, L)
    assert gpu_loss(Ui) == pytest.approx(loss, rel=1e-12)
    win = workloads.adjoint_window()
    wet = (U0[3] < -20.0)
    cand = np.argwhere(wet[win]) + np.array([win[0].start, win[1].start])
    rng = np.random.default_rng(9)
    pick = cand[rng.choice(len(cand), 64, replace=False)]
    eps = 1e-6
    fd_floor = 10 * np.finfo(float).eps * max(loss, 1.0) / eps
    for j, i in pick:
        Up = Ui.copy(); Up[0, j, i] += eps
        Um = Ui.copy(); Um[0, j, i] -= eps
        fd = (gpu_loss(Up) - gpu_loss(Um)) / (2 * eps)
        assert grad[0, j, i] == pytest.approx(fd, rel=1e-6, abs=fd_floor), (i, j, grad[0, j, i], fd)
    d.close()
