"""Batched linear leapfrog: each instance of a batch must equal, bit for bit,
the same initial condition advanced alone through domain%evolve_one_step
(one kernel code path; instances share only ELV and the metrics), for every
tile configuration the autotuner may pick; and instance 0 must equal the
oracle."""
import numpy as np
import pytest

from ptha_b200 import workloads
from pairs import oracle_from_kw


def _ics(U, B, seed=11):
    rng = np.random.default_rng(seed)
    ny, nx = U.shape[1:]
    out = np.zeros((B, 3, ny, nx))
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny))
    for b in range(B):
        cx, cy = rng.uniform(0.3, 0.7) * nx, rng.uniform(0.3, 0.7) * ny
        amp = rng.uniform(0.5, 3.0)
        L = rng.uniform(4, 10)
        out[b, 0] = amp * (np.exp(-((ii - cx - L / 4) ** 2 + (jj - cy) ** 2) / (2 * (L / 6) ** 2))
                           - np.exp(-((ii - cx + L / 4) ** 2 + (jj - cy) ** 2) / (2 * (L / 6) ** 2)))
        out[b, 0] = np.where(U[3] > 0, 0.0, out[b, 0])
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("real32", [False, True])
def test_batch_equals_single_instances(real32):
    from ptha_b200 import Domain
    from ptha_b200.batch import Batch
    kw, U = workloads.spherical_patch(nx=150, ny=90)
    kw.update(timestepping_method="linear")
    rb = 4 if real32 else 8
    grid = Domain(**kw, real_bytes=rb)
    grid.set_U(U)
    dt = 0.9 * grid.linear_timestep_max()
    B = 7
    ics = _ics(U, B)
    nsteps = 40
    ref = []
    for b in range(B):
        d = Domain(**kw, real_bytes=rb)
        Ub = U.copy()
        Ub[:3] = ics[b]
        d.set_U(Ub)
        d.evolve_steps(nsteps, dt)
        ref.append((d.get_U()[:3], d.max_stage()))
        d.close()
    from ptha_b200._lib import lib
    import ctypes
    for cfg in range(Batch.tile_config_count()):
        bt = Batch(grid, B)
        bt.set_U(ics)
        bt.set_tile_config(cfg)
        bt.evolve(nsteps, dt)   # graph-replayed
        got = bt.get_U()
        mx = bt.max_stage()
        for b in range(B):
            assert np.array_equal(got[b], ref[b][0]), (cfg, b)
            assert np.array_equal(mx[b], ref[b][1]), (cfg, b)
        bt.close()


@pytest.mark.gpu
def test_batch_instance_matches_oracle_and_gauges():
    from ptha_b200 import Domain
    from ptha_b200.batch import Batch
    kw, U = workloads.spherical_patch(nx=120, ny=80)
    kw.update(timestepping_method="linear")
    grid = Domain(**kw)
    grid.set_U(U)
    dt = grid.linear_timestep_max()
    B = 3
    ics = _ics(U, B, seed=5)
    bt = Batch(grid, B)
    bt.set_U(ics)
    m = grid.metrics()
    gx = m["x"][[20, 60, 100]]
    gy = m["y"][[20, 40, 60]]
    gauges = np.array([[x, y] for x in gx for y in gy])
    bt.gauges_setup(gauges, capacity=64)
    cfg, ms = bt.tune()
    assert 0 <= cfg < 5 and ms > 0
    bt.evolve(33, dt)
    o = oracle_from_kw(kw)
    o.U[:] = U
    o.U[:3] = ics[1]
    cols = [c for c in (20, 60, 100) for _ in (20, 40, 60)]
    rows = [r for _ in (20, 60, 100) for r in (20, 40, 60)]
    series = []
    for _ in range(33):
        o.evolve_one_step(dt)
        series.append(o.U[0][rows, cols].copy())
    got = bt.get_U(1, 1)[0]
    assert np.array_equal(got, o.U[:3])
    rec = bt.gauges_read()
    assert rec.shape == (33, B, 9)
    assert np.array_equal(rec[:, 1, :], np.array(series))
    t_, n_ = bt.time()
    assert n_ == 33 and t_ == pytest.approx(33 * dt, rel=1e-12)
    bt.close()
