"""max_speed on the staggered grid along the last column and row.

update_max_quantities (domain_mod.f90:2297-2326) takes the face depths as
0.5_dp * sum(x(i:ip1)) with ip1 = min(i+1, nx) (jp1 likewise): on the last
column the slice holds the cell alone, so depth_E is half the cell's own
depth there (and depth_N on the last row).  The expected values here are a
numpy restatement of those slice sums, written independently of the oracle
and of the kernels, so that neither can pass by sharing a mistake.
"""
import numpy as np
import pytest

from oracle import oracle as orc

MAD = 1.0e-5


def _slice_half_sum(d, axis):
    """0.5 * sum(d(i:min(i+1, n))) along `axis` (0: j, 1: i)."""
    out = np.empty_like(d)
    if axis == 1:
        out[:, :-1] = 0.5 * (d[:, :-1] + d[:, 1:])
        out[:, -1] = 0.5 * d[:, -1]
    else:
        out[:-1, :] = 0.5 * (d[:-1, :] + d[1:, :])
        out[-1, :] = 0.5 * d[-1, :]
    return out


def staggered_speed(U, msl, truely_linear):
    s, uh, vh, e = (np.asarray(U[k]) for k in range(4))
    one = s.dtype.type(1)
    d = (s.dtype.type(msl) - e) if truely_linear else (s - e)
    dE = _slice_half_sum(d, 1)
    dN = _slice_half_sum(d, 0)
    dEi = np.where(dE > s.dtype.type(MAD), one / np.where(dE > 0, dE, one), 0).astype(s.dtype)
    dNi = np.where(dN > s.dtype.type(MAD), one / np.where(dN > 0, dN, one), 0).astype(s.dtype)
    return np.sqrt(uh * uh * (dEi * dEi) + vh * vh * (dNi * dNi))


def _case(real32=False, nx=40, ny=30):
    dt_ = np.float32 if real32 else np.float64
    rng = np.random.default_rng(11)
    U = np.zeros((4, ny, nx), dt_)
    U[3] = -100.0 + rng.uniform(-5.0, 5.0, (ny, nx))
    U[0] = rng.uniform(-0.2, 0.2, (ny, nx))
    U[1] = rng.uniform(-3.0, 3.0, (ny, nx))
    U[2] = rng.uniform(-3.0, 3.0, (ny, nx))
    kw = dict(nx=(nx, ny), lw=(nx * 1000.0, ny * 1000.0), lower_left=(0.0, 0.0), timestepping_method="linear")
    return kw, U


@pytest.mark.parametrize("truely_linear", [True, False])
def test_oracle_staggered_max_speed_edges(truely_linear):
    kw, U = _case()
    nx, ny = kw["nx"]
    o = orc.OracleDomain(nx, ny, kw["lw"], timestepping_method="linear", truely_linear=truely_linear)
    o.U[:] = U
    o.c.max_U_extra = 2
    dt = 0.5 * o.linear_timestep_max()
    o.evolve_one_step(dt)
    expect = np.maximum(staggered_speed(U, 0.0, truely_linear), staggered_speed(o.U, 0.0, truely_linear))
    np.testing.assert_array_equal(o.max_U_extra[1], expect)
    # the edge values really differ from a doubled last-cell depth
    assert np.all(expect[:, -1] > 0) and np.all(expect[-1, :] > 0)


@pytest.mark.gpu
@pytest.mark.parametrize("real32", [False, True])
@pytest.mark.parametrize("truely_linear", [True, False])
def test_gpu_staggered_max_speed_edges(truely_linear, real32):
    from ptha_b200 import Domain
    kw, U = _case(real32)
    g = Domain(**kw, linear_solver_is_truely_linear=truely_linear, real_bytes=4 if real32 else 8)
    g.set_U(U.astype(np.float64))
    g.set_max_U_variables(("max_speed",))
    o = orc.OracleDomain(kw["nx"][0], kw["nx"][1], kw["lw"], timestepping_method="linear",
                         truely_linear=truely_linear)
    o.U[:] = U
    dt = 0.5 * o.linear_timestep_max()
    g.evolve_one_step(dt)
    U1 = g.get_U().astype(U.dtype)
    expect = np.maximum(staggered_speed(U, 0.0, truely_linear), staggered_speed(U1, 0.0, truely_linear))
    got = np.asarray(g.max_U("max_speed")).astype(U.dtype)
    np.testing.assert_array_equal(got, expect)
    g.close()
