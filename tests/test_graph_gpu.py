"""evolve_steps replays a CUDA graph of a few steps for long runs; the
result must be identical to issuing evolve_one_step one step at a time
(state, max_stage, gauges, time and step counters)."""
import numpy as np
import pytest

from ptha_b200 import Domain, workloads

pytestmark = pytest.mark.gpu


def _linear():
    kw, U, gauges = workloads.linear_gaussian_basin(n=96, dx=1000.0)
    return kw, U, gauges, None


def _rk2():
    kw, U, _, nsq = workloads.rk2_beach(n=96, dx=10.0 * 2048 / 96, toe=17580.0 * 96 / 2048)
    lw = kw["lw"]
    g = [0.25, 0.5, 0.75]
    gauges = [[fx * lw[0], fy * lw[1]] for fy in g for fx in g]
    return kw, U, gauges, nsq


@pytest.mark.parametrize("case", ["linear", "rk2"])
def test_graph_replay_equals_single_steps(case):
    kw, U, gauges, nsq = _linear() if case == "linear" else _rk2()
    out = []
    for mode in ("one", "steps"):
        d = Domain(**kw)
        d.set_U(U)
        if nsq is not None:
            d.set_manning_squared(nsq)
        d.gauges_setup(gauges, capacity=200)
        dt = d.linear_timestep_max() if case == "linear" else None
        if mode == "one":
            for _ in range(41):
                d.evolve_one_step(dt)
        else:
            d.evolve_steps(41, dt)   # 1 eager + 6 graph replays of 6 + 4 eager
        st = d.state()
        out.append((d.get_U(), d.max_stage(), d.gauges_read(), st.time, st.nsteps_advanced))
        d.close()
    a, b = out
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[2], b[2])
    assert a[3] == b[3] and a[4] == b[4] == 41


def test_graph_after_single_steps_moved_the_state_buffer():
    """A replayed graph reads the state buffers it was captured with: after
    single steps have rotated the state to another buffer (and set_U wrote
    there), evolve_steps must capture again rather than replay from the old
    buffer.  Compared with the same steps taken one by one."""
    kw, U, gauges, _ = _linear()
    rng = np.random.default_rng(3)
    U2 = U.copy()
    U2[0] = U2[0] + 0.1 * rng.standard_normal(U2[0].shape) * (U2[3] < 0)
    d = Domain(**kw)
    e = Domain(**kw)
    dt = d.linear_timestep_max()
    for x in (d, e):
        x.set_U(U)
    d.evolve_steps(20, dt)          # 1 single + 18 replayed + 1 single: the buffer rotates
    for _ in range(20):
        e.evolve_one_step(dt)
    for x in (d, e):
        x.set_U(U2)
    d.evolve_steps(24, dt)
    for _ in range(24):
        e.evolve_one_step(dt)
    np.testing.assert_array_equal(d.get_U(), e.get_U())
    d.close()
    e.close()


def test_batch_graph_after_odd_steps():
    from ptha_b200.batch import Batch
    kw, U = workloads.spherical_patch(nx=64, ny=48)
    kw.update(timestepping_method="linear")
    grid = Domain(**kw)
    grid.set_U(U)
    dt = grid.linear_timestep_max()
    ic = U[None, :3].copy()
    out = []
    # evolve(3) leaves the state in the other buffer than its 2-step graph
    # started from; evolve(2) must not replay that graph
    for pattern in ((3, 2, 3, 2), (1,) * 10):
        b = Batch(grid, 1)
        b.set_U(ic)
        for n in pattern:
            b.evolve(n, dt)
        out.append(b.get_U())
        b.close()
    np.testing.assert_array_equal(out[0], out[1])


def test_md_replay_refuses_a_moved_state_buffer():
    from ptha_b200 import Multidomain, SwalsError
    from nest_cases import two_level_nest
    specs = two_level_nest(ratio=3, child_method="rk2", parent_method="linear")
    md = Multidomain(specs, use_wetdry_limiting=True, flux_correction=True)
    for d in md.domains:
        U = np.zeros((4, d.nx[1], d.nx[0]))
        U[3] = -50.0
        d.set_U(U)
    md.capture_graph(3, 10.0)
    md.replay(1)
    md.evolve_one_step(10.0)     # the linear parent rotates to another buffer
    with pytest.raises(SwalsError):
        md.replay(1)
    md.close()
