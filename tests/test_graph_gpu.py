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
