"""compute_domain_statistics_new and volume_in_priority_domain on the GPU
against the oracle: max/min stage and speed equal exactly (order-free), the
energies and the volume within 1e-12 relative (the GPU adds each row's terms
in a warp tree, the reference in column order)."""
import numpy as np
import pytest

from ptha_b200 import workloads

from pairs import make_pair

pytestmark = pytest.mark.gpu


def _check(g, o, mask=None):
    if mask is not None:
        g.set_priority_mask(mask)
    s = g.compute_domain_statistics()
    r = o.domain_statistics(mask)
    keys = ["maxstage", "maxspeed", "minstage", "minspeed", "energy_potential_on_rho", "energy_kinetic_on_rho",
            "energy_total_on_rho"]
    for k, ref in zip(keys[:4], r[:4]):
        assert s[k] == ref, (k, s[k], ref)
    for k, ref in zip(keys[4:], r[4:]):
        assert s[k] == pytest.approx(ref, rel=1e-12, abs=1e-9 * max(1.0, abs(r[6]))), (k, s[k], ref)
    # volume_in_priority_domain: row sums in a warp tree vs column order.
    v = g.volume_in_priority_domain()
    assert v == pytest.approx(o.volume_in_priority_domain(mask), rel=1e-12, abs=1e-12 * abs(o.volume_interior()))


def test_linear_statistics():
    kw, U, _ = workloads.linear_gaussian_basin(n=200, dx=2000.0)
    g, o = make_pair(kw, U)
    dt = g.linear_timestep_max()
    for _ in range(30):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    _check(g, o)
    rng = np.random.default_rng(3)
    _check(g, o, mask=rng.random((200, 200)) > 0.3)


def test_rk2_statistics():
    n = 160
    kw, U, _, nsq = workloads.rk2_beach(n=n, dx=10.0 * 2048 / n, toe=17580.0 * n / 2048)
    g, o = make_pair(kw, U, manning_sq=nsq)
    for _ in range(40):
        g.evolve_one_step()
        o.evolve_one_step()
    assert np.array_equal(g.get_U(), o.U)
    _check(g, o)
