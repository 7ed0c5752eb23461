"""Groups of multidomains advanced in one graph launch (the batched form of
the nested configuration: many sources on the same nest).  Every member of
a replayed group must equal, bit for bit, the same multidomain advanced on
its own (md steps issued one by one), and a member must equal the oracle's
multidomain step (multidomain_mod.f90:1093-1212)."""
import numpy as np
import pytest

from oracle.multidomain import OracleMultidomain
from oracle.oracle import OracleDomain
from ptha_b200 import Multidomain, MultidomainGroup, SwalsError, workloads

from nest_cases import two_level_nest

pytestmark = pytest.mark.gpu


def _ic(specs, cx):
    out = []
    for k, s in enumerate(specs):
        X, Y = np.meshgrid(s.x(), s.y())
        U = np.zeros((4, s.nx[1], s.nx[0]))
        elv = np.clip(-50.0 + (X - 25000.0) / 200.0, -50.0, 5.0)
        if k == 0:
            elv[:2, :] = 100.0
            elv[-2:, :] = 100.0
            elv[:, :2] = 100.0
            elv[:, -2:] = 100.0
        U[3] = elv
        U[0] = np.maximum(np.exp(-((X - cx) ** 2 + (Y - 20000.0) ** 2) / (2 * 4000.0 ** 2)), elv)
        out.append(U)
    return out


def _member(cx, kw=None):
    specs = two_level_nest(ratio=3, child_method="rk2", parent_method="linear")
    md = Multidomain(specs, domain_kwargs=kw, use_wetdry_limiting=True, flux_correction=True)
    for d, U in zip(md.domains, _ic(specs, cx)):
        d.set_U(U)
        if d.timestepping_method == "rk2":
            d.set_manning_squared(0.025 ** 2)
    return specs, md


@pytest.mark.parametrize("precisions", ["fp64", "fp32_parent"])
def test_group_members_equal_lone_multidomains(precisions):
    kw = None if precisions == "fp64" else [dict(real_bytes=4), dict(real_bytes=8)]
    centres = (15000.0, 20000.0, 26000.0)
    group_mds = [_member(cx, kw)[1] for cx in centres]
    lone = [_member(cx, kw)[1] for cx in centres]
    dt = 10.0
    g = MultidomainGroup(group_mds, 3, dt)
    g.replay(2)
    for md in lone:
        for _ in range(6):
            md.evolve_one_step(dt)
    for q, (a, b) in enumerate(zip(group_mds, lone)):
        a.synchronize()
        b.synchronize()
        assert a.time == b.time == pytest.approx(60.0)
        for k, (da, db) in enumerate(zip(a.domains, b.domains)):
            np.testing.assert_array_equal(da.get_U(), db.get_U(), err_msg=f"member {q} domain {k}")
            np.testing.assert_array_equal(da.max_stage(), db.max_stage())
            assert da.time == db.time
    # a member taking single steps in between moves its buffers: refused
    group_mds[1].evolve_one_step(dt)
    with pytest.raises(SwalsError):
        g.replay(1)
    g.close()
    for md in group_mds + lone:
        md.close()


def test_group_member_matches_oracle():
    specs, md = _member(18000.0)
    _, other = _member(24000.0)
    odoms = [OracleDomain(s.nx[0], s.nx[1], s.lw, s.lower_left, timestepping_method=s.timestepping_method,
                          boundary_exterior=tuple(not b for b in s.is_nesting_boundary)) for s in specs]
    omd = OracleMultidomain(odoms, [s.timestepping_method for s in specs], [s.dx for s in specs], md.exchanges,
                            refinement=[s.timestepping_refinement_factor for s in specs],
                            priority_index=[s.priority_domain_index for s in specs], flux_correction=True)
    for od, U in zip(odoms, _ic(specs, 18000.0)):
        od.U[:] = U
        if od.c.method == 1:
            od.manning_squared[:] = 0.025 ** 2
    dt = 10.0
    g = MultidomainGroup([md, other], 3, dt)
    g.replay(1)
    for _ in range(3):
        omd.evolve_one_step(dt)
    md.synchronize()
    for k, (d, od) in enumerate(zip(md.domains, odoms)):
        np.testing.assert_array_equal(d.get_U(), od.U, err_msg=f"domain {k}")
    g.close()
    md.close()
    other.close()


def test_nested_configuration_group_small():
    """The four-domain nested configuration, shrunk 3x, two sources in a
    group against the same two advanced alone."""
    import math
    kw = [dict(real_bytes=4, spherical=True), dict(spherical=True), dict(spherical=True), dict(spherical=True)]

    def build(seed, nts):
        sp, co = workloads.nested_specs(nts, scale=3)
        md = Multidomain(sp, domain_kwargs=kw, use_wetdry_limiting=True, flux_correction=True,
                         periodic_xs=(0.0, 360.0))
        for k, (s_, d) in enumerate(zip(sp, md.domains)):
            d.set_U(workloads.nested_initial_state(s_, k, co, source_seed=seed))
            if d.timestepping_method == "rk2":
                d.set_manning_squared(0.025 ** 2)
        return md

    probe = build(11, (1, 1, 1, 1))
    dt = probe.domains[0].linear_timestep_max()
    nts = [max(1, int(math.ceil(dt / (d.stationary_timestep_max() if d.timestepping_method == "rk2" else dt))))
           for d in probe.domains]
    probe.close()
    grouped = [build(11 + q, nts) for q in range(2)]
    lone = [build(11 + q, nts) for q in range(2)]
    g = MultidomainGroup(grouped, 3, dt)
    g.replay(1)
    for md in lone:
        for _ in range(3):
            md.evolve_one_step(dt)
    for a, b in zip(grouped, lone):
        for da, db in zip(a.domains, b.domains):
            np.testing.assert_array_equal(da.get_U(), db.get_U())
    g.close()
    for md in grouped + lone:
        md.close()
