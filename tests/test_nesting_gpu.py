"""GPU nesting exchange (swals_gpu_md_*) against the oracle, bit for bit.

* the reference's nested-comms unit test (nested_grid_comms_mod.f90:2694-3056)
  on two GPU domains: packed buffers and received states equal the oracle's;
* the planar-field exchange of the 4-domain nest (multidomain_mod.f90:
  4089-4176) with the metadata from ptha_b200.nesting;
* multidomain steps with flux integrals and flux correction (a 'linear'
  parent with an 'rk2' child, and an all-'rk2' wet/dry nest): every domain's
  state and every flux error equal the oracle's after each step, and the
  corrected multidomain conserves mass.
"""
import numpy as np
import pytest

from oracle.multidomain import OracleComm, OracleMultidomain
from oracle.oracle import OracleDomain
from ptha_b200 import Domain, Multidomain
from ptha_b200 import nesting as nest

from nest_cases import nested_comms_case, planar_values, two_level_nest
from test_nesting_metadata import four_domain_nest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("r", [1, 2, 3, 4, 5, 7, 101])
def test_nested_comms_gpu(r):
    c = nested_comms_case(r)
    parent = Domain(c["nx1"], (20.0, 15.0), (0.0, 0.0), "rk2")
    child = Domain(c["nx2"], (9.0, 8.0), c["ll2"], "rk2")
    parent.set_U(c["U1"])
    child.set_U(c["U2"])
    ex = [nest.Exchange(sender=1, receiver=0, send_box=c["child_send"], recv_box=c["parent_recv"], recv_row=0,
                        send_row=0),
          nest.Exchange(sender=0, receiver=1, send_box=c["parent_send"], recv_box=c["child_recv"], recv_row=0,
                        send_row=0)]
    md = Multidomain.from_tables([parent, child], [c["dx1"], c["dx2"]], ex, use_wetdry_limiting=False)
    md.send_halos()
    # Oracle: the same two exchanges as send-only / recv-only comms.
    o_child = OracleComm(c["dx2"], c["dx1"], send_inds=list(c["child_send"]) + [1, 4], send_only=True,
                         use_wetdry_limiting=False)
    o_parent = OracleComm(c["dx1"], c["dx2"], send_inds=list(c["parent_send"]) + [1, 4], send_only=True,
                          use_wetdry_limiting=False)
    U1, U2 = c["U1"].copy(), c["U2"].copy()
    b_child = o_child.pack(U2).copy()
    b_parent = o_parent.pack(U1).copy()
    g0, g1 = md.buffer(0), md.buffer(1)
    assert g0.shape == b_child.shape and g1.shape == b_parent.shape
    np.testing.assert_array_equal(g0[:-1], b_child[:-1])
    np.testing.assert_array_equal(g1[:-1], b_parent[:-1])
    md.recv_halos()
    r_parent = OracleComm(c["dx1"], c["dx2"], recv_inds=list(c["parent_recv"]) + [1, 4], recv_only=True,
                          use_wetdry_limiting=False)
    r_child = OracleComm(c["dx2"], c["dx1"], recv_inds=list(c["child_recv"]) + [1, 4], recv_only=True,
                         use_wetdry_limiting=False)
    r_parent.unpack(b_child, U1)
    r_child.unpack(b_parent, U2)
    np.testing.assert_array_equal(parent.get_U(), U1)
    np.testing.assert_array_equal(child.get_U(), U2)
    if r % 2 == 1:
        assert np.max(np.abs(child.get_U() - c["U2"]) / c["U2"]) <= 1e-14
    md.close()


def test_planar_field_exchange_gpu():
    specs = four_domain_nest()
    md = Multidomain(specs, extra_halo_buffer=0, extra_cells_in_halo=0, use_wetdry_limiting=False,
                     flux_correction=False)
    global_ll = specs[0].interior_bounding_box[0]
    odoms = [OracleDomain(s.nx[0], s.nx[1], s.lw, s.lower_left, timestepping_method=s.timestepping_method,
                          boundary_exterior=tuple(not b for b in s.is_nesting_boundary)) for s in specs]
    omd = OracleMultidomain(odoms, [s.timestepping_method for s in specs], [s.dx for s in specs], md.exchanges,
                            use_wetdry_limiting=False, flux_correction=False)
    for k, (s, d, od) in enumerate(zip(specs, md.domains, odoms)):
        U = planar_values(s, k + 1, global_ll)
        d.set_U(U)
        od.U[:] = U
    md.send_halos()
    md.recv_halos()
    for k in range(len(odoms)):
        omd.send_halos(k)
    omd.recv_halos()
    for k, (s, d, od) in enumerate(zip(specs, md.domains, odoms)):
        U = d.get_U()
        np.testing.assert_array_equal(U, od.U)
        active = nest._in_active_region(s.priority_domain_index, s.priority_domain_image, k + 1, 1,
                                        s.nest_layer_width)
        expect = planar_values(s, s.priority_domain_index.T.astype(np.float64), global_ll)
        err = np.abs(U - expect)[:, active.T].max()
        assert err * err <= np.spacing(1.0)
    md.close()


def _ic(specs, wetdry):
    """Stage: a Gaussian hump; elevation: flat -50 m, or a beach rising
    eastward through the child (wet/dry); the outer two rings of the parent
    are +100 m walls."""
    out = []
    for k, s in enumerate(specs):
        x = s.x()
        y = s.y()
        X, Y = np.meshgrid(x, y)
        U = np.zeros((4, s.nx[1], s.nx[0]))
        cx, cy = 20000.0, 20000.0
        eta = 1.0 * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * 4000.0 ** 2))
        if wetdry:
            elv = np.clip(-50.0 + (X - 25000.0) / 200.0, -50.0, 5.0)
        else:
            elv = np.full_like(X, -50.0)
        if k == 0:
            elv[:2, :] = 100.0
            elv[-2:, :] = 100.0
            elv[:, :2] = 100.0
            elv[:, -2:] = 100.0
        U[3] = elv
        U[0] = np.maximum(eta, elv)
        out.append(U)
    return out


def _run_pair(specs, wetdry, nsteps, fp_kwargs=None):
    kw = [dict(record_max_stage=True) for _ in specs]
    md = Multidomain(specs, domain_kwargs=kw, use_wetdry_limiting=True, flux_correction=True)
    odoms = [OracleDomain(s.nx[0], s.nx[1], s.lw, s.lower_left, timestepping_method=s.timestepping_method,
                          boundary_exterior=tuple(not b for b in s.is_nesting_boundary)) for s in specs]
    omd = OracleMultidomain(odoms, [s.timestepping_method for s in specs], [s.dx for s in specs], md.exchanges,
                            refinement=[s.timestepping_refinement_factor for s in specs],
                            priority_index=[s.priority_domain_index for s in specs], use_wetdry_limiting=True,
                            flux_correction=True)
    Us = _ic(specs, wetdry)
    for d, od, U in zip(md.domains, odoms, Us):
        d.set_U(U)
        od.U[:] = U
        n2 = np.full((U.shape[1], U.shape[2]), 0.025 ** 2)
        if d.timestepping_method in ("rk2", "euler"):
            d.set_manning_squared(n2)
            od.manning_squared[:] = n2
    # Fixed md step from the oracle's stationary limits (multidomain_mod.f90:2575-2660).
    lim = []
    for s, od in zip(specs, odoms):
        ts = od.linear_timestep_max() if s.timestepping_method == "linear" else od.nonlinear_stationary_timestep_max()
        lim.append(ts * s.timestepping_refinement_factor)
    dt = 0.5 * min(lim)
    vol0 = None
    for step in range(nsteps):
        md.evolve_one_step(dt)
        omd.evolve_one_step(dt)
        for k, (d, od) in enumerate(zip(md.domains, odoms)):
            np.testing.assert_array_equal(d.get_U(), od.U, err_msg=f"domain {k} step {step}")
        for q in range(len(md.exchanges)):
            np.testing.assert_array_equal(md.flux(q, "error"), omd.recv[q].recv_error, err_msg=f"exchange {q}")
    return md, omd


def test_linear_parent_rk2_child_steps():
    specs = two_level_nest(ratio=3, child_method="rk2", parent_method="linear")
    md, omd = _run_pair(specs, wetdry=False, nsteps=6)
    assert md.time == pytest.approx(omd.time)
    md.close()


def test_rk2_wetdry_nest_steps():
    specs = two_level_nest(ratio=3, child_method="rk2", parent_method="rk2", child_nt=2)
    md, omd = _run_pair(specs, wetdry=True, nsteps=6)
    md.close()


def test_md_graph_replay_matches_steps():
    """Three md steps captured as one CUDA graph and replayed twice equal six
    md steps issued one by one, bit for bit, including the domain times."""
    res = []
    for mode in ("steps", "graph"):
        specs = two_level_nest(ratio=3, child_method="rk2", parent_method="linear")
        md = Multidomain(specs, use_wetdry_limiting=True, flux_correction=True)
        for d, U in zip(md.domains, _ic(specs, False)):
            d.set_U(U)
            if d.timestepping_method == "rk2":
                d.set_manning_squared(0.025 ** 2)
        dt = 10.0
        if mode == "steps":
            for _ in range(6):
                md.evolve_one_step(dt)
        else:
            md.capture_graph(3, dt)
            md.replay(2)
        md.synchronize()
        res.append(([d.get_U() for d in md.domains], [d.time for d in md.domains], md.time,
                    [d.max_stage() for d in md.domains]))
        md.close()
    for a, b in zip(res[0][0], res[1][0]):
        np.testing.assert_array_equal(a, b)
    # the update before the first step is in the graph but acts on its
    # first replay only
    for a, b in zip(res[0][3], res[1][3]):
        np.testing.assert_array_equal(a, b)
    assert res[0][1] == res[1][1]
    assert res[0][2] == res[1][2] == pytest.approx(60.0)


def test_mixed_precision_nest_close_to_fp64():
    """An FP32 'linear' parent with an FP64 'rk2' child (the precisions of
    the nested configuration) stays within FP32 round-off of the all-FP64
    oracle over several md steps."""
    specs = two_level_nest(ratio=3, child_method="rk2", parent_method="linear")
    kw = [dict(real_bytes=4), dict(real_bytes=8)]
    md = Multidomain(specs, domain_kwargs=kw, use_wetdry_limiting=True, flux_correction=True)
    odoms = [OracleDomain(s.nx[0], s.nx[1], s.lw, s.lower_left, timestepping_method=s.timestepping_method,
                          boundary_exterior=tuple(not b for b in s.is_nesting_boundary)) for s in specs]
    omd = OracleMultidomain(odoms, [s.timestepping_method for s in specs], [s.dx for s in specs], md.exchanges,
                            refinement=[s.timestepping_refinement_factor for s in specs],
                            priority_index=[s.priority_domain_index for s in specs], flux_correction=True)
    for d, od, U in zip(md.domains, odoms, _ic(specs, False)):
        d.set_U(U)
        od.U[:] = U
        if d.timestepping_method == "rk2":
            d.set_manning_squared(0.025 ** 2)
            od.manning_squared[:] = 0.025 ** 2
    dt = 10.0
    for _ in range(8):
        md.evolve_one_step(dt)
        omd.evolve_one_step(dt)
    for k, (d, od) in enumerate(zip(md.domains, odoms)):
        U = d.get_U().astype(np.float64)
        wet = od.U[3] < 0
        err = np.abs(U[0] - od.U[0])[wet].max()
        assert err <= 2e-5 * max(1.0, np.abs(od.U[0][wet]).max()), (k, err)
    md.close()


def test_periodic_exchange_gpu():
    """The reference's periodic multidomain test on the GPU: the halos of a
    domain periodic in x and y come from its own interior (self-exchanges),
    equal to the oracle's and within the reference's tolerance."""
    from test_nesting_oracle import periodic_case, periodic_check
    s, ex, pxs, pys, X, Y, U = periodic_case()
    fresh = nest.NestDomain((-10.0, -80.0), (360.0, 170.0), (200, 200), "euler", 1)   # setup widens its specs
    md = Multidomain([fresh], use_wetdry_limiting=False, flux_correction=False, periodic_xs=pxs, periodic_ys=pys)
    assert [(e.send_box, e.recv_box) for e in md.exchanges] == [(e.send_box, e.recv_box) for e in ex]
    md.domains[0].set_U(U)
    md.send_halos()
    md.recv_halos()
    od = OracleDomain(s.nx[0], s.nx[1], s.lw, s.lower_left, timestepping_method="euler",
                      boundary_exterior=tuple(not b for b in s.is_nesting_boundary))
    omd = OracleMultidomain([od], ["euler"], [s.dx], ex, use_wetdry_limiting=False, flux_correction=False)
    od.U[:] = U
    omd.send_halos(0)
    omd.recv_halos()
    G = md.domains[0].get_U()
    np.testing.assert_array_equal(G, od.U)
    assert periodic_check(G, X, Y, pxs, pys) > 0
    md.close()


@pytest.mark.parametrize("method", ["linear", "rk2"])
def test_periodic_channel_steps(method):
    """A wave crossing the periodic seam of an x-periodic channel (walls north
    and south): md steps equal the oracle's bit for bit, and the mass in the
    priority cells is conserved."""
    pxs = (0.0, 100000.0)
    s = nest.NestDomain((0.0, 0.0), (100000.0, 40000.0), (100, 40), method, 1)
    ex = nest.setup_multidomain([s], periodic_xs=pxs)
    md = Multidomain([nest.NestDomain((0.0, 0.0), (100000.0, 40000.0), (100, 40), method, 1)],
                     use_wetdry_limiting=True, flux_correction=True, periodic_xs=pxs)
    assert md.specs[0].nx == s.nx and [e.send_box for e in md.exchanges] == [e.send_box for e in ex]
    X, Y = np.meshgrid(s.x(), s.y())
    U = np.zeros((4, s.nx[1], s.nx[0]))
    U[3] = -100.0
    U[3][:2, :] = 50.0
    U[3][-2:, :] = 50.0
    U[0] = np.maximum(U[3], 0.5 * np.exp(-((X - 90000.0) ** 2 + (Y - 20000.0) ** 2) / (2 * 5000.0 ** 2)))
    od = OracleDomain(s.nx[0], s.nx[1], s.lw, s.lower_left, timestepping_method=method,
                      boundary_exterior=tuple(not b for b in s.is_nesting_boundary))
    omd = OracleMultidomain([od], [method], [s.dx], ex, refinement=[1], priority_index=[s.priority_domain_index],
                            use_wetdry_limiting=True, flux_correction=True)
    md.domains[0].set_U(U)
    od.U[:] = U
    if method == "rk2":
        md.domains[0].set_manning_squared(0.025 ** 2)
        od.manning_squared[:] = 0.025 ** 2
    dt = 0.5 * (od.linear_timestep_max() if method == "linear" else od.nonlinear_stationary_timestep_max())
    # one exchange first, so that the halos are the periodic images (as the
    # reference's periodic test does); mass over the priority cells that
    # are not periodic copies (is_priority_domain_not_periodic)
    md.send_halos()
    md.recv_halos()
    omd.send_halos(0)
    omd.recv_halos()
    np.testing.assert_array_equal(md.domains[0].get_U(), od.U)
    pr = (s.priority_domain_index.T == 1) & (X > pxs[0]) & (X < pxs[1])
    v0 = float(np.sum((od.U[0] - od.U[3])[pr]))
    for step in range(60):
        md.evolve_one_step(dt)
        omd.evolve_one_step(dt)
    G = md.domains[0].get_U()
    np.testing.assert_array_equal(G, od.U)
    v1 = float(np.sum((G[0] - G[3])[pr]))
    assert abs(v1 - v0) <= 1e-11 * abs(v0)
    # the wave went through the seam: the west end has moved
    assert np.max(np.abs(G[0][5:-5, 3:15])) > 1e-3
    md.close()
