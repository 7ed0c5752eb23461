"""The nesting oracle against the reference's own nesting unit tests.

* test_nested_grid_comms_mod (nested_grid_comms_mod.f90:2694-3056): for nest
  ratios 1, 2, 3, 4, 5, 7, 101 -- cell ratios and fine/coarse roles, matching
  send/receive buffer sizes, packed values inside [8, 32] (coarse) and
  [8 - dx, 32 + dx] (fine, even ratios), exact preservation of a linear field
  for odd ratios (relative 1e-14), and the time round trip.
* test_multidomain_mod1's planar-field exchange (multidomain_mod.f90:
  4089-4176): after send/recv every active cell of every domain holds the
  plane of its priority domain, err^2 < spacing(1).
"""
import numpy as np
import pytest

from oracle.multidomain import OracleComm, OracleMultidomain
from oracle.oracle import OracleDomain
from ptha_b200 import nesting as nest

from nest_cases import nested_comms_case, planar_values
from test_nesting_metadata import four_domain_nest


@pytest.mark.parametrize("r", [1, 2, 3, 4, 5, 7, 101])
def test_nested_comms_known_answers(r):
    c = nested_comms_case(r)
    child = OracleComm(c["dx2"], c["dx1"], send_inds=list(c["child_send"]) + [1, 4],
                       recv_inds=list(c["child_recv"]) + [1, 4], use_wetdry_limiting=False)
    parent = OracleComm(c["dx1"], c["dx2"], send_inds=list(c["parent_send"]) + [1, 4],
                        recv_inds=list(c["parent_recv"]) + [1, 4], use_wetdry_limiting=False)
    assert np.allclose(child.c.cell_ratios[:], [1.0 / r] * 2, atol=1e-6)
    assert np.allclose(parent.c.cell_ratios[:], [float(r)] * 2, atol=1e-6)
    assert parent.c.nsend == child.c.nrecv
    assert child.c.nsend == parent.c.nrecv
    if r > 1:
        assert not parent.c.my_domain_is_finer and child.c.my_domain_is_finer
    U1, U2 = c["U1"].copy(), c["U2"].copy()
    bp = parent.pack(U1).copy()
    bc = child.pack(U2).copy()
    err_tol = 1e-14
    strd = 5
    vals = bp[:parent.c.nsend_interior:strd]
    assert vals.max() / 32.0 <= 1 + err_tol and vals.min() / 8.0 >= 1 - err_tol
    off = c["dx2"][0] if r % 2 == 0 else 0.0
    vals = bc[:child.c.nsend_interior]
    assert vals.max() / (32.0 + off) <= 1 + err_tol and vals.min() / (8.0 - off) >= 1 - err_tol
    parent.unpack(bc, U1)
    child.unpack(bp, U2)
    if r % 2 == 1:
        for U, U0 in ((U1, c["U1"]), (U2, c["U2"])):
            assert np.max(np.abs(U - U0) / U0) <= err_tol
    # Time round trip
    bp = parent.pack(U1, time=2.0).copy()
    bc = child.pack(U2, time=3.0).copy()
    assert parent.unpack(bc, U1) == 3.0
    assert child.unpack(bp, U2) == 2.0


def oracle_nest4():
    specs = four_domain_nest()
    ex = nest.setup_multidomain(specs, extra_halo_buffer=0, extra_cells_in_halo=0)
    doms = [OracleDomain(s.nx[0], s.nx[1], s.lw, s.lower_left, timestepping_method=s.timestepping_method,
                         boundary_exterior=tuple(not b for b in s.is_nesting_boundary)) for s in specs]
    return specs, ex, doms


def test_planar_field_exchange():
    specs, ex, doms = oracle_nest4()
    global_ll = specs[0].interior_bounding_box[0]
    md = OracleMultidomain(doms, [s.timestepping_method for s in specs], [s.dx for s in specs], ex,
                           use_wetdry_limiting=False, flux_correction=False)
    for k, (s, d) in enumerate(zip(specs, doms)):
        d.U[:] = planar_values(s, k + 1, global_ll)
    for k in range(len(doms)):
        md.send_halos(k)
    md.recv_halos()
    for k, (s, d) in enumerate(zip(specs, doms)):
        active = nest._in_active_region(s.priority_domain_index, s.priority_domain_image, k + 1, 1,
                                        s.nest_layer_width)
        expect = planar_values(s, s.priority_domain_index.T.astype(np.float64), global_ll)
        err = np.abs(d.U - expect)[:, active.T].max()
        assert err * err <= np.spacing(1.0), (k, err)


def _priority_volume(specs, doms):
    """Water volume over each domain's priority cells."""
    v = 0.0
    for k, (s, d) in enumerate(zip(specs, doms)):
        pr = (s.priority_domain_index.T == k + 1)
        dep = d.U[0] - d.U[3]
        v += float(np.sum((dep * d.area[:, None])[pr]))
    return v


@pytest.mark.parametrize("parent,child,nt,wetdry", [("linear", "rk2", 3, False), ("rk2", "rk2", 2, True)])
def test_flux_correction_conserves_mass(parent, child, nt, wetdry):
    """Flux correction makes the nested solution conserve mass to round-off
    (the purpose of nesting_flux_correction_everywhere); without it the
    coarse/fine flux mismatch leaks mass."""
    from nest_cases import two_level_nest
    from test_nesting_gpu import _ic
    drift = {}
    for fc in (False, True):
        specs = two_level_nest(3, child, parent, nt)
        ex = nest.setup_multidomain(specs)
        doms = [OracleDomain(s.nx[0], s.nx[1], s.lw, s.lower_left, timestepping_method=s.timestepping_method,
                             boundary_exterior=tuple(not b for b in s.is_nesting_boundary)) for s in specs]
        md = OracleMultidomain(doms, [s.timestepping_method for s in specs], [s.dx for s in specs], ex,
                               refinement=[s.timestepping_refinement_factor for s in specs],
                               priority_index=[s.priority_domain_index for s in specs], flux_correction=fc)
        for d, U in zip(doms, _ic(specs, wetdry)):
            d.U[:] = U
            d.manning_squared[:] = 0.025 ** 2
        lim = [(d.linear_timestep_max() if s.timestepping_method == "linear" else d.nonlinear_stationary_timestep_max())
               * s.timestepping_refinement_factor for s, d in zip(specs, doms)]
        dt = 0.5 * min(lim)
        v0 = _priority_volume(specs, doms)
        for _ in range(10):
            md.evolve_one_step(dt)
        drift[fc] = abs(_priority_volume(specs, doms) - v0) / v0
    assert drift[True] < 1e-13
    assert drift[False] > 1e-8


def periodic_case():
    """test_multidomain_mod_periodic (multidomain_mod.f90:4185-4298): one
    200 x 200 'euler' domain over lon -10..350, lat -80..90, periodic in both
    directions, U(i,j,k) = x + y^2 + k."""
    pxs, pys = (-10.0, 350.0), (-80.0, 90.0)
    s = nest.NestDomain((-10.0, -80.0), (360.0, 170.0), (200, 200), "euler", 1)
    ex = nest.setup_multidomain([s], periodic_xs=pxs, periodic_ys=pys)
    X, Y = np.meshgrid(s.x(), s.y())
    U = np.stack([X + Y * Y + k for k in (1.0, 2.0, 3.0, 4.0)])
    return s, ex, pxs, pys, X, Y, U


def periodic_check(U, X, Y, pxs, pys):
    """The reference test's acceptance: every cell holds the field at its
    periodic image, within its heuristic tolerance."""
    px, _ = nest._periodic_shift(X.ravel(), *pxs, True)
    py, _ = nest._periodic_shift(Y.ravel(), *pys, True)
    px, py = px.reshape(X.shape), py.reshape(Y.shape)
    tv = px + py * py
    err = np.max(np.abs(U - (tv[None] + np.arange(1.0, 5.0)[:, None, None])), axis=0)
    xc, yc = np.abs(px - X), np.abs(py - Y)
    tol = 1e-10 + 40.0 * (np.spacing(np.abs(px) + np.abs(py * py)) + (np.spacing(xc) + 2.0 * yc * np.spacing(yc)))
    assert np.all(err <= tol), float(err.max())
    return int(np.count_nonzero((xc > 0) | (yc > 0)))


def test_periodic_exchange():
    s, ex, pxs, pys, X, Y, U = periodic_case()
    assert all(e.sender == 0 and e.receiver == 0 for e in ex)
    d = OracleDomain(s.nx[0], s.nx[1], s.lw, s.lower_left, timestepping_method="euler",
                     boundary_exterior=tuple(not b for b in s.is_nesting_boundary))
    md = OracleMultidomain([d], ["euler"], [s.dx], ex, use_wetdry_limiting=False, flux_correction=False)
    d.U[:] = U
    md.send_halos(0)
    md.recv_halos()
    assert periodic_check(d.U, X, Y, pxs, pys) > 0
