"""Nesting metadata builder against the reference's own known answers.

The 4-domain nest of ``test_multidomain_mod1`` (multidomain_mod.f90:3814-3993):
a 360x210 'euler' parent, two ratio-3 'rk2' children side by side (one with
timestepping_refinement_factor 2), and a ratio-9 'rk2' grandchild
(refinement factor 5), set up with extra_cells_in_halo=0 and
extra_halo_buffer=0.  The expected receive boxes below are the reference
test's tables (rows of: priority domain index, image, iL, iU, jL, jU).
"""
import numpy as np
import pytest

from ptha_b200 import nesting as nest


def _nint(v):
    return np.floor(np.abs(v) + 0.5) * np.sign(v)


def four_domain_nest():
    """The domains of test_multidomain_mod1, built with the same expressions
    (including its single-precision literal 1.1)."""
    global_lw = np.array([641000.0, 367000.0])
    global_ll = np.array([185985.0, 8795845.0])
    global_nx = np.array([360, 210])
    ratio = 3
    inner_lw = global_lw * (1.0 / ratio)
    inner_ll = global_ll + inner_lw
    dx1 = global_lw / global_nx
    d1 = nest.NestDomain(tuple(global_ll), tuple(global_lw), tuple(int(v) for v in global_nx), "euler", 1)
    lw2 = _nint(inner_lw / dx1) * dx1
    dx2 = dx1 / float(ratio)
    d2 = nest.NestDomain(tuple(global_ll), tuple(lw2), tuple(int(v) for v in _nint(lw2 / dx2)), "rk2", 1)
    ll3 = global_ll + _nint((inner_ll - global_ll) / dx1) * dx1
    lw3 = _nint(inner_lw / dx1) * dx1
    dx3 = dx1 / float(ratio)
    d3 = nest.NestDomain(tuple(ll3), tuple(lw3), tuple(int(v) for v in _nint(lw3 / dx3)), "rk2", 2)
    lw4 = _nint(lw3 * np.array([0.3, 0.5]) / dx1) * dx1
    one_point_one = float(np.float32(1.1))
    ll4 = global_ll + _nint(one_point_one * lw2 / dx1) * dx1
    dx4 = dx1 / float(ratio * ratio)
    d4 = nest.NestDomain(tuple(ll4), tuple(lw4), tuple(int(v) for v in _nint(lw4 / dx4)), "rk2", 5)
    return [d1, d2, d3, d4]


EXPECTED = {
    1: [[0, 0, 1, 118, 1, 68], [2, 1, 119, 120, 1, 68], [1, 1, 121, 360, 1, 70], [2, 1, 1, 120, 69, 70],
        [3, 1, 121, 240, 71, 72], [3, 1, 121, 122, 73, 138], [0, 0, 123, 238, 73, 138], [3, 1, 239, 240, 73, 138],
        [1, 1, 1, 120, 71, 140], [1, 1, 241, 360, 71, 140], [3, 1, 121, 240, 139, 140], [1, 1, 1, 360, 141, 210]],
    2: [[2, 1, 1, 360, 1, 210], [1, 1, 361, 366, 1, 210], [1, 1, 1, 360, 211, 216], [3, 1, 361, 366, 211, 216]],
    3: [[2, 1, 1, 9, 1, 9], [1, 1, 10, 378, 1, 9], [3, 1, 10, 369, 10, 30], [4, 1, 46, 153, 31, 39],
        [4, 1, 46, 54, 40, 126], [0, 0, 55, 144, 40, 126], [4, 1, 145, 153, 40, 126], [3, 1, 10, 45, 31, 135],
        [3, 1, 154, 369, 31, 135], [4, 1, 46, 153, 127, 135], [1, 1, 1, 9, 10, 219], [1, 1, 370, 378, 10, 219],
        [3, 1, 10, 369, 136, 219], [1, 1, 1, 378, 220, 228]],
    4: [[3, 1, 1, 366, 1, 21], [3, 1, 1, 21, 22, 336], [4, 1, 22, 345, 22, 336], [3, 1, 346, 366, 22, 336],
        [3, 1, 1, 366, 337, 357]],
}


@pytest.fixture(scope="module")
def nest4():
    doms = four_domain_nest()
    ex = nest.setup_multidomain(doms, extra_halo_buffer=0, extra_cells_in_halo=0)
    return doms, ex


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_recv_metadata_known_answers(nest4, k):
    doms, _ = nest4
    np.testing.assert_array_equal(doms[k - 1].recv_metadata, np.array(EXPECTED[k]))


def test_layer_widths_and_sizes(nest4):
    doms, _ = nest4
    # euler parent: 2 cells; rk2 children: ceil(4*nt/3)*3, nt = 1, 2, 5
    # (the grandchild's neighbours are ratio-3 coarser, so it rounds to 3s).
    assert [d.nest_layer_width for d in doms] == [2, 6, 9, 21]
    assert doms[0].is_nesting_boundary == (False, False, False, False)
    assert doms[1].nx == (366, 216)
    assert doms[2].nx == (378, 228)
    assert doms[3].nx == (366, 357)


def test_exchanges_pair_send_and_recv_boxes(nest4):
    """Every real receive box has one send box covering the same area
    (multidomain_mod.f90:3180-3300 checks this to round-off)."""
    doms, ex = nest4
    nreal = sum(int(((m[:, 0] != k + 1) & (m[:, 0] > 0)).sum()) for k, m in enumerate(d.recv_metadata for d in doms))
    assert len(ex) == nreal
    for e in ex:
        s, r = doms[e.sender], doms[e.receiver]
        sx, sy = s.x(), s.y()
        rx, ry = r.x(), r.y()
        iL, iU, jL, jU = e.send_box
        a = (sx[iL - 1] - 0.5 * s.dx[0], sx[iU - 1] + 0.5 * s.dx[0], sy[jL - 1] - 0.5 * s.dx[1], sy[jU - 1] + 0.5 * s.dx[1])
        iL, iU, jL, jU = e.recv_box
        b = (rx[iL - 1] - 0.5 * r.dx[0], rx[iU - 1] + 0.5 * r.dx[0], ry[jL - 1] - 0.5 * r.dx[1], ry[jU - 1] + 0.5 * r.dx[1])
        tol = 100 * np.spacing(max(abs(v) for v in a))
        assert np.all(np.abs(np.array(a) - np.array(b)) <= tol), (e, a, b)
        rx_, ry_ = nest.exchange_cell_ratios(doms, e)
        ns = (e.send_box[1] - e.send_box[0] + 1, e.send_box[3] - e.send_box[2] + 1)
        nr = (e.recv_box[1] - e.recv_box[0] + 1, e.recv_box[3] - e.recv_box[2] + 1)
        if s.dx[0] > r.dx[0]:
            assert (ns[0] * rx_, ns[1] * ry_) == nr
        else:
            assert (nr[0] * rx_, nr[1] * ry_) == ns


def test_priority_cells_are_not_received(nest4):
    """A domain never receives into its own priority cells."""
    doms, ex = nest4
    for e in ex:
        d = doms[e.receiver]
        iL, iU, jL, jU = e.recv_box
        assert np.all(d.priority_domain_index[iL - 1:iU, jL - 1:jU] == e.sender + 1)
