"""The library's native nesting metadata builder (swals_md_build_metadata,
multidomain_mod.f90:2663-3553) against the reference's known answers and
against the numpy restatement (ptha_b200.nesting.setup_multidomain), field
by field: widened extents, layer widths, nesting boundaries, parent ratios,
priority-domain arrays, receive boxes and the exchange list.  Host code:
runs without a GPU."""
import copy

import numpy as np
import pytest

from ptha_b200 import _lib
from ptha_b200 import nesting as nest

from nest_cases import two_level_nest
from test_nesting_metadata import EXPECTED, four_domain_nest


def _both(doms, **kw):
    a, b = copy.deepcopy(doms), copy.deepcopy(doms)
    ea = nest.setup_multidomain(a, **kw)
    eb = nest.setup_multidomain_native(b, **kw)
    return a, ea, b, eb


def _same(a, ea, b, eb):
    for da, db in zip(a, b):
        assert da.nx == db.nx and da.lw == db.lw and da.lower_left == db.lower_left
        assert da.dx == db.dx
        assert da.nest_layer_width == db.nest_layer_width
        assert da.is_nesting_boundary == db.is_nesting_boundary
        assert da.max_parent_dx_ratio == db.max_parent_dx_ratio
        np.testing.assert_array_equal(da.interior_bounding_box, db.interior_bounding_box)
        np.testing.assert_array_equal(da.priority_domain_index, db.priority_domain_index)
        np.testing.assert_array_equal(da.priority_domain_image, db.priority_domain_image)
        np.testing.assert_array_equal(da.recv_metadata, db.recv_metadata)
    assert ea == eb


def test_four_domain_nest_known_answers():
    a, ea, b, eb = _both(four_domain_nest(), extra_halo_buffer=0, extra_cells_in_halo=0)
    for k in EXPECTED:
        np.testing.assert_array_equal(b[k - 1].recv_metadata, np.array(EXPECTED[k]))
    _same(a, ea, b, eb)


@pytest.mark.parametrize("case", [
    dict(ratio=3, child_method="rk2", parent_method="linear"),
    dict(ratio=3, child_method="rk2", parent_method="rk2", child_nt=2),
    dict(ratio=5, child_method="midpoint", parent_method="leapfrog_nonlinear"),
    dict(ratio=2, child_method="rk2n", parent_method="leapfrog_linear_plus_nonlinear_friction", n=(50, 45)),
])
def test_two_level_nests(case):
    _same(*_both(two_level_nest(**case)))


def test_default_halo_settings_and_eddy_viscosity():
    doms = four_domain_nest()
    doms[1].use_eddy_viscosity = True
    doms[2].minimum_nesting_layer_thickness = 9
    _same(*_both(doms))


def test_periodic():
    pxs, pys = (-10.0, 350.0), (-80.0, 90.0)
    s = nest.NestDomain((-10.0, -80.0), (360.0, 170.0), (200, 200), "euler", 1)
    _same(*_both([s], periodic_xs=pxs, periodic_ys=pys))
    c = nest.NestDomain((0.0, 0.0), (100000.0, 40000.0), (100, 40), "linear", 1)
    _same(*_both([c], periodic_xs=(0.0, 100000.0)))


def test_errors():
    with pytest.raises(_lib.SwalsError):   # two domains with the same cell size overlap
        nest.setup_multidomain_native([nest.NestDomain((0.0, 0.0), (10.0, 10.0), (10, 10), "rk2", 1),
                                       nest.NestDomain((5.0, 5.0), (10.0, 10.0), (10, 10), "rk2", 1)])
    with pytest.raises(_lib.SwalsError):   # unknown method
        nest.setup_multidomain_native([nest.NestDomain((0.0, 0.0), (10.0, 10.0), (10, 10), "nope", 1)])
