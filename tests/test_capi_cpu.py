"""C-ABI checks that need no GPU: the library builds and loads, exports every
symbol include/swals_gpu.h declares, and rejects invalid descriptors the way
the reference's generic_stop paths do (as status codes)."""
import ctypes
import os
import re

import pytest

from ptha_b200 import _lib
from ptha_b200._lib import SwalsError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names.update(re.findall(r"^\s*(?:int|const char \*|void)\s+\**(swals_gpu_\w+)\s*\(", txt, re.M))
    return sorted(names)


def test_header_declares_symbols():
    syms = declared_symbols()
    assert "swals_gpu_evolve_one_step" in syms
    assert len(syms) >= 25


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    # and the Python binding covers the same set
    assert set(declared_symbols()) <= set(_lib.EXPORTED)


def test_version_string():
    assert b"sm_100a" in _lib.lib().swals_gpu_version()


def _create(**over):
    from ptha_b200 import Domain
    kw = dict(nx=(16, 16), lw=(16.0, 16.0), timestepping_method="linear")
    kw.update(over)
    return Domain(**kw)


def test_unknown_method_is_rejected():
    with pytest.raises(SwalsError) as e:
        _create(timestepping_method="not_a_method")
    assert e.value.code == 2 and "not recognized" in str(e.value)


@pytest.mark.parametrize("m", ["cliffs"])
def test_valid_but_unimplemented_methods(m):
    with pytest.raises(SwalsError) as e:
        _create(timestepping_method=m)
    assert e.value.code == 3


def test_host_callbacks_are_rejected():
    with pytest.raises(SwalsError) as e:
        _create(boundary_subroutine=lambda d: None)
    assert e.value.code == 6
    with pytest.raises(SwalsError) as e:
        _create(forcing_subroutine=lambda d, dt: None)
    assert e.value.code == 6


def test_coriolis_requires_spherical():
    with pytest.raises(SwalsError) as e:
        _create(coriolis=True, spherical=False)
    assert e.value.code == 1


def test_trailing_blanks_in_method_string_are_ignored_like_fortran_trim():
    # A Fortran character(len=charlen) is blank padded; TRIM() comparison ignores that.
    try:
        _create(timestepping_method="linear" + " " * 20)
    except SwalsError as e:
        assert e.code == 9  # only the missing device stops it on a CPU box
        return
    # on a GPU box the domain is created


def test_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(SwalsError) as e:
        _create()
    assert e.value.code == 9


def test_boundary_kind_checks():
    import torch
    # Flather is a known kind: on a CPU box only the missing device stops it.
    if not torch.cuda.is_available():
        with pytest.raises(SwalsError) as e:
            _create(boundary_kind=_lib.BC_FLATHER)
        assert e.value.code == 9
    with pytest.raises(SwalsError) as e:
        _create(boundary_kind=4)
    assert e.value.code == 1
    with pytest.raises(SwalsError) as e:
        _create(boundary_kind=_lib.BC_FLATHER, boundary_function_kind=7)
    assert e.value.code == 6
    with pytest.raises(SwalsError) as e:
        _create(boundary_kind=_lib.BC_FLATHER, exterior_cells_width=1)
    assert e.value.code == 3


def test_flux_method_checks():
    with pytest.raises(SwalsError) as e:
        _create(timestepping_method="rk2", compute_fluxes_inner_method="EEC")
    assert e.value.code == 3


@pytest.mark.parametrize("region", [dict(xU=17), dict(yU=20), dict(xL=9, xU=8), dict(yL=12, yU=3)])
def test_update_region_outside_the_grid_is_rejected(region):
    """xL..xU, yL..yU must lie inside 1..nx, 1..ny (the reference's loop
    bounds); checked before any device work."""
    with pytest.raises(SwalsError) as e:
        _create(**region)
    assert e.value.code == 1 and "update region" in str(e.value)
