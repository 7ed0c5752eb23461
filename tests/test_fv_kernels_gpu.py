"""Every form of the finite-volume stage kernels against the oracle, bit for bit.

The FV stages (DE1_low_fr_diffusion fluxes, theta wet/dry limiter,
update_U with Manning friction; domain_mod.f90:1360-1582,
domain_mod_compute_fluxes_DE1_inner_include.f90,
domain_mod_update_U_DE1_inner_include.f90) run in one of three kernel forms:
shared-memory tiles (SWALS_FV_KERNEL=tile), register-streaming warp strips
(SWALS_FV_STREAM=stream) and streaming strips with their carried rows in
shared memory, one warp (SWALS_FV_STREAM=srow) or the CTA's four warps
(SWALS_FV_STREAM=crow) per strip; by default grids of 1.5 M cells and more
take the CTA-wide strips, smaller ones the one-warp shared-memory rows for
FP64 update stages and registers for the rest.  Adaptive steps add a flux
pass that stores each cell's dt-independent update terms and a per-cell
update once dt is known.  Each form runs here on widths that cut the 28-
and 124-column strips every way (one partial strip, exactly one or two
strips, ragged last strips) and heights that leave short last segments, on a beach where
a wave runs up and the wet/dry front moves, with rk2 (adaptive and fixed
dt), euler, midpoint and rk2n, and on a spherical patch with Coriolis; FP64
against the IEEE-strict oracle, FP32 against the default form bit for bit.
"""
import numpy as np
import pytest

from pairs import make_pair

pytestmark = pytest.mark.gpu

FORMS = {
    "default": {},
    "tile": {"SWALS_FV_KERNEL": "tile"},
    "stream": {"SWALS_FV_STREAM": "stream"},
    "srow": {"SWALS_FV_STREAM": "srow"},
    "crow": {"SWALS_FV_STREAM": "crow"},
}


def _set_form(monkeypatch, form):
    for k in ("SWALS_FV_KERNEL", "SWALS_FV_STREAM"):
        monkeypatch.delenv(k, raising=False)
    for k, v in FORMS[form].items():
        monkeypatch.setenv(k, v)


def _beach(nx, ny, dx=40.0, depth=20.0, seed=5, method="rk2"):
    """A plane beach rising along x (slope 1/20, to +5 m) with seeded
    bumps, a 1.5 m hump offshore that runs up the beach, Manning n 0.03;
    no boundary routine (the outer cells stay put)."""
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    X, Y = np.meshgrid(x, y)
    elv = np.clip(-depth + (X - 0.45 * nx * dx) / 20.0, -depth, 5.0)
    for _ in range(6):
        bx, by = rng.uniform(0, nx * dx), rng.uniform(0, ny * dx)
        elv = elv + 0.8 * np.exp(-((X - bx) ** 2 + (Y - by) ** 2) / (2.0 * (3.0 * dx) ** 2))
    U = np.zeros((4, ny, nx))
    U[3] = elv
    hump = 1.5 * np.exp(-((X - 0.3 * nx * dx) ** 2 + (Y - 0.5 * ny * dx) ** 2) / (2.0 * (4.0 * dx) ** 2))
    U[0] = np.where(elv < 0.0, hump, elv)
    U[0] = np.maximum(U[0], elv)
    kw = dict(nx=(nx, ny), lw=(nx * dx, ny * dx), lower_left=(0.0, 0.0), timestepping_method=method)
    return kw, U, np.full((ny, nx), 0.03 ** 2)


def _assert_exact(g, o, tag):
    Ug = g.get_U()
    for k, name in enumerate(("STG", "UH", "VH")):
        np.testing.assert_array_equal(Ug[k], o.U[k], err_msg=f"{tag} {name}")
    np.testing.assert_array_equal(g.max_stage(), o.max_stage, err_msg=f"{tag} max_stage")
    st = g.state()
    assert st.time == o.time, tag
    assert st.negative_depth_fix_counter == o.negative_depth_fix_counter, tag
    return Ug


@pytest.mark.parametrize("form", list(FORMS))
@pytest.mark.parametrize("shape", [(30, 25), (56, 40), (97, 61), (124, 37), (130, 150)])
@pytest.mark.parametrize("adaptive", [True, False])
def test_rk2_form_matches_oracle(form, shape, adaptive, monkeypatch):
    _set_form(monkeypatch, form)
    kw, U, nsq = _beach(*shape)
    g, o = make_pair(kw, U, manning_sq=nsq)
    dt = None if adaptive else 0.5 * o.nonlinear_stationary_timestep_max()
    for _ in range(80):
        g.evolve_one_step(dt)
        o.evolve_one_step(dt)
    Ug = _assert_exact(g, o, f"rk2 {form} {shape} adaptive={adaptive}")
    if adaptive:   # the wave has reached the beach: the wet/dry branches ran
        wet0 = (U[0] - U[3]) > 1e-5
        assert np.any(((Ug[0] - U[3]) > 1e-5) & ~wet0), "the front never moved"
    g.close()


@pytest.mark.parametrize("form", list(FORMS))
@pytest.mark.parametrize("method", ["euler", "midpoint", "rk2n"])
def test_other_fv_methods_form_matches_oracle(form, method, monkeypatch):
    _set_form(monkeypatch, form)
    kw, U, nsq = _beach(97, 61, method=method)
    g, o = make_pair(kw, U, manning_sq=nsq)
    for _ in range(60):
        g.evolve_one_step()
        o.evolve_one_step()
    _assert_exact(g, o, f"{method} {form}")
    g.close()


@pytest.mark.parametrize("form", list(FORMS))
def test_rk2_form_spherical_coriolis(form, monkeypatch):
    from ptha_b200 import workloads
    _set_form(monkeypatch, form)
    kw, U = workloads.spherical_patch(nx=101, ny=67)
    kw.update(timestepping_method="rk2", coriolis=True)
    g, o = make_pair(kw, U, manning_sq=np.full(U[0].shape, 0.025 ** 2))
    for _ in range(60):
        g.evolve_one_step()
        o.evolve_one_step()
    _assert_exact(g, o, f"rk2 spherical coriolis {form}")
    g.close()


@pytest.mark.parametrize("adaptive", [True, False])
def test_fp32_forms_agree_bit_for_bit(adaptive, monkeypatch):
    """FP32 state: every form gives the default form's bits."""
    from ptha_b200 import Domain
    kw, U, nsq = _beach(97, 61)
    out = {}
    for form in FORMS:
        _set_form(monkeypatch, form)
        g = Domain(**kw, real_bytes=4)
        g.set_U(U)
        g.set_manning_squared(nsq)
        dt = None if adaptive else 0.02
        for _ in range(80):
            g.evolve_one_step(dt)
        out[form] = (g.get_U(), g.max_stage(), g.state().time)
        g.close()
    for form in FORMS:
        for k in range(3):
            np.testing.assert_array_equal(out[form][0][k], out["default"][0][k], err_msg=f"{form} {k}")
        np.testing.assert_array_equal(out[form][1], out["default"][1], err_msg=f"{form} max_stage")
        assert out[form][2] == out["default"][2], form


@pytest.mark.parametrize("form", ["crow", "srow", "stream"])
@pytest.mark.parametrize("rows", [1, 5, 16, 24, 80])
def test_segment_rows_match_oracle(form, rows, monkeypatch):
    """Any number of rows per strip segment (SWALS_FV_ROWS; chosen from the
    grid otherwise) gives the oracle's bits, segments of more than 64 rows
    (whose row constants are not kept in shared memory) included."""
    _set_form(monkeypatch, form)
    monkeypatch.setenv("SWALS_FV_ROWS", str(rows))
    kw, U, nsq = _beach(97, 61 if rows <= 24 else 150)   # 150 rows: segments of 80 and 70
    g, o = make_pair(kw, U, manning_sq=nsq)
    for _ in range(40):
        g.evolve_one_step()
        o.evolve_one_step()
    _assert_exact(g, o, f"rk2 {form} rows={rows}")
    g.close()
