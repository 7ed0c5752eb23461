"""Test helpers: build the same SWALS domain on the GPU (C ABI) and in the
CPU oracle, from one set of Domain keyword arguments."""
import numpy as np

from oracle import oracle as orc


def oracle_from_kw(kw, real32=False, variant="strict"):
    nx, ny = kw["nx"]
    return orc.OracleDomain(
        nx, ny, kw["lw"], lower_left=kw.get("lower_left", (0.0, 0.0)),
        timestepping_method=kw.get("timestepping_method", "rk2"),
        spherical=kw.get("spherical", False), coriolis=kw.get("coriolis"),
        nofriction=kw.get("nofriction", False),
        truely_linear=kw.get("linear_solver_is_truely_linear", True),
        friction_type=kw.get("friction_type", "manning"), cfl=kw.get("cfl"), theta=kw.get("theta"),
        msl_linear=kw.get("msl_linear", 0.0), linear_friction_coeff=kw.get("linear_friction_coeff", 0.0),
        boundary_exterior=kw.get("boundary_exterior", (True, True, True, True)),
        bc_kind=kw.get("boundary_kind", 0), bf_kind=kw.get("boundary_function_kind", 0),
        bf_params=kw.get("boundary_function_params", ()),
        xL=kw.get("xL", 0), xU=kw.get("xU", 0), yL=kw.get("yL", 0), yU=kw.get("yU", 0),
        compute_fluxes_inner_method=kw.get("compute_fluxes_inner_method", "DE1_low_fr_diffusion"),
        real32=real32, variant=variant)


def make_pair(kw, U, manning_sq=None, real32=False, oracle_real32=False):
    from ptha_b200 import Domain
    g = Domain(**kw, real_bytes=4 if real32 else 8)
    g.set_U(U)
    o = oracle_from_kw(kw, real32=oracle_real32)
    o.U[:] = U
    if manning_sq is not None:
        g.set_manning_squared(manning_sq)
        o.manning_squared[:] = manning_sq
    return g, o


def rel_err(a, b, floor=1.0, mask=None):
    """max|a-b| / max(max|b|, floor), optionally over a mask of cells.
    Wall cells (elevation 1e6) are excluded by the callers so that their
    large stage does not hide errors in the water."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if mask is not None:
        a = a[..., mask]
        b = b[..., mask]
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), floor))


def water_mask(elv):
    return np.asarray(elv) < 0.5e6


def report(tag, g, o):
    U = g.get_U()
    out = {}
    m = water_mask(o.U[3])
    for k, name in enumerate(["STG", "UH", "VH", "ELV"]):
        out[name] = rel_err(U[k], o.U[k], mask=m)
        out[name + "_exact"] = float(np.mean(U[k].astype(np.float64) == o.U[k].astype(np.float64)))
    print(tag, out)
    return U, out
