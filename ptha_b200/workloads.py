"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference publishes no datasets for this path; these generators stand in
for them with the stated sizes, bathymetry shapes and seeds.  Each returns a
dict of Domain keyword arguments plus initial arrays in the (4, ny, nx) layout.
"""
from __future__ import annotations

import numpy as np

from ._lib import BC_NONE, BC_STAGE_TRANSMISSIVE_NORMAL_MOMENTUM, BF_SOLITARY_WEST_WALLS

WALL = 1.0e6
GRAVITY = 9.8


def cell_centres(n, lw, ll):
    return ll + ((np.arange(1, n + 1) - 0.5) / n) * lw


def linear_gaussian_basin(n=400, dx=1000.0, depth=4000.0, amp=1.0, sigma=20.0e3, wall_cells=2):
    """Plain linear leapfrog: Cartesian n x n, flat bed, Gaussian hump, walls
    made by raising the outer `wall_cells` rows/columns to +100 m (the
    reference's wall idiom), 9 gauges on a 3x3 lattice at 1/4, 1/2, 3/4."""
    lw = n * dx
    x = cell_centres(n, lw, 0.0)
    X, Y = np.meshgrid(x, x)
    U = np.zeros((4, n, n))
    U[3] = -depth
    U[3][:wall_cells, :] = 100.0
    U[3][-wall_cells:, :] = 100.0
    U[3][:, :wall_cells] = 100.0
    U[3][:, -wall_cells:] = 100.0
    c = lw / 2.0
    U[0] = amp * np.exp(-((X - c) ** 2 + (Y - c) ** 2) / (2.0 * sigma ** 2))
    U[0] = np.maximum(U[0], np.minimum(U[3], U[0]))
    g = np.array([lw / 4, lw / 2, 3 * lw / 4])
    gauges = np.array([[gx, gy] for gy in g for gx in g])
    return dict(nx=(n, n), lw=(lw, lw), lower_left=(0.0, 0.0), timestepping_method="linear"), U, gauges


def rk2_beach(n=2048, dx=10.0, depth=50.0, top=10.0, slope=1.0 / 40.0, toe=17580.0, n_bumps=30,
              bump_amp=0.5, bump_sigma=50.0, seed=2, H_over_d=0.1, manning_n=0.025):
    """Nonlinear FV rk2 with wetting/drying: planar beach rising from -depth to
    +top along x, seeded Gaussian roughness, Manning friction, solitary wave
    entering through the west boundary; walls elsewhere."""
    lw = n * dx
    x = cell_centres(n, lw, 0.0)
    X, Y = np.meshgrid(x, x)
    elv = np.clip(-depth + (X - toe) * slope, -depth, top)
    rng = np.random.default_rng(seed)
    cx = rng.uniform(0.0, lw, n_bumps)
    cy = rng.uniform(0.0, lw, n_bumps)
    for bx, by in zip(cx, cy):
        elv = elv + bump_amp * np.exp(-((X - bx) ** 2 + (Y - by) ** 2) / (2.0 * bump_sigma ** 2))
    elv[:, 0] = -depth
    elv[0, :] = WALL
    elv[-1, :] = WALL
    elv[:, -1] = WALL
    U = np.zeros((4, n, n))
    U[3] = elv
    U[0] = np.maximum(elv, 0.0)
    U[0][0, :] = WALL
    U[0][-1, :] = WALL
    U[0][:, -1] = WALL
    H = H_over_d * depth
    k = np.sqrt(3.0 * H / (4.0 * depth ** 3))
    x0 = x[0] - 5.0 / k
    g = np.array([toe - 1500.0, toe + 800.0, toe + 1800.0])
    gy = np.array([lw / 4, lw / 2, 3 * lw / 4])
    gauges = np.array([[a, b] for b in gy for a in g])
    kw = dict(nx=(n, n), lw=(lw, lw), lower_left=(0.0, 0.0), timestepping_method="rk2",
              boundary_kind=BC_STAGE_TRANSMISSIVE_NORMAL_MOMENTUM, boundary_function_kind=BF_SOLITARY_WEST_WALLS,
              boundary_function_params=(H, depth, x0))
    return kw, U, gauges, manning_n ** 2


def spherical_patch(nx=120, ny=80, dlon=1.0 / 30.0, ll=(150.0, -30.0), depth_range=(-6000.0, -10.0), seed=6):
    """Small spherical grid with a smoothed random bathymetry and land mask."""
    rng = np.random.default_rng(seed)
    f = rng.standard_normal((ny, nx))
    # separable box smoothing (cheap, deterministic)
    for _ in range(6):
        f = (np.roll(f, 1, 0) + f + np.roll(f, -1, 0)) / 3.0
        f = (np.roll(f, 1, 1) + f + np.roll(f, -1, 1)) / 3.0
    lo, hi = np.percentile(f, [1, 99])
    elv = depth_range[0] + (f - lo) / (hi - lo) * (depth_range[1] - depth_range[0])
    elv = np.clip(elv, depth_range[0], depth_range[1])
    land = f > (lo + 0.85 * (hi - lo))
    elv[land] = 100.0
    elv[:2, :] = 100.0
    elv[-2:, :] = 100.0
    elv[:, :2] = 100.0
    elv[:, -2:] = 100.0
    lw = (nx * dlon, ny * dlon)
    lon = cell_centres(nx, lw[0], ll[0])
    lat = cell_centres(ny, lw[1], ll[1])
    LON, LAT = np.meshgrid(lon, lat)
    U = np.zeros((4, ny, nx))
    U[3] = elv
    c0 = (lon[nx // 2], lat[ny // 2])
    U[0] = 1.5 * np.exp(-(((LON - c0[0]) * 60) ** 2 + ((LAT - c0[1]) * 60) ** 2) / (2.0 * 6.0 ** 2))
    U[0] = np.where(elv > 0, 0.0, U[0])
    return dict(nx=(nx, ny), lw=lw, lower_left=ll, spherical=True), U


def dipoles(lon, lat, count, seed, band=((150.0, -40.0), (190.0, -10.0)), width_km=400.0):
    """Compact dipole uplift patches in a band: a random centre within
    width_km of the band's axis, extent L in U[50, 200] km, amplitude A in
    U[0.5, 3] m, eta = A [G(s - L/4, n) - G(s + L/4, n)] with Gaussians of
    sigma L/6 in band-aligned coordinates; evaluated within 3L of the centre
    (zero beyond).  Returns `count` (ny, nx) arrays."""
    rng = np.random.default_rng(seed)
    (x0, y0), (x1, y1) = band
    km_deg = 111.19
    ang = np.arctan2(y1 - y0, x1 - x0)
    out = []
    for _ in range(count):
        t = rng.uniform(0.0, 1.0)
        off = rng.uniform(-0.5, 0.5) * width_km / km_deg
        cx = x0 + t * (x1 - x0) - off * np.sin(ang)
        cy = y0 + t * (y1 - y0) + off * np.cos(ang)
        L = rng.uniform(50.0, 200.0)
        A = rng.uniform(0.5, 3.0)
        eta = np.zeros((len(lat), len(lon)))
        r_deg = 3.0 * L / km_deg
        ii = np.flatnonzero(np.abs(lon - cx) <= r_deg / max(np.cos(np.deg2rad(cy)), 0.2))
        jj = np.flatnonzero(np.abs(lat - cy) <= r_deg)
        if len(ii) and len(jj):
            LON, LAT = np.meshgrid(lon[ii], lat[jj])
            dx = (LON - cx) * km_deg * np.cos(np.deg2rad(cy))
            dy = (LAT - cy) * km_deg
            s_ = dx * np.cos(ang) + dy * np.sin(ang)
            n_ = -dx * np.sin(ang) + dy * np.cos(ang)
            sg = L / 6.0
            eta[np.ix_(jj, ii)] = A * (np.exp(-((s_ - L / 4) ** 2 + n_ ** 2) / (2 * sg ** 2)) -
                                       np.exp(-((s_ + L / 4) ** 2 + n_ ** 2) / (2 * sg ** 2)))
        out.append(eta)
    return out


def coast_elevation(lon, lat, coasts):
    """Deep ocean (-4000 m) shoaling over a 60 km shelf slope to -50 m, then a
    1/40 coastal ramp to +10 m, for each straight coastline (lon0, lat0,
    bearing of the seaward normal, (lon_min, lon_max, lat_min, lat_max) of
    the region it shapes)."""
    km = 111.19
    elv = np.full(np.broadcast(lon, lat).shape, -4000.0)
    for (x0, y0, ang, box) in coasts:
        inside = (lon >= box[0]) & (lon <= box[1]) & (lat >= box[2]) & (lat <= box[3])
        d = ((lon - x0) * np.cos(np.deg2rad(y0)) * np.cos(ang) + (lat - y0) * np.sin(ang)) * km
        ramp = np.clip(-50.0 - (d * 1000.0) / 40.0, -50.0, 10.0)           # within ~2.4 km of the coast
        shelf = np.clip(-50.0 - d * (3950.0 / 60.0), -4000.0, -50.0)        # 60 km shelf slope
        e = np.where(d <= 0.0, ramp, shelf)
        elv = np.where(inside, np.maximum(elv, e), elv)
    return elv


def batched_grid(nx=3600, ny=2400):
    """The batched linear configuration's grid: spherical, 1 arcmin at
    3600 x 2400 (lon 140E.., lat 45S..), smoothed random bathymetry from
    -6000 to -10 m with land at +100 m (seed 3).  Returns the Domain keyword
    arguments (FP32 'linear'), U (4, ny, nx), cell-centre lon and lat."""
    dl = 1.0 / 60.0 * (3600 / nx)
    gkw, U0 = spherical_patch(nx=nx, ny=ny, dlon=dl, ll=(140.0, -45.0), seed=3)
    gkw = dict(gkw, timestepping_method="linear", real_bytes=4)
    lon = gkw["lower_left"][0] + (np.arange(nx) + 0.5) * dl
    lat = gkw["lower_left"][1] + (np.arange(ny) + 0.5) * dl
    return gkw, U0, lon, lat


def batched_instance_stage(lon, lat, wet, q, nbatch):
    """Initial stage of instance q of a batch of nbatch: one dipole whose
    seed depends on q only (so the instances do not depend on how a batch is
    split over ranks or chunks), zero on land."""
    seeds = np.random.default_rng(4).integers(0, 2 ** 31, size=nbatch)
    eta = dipoles(lon, lat, 1, seed=int(seeds[q]))[0]
    return np.where(wet, eta, 0.0)


def batched_gauges(lon, lat, wet, n=200, seed=5):
    """n gauges at random wet cells (lon, lat pairs)."""
    gr = np.random.default_rng(seed)
    wj, wi = np.nonzero(wet)
    pick = gr.choice(wj.size, size=n, replace=False)
    return np.stack([lon[wi[pick]], lat[wj[pick]]], axis=1)


def adjoint_case(nx=1200, ny=800):
    """The adjoint configuration: spherical 2 arcmin at 1200 x 800 (FP64
    'linear'), smoothed random bathymetry (seed 6), 30 gauges at random wet
    cells (seed 7), a hidden dipole source (seed 8) whose waveforms are the
    target.  Returns (Domain kwargs, U0 (4, ny, nx), gauges (30, 2), the
    hidden source's initial stage (ny, nx), gauge cell indices (30, 2) as
    (row, column))."""
    dl = 2.0 / 60.0 * (1200 / nx)
    gkw, U0 = spherical_patch(nx=nx, ny=ny, dlon=dl, ll=(150.0, -40.0), seed=6)
    gkw = dict(gkw, timestepping_method="linear")
    lon = gkw["lower_left"][0] + (np.arange(nx) + 0.5) * dl
    lat = gkw["lower_left"][1] + (np.arange(ny) + 0.5) * dl
    wet = U0[3] < 0
    rng = np.random.default_rng(7)
    wi = np.argwhere(wet)
    pick = wi[rng.choice(len(wi), 30, replace=False)]
    gauges = np.stack([lon[pick[:, 1]], lat[pick[:, 0]]], axis=1)
    eta_t = dipoles(lon, lat, 1, seed=8, band=((lon[0] + 5, lat[0] + 5), (lon[-1] - 5, lat[-1] - 5)))[0]
    return gkw, U0, gauges, np.where(wet, eta_t, 0.0), pick


def adjoint_window(nx=1200, ny=800):
    """The 300 x 200 source window of the adjoint configuration (rows,
    columns), centred on the grid, scaled with the grid."""
    wy, wx = ny * 200 // 800, nx * 300 // 1200
    j0, i0 = (ny - wy) // 2, (nx - wx) // 2
    return slice(j0, j0 + wy), slice(i0, i0 + wx)


NEST_COARSE = 1.0 / 15.0     # coarse cell of the nested configuration (4 arcmin)


def nested_specs(nts=(1, 1, 1, 1), scale=1):
    """The nested configuration's four domains (interior extents): a coarse
    'linear' band 5400 x 1800 at 4 arcmin over 0-360 x 60S-60N, one
    ratio-3 'rk2' 900 x 900 domain and two ratio-9 'rk2' wet/dry domains
    (1197 x 801 and 702 x 1098: the nearest sizes that are whole parent
    cells).  `scale` 3, 5 or 15 shrinks every domain by that factor (same
    geometry, coarser cells, nested edges still on parent cell edges) for
    quick checks.  Returns NestDomain objects and the coastlines of
    coast_elevation."""
    import math
    from .nesting import NestDomain
    if scale not in (1, 3, 5, 15):
        raise ValueError("scale must be 1, 3, 5 or 15 (nested edges on parent cell edges)")
    c = NEST_COARSE * scale
    f3, f9 = c / 3.0, c / 9.0
    n = lambda v: v // scale                    # noqa: E731
    n9 = lambda v: max(9, v // scale // 9 * 9)  # noqa: E731  (whole parent cells)
    specs = [
        NestDomain((0.0, -60.0), (n(5400) * c, n(1800) * c), (n(5400), n(1800)), "linear", nts[0]),
        NestDomain((140.0, -40.0), (n(900) * f3, n(900) * f3), (n(900), n(900)), "rk2", nts[1]),
        NestDomain((141.0 + 2 * c, -39.0), (n9(1197) * f9, n9(801) * f9), (n9(1197), n9(801)), "rk2", nts[2]),
        NestDomain((152.0, -35.0), (n9(702) * f9, n9(1098) * f9), (n9(702), n9(1098)), "rk2", nts[3]),
    ]
    coasts = [(141.0 + 2 * c + n9(1197) * f9 * 0.75, -39.0 + n9(801) * f9 * 0.5, 0.0,
               (140.5, 151.0, -39.5, -32.5)),
              (152.0 + n9(702) * f9 * 0.5, -35.0 + n9(1098) * f9 * 0.8, math.pi / 2,
               (151.5, 157.7, -35.5, -26.3))]
    return specs, coasts


def nested_elevation(spec, k, coasts):
    """Elevation (ny, nx) of domain k of the nested configuration (after
    setup widened it): coastal ramps, walls on the coarse band's north and
    south rings."""
    lon, lat = spec.x(), spec.y()
    LON, LAT = np.meshgrid(lon, lat)
    elv = coast_elevation(LON, LAT, coasts)
    if k == 0:
        elv[:2, :] = 100.0
        elv[-2:, :] = 100.0
    return elv


def nested_initial_state(spec, k, coasts, source_seed=11, elevation=None):
    """U (4, ny, nx) of domain k of the nested configuration (after setup
    widened it): nested_elevation (or the one given), one dipole source
    (seed source_seed) on the wet cells, stage = elevation on land.  Source
    seeds 11, 12, ... are the instances of the batched (16-source) form."""
    lon, lat = spec.x(), spec.y()
    elv = nested_elevation(spec, k, coasts) if elevation is None else elevation
    eta = dipoles(lon, lat, 1, seed=source_seed, band=((144.0, -37.0), (150.0, -30.0)))[0]
    U = np.zeros((4, spec.nx[1], spec.nx[0]))
    U[3] = elv
    U[0] = np.where(elv < 0, eta, elv)
    return U
