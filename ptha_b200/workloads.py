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
