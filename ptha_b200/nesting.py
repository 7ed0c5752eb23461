"""Multidomain nesting metadata: which cells of each domain receive data from
which other domain, and which cells are sent.

This is the host-side setup of SWALS's ``multidomain_type`` for one process
(``multidomain_mod.f90:2663-3553``), restated in numpy so that a caller of the
GPU path can build the exchange tables the device kernels consume:

* each domain's nesting-layer width (``compute_multidomain_nesting_layer_width``,
  ``multidomain_mod.f90:620-716``; ``get_domain_nesting_layer_thickness``
  ``:1803-1852``), after which nesting boundaries are widened by that many
  cells (``:2860-2895``);
* the priority domain of every cell (``find_priority_domain_containing_xy``
  ``:1538-1677``: the finest domain whose interior bounding box contains the
  cell centre);
* the receive boxes (``convert_priority_domain_info_to_boxes`` ``:718-958``:
  row-wise run-length encoding of the priority domain within
  ``nest_layer_width`` of the domain's own priority cells, rows merged while
  their runs match);
* the matching send boxes (``:3090-3140``: the sender's cells whose centres
  lie inside the receive box's edges).

All coordinates are computed with the reference's expressions in IEEE double
so that the integer boxes match the reference's bit for bit (the reference's
own known answers for its 4-domain nest are re-encoded in
``tests/test_nesting_metadata.py``).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from fractions import Fraction
from typing import List, Optional, Sequence, Tuple

import numpy as np

HUGE = float(np.finfo(np.float64).max)
NULL_INDEX = 0  # multidomain_mod.f90:165
NULL_IMAGE = 0

# timestepping_metadata_mod.f90:60-160 -- cells of halo consumed by one
# evolve_one_step, and whether the method uses a staggered grid.
NESTING_THICKNESS = {
    "rk2": 4, "rk2n": 10, "midpoint": 4, "euler": 2, "linear": 2,
    "leapfrog_linear_plus_nonlinear_friction": 2, "cliffs": 2, "leapfrog_nonlinear": 3,
}
STAGGERED = {
    "rk2": 0, "rk2n": 0, "midpoint": 0, "euler": 0, "linear": 1,
    "leapfrog_linear_plus_nonlinear_friction": 1, "cliffs": 0, "leapfrog_nonlinear": 1,
}
# Methods whose nesting flux correction acts on the mass (STG) only
# (timestepping_metadata_mod.f90:189).
FLUX_CORRECTION_MASS_ONLY = {"linear", "leapfrog_linear_plus_nonlinear_friction", "leapfrog_nonlinear"}

EXTRA_CELLS_IN_HALO_DEFAULT = 1  # multidomain_mod.f90:102
EXTRA_HALO_BUFFER_DEFAULT = 0    # multidomain_mod.f90:90


@dataclass
class NestDomain:
    """The geometry fields of ``domain_type`` that nesting setup reads and
    writes.  ``lower_left``, ``lw`` and ``nx`` are the interior extent before
    setup; setup widens them on nesting boundaries."""
    lower_left: Tuple[float, float]
    lw: Tuple[float, float]
    nx: Tuple[int, int]
    timestepping_method: str = "rk2"
    timestepping_refinement_factor: int = 1
    minimum_nesting_layer_thickness: int = 0
    use_eddy_viscosity: bool = False
    # Filled by setup_multidomain:
    dx: Tuple[float, float] = (0.0, 0.0)
    interior_bounding_box: Optional[np.ndarray] = None   # (4, 2): ll, lr, ur, ul
    max_parent_dx_ratio: float = 1.0
    is_nesting_boundary: Tuple[bool, bool, bool, bool] = (False, False, False, False)  # N, E, S, W
    nest_layer_width: int = 0
    priority_domain_index: Optional[np.ndarray] = None   # (nx, ny), 1-based domain indices
    priority_domain_image: Optional[np.ndarray] = None
    recv_metadata: Optional[np.ndarray] = None   # (nbox, 6): ind, img, iL, iU, jL, jU
    send_metadata: Optional[np.ndarray] = None   # (nbox, 8)

    @property
    def is_staggered_grid(self) -> int:
        return STAGGERED[self.timestepping_method]

    def x(self) -> np.ndarray:
        """domain%x (domain_mod.f90:941): ll + ((i - 1/2)/nx) * lw."""
        i = np.arange(1, self.nx[0] + 1, dtype=np.float64)
        return self.lower_left[0] + ((i - 0.5) / (self.nx[0] * 1.0)) * self.lw[0]

    def y(self) -> np.ndarray:
        j = np.arange(1, self.nx[1] + 1, dtype=np.float64)
        return self.lower_left[1] + ((j - 0.5) / (self.nx[1] * 1.0)) * self.lw[1]


@dataclass
class Exchange:
    """One receive box and the send box that feeds it.  Boxes are 1-based,
    inclusive ``(iL, iU, jL, jU)`` in the reference's index convention."""
    sender: int            # 0-based domain index
    receiver: int
    send_box: Tuple[int, int, int, int]
    recv_box: Tuple[int, int, int, int]
    recv_row: int          # row of the receiver's recv_metadata (0-based)
    send_row: int          # row of the sender's send_metadata (0-based)


def domain_xs_ys(d: NestDomain) -> Tuple[np.ndarray, np.ndarray]:
    """get_domain_xs_ys (multidomain_mod.f90:1854-1880): ll + (i - 1/2)*lw/nx."""
    i = np.arange(1, d.nx[0] + 1, dtype=np.float64)
    j = np.arange(1, d.nx[1] + 1, dtype=np.float64)
    xs = d.lower_left[0] + ((i - 0.5) * d.lw[0]) / d.nx[0]
    ys = d.lower_left[1] + ((j - 0.5) * d.lw[1]) / d.nx[1]
    return xs, ys


def _periodic_shift(v: np.ndarray, lo: float, hi: float, adjust: bool):
    """check_periodic for one coordinate array (multidomain_mod.f90:280-346).
    The shift is added in 128-bit precision and rounded to double, which is
    the correctly rounded sum of the two doubles."""
    v = np.array(v, dtype=np.float64, copy=True)
    below = v < lo
    above = v > hi
    if adjust:
        span = hi - lo
        for idx in np.flatnonzero(below):
            v[idx] = float(Fraction(span) + Fraction(float(v[idx])))
        for idx in np.flatnonzero(above):
            v[idx] = float(Fraction(-span) + Fraction(float(v[idx])))
    return v, below | above


def _inside_rectangle(bbox: np.ndarray, px: np.ndarray, py: np.ndarray) -> np.ndarray:
    """point_in_poly (util/points_in_poly_mod.f90:31-58) for the 4-vertex
    bounding box ll, lr, ur, ul: the crossing test evaluated edge by edge."""
    vx, vy = bbox[:, 0], bbox[:, 1]
    inside = np.zeros(px.shape, dtype=bool)
    for i in range(4):
        j = 3 if i == 0 else i - 1
        crosses = (vy[i] > py) != (vy[j] > py)
        with np.errstate(divide="ignore", invalid="ignore"):
            g0 = (vx[j] - vx[i]) * (py - vy[i]) / (vy[j] - vy[i]) + vx[i]
        inside ^= crosses & (px < g0)
    return inside


def find_priority_domain_containing_xy(domains: Sequence[NestDomain], xs, ys, periodic_xs, periodic_ys,
                                       error_domain_overlap_same_dx: bool = True):
    """multidomain_mod.f90:1538-1677.  Returns (index, image, dx) per point:
    the domain with the smallest cell area whose interior bounding box holds
    the point (1-based index; -1 where no domain holds it)."""
    xs = np.asarray(xs, dtype=np.float64)
    ys = np.asarray(ys, dtype=np.float64)
    n = xs.size
    ind = np.full(n, -1, dtype=np.int64)
    img = np.full(n, -1, dtype=np.int64)
    big = -math.sqrt(HUGE - 1.0e6)
    ddx = np.full((n, 2), big, dtype=np.float64)
    px, _ = _periodic_shift(xs, periodic_xs[0], periodic_xs[1], True)
    py, _ = _periodic_shift(ys, periodic_ys[0], periodic_ys[1], True)
    for di, d in enumerate(domains):
        bbox = d.interior_bounding_box
        if np.all(bbox == 0.0):
            continue
        inside = _inside_rectangle(bbox, px, py)
        area1 = d.dx[0] * d.dx[1]
        area2 = ddx[:, 0] * ddx[:, 1]
        take = inside & (area1 < area2)
        if error_domain_overlap_same_dx:
            clash = inside & ~take & (np.abs(area1 - area2) < 1.0e-2 * np.minimum(area1, area2))
            if np.any(clash):
                k = int(np.flatnonzero(clash)[0])
                raise ValueError(f"domains with the same cell size overlap around ({xs[k]}, {ys[k]})")
        ind[take] = di + 1
        img[take] = 1
        ddx[take, 0] = d.dx[0]
        ddx[take, 1] = d.dx[1]
    return ind, img, ddx


def _boundary_points(d: NestDomain, boundary: int, width: int):
    """find_priority_nesting_domains_along_a_boundary (multidomain_mod.f90:
    1679-1800): the cell centres ``width`` cells outside boundary 1..4
    (N, E, S, W), extended by ``width`` cells past each end."""
    dxs, dys = domain_xs_ys(d)
    dx, dy = d.dx
    if boundary in (1, 3):
        n1 = d.nx[0]
        n2 = n1 + 2 * width
        xs = np.empty(n2)
        xs[width:n2 - width] = dxs
        for i in range(1, width + 1):
            xs[i - 1] = dxs[0] - (width - (i - 1)) * dx
            xs[n2 - (width - i) - 1] = dxs[n1 - 1] + i * dx
        yv = dys[d.nx[1] - 1] + dy * width if boundary == 1 else dys[0] - dy * width
        ys = np.full(n2, yv)
    else:
        n1 = d.nx[1]
        n2 = n1 + 2 * width
        ys = np.empty(n2)
        ys[width:n2 - width] = dys
        for i in range(1, width + 1):
            ys[i - 1] = dys[0] - (width - (i - 1)) * dy
            ys[n2 - (width - i) - 1] = dys[n1 - 1] + i * dy
        xv = dxs[d.nx[0] - 1] + dx * width if boundary == 2 else dxs[0] - dx * width
        xs = np.full(n2, xv)
    return xs, ys


def nesting_layer_thickness(d: NestDomain, max_parent_dx_ratio: float, extra_halo_buffer: int,
                            extra_cells_in_halo: int) -> int:
    """get_domain_nesting_layer_thickness (multidomain_mod.f90:1803-1852)."""
    required = NESTING_THICKNESS[d.timestepping_method]
    if d.use_eddy_viscosity:
        required = (required * 3) // 2
    thickness = required * d.timestepping_refinement_factor + extra_cells_in_halo
    if thickness < d.minimum_nesting_layer_thickness:
        thickness = d.minimum_nesting_layer_thickness
    r = _nint(max_parent_dx_ratio)
    if r > 1:
        thickness = (math.ceil(thickness * 1.0 / max_parent_dx_ratio) + extra_halo_buffer) * r
    else:
        thickness = math.ceil(thickness * 1.0 / max_parent_dx_ratio) * r
    return int(thickness)


def _nint(v: float) -> int:
    """Fortran NINT: round half away from zero."""
    return int(math.floor(abs(v) + 0.5)) * (1 if v >= 0 else -1)


def _in_active_region(pind: np.ndarray, pimg: np.ndarray, myindex: int, myimage: int, halo: int) -> np.ndarray:
    """is_in_active_region (multidomain_mod.f90:2021-2045) for every cell: a
    cell of the domain's own priority region lies within ``halo`` cells
    (Chebyshev distance)."""
    mine = (pind == myindex) & (pimg == myimage)
    nx, ny = mine.shape
    # Dilate the mask by `halo` in each direction with a 2-D prefix sum.
    c = np.zeros((nx + 1, ny + 1), dtype=np.int64)
    c[1:, 1:] = np.cumsum(np.cumsum(mine.astype(np.int64), axis=0), axis=1)
    i = np.arange(nx)
    j = np.arange(ny)
    i0 = np.maximum(i - halo, 0)[:, None]
    i1 = np.minimum(i + halo, nx - 1)[:, None] + 1
    j0 = np.maximum(j - halo, 0)[None, :]
    j1 = np.minimum(j + halo, ny - 1)[None, :] + 1
    s = c[i1, j1] - c[i0, j1] - c[i1, j0] + c[i0, j0]
    return s > 0


def convert_priority_domain_info_to_boxes(pind: np.ndarray, pimg: np.ndarray, halo_width: int, myimage: int,
                                          myindex: int, xs: np.ndarray, ys: np.ndarray, periodic_xs,
                                          periodic_ys) -> np.ndarray:
    """multidomain_mod.f90:718-958.  Rows of (ind, img, iL, iU, jL, jU),
    1-based, in the order the reference emits them: a box is closed (and
    appended) on the first row where its run no longer appears, and boxes
    still open at the last row are appended last, in creation order."""
    nx, ny = pind.shape
    in_px = (xs < periodic_xs[0]) | (xs > periodic_xs[1])
    in_py = (ys < periodic_ys[0]) | (ys > periodic_ys[1])
    active = _in_active_region(pind, pimg, myindex, myimage, halo_width)
    final: List[List[int]] = []
    cand: List[List[int]] = []
    for j in range(ny):
        nind = np.where(active[:, j], pind[:, j], NULL_INDEX)
        nimg = np.where(active[:, j], pimg[:, j], NULL_IMAGE)
        # Run-length encoding on (ind, img, periodic-x flag).
        brk = np.flatnonzero((nind[1:] != nind[:-1]) | (nimg[1:] != nimg[:-1]) | (in_px[1:] != in_px[:-1]))
        starts = np.concatenate(([0], brk + 1))
        ends = np.concatenate((brk, [nx - 1]))
        runs = [(int(nind[s]), int(nimg[s]), int(s) + 1, int(e) + 1) for s, e in zip(starts, ends)]
        if j == 0:
            cand = [[a, b, s, e, 1, -1] for (a, b, s, e) in runs]
            continue
        row_key = {(a, b, s, e, bool(in_py[j])) for (a, b, s, e) in runs}
        cand_key = [(c[0], c[1], c[2], c[3], bool(in_py[j - 1])) for c in cand]
        cand_set = set(cand_key)
        new = [r for r in runs if (r[0], r[1], r[2], r[3], bool(in_py[j])) not in cand_set]
        keep = []
        for c, k in zip(cand, cand_key):
            if k in row_key:
                keep.append(c)
            else:
                c[5] = j  # ends at the previous (1-based j) row
                final.append(c)
        cand = keep + [[a, b, s, e, j + 1, -1] for (a, b, s, e) in new]
        if j == ny - 1:
            for c in cand:
                c[5] = ny
            final.extend(cand)
            cand = []
    if ny == 1:
        for c in cand:
            c[5] = 1
        final.extend(cand)
    out = np.array(final, dtype=np.int64).reshape(-1, 6)
    for b in out:
        if b[0] == 0:
            continue
        i1, i2, j1, j2 = b[2] - 1, b[3], b[4] - 1, b[5]
        if (np.any(pind[i1:i2, j1:j2] != b[0]) or np.any(pimg[i1:i2, j1:j2] != b[1])
                or np.any(in_px[i1:i2] != in_px[i1]) or np.any(in_py[j1:j2] != in_py[j1])):
            raise RuntimeError("inconsistent box in priority-domain metadata")
    return out


def _create_bbox(domains: Sequence[NestDomain]) -> None:
    """create_all_bbox_and_dx (multidomain_mod.f90:960-1060)."""
    for d in domains:
        if d.interior_bounding_box is None or np.all(d.interior_bounding_box == 0.0):
            ll = np.asarray(d.lower_left, dtype=np.float64)
            lw = np.asarray(d.lw, dtype=np.float64)
            d.interior_bounding_box = np.array([ll, ll + lw * np.array([1.0, 0.0]), ll + lw,
                                                ll + lw * np.array([0.0, 1.0])])


def setup_multidomain(domains: Sequence[NestDomain], extra_halo_buffer: int = EXTRA_HALO_BUFFER_DEFAULT,
                      extra_cells_in_halo: int = EXTRA_CELLS_IN_HALO_DEFAULT,
                      periodic_xs=(-HUGE, HUGE), periodic_ys=(-HUGE, HUGE)) -> List[Exchange]:
    """setup_multidomain + setup_multidomain_domains for one image
    (multidomain_mod.f90:2663-2780, 2781-3553).  Mutates the domains
    (widened extents, metadata) and returns the exchanges in the reference's
    receive order (domain by domain, recv_metadata row by row)."""
    for d in domains:
        d.dx = (d.lw[0] / (1.0 * d.nx[0]), d.lw[1] / (1.0 * d.nx[1]))
    _create_bbox(domains)

    # Nesting-layer width (multidomain_mod.f90:636-716).
    for d in domains:
        mpdr = 1.0
        nesting = []
        for b in (1, 2, 3, 4):
            xs, ys = _boundary_points(d, b, 1)
            ind, img, ddx = find_priority_domain_containing_xy(domains, xs, ys, periodic_xs, periodic_ys)
            dxtmp = ddx.max(axis=0)
            if np.all(dxtmp > 0):
                nrtmp = [float(_nint(dxtmp[k] / d.dx[k])) for k in range(2)]
                mpdr = max(mpdr, max(nrtmp))
            nesting.append(bool(np.any(img > 0)))
        d.max_parent_dx_ratio = mpdr
        d.is_nesting_boundary = tuple(nesting)
        d.nest_layer_width = nesting_layer_thickness(d, mpdr, extra_halo_buffer, extra_cells_in_halo)

    # Widen the nesting boundaries (multidomain_mod.f90:2860-2895).
    for d in domains:
        w = d.nest_layer_width
        for b in (1, 2, 3, 4):
            if not d.is_nesting_boundary[b - 1]:
                continue
            lw, nx, ll, dx = list(d.lw), list(d.nx), list(d.lower_left), d.dx
            if b in (2, 4):
                lw[0] = lw[0] + w * dx[0]
                nx[0] = nx[0] + w
            if b in (1, 3):
                lw[1] = lw[1] + w * dx[1]
                nx[1] = nx[1] + w
            if b == 3:
                ll[1] = ll[1] - w * dx[1]
            if b == 4:
                ll[0] = ll[0] - w * dx[0]
            d.lw, d.nx, d.lower_left = tuple(lw), tuple(nx), tuple(ll)

    # Priority domains and receive boxes (:2897-3030).
    for jd, d in enumerate(domains):
        xs, ys = domain_xs_ys(d)
        nx, ny = d.nx
        pind = np.empty((nx, ny), dtype=np.int64)
        pimg = np.empty((nx, ny), dtype=np.int64)
        for jj in range(ny):
            ind, img, ddx = find_priority_domain_containing_xy(domains, xs, np.full(nx, ys[jj]), periodic_xs,
                                                               periodic_ys)
            if np.any(ind < 0):
                raise ValueError(f"domain {jd + 1}: cells outside every domain (row {jj + 1})")
            for k in range(2):
                if np.any(ddx[:, k] > 1.0001 * d.max_parent_dx_ratio * d.dx[k]):
                    raise ValueError(f"domain {jd + 1}: nesting boundary overlaps a domain coarser than its parent")
            pind[:, jj] = ind
            pimg[:, jj] = img
        d.priority_domain_index = pind
        d.priority_domain_image = pimg
        d.recv_metadata = convert_priority_domain_info_to_boxes(pind, pimg, d.nest_layer_width, 1, jd + 1, xs, ys,
                                                                periodic_xs, periodic_ys)

    # Receive rows as coordinates; flag the rows that need communication
    # (:3050-3080).
    recv_rows = []  # per domain: list of (ind, img, xlo, xhi, ylo, yhi, comm_counter, in_periodic)
    for jd, d in enumerate(domains):
        x, y = d.x(), d.y()
        rows = []
        counter = 0
        for b in d.recv_metadata:
            txs = np.array([x[b[2] - 1], x[b[3] - 1]])
            tys = np.array([y[b[4] - 1], y[b[5] - 1]])
            _, pa = _periodic_shift(np.array([txs[0]]), *periodic_xs, False)
            _, pb = _periodic_shift(np.array([tys[0]]), *periodic_ys, False)
            _, pc = _periodic_shift(np.array([txs[1]]), *periodic_xs, False)
            _, pd = _periodic_shift(np.array([tys[1]]), *periodic_ys, False)
            # check_periodic is called on (x1, y1) then (x2, y2); the flag
            # kept is the second call's.
            in_per = bool(pc[0] or pd[0])
            xlo, xhi = txs[0] - 0.5 * d.dx[0], txs[1] + 0.5 * d.dx[0]
            ylo, yhi = tys[0] - 0.5 * d.dx[1], tys[1] + 0.5 * d.dx[1]
            real = not (((not in_per) and b[0] == jd + 1 and b[1] == 1) or b[0] < 1)
            cnt = -1
            if real:
                counter += 1
                cnt = counter
            rows.append([int(b[0]), int(b[1]), xlo, xhi, ylo, yhi, cnt])
        recv_rows.append(rows)

    # Send metadata (:3090-3140).
    for jd, d in enumerate(domains):
        x, y = d.x(), d.y()
        smeta = []
        for jj, rows in enumerate(recv_rows):
            for i, r in enumerate(rows):
                if r[0] != jd + 1 or r[1] != 1:
                    continue
                tdx = domains[jj].dx
                txs = np.array([r[2] + 0.5 * tdx[0], r[3] - 0.5 * tdx[0]])
                tys = np.array([r[4] + 0.5 * tdx[1], r[5] - 0.5 * tdx[1]])
                p1x, f1x = _periodic_shift(txs[:1], *periodic_xs, True)
                p1y, f1y = _periodic_shift(tys[:1], *periodic_ys, True)
                p2x, f2x = _periodic_shift(txs[1:], *periodic_xs, True)
                p2y, f2y = _periodic_shift(tys[1:], *periodic_ys, True)
                in_per = bool(f2x[0] or f2y[0])
                txs = np.array([p1x[0], p2x[0]]) - 0.5 * np.array([1.0, -1.0]) * tdx[0]
                tys = np.array([p1y[0], p2y[0]]) - 0.5 * np.array([1.0, -1.0]) * tdx[1]
                smeta.append([jj + 1, 1, int(np.count_nonzero(x < txs[0])) + 1, int(np.count_nonzero(x < txs[1])),
                              int(np.count_nonzero(y < tys[0])) + 1, int(np.count_nonzero(y < tys[1])), i,
                              int(in_per)])
        d.send_metadata = np.array(smeta, dtype=np.int64).reshape(-1, 8)

    # Pair the real receive rows with their send rows (:3170-3330).
    exchanges: List[Exchange] = []
    send_index = {}
    for jd, d in enumerate(domains):
        for srow, s in enumerate(d.send_metadata):
            n_ind, recv_row, in_per = int(s[0]) - 1, int(s[6]), bool(s[7])
            if (not in_per and n_ind == jd) or s[0] < 1:
                continue
            send_index[(n_ind, recv_row)] = (jd, srow)
    for jd, rows in enumerate(recv_rows):
        for i, r in enumerate(rows):
            if r[6] < 1:
                continue
            sender, srow = send_index[(jd, i)]
            s = domains[sender].send_metadata[srow]
            b = domains[jd].recv_metadata[i]
            exchanges.append(Exchange(sender=sender, receiver=jd,
                                      send_box=(int(s[2]), int(s[3]), int(s[4]), int(s[5])),
                                      recv_box=(int(b[2]), int(b[3]), int(b[4]), int(b[5])),
                                      recv_row=i, send_row=srow))
    return exchanges


class _NestDomainDesc(ctypes.Structure):
    """swals_nest_domain_desc (include/swals_gpu.h)."""
    _fields_ = [("lower_left", ctypes.c_double * 2), ("lw", ctypes.c_double * 2), ("nx", ctypes.c_int32 * 2),
                ("timestepping_refinement_factor", ctypes.c_int32),
                ("minimum_nesting_layer_thickness", ctypes.c_int32), ("use_eddy_viscosity", ctypes.c_int32),
                ("nest_layer_width", ctypes.c_int32), ("is_nesting_boundary", ctypes.c_int32 * 4),
                ("max_parent_dx_ratio", ctypes.c_double), ("interior_bounding_box", ctypes.c_double * 8),
                ("timestepping_method", ctypes.c_char * 64)]


class _MdExchange(ctypes.Structure):
    _fields_ = [("sender", ctypes.c_int32), ("receiver", ctypes.c_int32), ("send_box", ctypes.c_int32 * 4),
                ("recv_box", ctypes.c_int32 * 4), ("recv_row", ctypes.c_int32), ("send_row", ctypes.c_int32)]


def setup_multidomain_native(domains: Sequence[NestDomain], extra_halo_buffer: int = EXTRA_HALO_BUFFER_DEFAULT,
                             extra_cells_in_halo: int = EXTRA_CELLS_IN_HALO_DEFAULT,
                             periodic_xs=(-HUGE, HUGE), periodic_ys=(-HUGE, HUGE)) -> List[Exchange]:
    """setup_multidomain through the library's native builder
    (swals_md_build_metadata): the same fields of the domains are set and the
    same exchanges returned as by setup_multidomain (send_metadata is not
    kept)."""
    from . import _lib
    L = _lib.lib()
    n = len(domains)
    descs = (_NestDomainDesc * n)()
    for c, d in zip(descs, domains):
        c.lower_left[:] = [float(v) for v in d.lower_left]
        c.lw[:] = [float(v) for v in d.lw]
        c.nx[:] = [int(v) for v in d.nx]
        c.timestepping_refinement_factor = int(d.timestepping_refinement_factor)
        c.minimum_nesting_layer_thickness = int(d.minimum_nesting_layer_thickness)
        c.use_eddy_viscosity = int(bool(d.use_eddy_viscosity))
        if d.interior_bounding_box is not None:
            c.interior_bounding_box[:] = [float(v) for v in np.asarray(d.interior_bounding_box).reshape(-1)]
        c.timestepping_method = d.timestepping_method.encode()
    handle = ctypes.c_void_p()
    pxs = (ctypes.c_double * 2)(*periodic_xs)
    pys = (ctypes.c_double * 2)(*periodic_ys)
    _lib.check(L.swals_md_build_metadata(descs, n, int(extra_halo_buffer), int(extra_cells_in_halo), pxs, pys,
                                         ctypes.byref(handle)))
    try:
        for c, d in zip(descs, domains):
            d.dx = (d.lw[0] / (1.0 * d.nx[0]), d.lw[1] / (1.0 * d.nx[1]))   # before widening, as setup records it
            d.interior_bounding_box = np.array(c.interior_bounding_box[:], dtype=np.float64).reshape(4, 2)
            d.max_parent_dx_ratio = float(c.max_parent_dx_ratio)
            d.is_nesting_boundary = tuple(bool(v) for v in c.is_nesting_boundary)
            d.nest_layer_width = int(c.nest_layer_width)
            d.lower_left, d.lw, d.nx = tuple(c.lower_left[:]), tuple(c.lw[:]), tuple(int(v) for v in c.nx)
        for k, d in enumerate(domains):
            nx, ny = d.nx
            ind = np.empty(nx * ny, dtype=np.int32)
            img = np.empty(nx * ny, dtype=np.int32)
            _lib.check(L.swals_md_metadata_priority(handle, k, ind.ctypes.data, img.ctypes.data))
            d.priority_domain_index = ind.reshape(ny, nx).T.astype(np.int64)
            d.priority_domain_image = img.reshape(ny, nx).T.astype(np.int64)
            cnt = ctypes.c_int32()
            _lib.check(L.swals_md_metadata_recv_boxes(handle, k, None, 0, ctypes.byref(cnt)))
            rows = np.empty((cnt.value, 6), dtype=np.int64)
            _lib.check(L.swals_md_metadata_recv_boxes(handle, k, rows.ctypes.data, cnt.value, ctypes.byref(cnt)))
            d.recv_metadata = rows
            d.send_metadata = None
        cnt = ctypes.c_int32()
        _lib.check(L.swals_md_metadata_exchanges(handle, None, 0, ctypes.byref(cnt)))
        exs = (_MdExchange * max(cnt.value, 1))()
        _lib.check(L.swals_md_metadata_exchanges(handle, exs, cnt.value, ctypes.byref(cnt)))
        return [Exchange(sender=e.sender, receiver=e.receiver, send_box=tuple(e.send_box[:]),
                         recv_box=tuple(e.recv_box[:]), recv_row=e.recv_row, send_row=e.send_row)
                for e in exs[:cnt.value]]
    finally:
        L.swals_md_metadata_free(handle)


def exchange_cell_ratios(domains: Sequence[NestDomain], e: Exchange) -> Tuple[int, int]:
    """The integer refinement (>= 1) in x and y between the two sides of an
    exchange, with the checks of initialise_two_way_nesting_comms
    (nested_grid_comms_mod.f90:372-430): the coarser cell must be an integer
    number of finer cells in both directions, and the same side coarser in
    both."""
    ds, dr = domains[e.sender].dx, domains[e.receiver].dx
    ratios = [ds[k] / dr[k] for k in range(2)]
    if not (all(x >= 1.0 - 1e-6 for x in ratios) or all(x <= 1.0 + 1e-6 for x in ratios)):
        raise ValueError(f"cell ratios {ratios} are not consistently coarser or finer")
    r = [max(x, 1.0 / x) for x in ratios]
    rr = [_nint(x) for x in r]
    for k in range(2):
        if abs(r[k] - rr[k]) > min(0.499, max(1e-6, 100 * float(np.spacing(r[k])))):
            raise ValueError(f"non-integer cell ratio {ratios}")
    return rr[0], rr[1]
