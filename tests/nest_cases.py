"""Shared set-ups for the nesting tests (oracle and GPU)."""
import numpy as np

from ptha_b200 import nesting as nest


def nested_comms_case(r):
    """The two domains and boxes of test_nested_grid_comms_mod_workhorse
    (nested_grid_comms_mod.f90:2694-2800) for nest ratio r: a 20x15 parent
    (dx 1, lower-left (0,0)) and a (9r)x(8r) child (dx 1/r, lower-left
    (3,4)); U(i,j,k) = x + y + k^2 on both."""
    nx1 = (20, 15)
    dx1 = (1.0, 1.0)
    ll2 = (3.0, 4.0)
    nx2 = (9 * r, 8 * r)
    dx2 = (dx1[0] / r, dx1[1] / r)
    U1 = np.zeros((4, nx1[1], nx1[0]))
    U2 = np.zeros((4, nx2[1], nx2[0]))
    for k in range(1, 5):
        i = np.arange(1, nx1[0] + 1)
        j = np.arange(1, nx1[1] + 1)
        x = 0.0 + (i - 0.5) * dx1[0]
        y = 0.0 + (j - 0.5) * dx1[1]
        U1[k - 1] = x[None, :] + y[:, None] + k * k
        i = np.arange(1, nx2[0] + 1)
        j = np.arange(1, nx2[1] + 1)
        x = ll2[0] + (i - 0.5) * dx2[0]
        y = ll2[1] + (j - 0.5) * dx2[1]
        U2[k - 1] = x[None, :] + y[:, None] + k * k
    xi = int(round((ll2[0] - 0.0) / dx1[0])) + 1
    yi = int(round((ll2[1] - 0.0) / dx1[1])) + 1
    # child -> parent and parent -> child, as (send box, recv box) pairs
    child_send = (r + 1, r * 2 + r, r + 1, nx2[1] - r)
    parent_recv = (xi + 1, xi + 2, yi + 1, yi + nx2[1] // r - 1 - 1)
    parent_send = (xi, xi, yi, yi + nx2[1] // r - 1)
    child_recv = (1, r, 1, nx2[1])
    return dict(nx1=nx1, dx1=dx1, nx2=nx2, dx2=dx2, ll2=ll2, U1=U1, U2=U2, child_send=child_send,
                parent_recv=parent_recv, parent_send=parent_send, child_recv=child_recv)


def planar_values(d: nest.NestDomain, index_grid, global_ll, c1=0.0001, c2=0.00003):
    """U(i,j,1:4) = (x-ll1)*c1 + (y-ll2)*c2 + index + [0,3,6,9]
    (multidomain_mod.f90:4089-4100), shape (4, ny, nx)."""
    x, y = d.x(), d.y()
    base = ((x[None, :] - global_ll[0]) * c1 + (y[:, None] - global_ll[1]) * c2) + index_grid
    return np.stack([base + 0.0, base + 3.0, base + 6.0, base + 9.0])


def two_level_nest(ratio=3, child_method="rk2", parent_method="linear", child_nt=None, n=(60, 40), dx=1000.0):
    """A small two-level nest used for stepping tests: a parent over
    n[0] x n[1] cells of size dx, and a ratio-`ratio` child over its middle."""
    lw = (n[0] * dx, n[1] * dx)
    parent = nest.NestDomain((0.0, 0.0), lw, n, parent_method, 1)
    c0 = (n[0] // 3, n[1] // 4)
    cw = (n[0] // 3, n[1] // 2)
    cl = (c0[0] * dx, c0[1] * dx)
    clw = (cw[0] * dx, cw[1] * dx)
    nt = child_nt if child_nt is not None else ratio
    child = nest.NestDomain(cl, clw, (cw[0] * ratio, cw[1] * ratio), child_method, nt)
    return [parent, child]
