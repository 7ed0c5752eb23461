"""The allocation-free volume_interior entry point against the allocating one.

swals_gpu_volume_interior_noalloc exists for callers that cannot call
cudaMalloc (code running under CUDA graph capture, hosts whose device memory
belongs to another allocator, loops that cannot take cudaMalloc's device-wide
synchronisation).  It must give the same volume as swals_gpu_volume_interior
on the same state, call after call, although its scratch is a shared fixed
device array.  Both entry points run the same row kernel with the same launch
shape and then add the row sums in row order in one thread, so the results
are compared for exact equality.  This file is collected last so that a
failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("real_bytes,ecw", [(8, 2), (8, 1), (4, 2), (4, 1)])
def test_noalloc_volume_interior_matches_allocating_entry_point(real_bytes, ecw):
    import torch
    from ptha_b200 import Domain, _lib, workloads

    n = 256
    kw, U, gauges, nsq = workloads.rk2_beach(n=n, dx=80.0, toe=17580.0 * n / 2048)
    d = Domain(**kw, real_bytes=real_bytes, exterior_cells_width=ecw)
    d.set_U(U)
    d.set_manning_squared(nsq)
    L = _lib.lib()
    tdt = torch.float64 if real_bytes == 8 else torch.float32
    area = torch.tensor(d.metrics()["area"], dtype=tdt, device="cuda")
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    stream = d.stream()

    for call in range(2):
        if call == 1:
            d.evolve_steps(25)   # a different state for the second call
        expected = d.volume_interior()          # allocating entry point (domain handle)
        (stg, uh, vh, elv), pitch = d.device_planes()
        rc = L.swals_gpu_volume_interior_noalloc(stg, elv, ctypes.c_void_p(area.data_ptr()), n, n, pitch,
                                                 real_bytes, ecw, ctypes.c_void_p(out.data_ptr()),
                                                 ctypes.c_void_p(stream))
        _lib.check(rc)
        d.synchronize()
        got = float(out.item())
        assert got == expected, (call, got, expected)

    # no interior rows (ny <= 2 * exterior_cells_width): the sum over an
    # empty range is 0, and the scratch's old contents are not read
    rc = L.swals_gpu_volume_interior_noalloc(stg, elv, ctypes.c_void_p(area.data_ptr()), n, 4, pitch, real_bytes, 2,
                                             ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    _lib.check(rc)
    d.synchronize()
    assert float(out.item()) == 0.0

    # sizes beyond the fixed scratch are refused before touching the device
    rc = L.swals_gpu_volume_interior_noalloc(stg, elv, ctypes.c_void_p(area.data_ptr()), n, 70000, pitch,
                                             real_bytes, 2, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    assert rc == 10 and "SWALS_NOALLOC_MAX_ROWS" in _lib.last_error()
    d.close()


@pytest.mark.gpu
@pytest.mark.parametrize("real_bytes", [8, 4])
def test_noalloc_volume_interior_without_exterior_cells(real_bytes):
    """exterior_cells_width = 0 sums every cell.  A domain treats 0 as its
    default width (2), so the allocating entry point cannot serve as the
    reference here: the sum is checked against numpy instead (row sums of
    stage - elevation in double, times area_cell_y, summed over rows; a
    different summation order, hence the round-off tolerance)."""
    import torch
    from ptha_b200 import Domain, _lib, workloads

    n = 192
    kw, U, gauges, nsq = workloads.rk2_beach(n=n, dx=80.0, toe=17580.0 * n / 2048)
    d = Domain(**kw, real_bytes=real_bytes)
    d.set_U(U)
    d.set_manning_squared(nsq)
    d.evolve_steps(15)
    L = _lib.lib()
    area_h = d.metrics()["area"].astype(np.float64 if real_bytes == 8 else np.float32)
    area = torch.tensor(area_h, device="cuda")
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    (stg, uh, vh, elv), pitch = d.device_planes()
    for _ in range(2):
        rc = L.swals_gpu_volume_interior_noalloc(stg, elv, ctypes.c_void_p(area.data_ptr()), n, n, pitch,
                                                 real_bytes, 0, ctypes.c_void_p(out.data_ptr()),
                                                 ctypes.c_void_p(d.stream()))
        _lib.check(rc)
        d.synchronize()
        Ud = d.get_U()
        rows = (Ud[0].astype(np.float64) - Ud[3].astype(np.float64)).sum(axis=1)
        expected = float(np.sum(area_h.astype(np.float64) * rows))
        assert float(out.item()) == pytest.approx(expected, rel=1e-13)
    d.close()
