"""The allocation-free volume_interior entry point against the allocating one.

swals_gpu_volume_interior_noalloc exists for callers that cannot call
cudaMalloc (code running under CUDA graph capture, hosts whose device memory
belongs to another allocator, loops that cannot take cudaMalloc's device-wide
synchronisation).  It must give the same volume as swals_gpu_volume_interior
on the same state, call after call, although its scratch is a shared fixed
device array.  This file is collected last so that a failure here comes
after every other test has run.
"""
import ctypes

import numpy as np
import pytest


@pytest.mark.gpu
def test_noalloc_volume_interior_matches_allocating_entry_point():
    import torch
    from ptha_b200 import Domain, _lib, workloads

    n = 256
    kw, U, gauges, nsq = workloads.rk2_beach(n=n, dx=80.0, toe=17580.0 * n / 2048)
    d = Domain(**kw)
    d.set_U(U)
    d.set_manning_squared(nsq)
    L = _lib.lib()
    area = torch.tensor(d.metrics()["area"], dtype=torch.float64, device="cuda")
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    stream = d.stream()

    for call in range(2):
        if call == 1:
            d.evolve_steps(25)   # a different state for the second call
        expected = d.volume_interior()          # allocating entry point (domain handle)
        (stg, uh, vh, elv), pitch = d.device_planes()
        rc = L.swals_gpu_volume_interior_noalloc(stg, elv, ctypes.c_void_p(area.data_ptr()), n, n, pitch, 8, 2,
                                                 ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
        _lib.check(rc)
        d.synchronize()
        got = float(out.item())
        # identical reduction order: equal to round-off of the final sum
        assert got == pytest.approx(expected, rel=1e-13, abs=1e-9), (call, got, expected)

    # sizes beyond the fixed scratch are refused before touching the device
    rc = L.swals_gpu_volume_interior_noalloc(stg, elv, ctypes.c_void_p(area.data_ptr()), n, 70000, pitch, 8, 2,
                                             ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    assert rc == 10 and "SWALS_NOALLOC_MAX_ROWS" in _lib.last_error()
    d.close()
