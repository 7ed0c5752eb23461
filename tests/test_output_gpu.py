"""REAL4 output staging against host-side conversion: the grid payload of
write_grids (util/netcdf_util_mod.f90:437-510) for several spatial strides
(start = stride/2 + 1) and the gauge series in the (station, time) order of
point_gauge_mod.f90:411-638, equal to numpy's float32 rounding of the FP64
(and FP32) state."""
import numpy as np
import pytest

from ptha_b200 import Domain, workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("real_bytes", [8, 4])
@pytest.mark.parametrize("stride", [1, 3, 4])
def test_grid_staging(real_bytes, stride):
    kw, U, gauges, nsq = workloads.rk2_beach(n=70, dx=10.0 * 2048 / 70, toe=17580.0 * 70 / 2048)
    d = Domain(**kw, real_bytes=real_bytes)
    d.set_U(U)
    d.set_manning_squared(nsq)
    for _ in range(30):
        d.evolve_one_step()
    names = ("stage", "uh", "vh", "elevation", "max_stage")
    got = d.stage_grids_real4(names, spatial_stride=stride)
    G = d.get_U()
    st = stride // 2
    ref = {n: G[k][st::stride, st::stride] for k, n in enumerate(names[:4])}
    ref["max_stage"] = d.max_stage()[st::stride, st::stride]
    for n in names:
        np.testing.assert_array_equal(got[n], ref[n].astype(np.float32), err_msg=n)
    one = d.stage_grids_real4(("vh",), spatial_stride=stride)
    np.testing.assert_array_equal(one["vh"], got["vh"])
    d.close()


def test_gauge_staging():
    kw, U, gauges = workloads.linear_gaussian_basin(n=120, dx=1000.0)
    d = Domain(**kw)
    d.set_U(U)
    d.gauges_setup(gauges, capacity=50)
    dt = d.linear_timestep_max()
    for _ in range(40):
        d.evolve_one_step(dt)
    series = d.gauges_read()                      # (records, gauges, 3) doubles
    r4 = d.gauges_read_real4()                    # (3, records, gauges) floats
    assert r4.shape == (3, series.shape[0], series.shape[1])
    np.testing.assert_array_equal(r4, np.transpose(series, (2, 0, 1)).astype(np.float32))
    d.close()
