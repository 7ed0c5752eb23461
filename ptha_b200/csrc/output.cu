// output.cu -- REAL4 output staging on the device.
//
// SWALS writes its grids and gauge series to netCDF in the output precision
// (REAL4 by default): write_grids (util/netcdf_util_mod.f90:437-510) stores
// U(start:nx:stride, start:ny:stride, k) with start = stride/2 + 1 for the
// flow variables it is asked for, and the point gauges
// (point_gauge_mod.f90:411-638) store per variable a (station, time) array.
// Here the conversion to REAL4 (round to nearest, as netCDF's own
// conversion) and the striding are done on the device into one staging
// buffer, so that a writer receives the variables contiguous, in the
// netCDF variables' Fortran order, in one device-to-host copy.
#include "domain_internal.h"
#include "swals_kernels.h"

#include <cstdio>

namespace {

template <typename R>
__global__ void grid_stage_kernel(const R *plane, int64_t P, int start, int stride, int cx, int cy, float *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= cx || j >= cy) return;
    out[(int64_t)j * cx + i] = (float)plane[(int64_t)(start + j * stride) * P + start + (int64_t)i * stride];
}

// records (t, gauge, var) -> out (var, t, gauge)
__global__ void gauge_stage_kernel(const double *rec, int ng, int nrec, float *out)
{
    const int64_t n = (int64_t)nrec * ng;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < 3 * n; q += (int64_t)gridDim.x * blockDim.x) {
        const int v = (int)(q / n);
        const int64_t tg = q - v * n;
        out[q] = (float)rec[tg * 3 + v];
    }
}

int stage_fail(int code, const char *msg)
{
    swals::set_last_error(msg);
    return code;
}

int ensure_stage(swals_domain *d, size_t floats)
{
    if (d->stage_cap >= floats) return SWALS_OK;
    if (d->stage_buf) cudaFree(d->stage_buf);
    d->stage_buf = nullptr;
    d->stage_cap = 0;
    if (cudaMalloc(&d->stage_buf, floats * sizeof(float)) != cudaSuccess)
        return stage_fail(SWALS_ERR_CUDA, "staging buffer allocation failed");
    d->stage_cap = floats;
    return SWALS_OK;
}

}  // namespace

extern "C" int swals_gpu_stage_grids_real4(swals_domain *d, int32_t var_mask, int32_t spatial_stride, float *host_out,
                                           int64_t capacity_floats, int32_t *count_xy)
{
    if (!d || !host_out) return stage_fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    if (spatial_stride < 1 || spatial_stride > (d->nx < d->ny ? d->nx : d->ny))
        return stage_fail(SWALS_ERR_INVALID_ARGUMENT, "spatial_stride must be in 1 .. min(nx, ny)");
    if (var_mask <= 0 || var_mask > 31) return stage_fail(SWALS_ERR_INVALID_ARGUMENT, "var_mask must select 1 to 5 variables");
    const int start = spatial_stride / 2;   // 0-based start = stride/2 + 1 - 1
    const int cx = (d->nx - 1 - start) / spatial_stride + 1, cy = (d->ny - 1 - start) / spatial_stride + 1;
    int nvar = 0;
    for (int k = 0; k < 5; k++) nvar += (var_mask >> k) & 1;
    const size_t per = (size_t)cx * cy, need = per * nvar;
    if ((int64_t)need > capacity_floats) {
        char msg[160];
        snprintf(msg, sizeof(msg), "host buffer holds %lld floats, %zu needed", (long long)capacity_floats, need);
        return stage_fail(SWALS_ERR_CAPACITY, msg);
    }
    int rc = ensure_stage(d, need);
    if (rc != SWALS_OK) return rc;
    const dim3 grid((cx + 127) / 128, cy);
    size_t off = 0;
    for (int k = 0; k < 5; k++) {
        if (!((var_mask >> k) & 1)) continue;
        const void *pl = (k == 4) ? d->max_stage : (k == 3) ? d->elv : d->planes[d->cur][k];
        if (d->fp64)
            grid_stage_kernel<double><<<grid, 128, 0, d->stream>>>((const double *)pl, d->pitch, start,
                                                                   spatial_stride, cx, cy, d->stage_buf + off);
        else
            grid_stage_kernel<float><<<grid, 128, 0, d->stream>>>((const float *)pl, d->pitch, start, spatial_stride,
                                                                  cx, cy, d->stage_buf + off);
        d->launches++;
        off += per;
    }
    cudaError_t e = cudaMemcpyAsync(host_out, d->stage_buf, need * sizeof(float), cudaMemcpyDeviceToHost, d->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
    if (e != cudaSuccess) return stage_fail(SWALS_ERR_CUDA, cudaGetErrorString(e));
    if (count_xy) { count_xy[0] = cx; count_xy[1] = cy; }
    return SWALS_OK;
}

extern "C" int swals_gpu_gauges_read_real4(swals_domain *d, float *out, int32_t max_records, int32_t *n_records)
{
    if (!d || !n_records) return stage_fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    int rec = 0;
    cudaError_t e = cudaMemcpyAsync(&rec, &d->sc->gauge_records, sizeof(int), cudaMemcpyDeviceToHost, d->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
    if (e != cudaSuccess) return stage_fail(SWALS_ERR_CUDA, cudaGetErrorString(e));
    const int valid = rec < d->gauge_capacity ? rec : d->gauge_capacity;
    const int ncopy = valid < max_records ? valid : max_records;
    *n_records = ncopy;
    if (ncopy > 0 && out && d->n_gauges > 0) {
        const size_t need = (size_t)3 * d->n_gauges * ncopy;
        int rc = ensure_stage(d, need);
        if (rc != SWALS_OK) return rc;
        gauge_stage_kernel<<<(int)((need + 255) / 256 < 1184 ? (need + 255) / 256 : 1184), 256, 0, d->stream>>>(
            d->d_records, d->n_gauges, ncopy, d->stage_buf);
        d->launches++;
        e = cudaMemcpyAsync(out, d->stage_buf, need * sizeof(float), cudaMemcpyDeviceToHost, d->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
        if (e != cudaSuccess) return stage_fail(SWALS_ERR_CUDA, cudaGetErrorString(e));
    }
    if (rec > d->gauge_capacity) {
        char msg[120];
        snprintf(msg, sizeof(msg), "gauge buffer full: %d records requested, capacity %d", rec, d->gauge_capacity);
        return stage_fail(SWALS_ERR_CAPACITY, msg);
    }
    return SWALS_OK;
}
