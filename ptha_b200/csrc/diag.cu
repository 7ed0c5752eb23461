// diag.cu -- diagnostics reductions: volume_interior and the stationary
// timestep limits (domain_mod.f90:1815-1849, 1906-1960).
#include "swals_kernels.h"

#include <cfloat>

namespace swals {
namespace {

// One warp per row: fixed-order warp tree of (double)STG - (double)ELV, then
// one thread adds area(j) * row sum in row order (deterministic).
template <typename R>
__global__ void row_volume_kernel(int nx, int ny, int64_t P, const R *stg, const R *elv, int n_ext, double *row_sums)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int r = n_ext + warp;
    if (r > ny - n_ext - 1) return;
    double acc = 0.0;
    for (int i = n_ext + lane; i <= nx - n_ext - 1; i += 32) {
        const int64_t o = (int64_t)r * P + i;
        acc += (double)stg[o] - (double)elv[o];
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) row_sums[r] = acc;
}

template <typename R>
__global__ void volume_total_kernel(int ny, int n_ext, const R *area, const double *row_sums, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double vol = 0.0;
    for (int r = n_ext; r <= ny - n_ext - 1; r++) vol = vol + (double)area[r] * row_sums[r];
    *out = vol;
}

template <typename R>
__global__ void timestep_min_kernel(int nx, int ny, int64_t P, const R *stg, const R *elv, const R *dxb,
                                    const R *dyl, R msl, int linear, double *block_min)
{
    __shared__ double red[32];
    double best = DBL_MAX;
    const int64_t n = (int64_t)nx * ny;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(q / nx), i = (int)(q - (int64_t)r * nx);
        const int64_t o = (int64_t)r * P + i;
        R sdx, sdy, dep;
        if (linear) {
            sdx = dxb[r] + dxb[r + 1];
            sdy = dyl[i] + dyl[i + 1];
            dep = rmax(msl - elv[o], K<R>::min_depth());
        } else {
            sdx = dxb[r + 1] + dxb[r];
            sdy = dyl[i + 1] + dyl[i];
            dep = rmax(stg[o] - elv[o], K<R>::min_depth());
        }
        R v = R(0.5) * rmin(sdx, sdy) / R(sqrt(K<R>::gravity() * dep));
        best = fmin(best, (double)v);
    }
    for (int o = 16; o > 0; o >>= 1) best = fmin(best, __shfl_down_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmin(m, red[w]);
        block_min[blockIdx.x] = m;
    }
}

__global__ void min_finalize_kernel(const double *block_min, int nb, double *out)
{
    if (threadIdx.x != 0) return;
    double m = DBL_MAX;
    for (int b = 0; b < nb; b++) m = fmin(m, block_min[b]);
    *out = m;
}

}  // namespace

template <typename R>
cudaError_t launch_volume_interior(int nx, int ny, int64_t pitch, const R *stg, const R *elv, const R *area,
                                   int n_ext, double *row_sums, double *out, cudaStream_t s)
{
    const int rows = ny - 2 * n_ext;
    if (rows > 0) {
        const int threads = 256;
        const int blocks = (rows * 32 + threads - 1) / threads;
        row_volume_kernel<R><<<blocks, threads, 0, s>>>(nx, ny, pitch, stg, elv, n_ext, row_sums);
    }
    volume_total_kernel<R><<<1, 32, 0, s>>>(ny, n_ext, area, row_sums, out);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_timestep_max(int nx, int ny, int64_t pitch, const R *stg, const R *elv, const R *dxb,
                                const R *dyl, double msl, int linear, double cfl, double *block_min, int max_blocks,
                                double *out, cudaStream_t s)
{
    (void)cfl;
    int nb = (int)((int64_t)nx * ny / 256 + 1);
    if (nb > max_blocks) nb = max_blocks;
    timestep_min_kernel<R><<<nb, 256, 0, s>>>(nx, ny, pitch, stg, elv, dxb, dyl, R(msl), linear, block_min);
    min_finalize_kernel<<<1, 32, 0, s>>>(block_min, nb, out);
    return cudaGetLastError();
}

template cudaError_t launch_volume_interior<double>(int, int, int64_t, const double *, const double *,
                                                    const double *, int, double *, double *, cudaStream_t);
template cudaError_t launch_volume_interior<float>(int, int, int64_t, const float *, const float *, const float *,
                                                   int, double *, double *, cudaStream_t);
template cudaError_t launch_timestep_max<double>(int, int, int64_t, const double *, const double *, const double *,
                                                 const double *, double, int, double, double *, int, double *,
                                                 cudaStream_t);
template cudaError_t launch_timestep_max<float>(int, int, int64_t, const float *, const float *, const float *,
                                                const float *, double, int, double, double *, int, double *,
                                                cudaStream_t);

}  // namespace swals
