// diag.cu -- diagnostics reductions: volume_interior and the stationary
// timestep limits (domain_mod.f90:1815-1849, 1906-1960).
#include "swals_kernels.h"

#include <cfloat>

namespace swals {
namespace {

// One warp per row: fixed-order warp tree of (double)STG - (double)ELV, then
// one thread adds area(j) * row sum in row order (deterministic).
template <typename R>
__global__ void row_volume_kernel(int nx, int ny, int64_t P, const R *stg, const R *elv, int n_ext, double *row_sums,
                                  const uint8_t *mask)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int r = n_ext + warp;
    if (r > ny - n_ext - 1) return;
    double acc = 0.0;
    for (int i = n_ext + lane; i <= nx - n_ext - 1; i += 32) {
        if (mask && !mask[(int64_t)r * nx + i]) continue;   // volume_in_priority_domain's mask
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

// compute_domain_statistics_new (domain_mod.f90:683-849), one warp per row
// j (ecw+1..ny-ecw): each lane accumulates the potential and kinetic energy
// terms of its cells, a warp tree combines them, and the row results go to
// out6[6*j ..]: {E_pot, E_kin, max stage, min stage, max speed^2, min speed^2}.
template <typename R>
__global__ void stats_row_kernel(int nx, int ny, int64_t P, const R *stg, const R *uh, const R *vh, const R *elv,
                                 const R *area, const uint8_t *mask, int ecw, int staggered, int tl, R msl,
                                 double *out6)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int j = ecw + warp;           // 0-based row
    if (j > ny - 1 - ecw) return;
    const R mad = K<R>::min_depth(), half = R(0.5), g = K<R>::gravity(), one = R(1), zero = R(0);
    double pe = 0.0, ke = 0.0;
    R mxs = -K<R>::huge(), mns = K<R>::huge(), mxv = zero, mnv = K<R>::huge();
    for (int i = ecw + lane; i <= nx - 1 - ecw; i += 32) {
        if (mask && !mask[(int64_t)j * nx + i]) continue;
        const int64_t o = (int64_t)j * P + i;
        const R s = stg[o], e = elv[o];
        const bool wet = tl ? (msl > e + mad) : (s > e + mad);
        const double w0 = (double)s + (double)e, d1 = (double)s - (double)e;
        const double e_flow = wet ? w0 * d1 : 0.0;
        const double w2 = (double)msl + (double)e, d3 = (double)msl - (double)e;
        const double e_const = (msl > e + mad) ? w2 * d3 : 0.0;
        pe += (double)(area[j] * g * half) * (e_flow - e_const);
        if (!wet) continue;
        mxs = (s > mxs) ? s : mxs;
        mns = (s < mns) ? s : mns;
        R speed_sq;
        const R u = uh[o], v = vh[o];
        if (staggered) {
            R dE, dN;
            if (tl) {
                dE = half * ((msl - e) + (msl - elv[o + 1]));
                dN = half * ((msl - e) + (msl - elv[o + P]));
            } else {
                dE = half * ((s - e) + (stg[o + 1] - elv[o + 1]));
                dN = half * ((s - e) + (stg[o + P] - elv[o + P]));
            }
            const R dEi = (dE > mad) ? one / dE : zero;
            const R dNi = (dN > mad) ? one / dN : zero;
            speed_sq = u * u * (dEi * dEi) + v * v * (dNi * dNi);
            ke += (double)(half * (area[j] * u * u * dEi + half * (area[j] + area[j + 1]) * v * v * dNi));
        } else {
            const R dc = s - e;
            speed_sq = (u * u + v * v) / (dc * dc);
            ke += (double)(area[j] * half * dc * speed_sq);
        }
        mxv = (speed_sq > mxv) ? speed_sq : mxv;
        mnv = (speed_sq < mnv) ? speed_sq : mnv;
    }
    for (int off = 16; off > 0; off >>= 1) {
        pe += __shfl_down_sync(0xffffffffu, pe, off);
        ke += __shfl_down_sync(0xffffffffu, ke, off);
        const R a = __shfl_down_sync(0xffffffffu, mxs, off); mxs = (a > mxs) ? a : mxs;
        const R b = __shfl_down_sync(0xffffffffu, mns, off); mns = (b < mns) ? b : mns;
        const R c = __shfl_down_sync(0xffffffffu, mxv, off); mxv = (c > mxv) ? c : mxv;
        const R d = __shfl_down_sync(0xffffffffu, mnv, off); mnv = (d < mnv) ? d : mnv;
    }
    if (lane == 0) {
        double *w = out6 + 6 * (int64_t)j;
        w[0] = pe; w[1] = ke; w[2] = (double)mxs; w[3] = (double)mns; w[4] = (double)mxv; w[5] = (double)mnv;
    }
}

template <typename R>
__global__ void stats_final_kernel(int ny, int ecw, const double *rows6, double *out7)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double pe = 0.0, ke = 0.0;
    R mxs = -K<R>::huge(), mns = K<R>::huge(), mxv = R(0), mnv = K<R>::huge();
    for (int j = ecw; j <= ny - 1 - ecw; j++) {
        const double *w = rows6 + 6 * (int64_t)j;
        pe = pe + w[0];
        ke = ke + w[1];
        mxs = (R(w[2]) > mxs) ? R(w[2]) : mxs;
        mns = (R(w[3]) < mns) ? R(w[3]) : mns;
        mxv = (R(w[4]) > mxv) ? R(w[4]) : mxv;
        mnv = (R(w[5]) < mnv) ? R(w[5]) : mnv;
    }
    out7[0] = (double)mxs;
    out7[1] = (double)R(sqrt((double)mxv));
    out7[2] = (double)mns;
    out7[3] = (double)R(sqrt((double)mnv));
    out7[4] = pe;
    out7[5] = ke;
    out7[6] = ke + pe;
}

}  // namespace

template <typename R>
cudaError_t launch_domain_statistics(int nx, int ny, int64_t P, const R *stg, const R *uh, const R *vh, const R *elv,
                                     const R *area, const uint8_t *mask, int ecw, int staggered, int tl, double msl,
                                     double *rows6, double *out7, cudaStream_t s)
{
    const int rows = ny - 2 * ecw;
    if (rows <= 0) return cudaErrorInvalidValue;
    const int threads = 256, blocks = (rows * 32 + threads - 1) / threads;
    stats_row_kernel<R><<<blocks, threads, 0, s>>>(nx, ny, P, stg, uh, vh, elv, area, mask, ecw, staggered, tl, R(msl),
                                                   rows6);
    stats_final_kernel<R><<<1, 32, 0, s>>>(ny, ecw, rows6, out7);
    return cudaGetLastError();
}

template cudaError_t launch_domain_statistics<double>(int, int, int64_t, const double *, const double *,
                                                      const double *, const double *, const double *, const uint8_t *,
                                                      int, int, int, double, double *, double *, cudaStream_t);
template cudaError_t launch_domain_statistics<float>(int, int, int64_t, const float *, const float *, const float *,
                                                     const float *, const float *, const uint8_t *, int, int, int,
                                                     double, double *, double *, cudaStream_t);

template <typename R>
cudaError_t launch_volume_interior(int nx, int ny, int64_t pitch, const R *stg, const R *elv, const R *area,
                                   int n_ext, double *row_sums, double *out, cudaStream_t s, const uint8_t *mask)
{
    const int rows = ny - 2 * n_ext;
    if (rows > 0) {
        const int threads = 256;
        const int blocks = (rows * 32 + threads - 1) / threads;
        row_volume_kernel<R><<<blocks, threads, 0, s>>>(nx, ny, pitch, stg, elv, n_ext, row_sums, mask);
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
                                                    const double *, int, double *, double *, cudaStream_t,
                                                    const uint8_t *);
template cudaError_t launch_volume_interior<float>(int, int, int64_t, const float *, const float *, const float *,
                                                   int, double *, double *, cudaStream_t, const uint8_t *);
template cudaError_t launch_timestep_max<double>(int, int, int64_t, const double *, const double *, const double *,
                                                 const double *, double, int, double, double *, int, double *,
                                                 cudaStream_t);
template cudaError_t launch_timestep_max<float>(int, int, int64_t, const float *, const float *, const float *,
                                                const float *, double, int, double, double *, int, double *,
                                                cudaStream_t);

}  // namespace swals
