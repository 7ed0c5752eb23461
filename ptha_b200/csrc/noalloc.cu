// noalloc.cu -- allocation-free variant of the volume_interior reduction.
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA graph is
// being captured (allocation is not allowed inside stream capture), hosts
// whose device memory is owned by another allocator (a framework's caching
// pool) and loops that cannot afford cudaMalloc's implicit device-wide
// synchronisation.  For them swals_gpu_volume_interior_noalloc computes
// domain%volume_interior (domain_mod.f90:1815-1849) from device arrays the
// caller already owns, with its per-row scratch in a fixed file-scope
// device array instead of an allocation.
//
// The scratch array is SWALS_NOALLOC_MAX_ROWS doubles (512 KiB), held by
// every GPU that loads the library until the process exits.  All calls on a
// device share it and it keeps the last call's partial sums; every row that
// a call reads is written by the same call first, so nothing has to be
// cleared between calls.  Calls whose kernels overlap on the GPU (different
// streams without ordering) race on the shared scratch.  The array's device
// address is looked up once per device and context (again after a device
// reset), never per call.
#include "swals_kernels.h"
#include "../../include/swals_gpu.h"

#include <cuda.h>   // CUcontext (type only; the function is fetched through the runtime)
#include <mutex>

namespace {

static __device__ __align__(256) double g_noalloc_row_sums[SWALS_NOALLOC_MAX_ROWS];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
// Device address of g_noalloc_row_sums, per device ordinal, and the context
// it was looked up in: after cudaDeviceReset (or any new primary context on
// that ordinal) the array lives at a new address, so a changed context
// means a fresh look-up rather than a stale pointer.
double *g_row_sums_dev[kMaxDevices] = {};
CUcontext g_row_sums_ctx[kMaxDevices] = {};

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);

CUcontext current_context()
{
    static CtxGetCurrentFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (CtxGetCurrentFn)p;
    }
    CUcontext c = nullptr;
    if (fn) fn(&c);
    return c;
}

template <typename R>
__global__ void noalloc_row_volume_kernel(int nx, int ny, int64_t P, const R *stg, const R *elv, int n_ext,
                                          double *row_sums)
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
__global__ void noalloc_volume_total_kernel(int ny, int n_ext, const R *area, const double *row_sums, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double vol = 0.0;
    for (int r = n_ext; r <= ny - n_ext - 1; r++) vol = vol + (double)area[r] * row_sums[r];
    *out = vol;
}

int noalloc_fail(int code, const char *msg)
{
    swals::set_last_error(msg);
    return code;
}

// Once per device, with that device current: the device address of the
// scratch array.  The host-side symbol is only a stand-in for it.
int scratch_for_current_device(double **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return noalloc_fail(SWALS_ERR_NO_DEVICE, "no current CUDA device");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    // A thread that has not used the runtime yet may have no context bound
    // (null): the look-up below binds the device's primary context.
    const CUcontext ctx = current_context();
    if (!g_row_sums_dev[dev] || !ctx || g_row_sums_ctx[dev] != ctx) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_row_sums);
        if (e != cudaSuccess || !p) return noalloc_fail(SWALS_ERR_CUDA, "cudaGetSymbolAddress failed for the scratch array");
        g_row_sums_dev[dev] = (double *)p;
        g_row_sums_ctx[dev] = current_context();
    }
    *out = g_row_sums_dev[dev];
    return SWALS_OK;
}

}  // namespace

extern "C" int swals_gpu_volume_interior_noalloc(const void *stg, const void *elv, const void *area, int32_t nx,
                                                 int32_t ny, int64_t pitch_elems, int32_t real_bytes,
                                                 int32_t exterior_cells_width, double *out_device, void *stream)
{
    if (!stg || !elv || !area || !out_device) return noalloc_fail(SWALS_ERR_INVALID_ARGUMENT, "NULL pointer argument");
    if (real_bytes != 8 && real_bytes != 4) return noalloc_fail(SWALS_ERR_INVALID_ARGUMENT, "real_bytes must be 4 or 8");
    if (nx < 1 || ny < 1 || pitch_elems < nx || exterior_cells_width < 0)
        return noalloc_fail(SWALS_ERR_INVALID_ARGUMENT, "invalid nx, ny, pitch or exterior_cells_width");
    if (ny > SWALS_NOALLOC_MAX_ROWS)
        return noalloc_fail(SWALS_ERR_CAPACITY,
                            "ny exceeds SWALS_NOALLOC_MAX_ROWS (65536): use swals_gpu_volume_interior instead");
    double *rows = nullptr;
    int rc = scratch_for_current_device(&rows);
    if (rc != SWALS_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int n_ext = exterior_cells_width;
    const int nrows = ny - 2 * n_ext;
    const int threads = 256;
    if (real_bytes == 8) {
        if (nrows > 0)
            noalloc_row_volume_kernel<double><<<(nrows * 32 + threads - 1) / threads, threads, 0, s>>>(
                nx, ny, pitch_elems, (const double *)stg, (const double *)elv, n_ext, rows);
        noalloc_volume_total_kernel<double><<<1, 32, 0, s>>>(ny, n_ext, (const double *)area, rows, out_device);
    } else {
        if (nrows > 0)
            noalloc_row_volume_kernel<float><<<(nrows * 32 + threads - 1) / threads, threads, 0, s>>>(
                nx, ny, pitch_elems, (const float *)stg, (const float *)elv, n_ext, rows);
        noalloc_volume_total_kernel<float><<<1, 32, 0, s>>>(ny, n_ext, (const float *)area, rows, out_device);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(SWALS_ERR_CUDA, cudaGetErrorString(e));
    return SWALS_OK;
}
