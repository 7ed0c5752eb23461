// batch.cu -- many independent linear-leapfrog initial conditions on one grid.
//
// A batch borrows the grid of a 'linear' domain (geometry, metrics, ELV,
// solver options) and owns `nbatch` copies of the state planes (STG, UH, VH;
// ping-pong) plus optional per-instance max_stage.  Each step is one launch
// of the linear leapfrog kernel over all instances (blockIdx.z = instance
// group), so ELV and the truly-linear face depths are read once per tile for
// several instances.  evolve() replays the step sequence from a CUDA graph.
// The reference has no batched form: a batch of B instances equals B
// independent domain%evolve_one_step sequences (domain_mod_linear_solver_
// include.f90:58-571), which the tests check instance by instance.
#include "domain_internal.h"

#include <cfloat>
#include <cstring>
#include <vector>

struct swals_batch {
    swals_domain *grid = nullptr;   // borrowed
    int nbatch = 0;
    void *pool = nullptr;
    void *state[2] = {nullptr, nullptr};  // each: nbatch x [STG, UH, VH] planes
    void *max_stage = nullptr;            // nbatch planes or null
    int cur = 0;
    int64_t plane = 0;        // elements per plane (pitch * ny)
    int64_t inst_stride = 0;  // elements per instance (3 planes)
    double time = 0.0;
    int64_t nsteps = 0;
    int tile_cfg = 0;
    // gauges
    int n_gauges = 0, capacity = 0, nrec = 0;
    int *d_sites = nullptr;
    double *d_records = nullptr;
    std::vector<int> h_sites;
    // graph of `graph_steps` steps (even, so the ping-pong parity is unchanged)
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    double graph_dt = 0.0;
    bool graph_gauges = false;
    int graph_cur = -1;       // state buffer the graph starts from (and returns to)
    int *d_rec = nullptr;     // device record counter used inside graphs
};

namespace {

using swals::api_cuda_fail;
using swals::api_fail;

#define BCK(call)                                                 \
    do {                                                          \
        cudaError_t _e = (call);                                  \
        if (_e != cudaSuccess) return api_cuda_fail(_e, #call);   \
    } while (0)

size_t esz(const swals_batch *b) { return b->grid->fp64 ? 8 : 4; }

template <typename R>
__global__ void fill_kernel_b(R *p, int64_t n, R v)
{
    int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q < n) p[q] = v;
}

// Gauge sampling for graph replay: the record index lives on the device.
template <typename R>
__global__ void batch_gauge_dev_kernel(int64_t P, const R *stg0, int64_t inst_stride, int nbatch, const int *site_ij,
                                       int n, double *records, const int *d_rec, int capacity)
{
    const int rec = *d_rec;
    if (rec >= capacity) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n * nbatch) return;
    const int b = q / n, gi = q - b * n;
    const int i = site_ij[2 * gi], r = site_ij[2 * gi + 1];
    records[((int64_t)rec * nbatch + b) * n + gi] = (double)stg0[(int64_t)b * inst_stride + (int64_t)r * P + i];
}

__global__ void inc_kernel(int *c) { *c += 1; }

template <typename R>
cudaError_t one_step(swals_batch *b, double dt, bool gauges_dev)
{
    using namespace swals;
    swals_domain *g = b->grid;
    const int in = b->cur, out = 1 - b->cur;
    StepPlanes<R> p;
    p.nx = g->nx; p.ny = g->ny; p.pitch = g->pitch;
    R *si = (R *)b->state[in], *so = (R *)b->state[out];
    p.stg = si; p.uh = si + b->plane; p.vh = si + 2 * b->plane;
    p.stg_o = so; p.uh_o = so + b->plane; p.vh_o = so + 2 * b->plane;
    p.elv = (R *)g->elv;
    p.max_stage = (R *)b->max_stage;
    p.manning_sq = nullptr;
    LaunchHook hook = hook_of(g);
    cudaError_t e = launch_linear_batch<R>(p, b->inst_stride, b->plane, b->nbatch, metrics_of<R>(g), g->cfg, R(dt),
                                           b->tile_cfg, g->stream, hook);
    if (e != cudaSuccess) return e;
    b->cur = out;
    if (b->n_gauges > 0 && gauges_dev) {
        const int tot = b->n_gauges * b->nbatch;
        hook(CAT_GAUGES, 0);
        batch_gauge_dev_kernel<R><<<(tot + 255) / 256, 256, 0, g->stream>>>(
            g->pitch, (const R *)b->state[b->cur], b->inst_stride, b->nbatch, b->d_sites, b->n_gauges, b->d_records,
            b->d_rec, b->capacity);
        inc_kernel<<<1, 1, 0, g->stream>>>(b->d_rec);
        hook(CAT_GAUGES, 1);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t step_any(swals_batch *b, double dt, bool gauges)
{
    return b->grid->fp64 ? one_step<double>(b, dt, gauges) : one_step<float>(b, dt, gauges);
}

void drop_graph(swals_batch *b)
{
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_steps = 0;
}

int build_graph(swals_batch *b, int steps, double dt, bool gauges)
{
    drop_graph(b);
    cudaStream_t s = b->grid->stream;
    const int cur0 = b->cur;
    const int64_t launches0 = b->grid->launches;
    cudaGraph_t graph = nullptr;
    BCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < steps && e == cudaSuccess; k++) e = step_any(b, dt, gauges);
    cudaError_t e2 = cudaStreamEndCapture(s, &graph);
    b->cur = cur0;  // capture does not execute; restore the buffer parity
    b->grid->launches = launches0;
    if (e != cudaSuccess) return api_cuda_fail(e, "batch step capture");
    if (e2 != cudaSuccess) return api_cuda_fail(e2, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&b->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return api_cuda_fail(e, "cudaGraphInstantiate");
    b->graph_steps = steps;
    b->graph_dt = dt;
    b->graph_gauges = gauges;
    b->graph_cur = cur0;
    return SWALS_OK;
}

int copy_instances(swals_batch *b, int first, int count, void *host, int nvar, bool to_dev, bool max_plane)
{
    swals_domain *g = b->grid;
    const size_t es = esz(b);
    const size_t hplane = (size_t)g->nx * g->ny * es;
    for (int q = 0; q < count; q++) {
        for (int v = 0; v < nvar; v++) {
            char *dev;
            if (max_plane) dev = (char *)b->max_stage + ((size_t)(first + q) * b->plane) * es;
            else dev = (char *)b->state[b->cur] + ((size_t)(first + q) * b->inst_stride + v * b->plane) * es;
            char *h = (char *)host + ((size_t)q * nvar + v) * hplane;
            if (to_dev)
                BCK(cudaMemcpy2DAsync(dev, g->pitch * es, h, g->nx * es, g->nx * es, g->ny, cudaMemcpyHostToDevice,
                                      g->stream));
            else
                BCK(cudaMemcpy2DAsync(h, g->nx * es, dev, g->pitch * es, g->nx * es, g->ny, cudaMemcpyDeviceToHost,
                                      g->stream));
        }
    }
    BCK(cudaStreamSynchronize(g->stream));
    return to_dev ? SWALS_OK : swals::api_check_bulk_waits(g->stream);
}

}  // namespace

extern "C" {

int swals_gpu_batch_create(swals_domain *grid, int32_t nbatch, int32_t record_max_stage, swals_batch **out)
{
    if (!grid || !out || nbatch < 1) return api_fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    *out = nullptr;
    if (strncmp(grid->desc.timestepping_method, "linear", 6) != 0 || grid->desc.timestepping_method[6] > ' ')
        return api_fail(SWALS_ERR_UNSUPPORTED, "batches are implemented for timestepping_method='linear' only");
    if (grid->cfg.n_forcing)
        return swals::api_fail(SWALS_ERR_UNSUPPORTED, "forcing patches are not supported here");
    if (grid->cfg.bc_kind != SWALS_BC_NONE)
        return api_fail(SWALS_ERR_UNSUPPORTED, "batches support walls via elevation only (no boundary routine)");
    swals_batch *b = new swals_batch();
    b->grid = grid;
    b->nbatch = nbatch;
    b->plane = grid->pitch * (int64_t)grid->ny;
    b->inst_stride = 3 * b->plane;
    const size_t es = esz(b);
    const size_t state_bytes = (size_t)nbatch * b->inst_stride * es;
    const size_t max_bytes = record_max_stage ? (size_t)nbatch * b->plane * es : 0;
    size_t total = 2 * state_bytes + max_bytes + 256;
    cudaError_t e = cudaMalloc(&b->pool, total);
    if (e != cudaSuccess) {
        delete b;
        return api_cuda_fail(e, "batch allocation");
    }
    b->state[0] = b->pool;
    b->state[1] = (char *)b->pool + state_bytes;
    b->max_stage = record_max_stage ? (char *)b->pool + 2 * state_bytes : nullptr;
    b->d_rec = (int *)((char *)b->pool + 2 * state_bytes + max_bytes);
    e = cudaMemsetAsync(b->pool, 0, total, grid->stream);
    if (e == cudaSuccess && b->max_stage) {
        const float init = -0.99f * FLT_MAX;
        const int64_t n = (int64_t)nbatch * b->plane;
        const unsigned blocks = (unsigned)((n + 255) / 256);
        if (grid->fp64) fill_kernel_b<double><<<blocks, 256, 0, grid->stream>>>((double *)b->max_stage, n, (double)init);
        else fill_kernel_b<float><<<blocks, 256, 0, grid->stream>>>((float *)b->max_stage, n, init);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(grid->stream);
    if (e != cudaSuccess) {
        cudaFree(b->pool);
        delete b;
        return api_cuda_fail(e, "batch initialisation");
    }
    *out = b;
    return SWALS_OK;
}

int swals_gpu_batch_destroy(swals_batch *b)
{
    if (!b) return SWALS_OK;
    cudaStreamSynchronize(b->grid->stream);
    drop_graph(b);
    if (b->d_sites) cudaFree(b->d_sites);
    if (b->d_records) cudaFree(b->d_records);
    cudaFree(b->pool);
    delete b;
    return SWALS_OK;
}

int swals_gpu_batch_upload_U(swals_batch *b, int32_t first, int32_t count, const void *U3)
{
    if (!b || !U3 || first < 0 || count < 0 || first + count > b->nbatch)
        return api_fail(SWALS_ERR_INVALID_ARGUMENT, "bad instance range");
    return copy_instances(b, first, count, (void *)U3, 3, true, false);
}

int swals_gpu_batch_download_U(swals_batch *b, int32_t first, int32_t count, void *U3)
{
    if (!b || !U3 || first < 0 || count < 0 || first + count > b->nbatch)
        return api_fail(SWALS_ERR_INVALID_ARGUMENT, "bad instance range");
    return copy_instances(b, first, count, U3, 3, false, false);
}

int swals_gpu_batch_download_max_stage(swals_batch *b, int32_t first, int32_t count, void *host)
{
    if (!b || !host || first < 0 || count < 0 || first + count > b->nbatch)
        return api_fail(SWALS_ERR_INVALID_ARGUMENT, "bad instance range");
    if (!b->max_stage) return api_fail(SWALS_ERR_INVALID_ARGUMENT, "batch created without max_stage");
    return copy_instances(b, first, count, host, 1, false, true);
}

int swals_gpu_batch_device_state(swals_batch *b, void **stg0, int64_t *pitch_elems, int64_t *plane_elems,
                                 int64_t *instance_stride_elems)
{
    if (!b) return api_fail(SWALS_ERR_INVALID_ARGUMENT, "NULL batch");
    if (stg0) *stg0 = b->state[b->cur];
    if (pitch_elems) *pitch_elems = b->grid->pitch;
    if (plane_elems) *plane_elems = b->plane;
    if (instance_stride_elems) *instance_stride_elems = b->inst_stride;
    return SWALS_OK;
}

int swals_gpu_batch_gauges_setup(swals_batch *b, const double *xy, int32_t n, int32_t capacity)
{
    if (!b || n < 0 || capacity < 0 || (n > 0 && !xy)) return api_fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    swals_domain *g = b->grid;
    drop_graph(b);
    if (b->d_sites) { cudaFree(b->d_sites); b->d_sites = nullptr; }
    if (b->d_records) { cudaFree(b->d_records); b->d_records = nullptr; }
    b->n_gauges = 0;
    b->h_sites.assign(2 * (size_t)n, 0);
    const int nxy[2] = {g->nx, g->ny};
    for (int q = 0; q < n; q++) {
        for (int k = 0; k < 2; k++) {
            double dx = g->desc.lw[k] / nxy[k];
            double qv;
            if (g->fp64) qv = (xy[2 * q + k] - g->desc.lower_left[k]) / dx;
            else qv = (double)(((float)xy[2 * q + k] - (float)g->desc.lower_left[k]) /
                               ((float)g->desc.lw[k] / ((float)nxy[k] * 1.0f)));
            int f = (int)floor(qv);
            if (nxy[k] - 1 < f) f = nxy[k] - 1;
            if (f < 0) return api_fail(SWALS_ERR_INVALID_ARGUMENT, "gauge outside the domain");
            b->h_sites[2 * q + k] = f;
        }
    }
    if (n > 0) {
        BCK(cudaMalloc(&b->d_sites, sizeof(int) * 2 * (size_t)n));
        BCK(cudaMemcpy(b->d_sites, b->h_sites.data(), sizeof(int) * 2 * (size_t)n, cudaMemcpyHostToDevice));
        if (capacity > 0) BCK(cudaMalloc(&b->d_records, sizeof(double) * (size_t)n * b->nbatch * capacity));
    }
    b->n_gauges = capacity > 0 ? n : 0;
    b->capacity = capacity;
    b->nrec = 0;
    BCK(cudaMemsetAsync(b->d_rec, 0, sizeof(int), g->stream));
    BCK(cudaStreamSynchronize(g->stream));
    return SWALS_OK;
}

int swals_gpu_batch_gauges_read(swals_batch *b, double *out, int32_t max_records, int32_t *n_records)
{
    if (!b || !n_records) return api_fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    swals_domain *g = b->grid;
    int rec = 0;
    BCK(cudaMemcpyAsync(&rec, b->d_rec, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
    BCK(cudaStreamSynchronize(g->stream));
    int valid = rec < b->capacity ? rec : b->capacity;
    int ncopy = valid < max_records ? valid : max_records;
    if (ncopy > 0 && out)
        BCK(cudaMemcpy(out, b->d_records, sizeof(double) * (size_t)b->n_gauges * b->nbatch * ncopy,
                       cudaMemcpyDeviceToHost));
    *n_records = ncopy;
    if (rec > b->capacity)
        return api_fail(SWALS_ERR_CAPACITY, "batch gauge buffer full");
    return SWALS_OK;
}

int swals_gpu_batch_evolve(swals_batch *b, int32_t nsteps, double dt)
{
    if (!b || nsteps < 0) return api_fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    const bool gauges = b->n_gauges > 0;
    if (b->nsteps == 0 && b->max_stage && nsteps > 0) {
        // update_max_quantities before the first step (domain_mod.f90:1719)
        swals_domain *g = b->grid;
        for (int q = 0; q < b->nbatch; q++) {
            cudaError_t e;
            if (g->fp64)
                e = swals::launch_update_max_stage<double>(g->nx, g->ny, g->pitch,
                        (const double *)b->state[b->cur] + q * b->inst_stride, (double *)b->max_stage + q * b->plane,
                        g->cfg, g->stream);
            else
                e = swals::launch_update_max_stage<float>(g->nx, g->ny, g->pitch,
                        (const float *)b->state[b->cur] + q * b->inst_stride, (float *)b->max_stage + q * b->plane,
                        g->cfg, g->stream);
            if (e != cudaSuccess) return api_cuda_fail(e, "max_stage before the first step");
        }
    }
    int done = 0;
    if (nsteps >= 2) {
        int gsteps = nsteps < 32 ? (nsteps & ~1) : 32;
        // an odd number of single steps since the capture flips the buffer
        // the graph would start from: capture again
        if (!b->graph || b->graph_steps != gsteps || b->graph_dt != dt || b->graph_gauges != gauges ||
            b->graph_cur != b->cur) {
            int rc = build_graph(b, gsteps, dt, gauges);
            if (rc) return rc;
        }
        while (nsteps - done >= b->graph_steps) {
            BCK(cudaGraphLaunch(b->graph, b->grid->stream));
            b->grid->launches += (int64_t)b->graph_steps * (gauges ? 3 : 1);
            done += b->graph_steps;
        }
    }
    for (; done < nsteps; done++) BCK(step_any(b, dt, gauges));
    for (int k = 0; k < nsteps; k++) {
        // domain%time advances by dt/2 twice per leapfrog step (:119, :571)
        if (b->grid->fp64) b->time = (b->time + (double)(dt * 0.5)) + (double)(0.5 * dt);
        else b->time = (b->time + (double)((float)dt * 0.5f)) + (double)(0.5f * (float)dt);
    }
    b->nsteps += nsteps;
    return SWALS_OK;
}

int swals_gpu_batch_time(swals_batch *b, double *time, int64_t *nsteps)
{
    if (!b) return api_fail(SWALS_ERR_INVALID_ARGUMENT, "NULL batch");
    if (time) *time = b->time;
    if (nsteps) *nsteps = b->nsteps;
    return SWALS_OK;
}

int swals_gpu_batch_tune(swals_batch *b, int32_t *cfg_out, double *ms_per_step_out)
{
    if (!b) return api_fail(SWALS_ERR_INVALID_ARGUMENT, "NULL batch");
    drop_graph(b);
    swals_domain *g = b->grid;
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    const int ncfg = swals::linear_tile_config_count();
    int best = 0;
    float best_ms = 1e30f;
    const int saved = b->tile_cfg;
    for (int c = 0; c < ncfg; c++) {
        b->tile_cfg = c;
        // dt = 0 steps leave the state unchanged but move the same bytes and
        // do the same arithmetic; an even count keeps the buffer parity.
        for (int k = 0; k < 2; k++) BCK(step_any(b, 0.0, false));
        BCK(cudaEventRecord(e0, g->stream));
        for (int k = 0; k < 6; k++) BCK(step_any(b, 0.0, false));
        BCK(cudaEventRecord(e1, g->stream));
        BCK(cudaEventSynchronize(e1));
        float ms = 0.f;
        BCK(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) { best_ms = ms; best = c; }
    }
    (void)saved;
    b->tile_cfg = best;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cfg_out) *cfg_out = best;
    if (ms_per_step_out) *ms_per_step_out = best_ms / 6.0;
    return SWALS_OK;
}

int swals_gpu_batch_tile_config_count(int32_t *n)
{
    if (!n) return api_fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    *n = swals::linear_tile_config_count();
    return SWALS_OK;
}

int swals_gpu_batch_set_tile_config(swals_batch *b, int32_t cfg)
{
    if (!b || cfg < 0 || cfg >= swals::linear_tile_config_count())
        return api_fail(SWALS_ERR_INVALID_ARGUMENT, "bad tile configuration");
    drop_graph(b);
    b->tile_cfg = cfg;
    return SWALS_OK;
}

}  // extern "C"
