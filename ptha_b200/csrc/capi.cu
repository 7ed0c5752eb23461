// capi.cu -- the extern "C" boundary (include/swals_gpu.h) and the device
// domain that stands behind it.
//
// swals_domain mirrors the parts of SWALS's domain_type (domain_mod.f90:137-
// 507) that the time-step hot path touches: geometry, solver options, the
// state arrays U / max_U(:,:,1) / manning_squared, and the scalar state
// (time, max_dt, nsteps_advanced, boundary-flux integrals).  The state lives
// on the device; the host only keeps descriptors and the 1-D metrics.
#include "domain_internal.h"

#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    return fail(e == cudaErrorMemoryAllocation ? SWALS_ERR_OUT_OF_MEMORY : SWALS_ERR_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
}

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t _e = (call);                                   \
        if (_e != cudaSuccess) return cuda_fail(_e, #call);        \
    } while (0)

int parse_method(const char *s, int *m, double *def_cfl, double *def_theta)
{
    struct { const char *name; int m; double cfl; double theta; } tab[] = {
        {"rk2", M_RK2, 0.99, 1.6},
        {"rk2n", M_RK2N, 0.99, 1.6},
        {"midpoint", M_MIDPOINT, 0.99, 1.6},
        {"euler", M_EULER, 0.9, 0.9},
        {"linear", M_LINEAR, 0.7, -1.0},
        {"leapfrog_linear_plus_nonlinear_friction", M_LF_LIN_NLFRIC, 0.7, -1.0},
        {"cliffs", M_CLIFFS, 0.7, -1.0},
        {"leapfrog_nonlinear", M_LF_NONLINEAR, 0.7, -1.0},
    };
    // Fortran compares TRIM()ed strings: ignore trailing blanks.
    std::string name(s);
    while (!name.empty() && (name.back() == ' ' || name.back() == '\0')) name.pop_back();
    for (auto &t : tab) {
        if (name == t.name) {
            *m = t.m;
            *def_cfl = t.cfl;
            *def_theta = t.theta;
            return 1;
        }
    }
    return 0;
}

// domain%compute_fluxes_inner_method (domain_mod.f90:1448-1484) -> fv::FLUX_*
// bits; empty = the default 'DE1_low_fr_diffusion'.  -1: not implemented.
int parse_flux_method(const char *s, size_t cap)
{
    std::string name(s, strnlen(s, cap));
    while (!name.empty() && name.back() == ' ') name.pop_back();
    if (name.empty() || name == "DE1_low_fr_diffusion") return 0;
    if (name == "DE1") return swals::FLUX_PLAIN_DIFFUSION;
    if (name == "DE1_upwind_transverse") return swals::FLUX_PLAIN_DIFFUSION | swals::FLUX_UPWIND_TRANSVERSE;
    if (name == "DE1_low_fr_diffusion_upwind_transverse") return swals::FLUX_UPWIND_TRANSVERSE;
    return -1;
}

bool is_staggered(int m) { return m == M_LINEAR || m == M_LF_LIN_NLFRIC || m == M_LF_NONLINEAR; }

}  // namespace

void swals::set_last_error(const char *msg) { g_last_error = msg; }
int swals::api_fail(int code, const char *msg) { g_last_error = msg; return code; }
int swals::api_cuda_fail(cudaError_t e, const char *what) { return cuda_fail(e, what); }
int swals::api_check_bulk_waits(cudaStream_t s)
{
    if (!swals::linear_bulk_launched()) return SWALS_OK;
    unsigned n = 0;
    cudaError_t e = swals::linear_wait_expired(&n, true, s);
    if (e != cudaSuccess) return cuda_fail(e, "reading the expired-wait count");
    if (n)
        return fail(SWALS_ERR_CUDA,
                    "%u bounded waits for bulk-copied rows ran out: rows of a linear step were not updated", n);
    return SWALS_OK;
}


namespace {

template <typename R>
void compute_geometry(swals_domain *d)
{
    // Host restatement of domain_mod.f90:925-1014 in the state precision R,
    // evaluating libm functions in double exactly as a C compiler would for
    // the reference's expressions.
    const int nx = d->nx, ny = d->ny;
    const swals_domain_desc &D = d->desc;
    const R one = R(1), half = R(0.5);
    const R radius_earth = R(6371000.0);
    const R pi = R(std::acos((double)R(-1.0)));
    const R deg2rad = pi / R(180.0);
    const R omega = R(7.292115e-05);
    const R dx1 = R(D.lw[0]) / (R(nx) * one);
    const R dx2 = R(D.lw[1]) / (R(ny) * one);
    std::vector<R> x(nx), y(ny), dxb(ny + 1), dyl(nx + 1), area(ny), cor(ny, R(0)), cor_be(ny + 1, R(0)),
        tanlat(ny, R(0));
    for (int i = 1; i <= nx; i++) x[i - 1] = R(D.lower_left[0]) + ((R(i) - half) / (R(nx) * one)) * R(D.lw[0]);
    for (int i = 1; i <= ny; i++) y[i - 1] = R(D.lower_left[1]) + ((R(i) - half) / (R(ny) * one)) * R(D.lw[1]);
    if (D.spherical) {
        for (int i = 0; i < ny; i++) tanlat[i] = R(std::tan((double)(y[i] * deg2rad))) / radius_earth;
        if (D.coriolis) {
            for (int i = 0; i < ny; i++) {
                cor[i] = (R(2.0) * R(std::sin((double)(y[i] * deg2rad)))) * omega;
                cor_be[i] = (R(2.0) * omega) * R(std::sin((double)((y[i] - half * dx2) * deg2rad)));
            }
            cor_be[ny] = (R(2.0) * omega) * R(std::sin((double)((y[ny - 1] + half * dx2) * deg2rad)));
        }
        for (int i = 0; i <= nx; i++) dyl[i] = (dx2 * deg2rad) * radius_earth;
        for (int i = 0; i <= ny; i++) {
            R coslat_be = (i < ny) ? R(std::cos((double)((y[i] - half * dx2) * deg2rad)))
                                   : R(std::cos((double)((y[ny - 1] + half * dx2) * deg2rad)));
            dxb[i] = ((dx1 * deg2rad) * radius_earth) * coslat_be;
        }
        // area_lonlat_rectangle(flat=.TRUE.), spherical_mod.f90:48-51
        for (int i = 0; i < ny; i++) {
            const R lat1 = y[i] - dx2 * half;
            R a = radius_earth * radius_earth;
            a = a * R(std::cos((double)((lat1 + R(0.5) * dx2) * deg2rad)));
            a = a * R(std::fabs((double)dx2));
            a = a * deg2rad;
            a = a * R(std::fmod(std::fabs((double)dx1), (double)R(360.0)));
            a = a * deg2rad;
            area[i] = a;
        }
    } else {
        for (int i = 0; i <= nx; i++) dyl[i] = dx2;
        for (int i = 0; i <= ny; i++) dxb[i] = dx1;
        for (int i = 0; i < ny; i++) area[i] = dx1 * dx2;
    }
    const std::vector<R> *src[8] = {&dxb, &dyl, &area, &cor, &cor_be, &tanlat, &x, &y};
    for (int k = 0; k < 8; k++) {
        d->h_metric[k].assign(src[k]->begin(), src[k]->end());
    }
}

template <typename R>
int upload_metrics_t(swals_domain *d)
{
    for (int k = 0; k < 8; k++) {
        std::vector<R> tmp(d->h_metric[k].begin(), d->h_metric[k].end());
        CK(cudaMemcpyAsync(d->metric[k], tmp.data(), tmp.size() * sizeof(R), cudaMemcpyHostToDevice, d->stream));
        CK(cudaStreamSynchronize(d->stream));
    }
    return SWALS_OK;
}


template <typename R>
__global__ void fill_kernel(R *p, int64_t n, R v)
{
    int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q < n) p[q] = v;
}

size_t esize(const swals_domain *d) { return d->fp64 ? 8 : 4; }

int copy_plane(swals_domain *d, void *dev, const void *host, bool to_dev)
{
    const size_t es = esize(d);
    if (to_dev)
        CK(cudaMemcpy2DAsync(dev, d->pitch * es, host, d->nx * es, d->nx * es, d->ny, cudaMemcpyHostToDevice,
                             d->stream));
    else
        CK(cudaMemcpy2DAsync((void *)host, d->nx * es, dev, d->pitch * es, d->nx * es, d->ny,
                             cudaMemcpyDeviceToHost, d->stream));
    return SWALS_OK;
}

void *plane_ptr(swals_domain *d, int k)
{
    if (k == 4) return d->elv;
    return d->planes[d->cur][k - 1];
}

cudaEvent_t take_event(swals_domain *d)
{
    if (!d->ev_pool.empty()) {
        cudaEvent_t e = d->ev_pool.back();
        d->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void on_launch(void *ctx, int cat, int phase)
{
    swals_domain *d = (swals_domain *)ctx;
    if (phase == 0) d->launches++;
    if (!d->timers_on) return;
    cudaEvent_t e = take_event(d);
    cudaEventRecord(e, d->stream);
    if (phase == 0) d->open_ev[cat] = e;
    else d->pending.push_back({cat, d->open_ev[cat], e});
}

}  // namespace

swals::LaunchHook swals::hook_of(swals_domain *d)
{
    swals::LaunchHook h;
    h.fn = on_launch;
    h.ctx = d;
    return h;
}

namespace {

template <typename R>
int evolve_t(swals_domain *d, double timestep, int has_dt)
{
    using namespace swals;
    const StepConfig &c = d->cfg;
    const LaunchHook hook = swals::hook_of(d);
    Metrics<R> m = swals::metrics_of<R>(d);
    R *max_stage = d->desc.record_max_stage ? (R *)d->max_stage : nullptr;
    auto max_u_after = [&](int every) {
        return launch_update_max_u<R>(d->nx, d->ny, d->pitch, (const R *)d->planes[d->cur][0],
                                      (const R *)d->planes[d->cur][1], (const R *)d->planes[d->cur][2],
                                      (const R *)d->elv, max_stage, c, d->max_u, d->sc, every, d->stream);
    };
    if (d->nsteps == 0 && max_stage) {
        // Gated on the device step count as well, so that a graph captured
        // from the first step does this only on its first replay.
        hook(CAT_MAXSTAGE, 0);
        cudaError_t e = d->max_u_generic ? max_u_after(0)
                                         : launch_update_max_stage_every<R>(d->nx, d->ny, d->pitch,
                                                                            (const R *)d->planes[d->cur][0],
                                                                            max_stage, c, d->sc, 0, d->stream);
        hook(CAT_MAXSTAGE, 1);
        if (e != cudaSuccess) return cuda_fail(e, "update_max_quantities");
    }
    cudaError_t e = cudaSuccess;
    bool gauges_fused = false;   // the step's own kernels recorded the gauges
    if (d->static_pending) {
        // static_before_time (domain_mod.f90:1706-1716): the clock decides
        // on the host, one read per step until it has passed.
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CK(cudaStreamIsCapturing(d->stream, &cs));
        if (cs != cudaStreamCaptureStatusNone)
            return fail(SWALS_ERR_UNSUPPORTED, "a step before static_before_time cannot be captured in a graph");
        double time0 = 0.0;
        CK(cudaMemcpyAsync(&time0, &d->sc->time, sizeof(double), cudaMemcpyDeviceToHost, d->stream));
        CK(cudaStreamSynchronize(d->stream));
        if (time0 < d->static_before_time) {
            e = launch_static_step(d->sc, timestep, has_dt, d->stream);
            if (e != cudaSuccess) return cuda_fail(e, "static step");
            d->nsteps++;
            return SWALS_OK;
        }
        d->static_pending = false;
    }
    // max_U_update_frequency > 1: the step kernels skip max_stage and one
    // kernel updates it after the steps the reference updates it after.
    R *const max_every = (max_stage && (d->max_U_update_frequency > 1 || d->max_u_generic)) ? max_stage : nullptr;
    if (max_every) max_stage = nullptr;
    if (d->method == M_LINEAR || d->method == M_LF_LIN_NLFRIC) {
        if (!has_dt)
            return fail(SWALS_ERR_TIMESTEP_REQUIRED, "ERROR: timestep must be provided for %s evolve_one_step",
                        d->desc.timestepping_method);
        const int in = d->cur, out = (d->cur + 1) % 3;
        StepPlanes<R> p;
        p.nx = d->nx; p.ny = d->ny; p.pitch = d->pitch;
        p.stg = (const R *)d->planes[in][0]; p.uh = (const R *)d->planes[in][1]; p.vh = (const R *)d->planes[in][2];
        p.stg_o = (R *)d->planes[out][0]; p.uh_o = (R *)d->planes[out][1]; p.vh_o = (R *)d->planes[out][2];
        p.elv = (R *)d->elv; p.max_stage = max_stage; p.manning_sq = (R *)d->manning_sq;
        if (!d->aux.stream) {
            cudaStreamCreateWithFlags(&d->aux.stream, cudaStreamNonBlocking);
            cudaEventCreateWithFlags(&d->aux.fork, cudaEventDisableTiming);
            cudaEventCreateWithFlags(&d->aux.join, cudaEventDisableTiming);
        }
        // the step kernel records the gauges when it is the step's last one
        StepConfig cg = c;
        cg.g_sites = d->d_sites;
        cg.g_n = d->n_gauges;
        cg.g_records = d->d_records;
        cg.g_capacity = d->gauge_capacity;
        gauges_fused = swals::linear_step_fuses_gauges(cg, d->nx, d->ny);
        e = launch_linear_step<R>(p, m, cg, R(timestep), d->sc, d->stream, hook, d->timers_on ? nullptr : &d->aux);
        if (e != cudaSuccess) return cuda_fail(e, "linear leapfrog step");
        if (d->cfg.fw) d->cfg.fw_ready = 1;
        d->cur = out;
    } else if (d->method == M_LF_NONLINEAR) {
        if (!has_dt)
            return fail(SWALS_ERR_TIMESTEP_REQUIRED, "ERROR: timestep must be provided for leapfrog_nonlinear "
                                                     "evolve_one_step");
        const int in = d->cur, out = (d->cur + 1) % 3;
        StepPlanes<R> p;
        p.nx = d->nx; p.ny = d->ny; p.pitch = d->pitch;
        p.stg = (const R *)d->planes[in][0]; p.uh = (const R *)d->planes[in][1]; p.vh = (const R *)d->planes[in][2];
        p.stg_o = (R *)d->planes[out][0]; p.uh_o = (R *)d->planes[out][1]; p.vh_o = (R *)d->planes[out][2];
        p.elv = (R *)d->elv; p.max_stage = max_stage; p.manning_sq = (R *)d->manning_sq;
        e = launch_leapfrog_nonlinear_step<R>(p, m, c, R(timestep), d->sc, d->stream, hook);
        if (e != cudaSuccess) return cuda_fail(e, "nonlinear leapfrog step");
        d->cur = out;
    } else if (d->method == M_RK2 || d->method == M_EULER || d->method == M_MIDPOINT || d->method == M_RK2N) {
        R *pl[3][3];
        for (int b = 0; b < 3; b++)
            for (int v = 0; v < 3; v++) pl[b][v] = (R *)d->planes[b][v];
        Rk2Buffers buf;
        buf.side = d->side;
        buf.partials = d->lines;
        buf.partials_len = 5 * (2 * d->nx + 2 * d->ny);
        buf.edges = d->edges;
        // the step's finalize kernel records the gauges from its final planes
        StepConfig cg = c;
        cg.g_sites = d->d_sites;
        cg.g_n = d->n_gauges;
        cg.g_records = d->d_records;
        cg.g_capacity = d->gauge_capacity;
        gauges_fused = d->n_gauges > 0;
        if (d->method == M_MIDPOINT)
            e = launch_midpoint_step<R>(pl, d->cur, (R *)d->elv, max_stage, (R *)d->manning_sq, d->nx, d->ny,
                                        d->pitch, m, cg, has_dt != 0, timestep, buf, d->sc, d->stream, hook);
        else if (d->method == M_RK2N)
            e = launch_rk2n_step<R>(pl, d->cur, (R *)d->elv, max_stage, (R *)d->manning_sq, d->nx, d->ny, d->pitch,
                                    m, cg, has_dt != 0, timestep, buf, d->sc, d->stream, hook);
        else
            e = launch_rk2_step<R>(pl, d->cur, (R *)d->elv, max_stage, (R *)d->manning_sq, d->nx, d->ny, d->pitch,
                                   m, cg, has_dt != 0, timestep, d->method == M_EULER, buf, d->sc, d->stream, hook);
        if (e != cudaSuccess) return cuda_fail(e, "finite-volume step");
    } else {
        return fail(SWALS_ERR_UNSUPPORTED, "timestepping_method '%s' is not implemented on the GPU path",
                    d->desc.timestepping_method);
    }
    if (max_every) {
        hook(CAT_MAXSTAGE, 0);
        max_stage = max_every;
        e = d->max_u_generic ? max_u_after(d->max_U_update_frequency)
                             : launch_update_max_stage_every<R>(d->nx, d->ny, d->pitch, (const R *)d->planes[d->cur][0],
                                                                max_every, c, d->sc, d->max_U_update_frequency,
                                                                d->stream);
        hook(CAT_MAXSTAGE, 1);
        if (e != cudaSuccess) return cuda_fail(e, "update_max_quantities");
    }
    if (d->n_gauges > 0 && !gauges_fused) {
        hook(CAT_GAUGES, 0);
        e = launch_gauges<R>(d->pitch, (const R *)d->planes[d->cur][0], (const R *)d->planes[d->cur][1],
                             (const R *)d->planes[d->cur][2], d->d_sites, d->n_gauges, d->d_records,
                             d->gauge_capacity, d->sc, d->stream);
        hook(CAT_GAUGES, 1);
        if (e != cudaSuccess) return cuda_fail(e, "gauges");
    }
    d->nsteps++;
    return SWALS_OK;
}

}  // namespace

extern "C" {

int swals_gpu_last_error(char *buf, size_t len)
{
    if (!buf || len == 0) return SWALS_ERR_INVALID_ARGUMENT;
    snprintf(buf, len, "%s", g_last_error.c_str());
    return SWALS_OK;
}

const char *swals_gpu_version(void) { return "swals-b200 0.1 (sm_100a)"; }

int swals_gpu_desc_init(swals_domain_desc *desc)
{
    if (!desc) return fail(SWALS_ERR_INVALID_ARGUMENT, "desc is NULL");
    memset(desc, 0, sizeof(*desc));
    desc->nx[0] = desc->nx[1] = -1;
    snprintf(desc->timestepping_method, sizeof(desc->timestepping_method), "%s", "rk2");
    desc->cfl = -DBL_MAX;
    desc->theta = -DBL_MAX;
    desc->msl_linear = 0.0;
    desc->linear_friction_coeff = 0.0;
    desc->maximum_timestep = 1.0e+20;
    desc->linear_solver_is_truely_linear = 1;
    desc->friction_type = SWALS_FRICTION_MANNING;
    desc->real_bytes = 8;
    for (int k = 0; k < 4; k++) desc->boundary_exterior[k] = 1;
    desc->boundary_kind = SWALS_BC_NONE;
    desc->record_max_stage = 1;
    desc->exterior_cells_width = 2;
    desc->device = -1;
    snprintf(desc->compute_fluxes_inner_method, sizeof(desc->compute_fluxes_inner_method), "%s",
             "DE1_low_fr_diffusion");
    return SWALS_OK;
}

int swals_gpu_domain_create(const swals_domain_desc *desc, swals_domain **out)
{
    if (!desc || !out) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (desc->has_host_boundary_subroutine || desc->has_host_forcing_subroutine)
        return fail(SWALS_ERR_UNSUPPORTED_CALLBACK,
                    "host boundary/forcing procedure pointers cannot run on the device; use a device boundary kind");
    int method;
    double def_cfl, def_theta;
    if (!parse_method(desc->timestepping_method, &method, &def_cfl, &def_theta))
        return fail(SWALS_ERR_UNKNOWN_METHOD, "timestepping_method: %s not recognized", desc->timestepping_method);
    if (!(method == M_LINEAR || method == M_RK2 || method == M_EULER || method == M_MIDPOINT || method == M_RK2N ||
          method == M_LF_LIN_NLFRIC || method == M_LF_NONLINEAR))
        return fail(SWALS_ERR_UNSUPPORTED, "timestepping_method '%s' is not implemented on the GPU path",
                    desc->timestepping_method);
    const int nx = desc->nx[0], ny = desc->nx[1];
    if (nx < 4 || ny < 4) return fail(SWALS_ERR_INVALID_ARGUMENT, "nx, ny must be >= 4 (got %d, %d)", nx, ny);
    {
        // The update region xL..xU, yL..yU (1-based, 0 = the full range) lies
        // inside the grid, as the reference's loop bounds assume; the kernels
        // index neighbours of its cells.
        const int xl = desc->xL > 0 ? desc->xL : 1, xu = desc->xU > 0 ? desc->xU : nx;
        const int yl = desc->yL > 0 ? desc->yL : 1, yu = desc->yU > 0 ? desc->yU : ny;
        if (xu > nx || yu > ny || xl > xu || yl > yu)
            return fail(SWALS_ERR_INVALID_ARGUMENT,
                        "update region xL..xU = %d..%d, yL..yU = %d..%d is not inside 1..%d, 1..%d", xl, xu, yl, yu,
                        nx, ny);
    }
    if (!(desc->real_bytes == 8 || desc->real_bytes == 4))
        return fail(SWALS_ERR_INVALID_ARGUMENT, "real_bytes must be 4 or 8");
    if (desc->coriolis && !desc->spherical)
        return fail(SWALS_ERR_INVALID_ARGUMENT, "Cannot define preprocessing flag CORIOLIS without also defining SPHERICAL");
    const int flux_variant = parse_flux_method(desc->compute_fluxes_inner_method,
                                               sizeof(desc->compute_fluxes_inner_method));
    if (flux_variant < 0)
        return fail(SWALS_ERR_UNSUPPORTED, "compute_fluxes_inner_method '%.64s' is not implemented on the GPU path",
                    desc->compute_fluxes_inner_method);
    if (desc->boundary_kind < 0 || desc->boundary_kind > 3)
        return fail(SWALS_ERR_INVALID_ARGUMENT, "unknown boundary_kind %d", desc->boundary_kind);
    if (desc->boundary_function_kind < 0 || desc->boundary_function_kind > 1)
        return fail(SWALS_ERR_UNSUPPORTED_CALLBACK, "unknown boundary_function_kind %d", desc->boundary_function_kind);
    if (is_staggered(method) && desc->boundary_kind == SWALS_BC_FLATHER && desc->exterior_cells_width == 1)
        return fail(SWALS_ERR_UNSUPPORTED, "flather_boundary with the linear solver needs exterior_cells_width >= 2");
    if (is_staggered(method) && desc->boundary_kind == SWALS_BC_TRANSMISSIVE)
        return fail(SWALS_ERR_UNSUPPORTED, "transmissive_boundary with the staggered linear solver is not implemented");
    if (desc->boundary_kind == SWALS_BC_STAGE_TRANSMISSIVE_NORMAL_MOMENTUM && desc->boundary_function_kind != 1)
        return fail(SWALS_ERR_UNSUPPORTED_CALLBACK, "boundary_function must be a device kind (SWALS_BF_*)");

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(SWALS_ERR_NO_DEVICE, "no CUDA device available (there is no CPU fallback)");

    if (desc->device >= ndev)
        return fail(SWALS_ERR_INVALID_ARGUMENT, "device %d does not exist (%d devices)", desc->device, ndev);
    if (desc->device >= 0) {
        cudaError_t se = cudaSetDevice(desc->device);
        if (se != cudaSuccess) return cuda_fail(se, "cudaSetDevice");
    }

    swals_domain *d = new swals_domain();
    d->desc = *desc;
    d->method = method;
    d->fp64 = (desc->real_bytes == 8);
    d->nx = nx;
    d->ny = ny;
    d->pitch = swals::round_up(nx, 32);
    if (d->desc.cfl == -DBL_MAX) d->desc.cfl = def_cfl;
    if (d->desc.theta == -DBL_MAX) d->desc.theta = def_theta;
    if (d->desc.maximum_timestep <= 0) d->desc.maximum_timestep = 1.0e20;
    if (d->desc.exterior_cells_width <= 0) d->desc.exterior_cells_width = 2;

    swals::StepConfig &c = d->cfg;
    c.xl = (desc->xL > 0 ? desc->xL : 1) - 1;
    c.xu = (desc->xU > 0 ? desc->xU : nx) - 1;
    c.yl = (desc->yL > 0 ? desc->yL : 1) - 1;
    c.yu = (desc->yU > 0 ? desc->yU : ny) - 1;
    for (int k = 0; k < 4; k++) c.bext[k] = desc->boundary_exterior[k] ? 1 : 0;
    c.bc_kind = desc->boundary_kind;
    c.flux_variant = flux_variant;
    c.bf.kind = desc->boundary_function_kind;
    for (int k = 0; k < 8; k++) c.bf.p[k] = desc->boundary_function_params[k];
    c.spherical = desc->spherical;
    c.coriolis = desc->coriolis;
    c.nofriction = desc->nofriction;
    c.chezy = (desc->friction_type == SWALS_FRICTION_CHEZY);
    c.truely_linear = desc->linear_solver_is_truely_linear;
    c.msl_linear = desc->msl_linear;
    c.linear_friction_coeff = desc->linear_friction_coeff;
    c.theta = d->desc.theta;
    c.cfl = d->desc.cfl;
    c.maximum_timestep = d->desc.maximum_timestep;
    c.exterior_cells_width = d->desc.exterior_cells_width;

    cudaError_t e = cudaGetDevice(&d->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete d;
        return cuda_fail(e, "stream creation");
    }
    // One pool: 3 state copies x 3 planes, ELV, max_stage, manning, metrics, scalars, ring/line buffers.
    const size_t es = esize(d);
    const size_t plane = (size_t)d->pitch * ny * es;
    const size_t metric_elems[8] = {(size_t)ny + 1, (size_t)nx + 1, (size_t)ny, (size_t)ny,
                                    (size_t)ny + 1, (size_t)ny, (size_t)nx, (size_t)ny};
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    size_t total = 12 * al(plane);
    for (int k = 0; k < 8; k++) total += al(metric_elems[k] * es);
    total += al(sizeof(swals::DevScalars));
    const size_t side_bytes = al((size_t)(4 * ny + 4 * nx) * 3 * es);
    const size_t lines_bytes = al((size_t)5 * (2 * nx + 2 * ny) * sizeof(double));   // 5 flux evaluations (rk2n)
    d->scratch_len = (nx > ny ? nx : ny) + 4096;
    const size_t scratch_bytes = al((size_t)d->scratch_len * sizeof(double));
    total += side_bytes + lines_bytes + scratch_bytes + al(64);
    // Stored stage-1 edge results of adaptive finite-volume steps.
    const size_t edge_bytes = (d->method == M_RK2 || d->method == M_EULER || d->method == M_MIDPOINT ||
                               d->method == M_RK2N)
                                  ? al((size_t)swals::rk2_edge_bytes(d->pitch, ny, (int)es)) : 0;
    total += edge_bytes;
    const size_t fw_bytes = (d->method == M_LF_LIN_NLFRIC || d->method == M_LF_NONLINEAR) ? 2 * al(plane) : 0;
    total += fw_bytes;   // friction_work
    const size_t nl_bytes = (d->method == M_LF_NONLINEAR) ? 9 * al((size_t)d->pitch * (ny + 1) * es) : 0;
    total += nl_bytes;   // leapfrog_nonlinear work planes
    e = cudaMalloc(&d->pool, total);
    if (e != cudaSuccess) {
        cudaStreamDestroy(d->stream);
        delete d;
        return cuda_fail(e, "device allocation of the domain");
    }
    d->pool_bytes = total;
    char *p = (char *)d->pool;
    for (int b = 0; b < 3; b++)
        for (int v = 0; v < 3; v++) { d->planes[b][v] = p; p += al(plane); }
    d->elv = p; p += al(plane);
    d->max_stage = p; p += al(plane);
    d->manning_sq = p; p += al(plane);
    for (int k = 0; k < 8; k++) { d->metric[k] = p; p += al(metric_elems[k] * es); }
    d->sc = (swals::DevScalars *)p; p += al(sizeof(swals::DevScalars));
    d->side = p; p += side_bytes;
    d->lines = (double *)p; p += lines_bytes;
    d->scratch = (double *)p; p += scratch_bytes;
    d->d_out = (double *)p; p += al(64);
    d->edges = edge_bytes ? (void *)p : nullptr; p += edge_bytes;
    d->cfg.ring = d->side;   // the staggered solver's Flather ring buffer (the side buffer is for FV stages)
    d->cfg.fw = fw_bytes ? (void *)p : nullptr; p += fw_bytes;
    d->cfg.nl_work = nl_bytes ? (void *)p : nullptr; p += nl_bytes;
    d->cfg.fw_ready = 0;

    int rc = SWALS_OK;
    if ((e = cudaMemsetAsync(d->pool, 0, total, d->stream)) != cudaSuccess) rc = cuda_fail(e, "memset");
    if (rc == SWALS_OK) {
        // max_U default: -0.99 * huge(real(1.0, output_precision)) in single precision (domain_mod.f90:1108)
        const float init = -0.99f * FLT_MAX;
        const int64_t n = d->pitch * (int64_t)ny;
        const int blocks = (int)((n + 255) / 256);
        if (d->fp64) fill_kernel<double><<<blocks, 256, 0, d->stream>>>((double *)d->max_stage, n, (double)init);
        else fill_kernel<float><<<blocks, 256, 0, d->stream>>>((float *)d->max_stage, n, init);
        if ((e = cudaGetLastError()) != cudaSuccess) rc = cuda_fail(e, "max_stage init");
    }
    if (rc == SWALS_OK) {
        if (d->fp64) { compute_geometry<double>(d); rc = upload_metrics_t<double>(d); }
        else { compute_geometry<float>(d); rc = upload_metrics_t<float>(d); }
    }
    if (rc == SWALS_OK && (e = cudaStreamSynchronize(d->stream)) != cudaSuccess) rc = cuda_fail(e, "create sync");
    if (rc != SWALS_OK) {
        cudaFree(d->pool);
        cudaStreamDestroy(d->stream);
        delete d;
        return rc;
    }
    *out = d;
    return SWALS_OK;
}

static void drop_step_graph(swals_domain *d)
{
    if (d->step_graph) cudaGraphExecDestroy(d->step_graph);
    d->step_graph = nullptr;
}

static void free_forcing(swals_domain *d)
{
    for (auto &f : d->forcing) {
        if (f.work) cudaFree(f.work);
        if (f.saved_max) cudaFree(f.saved_max);
    }
    d->forcing.clear();
    d->cfg.n_forcing = 0;
    d->cfg.forcing = nullptr;
}

int swals_gpu_domain_destroy(swals_domain *d)
{
    if (!d) return SWALS_OK;
    cudaStreamSynchronize(d->stream);
    free_forcing(d);
    if (d->stage_buf) cudaFree(d->stage_buf);
    if (d->eddy_visc) cudaFree(d->eddy_visc);
    if (d->max_u.planes) cudaFree(d->max_u.planes);
    for (auto &p : d->pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    for (auto e : d->ev_pool) cudaEventDestroy(e);
    if (d->d_sites) cudaFree(d->d_sites);
    if (d->d_records) cudaFree(d->d_records);
    if (d->ws) cudaFree(d->ws);
    if (d->prio_mask) cudaFree(d->prio_mask);
    if (d->stats_buf) cudaFree(d->stats_buf);
    drop_step_graph(d);
    for (auto &g : d->adj_graph)
        if (g) cudaGraphExecDestroy(g);
    if (d->aux.stream) {
        cudaStreamSynchronize(d->aux.stream);
        cudaStreamDestroy(d->aux.stream);
        cudaEventDestroy(d->aux.fork);
        cudaEventDestroy(d->aux.join);
    }
    cudaFree(d->pool);
    cudaStreamDestroy(d->stream);
    delete d;
    return SWALS_OK;
}

int swals_gpu_upload_U(swals_domain *d, const void *U)
{
    if (!d || !U) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    const size_t plane_host = (size_t)d->nx * d->ny * esize(d);
    for (int k = 1; k <= 4; k++) {
        int rc = copy_plane(d, plane_ptr(d, k), (const char *)U + (k - 1) * plane_host, true);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(d->stream));
    return SWALS_OK;
}

int swals_gpu_download_U(swals_domain *d, void *U)
{
    if (!d || !U) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    const size_t plane_host = (size_t)d->nx * d->ny * esize(d);
    for (int k = 1; k <= 4; k++) {
        int rc = copy_plane(d, plane_ptr(d, k), (char *)U + (k - 1) * plane_host, false);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(d->stream));
    return SWALS_OK;
}

int swals_gpu_upload_var(swals_domain *d, int32_t k, const void *host)
{
    if (!d || !host || k < 1 || k > 4) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    int rc = copy_plane(d, plane_ptr(d, k), host, true);
    if (rc) return rc;
    CK(cudaStreamSynchronize(d->stream));
    return SWALS_OK;
}

int swals_gpu_download_var(swals_domain *d, int32_t k, void *host)
{
    if (!d || !host || k < 1 || k > 4) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    int rc = copy_plane(d, plane_ptr(d, k), host, false);
    if (rc) return rc;
    CK(cudaStreamSynchronize(d->stream));
    return SWALS_OK;
}

int swals_gpu_upload_manning_squared(swals_domain *d, const void *host)
{
    if (!d || !host) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    int rc = copy_plane(d, d->manning_sq, host, true);
    if (rc) return rc;
    CK(cudaStreamSynchronize(d->stream));
    return SWALS_OK;
}

int swals_gpu_download_max_stage(swals_domain *d, void *host)
{
    if (!d || !host) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    int rc = copy_plane(d, d->max_stage, host, false);
    if (rc) return rc;
    CK(cudaStreamSynchronize(d->stream));
    return SWALS_OK;
}

int swals_gpu_get_metrics(swals_domain *d, double *x, double *y, double *dxb, double *dyl, double *area,
                          double *coriolis, double *coriolis_bottom_edge, double *tanlat)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    double *dst[8] = {dxb, dyl, area, coriolis, coriolis_bottom_edge, tanlat, x, y};
    for (int k = 0; k < 8; k++)
        if (dst[k]) memcpy(dst[k], d->h_metric[k].data(), d->h_metric[k].size() * sizeof(double));
    return SWALS_OK;
}

int swals_gpu_upload_metrics(swals_domain *d, const double *dxb, const double *dyl, const double *area,
                             const double *coriolis, const double *coriolis_bottom_edge, const double *tanlat)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    const double *src[6] = {dxb, dyl, area, coriolis, coriolis_bottom_edge, tanlat};
    for (int k = 0; k < 6; k++)
        if (src[k]) memcpy(d->h_metric[k].data(), src[k], d->h_metric[k].size() * sizeof(double));
    return d->fp64 ? upload_metrics_t<double>(d) : upload_metrics_t<float>(d);
}

int swals_gpu_evolve_one_step(swals_domain *d, double timestep, int32_t has_timestep)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    return d->fp64 ? evolve_t<double>(d, timestep, has_timestep) : evolve_t<float>(d, timestep, has_timestep);
}

// nsteps calls of evolve_one_step.  Long runs replay a CUDA graph of
// GRAPH_STEPS steps (a multiple of 3, so every method's state-buffer
// rotation returns to where it started): the sequence of launches is the
// same, without the per-launch host cost.  Timed (timers on) and first
// steps run one by one.
static constexpr int GRAPH_STEPS = 6;

int swals_gpu_evolve_steps(swals_domain *d, int32_t nsteps, double timestep, int32_t has_timestep)
{
    if (!d || nsteps < 0) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    int done = 0;
    auto eager = [&](int n) {
        for (int s = 0; s < n; s++) {
            int rc = swals_gpu_evolve_one_step(d, timestep, has_timestep);
            if (rc) return rc;
        }
        return (int)SWALS_OK;
    };
    if (d->nsteps == 0 && nsteps > 0) {
        int rc = eager(1);
        if (rc) return rc;
        done = 1;
    }
    const bool use_graph = !d->timers_on && !d->static_pending && (nsteps - done) >= 2 * GRAPH_STEPS;
    if (use_graph) {
        // The graph reads and writes the state buffers it was captured
        // with: it is valid only while the step sequence starts from the
        // same buffer (steps taken one by one in between rotate it).
        const bool same = d->step_graph && d->graph_dt == timestep && d->graph_has_dt == (has_timestep != 0) &&
                          d->graph_stream == d->stream && d->graph_gauges == d->n_gauges && d->graph_cur == d->cur;
        if (!same) {
            drop_step_graph(d);
            const int cur0 = d->cur;
            const int64_t n0 = d->nsteps, l0 = d->launches;
            CK(cudaStreamBeginCapture(d->stream, cudaStreamCaptureModeThreadLocal));
            int rc = SWALS_OK;
            for (int s = 0; s < GRAPH_STEPS && rc == SWALS_OK; s++)
                rc = d->fp64 ? evolve_t<double>(d, timestep, has_timestep) : evolve_t<float>(d, timestep, has_timestep);
            cudaGraph_t g = nullptr;
            cudaError_t ce = cudaStreamEndCapture(d->stream, &g);
            const bool back = (d->cur == cur0);
            d->graph_launches = d->launches - l0;
            d->cur = cur0;
            d->nsteps = n0;
            d->launches = l0;
            if (rc) { if (g) cudaGraphDestroy(g); return rc; }
            if (ce != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(ce, "cudaStreamEndCapture"); }
            if (!back) { cudaGraphDestroy(g); return eager(nsteps - done); }
            ce = cudaGraphInstantiate(&d->step_graph, g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
            d->graph_dt = timestep;
            d->graph_has_dt = has_timestep != 0;
            d->graph_stream = d->stream;
            d->graph_gauges = d->n_gauges;
            d->graph_cur = d->cur;
        }
        while (nsteps - done >= GRAPH_STEPS) {
            CK(cudaGraphLaunch(d->step_graph, d->stream));
            d->nsteps += GRAPH_STEPS;
            d->launches += d->graph_launches;
            done += GRAPH_STEPS;
        }
    }
    return eager(nsteps - done);
}

int swals_gpu_get_state(swals_domain *d, swals_domain_state *st)
{
    if (!d || !st) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    swals::DevScalars h;
    CK(cudaMemcpyAsync(&h, d->sc, sizeof(h), cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    st->time = h.time;
    st->max_dt = h.max_dt;
    st->dt_last_update = h.dt_last_update;
    st->evolve_step_dt = h.evolve_step_dt;
    st->nsteps_advanced = h.nsteps_advanced;
    st->negative_depth_fix_counter = h.negative_depth_fix_counter;
    for (int k = 0; k < 4; k++) st->boundary_flux_store[k] = h.boundary_flux_store[k];
    st->boundary_flux_evolve_integral = h.boundary_flux_evolve_integral;
    st->boundary_flux_time_integral = h.boundary_flux_time_integral;
    return SWALS_OK;
}

int swals_gpu_set_time(swals_domain *d, double time)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    CK(cudaMemcpyAsync(&d->sc->time, &time, sizeof(double), cudaMemcpyHostToDevice, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    return SWALS_OK;
}

int swals_gpu_synchronize(swals_domain *d)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    CK(cudaStreamSynchronize(d->stream));
    return swals::api_check_bulk_waits(d->stream);
}

static int timestep_max_impl(swals_domain *d, int linear, double *out)
{
    if (!d || !out) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaError_t e;
    const int max_blocks = 4096;
    if (d->fp64)
        e = swals::launch_timestep_max<double>(d->nx, d->ny, d->pitch, (const double *)d->planes[d->cur][0],
                                               (const double *)d->elv, (const double *)d->metric[0],
                                               (const double *)d->metric[1], d->desc.msl_linear, linear,
                                               d->desc.cfl, d->scratch, max_blocks, d->d_out, d->stream);
    else
        e = swals::launch_timestep_max<float>(d->nx, d->ny, d->pitch, (const float *)d->planes[d->cur][0],
                                              (const float *)d->elv, (const float *)d->metric[0],
                                              (const float *)d->metric[1], d->desc.msl_linear, linear,
                                              d->desc.cfl, d->scratch, max_blocks, d->d_out, d->stream);
    if (e != cudaSuccess) return cuda_fail(e, "timestep_max");
    double m;
    CK(cudaMemcpyAsync(&m, d->d_out, sizeof(double), cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    if (d->fp64) *out = m * d->desc.cfl;
    else *out = (double)((float)m * (float)d->desc.cfl);
    return SWALS_OK;
}

int swals_gpu_linear_timestep_max(swals_domain *d, double *out) { return timestep_max_impl(d, 1, out); }
int swals_gpu_nonlinear_stationary_timestep_max(swals_domain *d, double *out) { return timestep_max_impl(d, 0, out); }

int swals_gpu_stationary_timestep_max(swals_domain *d, double *out)
{
    // domain_mod.f90:1963-2016
    if (!d || !out) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    if (is_staggered(d->method)) {
        if (d->method == M_LF_NONLINEAR || !d->desc.linear_solver_is_truely_linear)
            return timestep_max_impl(d, 0, out);
        return timestep_max_impl(d, 1, out);
    }
    int rc = timestep_max_impl(d, 0, out);
    if (rc) return rc;
    if (d->method == M_RK2N) *out = *out * 0.5 * (5 - 1.0);
    else if (d->method == M_CLIFFS) (void)0;
    else *out = *out * 0.5;
    return SWALS_OK;
}

int swals_gpu_set_priority_mask(swals_domain *d, const uint8_t *mask)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    CK(cudaStreamSynchronize(d->stream));
    if (!mask) {
        if (d->prio_mask) cudaFree(d->prio_mask);
        d->prio_mask = nullptr;
        return SWALS_OK;
    }
    const size_t n = (size_t)d->nx * d->ny;
    if (!d->prio_mask) CK(cudaMalloc(&d->prio_mask, n));
    CK(cudaMemcpy(d->prio_mask, mask, n, cudaMemcpyHostToDevice));
    return SWALS_OK;
}

int swals_gpu_domain_statistics(swals_domain *d, swals_domain_stats *out)
{
    if (!d || !out) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    if (!d->stats_buf) CK(cudaMalloc(&d->stats_buf, sizeof(double) * (6 * (size_t)d->ny + 8)));
    const int ecw = d->desc.exterior_cells_width;
    const int staggered = is_staggered(d->method) ? 1 : 0;
    const int tl = (d->method == M_LINEAR || d->method == M_LF_LIN_NLFRIC) && d->desc.linear_solver_is_truely_linear;
    double *o7 = d->stats_buf + 6 * (size_t)d->ny;
    cudaError_t e;
    if (d->fp64)
        e = swals::launch_domain_statistics<double>(
            d->nx, d->ny, d->pitch, (const double *)d->planes[d->cur][0], (const double *)d->planes[d->cur][1],
            (const double *)d->planes[d->cur][2], (const double *)d->elv, (const double *)d->metric[2], d->prio_mask,
            ecw, staggered, tl, d->desc.msl_linear, d->stats_buf, o7, d->stream);
    else
        e = swals::launch_domain_statistics<float>(
            d->nx, d->ny, d->pitch, (const float *)d->planes[d->cur][0], (const float *)d->planes[d->cur][1],
            (const float *)d->planes[d->cur][2], (const float *)d->elv, (const float *)d->metric[2], d->prio_mask,
            ecw, staggered, tl, d->desc.msl_linear, d->stats_buf, o7, d->stream);
    if (e != cudaSuccess) return cuda_fail(e, "domain statistics");
    double h[7];
    CK(cudaMemcpyAsync(h, o7, sizeof(h), cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    out->maxstage = h[0]; out->maxspeed = h[1]; out->minstage = h[2]; out->minspeed = h[3];
    out->energy_potential_on_rho = h[4]; out->energy_kinetic_on_rho = h[5]; out->energy_total_on_rho = h[6];
    return SWALS_OK;
}

static int volume_impl(swals_domain *d, double *out, const uint8_t *mask)
{
    if (!d || !out) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaError_t e;
    const int n_ext = d->desc.exterior_cells_width;
    if (d->fp64)
        e = swals::launch_volume_interior<double>(d->nx, d->ny, d->pitch, (const double *)d->planes[d->cur][0],
                                                  (const double *)d->elv, (const double *)d->metric[2], n_ext,
                                                  d->scratch, d->d_out, d->stream, mask);
    else
        e = swals::launch_volume_interior<float>(d->nx, d->ny, d->pitch, (const float *)d->planes[d->cur][0],
                                                 (const float *)d->elv, (const float *)d->metric[2], n_ext,
                                                 d->scratch, d->d_out, d->stream, mask);
    if (e != cudaSuccess) return cuda_fail(e, "volume_interior");
    CK(cudaMemcpyAsync(out, d->d_out, sizeof(double), cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    return SWALS_OK;
}

int swals_gpu_forcing_patch_add(swals_domain *d, int32_t i0, int32_t i1, int32_t j0, int32_t j1, int32_t k0,
                                int32_t k1, double start_time, double end_time, const double *forcing_work,
                                int32_t *index_out)
{
    if (!d || !forcing_work) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    // apply_forcing_patch_base's checks (forcing_mod.f90:175-201)
    if (i0 > i1 || j0 > j1 || i0 < 1 || j0 < 1 || i1 > d->nx || j1 > d->ny)
        return fail(SWALS_ERR_INVALID_ARGUMENT, "Error in apply_forcing_patch: the forcing_patch does not have indices "
                                                "set correctly (%d:%d, %d:%d in a %d x %d domain)",
                    i0, i1, j0, j1, d->nx, d->ny);
    if (start_time > end_time)
        return fail(SWALS_ERR_INVALID_ARGUMENT,
                    "Error in apply_forcing_patch: the forcing_patch start/end times are not set correctly");
    if (!(k0 >= 1 && k0 <= 4 && k1 >= 1 && k1 <= 4 && k0 <= k1))
        return fail(SWALS_ERR_INVALID_ARGUMENT, "forcing_work has a 3rd dimension incompatible with domain%%U (%d:%d)",
                    k0, k1);
    const bool elevation_always = (d->method == M_EULER || is_staggered(d->method));
    if (k1 == 4 && !elevation_always)
        return fail(SWALS_ERR_UNSUPPORTED, "forcing the elevation with '%s' needs support_elevation_forcing "
                                           "(elevation in the backed-up state), which this GPU path does not implement",
                    d->desc.timestepping_method);
    if (is_staggered(d->method)) {
        // The leapfrog applies patches after its step kernel, so a patch
        // must stay clear of what that kernel used before the forcing: the
        // boundary ring, the boundary-flux lines when it forces momenta, and
        // a Flather ring's neighbours.
        const bool momenta = (k0 <= 3 && k1 >= 2);
        int m = 2;
        if (momenta) m = d->desc.exterior_cells_width + 2;
        if (d->cfg.bc_kind == SWALS_BC_FLATHER && m < 3) m = 3;
        if (i0 < m || j0 < m || i1 > d->nx - m + 1 || j1 > d->ny - m + 1)
            return fail(SWALS_ERR_UNSUPPORTED, "this leapfrog forcing patch must lie in i, j = %d..%d, %d..%d (clear "
                                               "of the boundary ring%s)",
                        m, d->nx - m + 1, m, d->ny - m + 1,
                        momenta ? " and the boundary-flux lines" : "");
    }
    const int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
    const size_t n = (size_t)ni * nj * nk, es = esize(d);
    CK(cudaStreamSynchronize(d->stream));   // no step in flight while the patch list changes
    swals::ForcingPatch f{};
    f.i0 = i0 - 1; f.i1 = i1 - 1; f.j0 = j0 - 1; f.j1 = j1 - 1; f.k0 = k0 - 1; f.k1 = k1 - 1;
    f.start_time = start_time;
    f.end_time = end_time;
    CK(cudaMalloc(&f.work, n * es));
    cudaError_t e;
    if (d->fp64) {
        e = cudaMemcpy(f.work, forcing_work, n * es, cudaMemcpyHostToDevice);
    } else {
        std::vector<float> tmp(forcing_work, forcing_work + n);
        e = cudaMemcpy(f.work, tmp.data(), n * es, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess && k0 == 1 && is_staggered(d->method) && d->desc.record_max_stage)
        e = cudaMalloc(&f.saved_max, (size_t)ni * nj * es);
    if (e != cudaSuccess) {
        cudaFree(f.work);
        if (f.saved_max) cudaFree(f.saved_max);
        return cuda_fail(e, "forcing patch upload");
    }
    d->forcing.push_back(f);
    d->cfg.n_forcing = (int)d->forcing.size();
    d->cfg.forcing = d->forcing.data();
    drop_step_graph(d);
    if (index_out) *index_out = d->cfg.n_forcing - 1;
    return SWALS_OK;
}

int swals_gpu_forcing_clear(swals_domain *d)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    CK(cudaStreamSynchronize(d->stream));
    free_forcing(d);
    drop_step_graph(d);
    return SWALS_OK;
}

int swals_gpu_set_eddy_viscosity(swals_domain *d, int32_t use_eddy_viscosity, double constant, double shiono_knight)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    CK(cudaStreamSynchronize(d->stream));
    drop_step_graph(d);
    if (!use_eddy_viscosity) {
        d->cfg.flux_variant &= ~swals::FLUX_EDDY;
        d->cfg.eddy_visc = nullptr;
        return SWALS_OK;
    }
    // timestepping_metadata(:)%eddy_viscosity_is_supported (timestepping_metadata_mod.f90:79-109)
    if (!(d->method == M_RK2 || d->method == M_RK2N || d->method == M_MIDPOINT || d->method == M_EULER))
        return fail(SWALS_ERR_UNSUPPORTED, "Eddy viscosity is not supported for the numerical scheme %s",
                    d->desc.timestepping_method);
    if (d->nx < 3) return fail(SWALS_ERR_INVALID_ARGUMENT, "eddy viscosity needs nx >= 3");
    if (!(constant >= 0.0) || !(shiono_knight >= 0.0))
        return fail(SWALS_ERR_INVALID_ARGUMENT, "eddy_visc_constants must be >= 0");
    if (!d->eddy_visc) CK(cudaMalloc(&d->eddy_visc, (size_t)d->pitch * d->ny * esize(d)));
    d->cfg.eddy_visc = d->eddy_visc;
    d->cfg.eddy_visc_constants[0] = constant;
    d->cfg.eddy_visc_constants[1] = shiono_knight;
    d->cfg.flux_variant |= swals::FLUX_EDDY;
    return SWALS_OK;
}

int swals_gpu_set_static_before_time(swals_domain *d, double static_before_time)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    CK(cudaStreamSynchronize(d->stream));
    drop_step_graph(d);
    d->static_before_time = static_before_time;
    d->static_pending = static_before_time > -DBL_MAX;
    return SWALS_OK;
}

int swals_gpu_set_max_U_update_frequency(swals_domain *d, int32_t every)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    if (every < 1) return fail(SWALS_ERR_INVALID_ARGUMENT, "max_U_update_frequency must be >= 1");
    CK(cudaStreamSynchronize(d->stream));
    drop_step_graph(d);
    d->max_U_update_frequency = every;
    return SWALS_OK;
}

int swals_gpu_set_max_U_variables(swals_domain *d, int32_t mask, int32_t stage_extrema_include_dry_cells,
                                  double arrival_stage_threshold_above_msl_linear)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    if (mask < 0 || mask > 31) return fail(SWALS_ERR_INVALID_ARGUMENT, "max_U_variables mask %d", mask);
    if (!d->desc.record_max_stage && (mask || !stage_extrema_include_dry_cells))
        return fail(SWALS_ERR_INVALID_ARGUMENT, "max_U_variables need record_max_stage (max_stage comes first)");
    if (d->nsteps > 0) return fail(SWALS_ERR_INVALID_ARGUMENT, "max_U_variables are set before the first step");
    CK(cudaStreamSynchronize(d->stream));
    drop_step_graph(d);
    const size_t es = esize(d);
    const int64_t plane = (int64_t)d->nx * d->ny;
    if (mask && !d->max_u.planes) CK(cudaMalloc(&d->max_u.planes, (size_t)plane * 5 * es));
    if (d->max_u.planes) {
        // -0.99 huge(real(1.0, output_precision)); min_stage starts at +0.99 huge (domain_mod.f90:1098-1117)
        const float init = -0.99f * FLT_MAX;
        const int blocks = (int)((plane + 255) / 256);
        for (int k = 0; k < 5; k++) {
            const float v = (k == 4) ? -init : init;
            char *p = (char *)d->max_u.planes + (size_t)k * plane * es;
            if (d->fp64) fill_kernel<double><<<blocks, 256, 0, d->stream>>>((double *)p, plane, (double)v);
            else fill_kernel<float><<<blocks, 256, 0, d->stream>>>((float *)p, plane, v);
        }
        CK(cudaGetLastError());
    }
    d->max_u.mask = mask;
    d->max_u.include_dry = stage_extrema_include_dry_cells ? 1 : 0;
    d->max_u.staggered = is_staggered(d->method) ? 1 : 0;
    d->max_u.truely_linear = (d->desc.linear_solver_is_truely_linear &&
                              (d->method == M_LINEAR || d->method == M_LF_LIN_NLFRIC)) ? 1 : 0;
    d->max_u.arrival = d->fp64 ? d->desc.msl_linear + arrival_stage_threshold_above_msl_linear
                               : (double)((float)d->desc.msl_linear + (float)arrival_stage_threshold_above_msl_linear);
    d->max_u.plane = plane;
    d->max_u_generic = mask != 0 || !stage_extrema_include_dry_cells;
    return SWALS_OK;
}

int swals_gpu_download_max_U(swals_domain *d, int32_t bit, double *host)
{
    if (!d || !host) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    int k = -1;
    for (int q = 0; q < 5; q++)
        if (bit == (1 << q)) k = q;
    if (k < 0 || !(d->max_u.mask & bit)) return fail(SWALS_ERR_INVALID_ARGUMENT, "max_U variable %d not recorded", bit);
    const size_t es = esize(d), n = (size_t)d->max_u.plane;
    std::vector<char> tmp(n * es);
    CK(cudaMemcpyAsync(tmp.data(), (char *)d->max_u.planes + (size_t)k * n * es, n * es, cudaMemcpyDeviceToHost,
                       d->stream));
    CK(cudaStreamSynchronize(d->stream));
    for (size_t q = 0; q < n; q++)
        host[q] = d->fp64 ? ((const double *)tmp.data())[q] : (double)((const float *)tmp.data())[q];
    return SWALS_OK;
}

int swals_gpu_apply_forcing(swals_domain *d, double dt)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    swals::ForcingClock clk{};
    clk.mode = swals::FORCE_EXPLICIT;
    clk.dt = dt;
    const swals::LaunchHook hook = swals::hook_of(d);
    cudaError_t e;
    if (d->fp64)
        e = swals::launch_forcing<double>(d->cfg, clk, d->pitch, (double *)d->planes[d->cur][0],
                                          (double *)d->planes[d->cur][1], (double *)d->planes[d->cur][2],
                                          (double *)d->elv, d->sc, d->stream, hook, swals::CAT_FINALIZE);
    else
        e = swals::launch_forcing<float>(d->cfg, clk, d->pitch, (float *)d->planes[d->cur][0],
                                         (float *)d->planes[d->cur][1], (float *)d->planes[d->cur][2],
                                         (float *)d->elv, d->sc, d->stream, hook, swals::CAT_FINALIZE);
    if (e != cudaSuccess) return cuda_fail(e, "apply_forcing");
    return SWALS_OK;
}

int swals_gpu_volume_interior(swals_domain *d, double *out) { return volume_impl(d, out, nullptr); }

int swals_gpu_volume_in_priority_domain(swals_domain *d, double *out)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    return volume_impl(d, out, d->prio_mask);
}

int swals_gpu_gauges_setup(swals_domain *d, const double *xy, int32_t n, int32_t capacity)
{
    if (!d || (n > 0 && !xy) || n < 0 || capacity < 0) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    cudaStreamSynchronize(d->stream);
    drop_step_graph(d);  // it holds the old gauge buffers
    if (d->d_sites) { cudaFree(d->d_sites); d->d_sites = nullptr; }
    if (d->d_records) { cudaFree(d->d_records); d->d_records = nullptr; }
    d->n_gauges = 0;
    d->h_sites.assign(2 * (size_t)n, 0);
    // point_gauge_mod.f90:336-347, evaluated in the state precision
    const double dx[2] = {d->desc.lw[0] / d->nx, d->desc.lw[1] / d->ny};
    const int nxy[2] = {d->nx, d->ny};
    for (int g = 0; g < n; g++) {
        for (int k = 0; k < 2; k++) {
            double q;
            if (d->fp64) q = (xy[2 * g + k] - d->desc.lower_left[k]) / dx[k];
            else {
                float dxf = (float)d->desc.lw[k] / ((float)nxy[k] * 1.0f);
                q = (double)(((float)xy[2 * g + k] - (float)d->desc.lower_left[k]) / dxf);
            }
            int f = (int)std::floor(q);
            if (nxy[k] - 1 < f) f = nxy[k] - 1;
            int site = 1 + f;
            if (site < 1 || site > nxy[k])
                return fail(SWALS_ERR_INVALID_ARGUMENT, "Gauge coordinate (%g, %g) is outside the domain",
                            xy[2 * g], xy[2 * g + 1]);
            d->h_sites[2 * g + k] = site - 1;
        }
    }
    if (n > 0) {
        CK(cudaMalloc(&d->d_sites, sizeof(int) * 2 * (size_t)n));
        CK(cudaMemcpy(d->d_sites, d->h_sites.data(), sizeof(int) * 2 * (size_t)n, cudaMemcpyHostToDevice));
        if (capacity > 0) CK(cudaMalloc(&d->d_records, sizeof(double) * 3 * (size_t)n * capacity));
    }
    d->n_gauges = (capacity > 0) ? n : 0;
    d->gauge_capacity = capacity;
    int zero = 0;
    CK(cudaMemcpyAsync(&d->sc->gauge_records, &zero, sizeof(int), cudaMemcpyHostToDevice, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    return SWALS_OK;
}

int swals_gpu_gauges_site_index(swals_domain *d, int32_t *site)
{
    if (!d || !site) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    for (size_t q = 0; q < d->h_sites.size(); q++) site[q] = d->h_sites[q] + 1;
    return SWALS_OK;
}

int swals_gpu_gauges_read(swals_domain *d, double *out, int32_t max_records, int32_t *n_records)
{
    if (!d || !n_records) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    int rec = 0;
    CK(cudaMemcpyAsync(&rec, &d->sc->gauge_records, sizeof(int), cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    int valid = rec < d->gauge_capacity ? rec : d->gauge_capacity;
    int ncopy = valid < max_records ? valid : max_records;
    if (ncopy > 0 && out)
        CK(cudaMemcpy(out, d->d_records, sizeof(double) * 3 * (size_t)d->n_gauges * ncopy, cudaMemcpyDeviceToHost));
    *n_records = ncopy;
    if (rec > d->gauge_capacity)
        return fail(SWALS_ERR_CAPACITY, "gauge buffer full: %d records requested, capacity %d", rec,
                    d->gauge_capacity);
    return SWALS_OK;
}

int swals_gpu_gauges_reset(swals_domain *d)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    int zero = 0;
    CK(cudaMemcpyAsync(&d->sc->gauge_records, &zero, sizeof(int), cudaMemcpyHostToDevice, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    return SWALS_OK;
}

int swals_gpu_timers_enable(swals_domain *d, int32_t enable)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    CK(cudaStreamSynchronize(d->stream));
    for (auto &p : d->pending) { d->ev_pool.push_back(p.a); d->ev_pool.push_back(p.b); }
    d->pending.clear();
    for (int c = 0; c < swals::CAT_COUNT; c++) { d->tot_ms[c] = 0.0; d->counts[c] = 0; }
    d->timers_on = enable != 0;
    return SWALS_OK;
}

int swals_gpu_timers_read(swals_domain *d, double *ms_out, int32_t n, int32_t *n_written)
{
    if (!d || !n_written || (n > 0 && !ms_out)) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    CK(cudaStreamSynchronize(d->stream));
    for (auto &p : d->pending) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, p.a, p.b));
        d->tot_ms[p.cat] += ms;
        d->counts[p.cat] += 1;
        d->ev_pool.push_back(p.a);
        d->ev_pool.push_back(p.b);
    }
    d->pending.clear();
    int w = 0;
    for (int c = 0; c < swals::CAT_COUNT && 2 * c + 1 < n; c++) {
        ms_out[2 * c] = d->tot_ms[c];
        ms_out[2 * c + 1] = (double)d->counts[c];
        w += 2;
    }
    *n_written = w;
    return SWALS_OK;
}

int swals_gpu_launch_count(swals_domain *d, int64_t *count)
{
    if (!d || !count) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    *count = d->launches;
    return SWALS_OK;
}

int swals_gpu_stream(swals_domain *d, void **stream_out)
{
    if (!d || !stream_out) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL argument");
    *stream_out = (void *)d->stream;
    return SWALS_OK;
}

int swals_gpu_device_planes(swals_domain *d, void **stg, void **uh, void **vh, void **elv, int64_t *pitch_elems)
{
    if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL domain");
    if (stg) *stg = d->planes[d->cur][0];
    if (uh) *uh = d->planes[d->cur][1];
    if (vh) *vh = d->planes[d->cur][2];
    if (elv) *elv = d->elv;
    if (pitch_elems) *pitch_elems = d->pitch;
    return SWALS_OK;
}

}  // extern "C"
