// domain_internal.h -- the device domain behind the C ABI, shared by the
// entry-point files (capi.cu, batch.cu, adjoint.cu).  Internal to the library.
#pragma once
#include <vector>

#include "swals_kernels.h"
#include "../../include/swals_gpu.h"

// timestepping_method codes (timestepping_metadata_mod.f90:135-232).
enum Method {
    M_RK2 = 1, M_RK2N, M_MIDPOINT, M_EULER, M_LINEAR, M_LF_LIN_NLFRIC, M_CLIFFS, M_LF_NONLINEAR
};

// The staggered leapfrog solvers ('linear',
// 'leapfrog_linear_plus_nonlinear_friction', 'leapfrog_nonlinear'): nesting
// treats them alike (staggered grid, mass-only flux correction,
// U(:,:,UH/VH) fluxes with lower index 2).
inline bool is_linear_leapfrog(int m) { return m == M_LINEAR || m == M_LF_LIN_NLFRIC || m == M_LF_NONLINEAR; }

// Mirrors the parts of SWALS's domain_type (domain_mod.f90:137-507) the time
// step touches: geometry, solver options, device planes and scalar state.
struct swals_domain {
    swals_domain_desc desc;
    int method = 0;
    bool fp64 = true;
    int nx = 0, ny = 0;
    int64_t pitch = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    void *pool = nullptr;
    size_t pool_bytes = 0;
    void *planes[3][3] = {};
    void *elv = nullptr, *max_stage = nullptr, *manning_sq = nullptr;
    void *metric[8] = {};  // dxb, dyl, area, cor, cor_be, tanlat, x, y
    std::vector<double> h_metric[8];
    swals::DevScalars *sc = nullptr;
    void *side = nullptr;
    double *lines = nullptr;
    double *scratch = nullptr;  // row sums / block minima
    int64_t scratch_len = 0;
    double *d_out = nullptr;    // small result slot
    void *edges = nullptr;      // stored stage-1 flux-pass results (finite-volume methods)
    int cur = 0;
    int64_t nsteps = 0;
    swals::StepConfig cfg{};
    // gauges
    int n_gauges = 0, gauge_capacity = 0;
    int *d_sites = nullptr;
    double *d_records = nullptr;
    std::vector<int> h_sites;
    // launch accounting and per-kernel event timers
    int64_t launches = 0;
    // Diagnostics: the domain's own priority cells (nx*ny bytes, i fastest)
    // and the statistics scratch.
    uint8_t *prio_mask = nullptr;
    double *stats_buf = nullptr;
    // Side stream for the leapfrog's bookkeeping kernel.
    swals::AuxStream aux;
    // Forcing patches (forcing_mod.f90), device buffers owned here;
    // cfg.forcing points at this vector's data.
    std::vector<swals::ForcingPatch> forcing;
    // REAL4 output staging buffer (floats), allocated on first use.
    float *stage_buf = nullptr;
    void *eddy_visc = nullptr;   // use_eddy_viscosity: one plane of pitch x ny reals
    double static_before_time = -1.7976931348623157e308;  // domain%static_before_time
    bool static_pending = false;   // static_before_time may still lie ahead (the host checks the clock)
    int max_U_update_frequency = 1;
    swals::MaxUConfig max_u{};     // optional max_U_variables (planes nx x ny, allocated when set)
    bool max_u_generic = false;     // max_stage and the options by max_u_kernel instead of the step kernels
    size_t stage_cap = 0;
    // Replayed graph of a few steps for evolve_steps.
    cudaGraphExec_t step_graph = nullptr;
    double graph_dt = 0.0;
    bool graph_has_dt = false;
    cudaStream_t graph_stream = nullptr;
    int graph_gauges = -1;
    int graph_cur = -1;            // state buffer the graph starts from (and returns to)
    int64_t graph_launches = 0;
    // misfit_gradient's replayed graphs (segments of K steps), valid for
    // (adj_K, adj_ng, adj_dt, ws).
    // [0] forward; [1 + 3 set] recompute into buffer set `set`;
    // [2 + 3 set + lc] adjoint from lambda buffer lc with set's residuals
    cudaGraphExec_t adj_graph[7] = {};
    int adj_K = 0, adj_ng = 0;
    double adj_dt = 0.0;
    void *adj_ws = nullptr;
    // Scratch of the adjoint entry points, kept between calls (grown on demand).
    void *ws = nullptr;
    size_t ws_bytes = 0;
    bool timers_on = false;
    std::vector<cudaEvent_t> ev_pool;
    struct Pending { int cat; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    cudaEvent_t open_ev[swals::CAT_COUNT] = {};
    double tot_ms[swals::CAT_COUNT] = {};
    int64_t counts[swals::CAT_COUNT] = {};
};

namespace swals {
int api_fail(int code, const char *msg);
int api_cuda_fail(cudaError_t e, const char *what);
// After work on stream s: SWALS_ERR_CUDA (and the count cleared) when
// bounded waits of bulk-copied linear rows ran out since the last check;
// SWALS_OK at once when no bulk-copy step was ever launched.
int api_check_bulk_waits(cudaStream_t s);
LaunchHook hook_of(swals_domain *d);

template <typename R>
inline Metrics<R> metrics_of(const swals_domain *d)
{
    Metrics<R> m;
    m.dxb = (const R *)d->metric[0];
    m.dyl = (const R *)d->metric[1];
    m.area = (const R *)d->metric[2];
    m.cor = (const R *)d->metric[3];
    m.cor_be = (const R *)d->metric[4];
    m.tanlat = (const R *)d->metric[5];
    m.x = (const R *)d->metric[6];
    m.y = (const R *)d->metric[7];
    return m;
}
}  // namespace swals
