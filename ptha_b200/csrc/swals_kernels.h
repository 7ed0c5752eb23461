// swals_kernels.h -- host-side launch interface of the SWALS CUDA kernels
// (internal to libswalsgpu; the public ABI is include/swals_gpu.h).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "swals_common.cuh"

namespace swals {

// Sets the message returned by swals_gpu_last_error (this thread).
void set_last_error(const char *msg);

// Kernel categories for the per-launch timers (include/swals_gpu.h).
enum LaunchCat {
    CAT_CFL = 0, CAT_STAGE1 = 1, CAT_BC1 = 2, CAT_STAGE2 = 3, CAT_BC2 = 4, CAT_FINALIZE = 5,
    CAT_LINEAR_EDGE = 6, CAT_LINEAR_MAIN = 7, CAT_GAUGES = 8, CAT_MAXSTAGE = 9, CAT_COUNT = 10
};

// Called before (phase 0) and after (phase 1) every kernel launch.
struct LaunchHook {
    void (*fn)(void *ctx, int cat, int phase) = nullptr;
    void *ctx = nullptr;
    void operator()(int cat, int phase) const { if (fn) fn(ctx, cat, phase); }
};

template <typename R>
struct StepPlanes {
    int nx, ny;
    int64_t pitch;          // elements
    const R *stg, *uh, *vh; // state read by the step
    R *stg_o, *uh_o, *vh_o; // state written by the step
    R *elv;
    R *max_stage;           // may be null
    R *manning_sq;          // rk2 family
};

// compute_fluxes_inner_method (compute_fluxes_alternatives_include.f90:11-64)
// as bits: 'DE1_low_fr_diffusion' 0, 'DE1' PLAIN_DIFFUSION,
// 'DE1_upwind_transverse' both, 'DE1_low_fr_diffusion_upwind_transverse'
// UPWIND_TRANSVERSE.
enum {
    FLUX_PLAIN_DIFFUSION = 1,    // reduced_momentum_diffusion = .false. (fr2 = 1)
    FLUX_UPWIND_TRANSVERSE = 2,  // upwind_transverse_momentum = .true.
    FLUX_EDDY = 4                // use_eddy_viscosity (the *_eddyvisc variants)
};

// forcing_patch_type (forcing_mod.f90:23-53) on the device: a 0-based
// inclusive box, variables k0..k1 (0 STG, 1 UH, 2 VH, 3 ELV), forcing_work as
// R planes (k, j, i) with i fastest; saved_max holds the leapfrog step's copy
// of max_stage over the box (patches that force STG).
struct ForcingPatch {
    int i0, i1, j0, j1, k0, k1;
    double start_time, end_time;
    void *work;
    void *saved_max;
};

// The time and timestep a forcing is applied with (domain%time after the
// update, and the update's dt).
enum { FORCE_FV_STAGE = 0, FORCE_LEAPFROG = 1, FORCE_EXPLICIT = 2 };
struct ForcingClock {
    int mode;
    int n_dt;               // FV: time = time0 + dt + ... (n_dt additions)
    double dt_extra;        // FV: then + dt * dt_extra when nonzero, which is also the update's dt
    int dt_from_cfl;        // FV: dt from the CFL maximum, else dt_fixed
    double dt_fixed;
    double max_dt_inv_init;
    double dt;              // FORCE_EXPLICIT: dt (time = domain%time); FORCE_LEAPFROG: dt (time = time0 + dt/2)
};

struct StepConfig {
    int xl, xu, yl, yu;     // 0-based inclusive active region (domain%xL-1 ...)
    int bext[4];            // boundary_exterior N,E,S,W
    int bc_kind;            // SWALS_BC_*
    BoundaryFn bf;
    int spherical, coriolis, nofriction, chezy, truely_linear;
    double msl_linear, linear_friction_coeff, theta, cfl, maximum_timestep;
    int exterior_cells_width;
    int flux_variant;       // compute_fluxes_inner_method as FLUX_* bits
    void *ring;             // linear + Flather: 2 (nx + ny - 2) x 2 reals of ring momenta
    void *fw;               // leapfrog_linear_plus_nonlinear_friction: friction_work (2 planes), else null
    int fw_ready;           // truely linear: friction_work already computed (friction_work_is_setup)
    void *nl_work;          // leapfrog_nonlinear: 9 work planes of pitch x (ny + 1)
    int n_forcing;          // forcing patches, applied in order (apply_forcing_patch_array)
    const ForcingPatch *forcing;
    void *eddy_visc;        // use_eddy_viscosity: one plane of per-cell eddy viscosity, else null
    double eddy_visc_constants[2];  // domain%eddy_visc_constants (constant, Shiono-Knight)
    // Point gauges the step records itself (finite-volume steps always, in
    // their finalize kernel; linear steps when linear_step_fuses_gauges):
    // 0-based (i, j) sites, records[rec][g][STG, UH, VH], capacity records.
    const int *g_sites;
    int g_n;
    double *g_records;
    int g_capacity;
};

// Forcing patches (forcing.cu): add each active patch's share of its
// forcing_work to the planes of k = STG, UH, VH, ELV.
template <typename R>
cudaError_t launch_forcing(const StepConfig &c, const ForcingClock &clk, int64_t pitch, R *stg, R *uh, R *vh,
                           R *elv, const DevScalars *sc, cudaStream_t s, const LaunchHook &hook, int cat);
// Leapfrog steps: copy max_stage over the STG patches' boxes before the step
// kernel; afterwards max_stage = max(copy, forced stage) there.
template <typename R>
cudaError_t launch_forcing_save_max(const StepConfig &c, int64_t pitch, const R *max_stage, cudaStream_t s,
                                    const LaunchHook &hook, int cat);
template <typename R>
cudaError_t launch_forcing_restore_max(const StepConfig &c, int64_t pitch, const R *stg, R *max_stage,
                                       cudaStream_t s, const LaunchHook &hook, int cat);

// compute_domain_statistics_new: rows6 is 6*ny doubles of scratch; out7 (device)
// receives {maxstage, maxspeed, minstage, minspeed, E_pot, E_kin, E_total}.
template <typename R>
cudaError_t launch_domain_statistics(int nx, int ny, int64_t P, const R *stg, const R *uh, const R *vh, const R *elv,
                                     const R *area, const uint8_t *mask, int ecw, int staggered, int tl, double msl,
                                     double *rows6, double *out7, cudaStream_t s);

// Gauges (0-based i, j site pairs) inside the window [i0, i1] x [r0, r1]:
// bit q set for gauge q.  Streaming kernels compute it once per warp segment
// so the per-row check costs nothing where there is no gauge.  With more than
// 64 gauges every bit is set and the callers test each gauge.
__device__ __forceinline__ unsigned long long gauges_in(const int *sites, int n, int i0, int i1, int r0, int r1)
{
    if (n > 64) return ~0ull;
    unsigned long long m = 0ull;
    for (int q = 0; q < n; q++) {
        const int gi = sites[2 * q], gj = sites[2 * q + 1];
        if (gi >= i0 && gi <= i1 && gj >= r0 && gj <= r1) m |= 1ull << q;
    }
    return m;
}

// Linear leapfrog, one full step (domain_mod_linear_solver_include.f90:58-571).
// With an auxiliary stream and two events, the one-block bookkeeping kernel
// (boundary-flux sums, time) runs beside the main kernel when no boundary
// routine writes the stage ring (the two then touch disjoint data).
struct AuxStream {
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
template <typename R>
cudaError_t launch_linear_step(const StepPlanes<R> &p, const Metrics<R> &m, const StepConfig &c,
                               R dt, DevScalars *sc, cudaStream_t s, const LaunchHook &hook,
                               const AuxStream *aux = nullptr);
// one_leapfrog_nonlinear_step (domain_mod_leapfrog_nonlinear_include.f90).
// flather_boundary on the ring after a leapfrog_nonlinear stage sweep (rk2.cu).
template <typename R>
cudaError_t launch_leapfrog_boundary(int nx, int ny, int64_t pitch, R *stg, R *uh, R *vh, R *elv, const Metrics<R> &m,
                                     const StepConfig &c, R dt, DevScalars *sc, cudaStream_t s);
template <typename R>
cudaError_t launch_leapfrog_nonlinear_step(const StepPlanes<R> &p, const Metrics<R> &m, const StepConfig &c, R dt,
                                           DevScalars *sc, cudaStream_t s, const LaunchHook &hook);

// The leapfrog's interior update alone (no boundary routine, boundary-flux
// sums, time or max_stage): the linear map x' = M x that the adjoint
// differentiates.  With n_sites > 0 the new stage at the sites (0-based i, j
// pairs) is written to rec.
template <typename R>
cudaError_t launch_linear_map(const StepPlanes<R> &p, const Metrics<R> &m, const StepConfig &c, R dt,
                              const int *sites, int n_sites, double *rec, cudaStream_t s, const LaunchHook &hook);

// Batched truly/not-truly linear leapfrog: `nbatch` instances whose planes
// follow instance 0's at `inst_stride` elements, sharing ELV and metrics
// (no boundary routine).  tile_cfg selects one of linear_tile_config_count()
// tile shapes.
template <typename R>
cudaError_t launch_linear_batch(const StepPlanes<R> &p0, int64_t inst_stride, int64_t max_stride, int nbatch,
                                const Metrics<R> &m, const StepConfig &c, R dt, int tile_cfg, cudaStream_t s,
                                const LaunchHook &hook);
int linear_tile_config_count();
// Whether launch_linear_step records the step's gauges itself (c.g_n > 0
// and the step's last kernel is the shared-memory tile kernel: no Flather
// fix-up, forcing or friction kernel after it); the caller then launches
// no gauge kernel.
bool linear_step_fuses_gauges(const StepConfig &c, int nx, int ny);

// Bounded waits of the bulk-copy linear rows that gave up on the current
// device since the count was last cleared (read on `s`, which is then
// synchronised); `clear` resets it.  A nonzero count means some rows of a
// step were not updated.
cudaError_t linear_wait_expired(unsigned *count, bool clear, cudaStream_t s);
// Whether a bulk-copy linear step has been launched in this process (the
// count above can only be nonzero then).
bool linear_bulk_launched();

// Batched gauges: records[rec][b][g] = STG of instance b at gauge g.
template <typename R>
cudaError_t launch_batch_gauges(int64_t pitch, const R *stg0, int64_t inst_stride, int nbatch, const int *site_ij,
                                int n, double *records, int rec, int capacity, cudaStream_t s);

// max_stage = max(max_stage, STG) over the active region (domain_mod.f90:2243-2290).
// update_max_quantities after a step when (nsteps_advanced - 1) % every == 0.
template <typename R>
cudaError_t launch_update_max_stage_every(int nx, int ny, int64_t pitch, const R *stg, R *max_stage,
                                          const StepConfig &c, const DevScalars *sc, int every, cudaStream_t s);
// The optional max_U_variables (bits: 1 time_of_max_stage, 2 max_speed,
// 4 max_flux, 8 arrival_time, 16 min_stage; planes of nx x ny elements in
// bit order, `plane` elements apart) and the flags update_max_quantities
// reads.
struct MaxUConfig {
    int mask;
    int include_dry;        // stage_extrema_include_dry_cells
    int staggered;          // is_staggered_grid
    int truely_linear;      // the staggered max_speed uses msl_linear depths
    double arrival;         // msl_linear + arrival_stage_threshold_above_msl_linear
    void *planes;
    int64_t plane;
};
template <typename R>
cudaError_t launch_update_max_u(int nx, int ny, int64_t pitch, const R *stg, const R *uh, const R *vh, const R *elv,
                                R *max_stage, const StepConfig &c, const MaxUConfig &mu, const DevScalars *sc,
                                int every, cudaStream_t s);
// A static step (before static_before_time): clock and counters only.
cudaError_t launch_static_step(DevScalars *sc, double dt, int has_dt, cudaStream_t s);
template <typename R>
cudaError_t launch_update_max_stage(int nx, int ny, int64_t pitch, const R *stg, R *max_stage,
                                    const StepConfig &c, cudaStream_t s);

// Gauge sampling: append [STG,UH,VH] at sites (point_gauge_mod.f90:208-245).
template <typename R>
cudaError_t launch_gauges(int64_t pitch, const R *stg, const R *uh, const R *vh, const int *site_ij, int n,
                          double *records, int capacity, DevScalars *sc, cudaStream_t s);

// rk2 / euler (timestepping_alternatives_include.f90:8-146).
struct Rk2Buffers {
    void *side;            // ring buffer used when a boundary routine is active
    void *partials;        // per-block partial sums (deterministic reductions)
    int64_t partials_len;
    void *edges = nullptr; // stored stage-1 flux-pass results (adaptive steps), or null
};

// Bytes of the stored stage-1 flux-pass results of a pitch x ny grid: per
// cell the three flux sums (real) and two explicit-source sums (double).
inline int64_t rk2_edge_bytes(int64_t pitch, int ny, int real_bytes)
{
    return (3 * (int64_t)real_bytes + 2 * 8) * pitch * (int64_t)ny + 512;
}

template <typename R>
cudaError_t launch_rk2_step(R *const planes[3][3], int &cur, R *elv, R *max_stage, R *manning_sq, int nx, int ny,
                            int64_t pitch, const Metrics<R> &m, const StepConfig &c, bool has_dt, double dt,
                            bool euler_only, const Rk2Buffers &buf, DevScalars *sc, cudaStream_t s,
                            const LaunchHook &hook);
// one_midpoint_step / one_rk2n_step (timestepping_alternatives_include.f90:
// 149-337) on the same stage kernels; the same arguments as launch_rk2_step.
template <typename R>
cudaError_t launch_midpoint_step(R *const planes[3][3], int &cur, R *elv, R *max_stage, R *manning_sq, int nx, int ny,
                                 int64_t pitch, const Metrics<R> &m, const StepConfig &c, bool has_dt, double dt,
                                 const Rk2Buffers &buf, DevScalars *sc, cudaStream_t s, const LaunchHook &hook);
template <typename R>
cudaError_t launch_rk2n_step(R *const planes[3][3], int &cur, R *elv, R *max_stage, R *manning_sq, int nx, int ny,
                             int64_t pitch, const Metrics<R> &m, const StepConfig &c, bool has_dt, double dt,
                             const Rk2Buffers &buf, DevScalars *sc, cudaStream_t s, const LaunchHook &hook);

// Reductions used by diagnostics.
template <typename R>
cudaError_t launch_volume_interior(int nx, int ny, int64_t pitch, const R *stg, const R *elv, const R *area,
                                   int n_ext, double *row_sums, double *out, cudaStream_t s,
                                   const uint8_t *mask = nullptr);
template <typename R>
cudaError_t launch_timestep_max(int nx, int ny, int64_t pitch, const R *stg, const R *elv, const R *dxb,
                                const R *dyl, double msl, int linear, double cfl, double *block_min,
                                int max_blocks, double *out, cudaStream_t s);

}  // namespace swals
