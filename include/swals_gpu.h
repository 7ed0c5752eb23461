/*
 * swals_gpu.h -- C ABI of the B200 (sm_100a) implementation of the SWALS
 * shallow-water time-step hot path.
 *
 * The reference (GeoscienceAustralia/ptha, propagation/SWALS) has no device
 * boundary: Fortran type-bound procedures of domain_type / multidomain_type
 * advance host arrays.  This header is the drop-in boundary a Fortran
 * ISO_C_BINDING shim (or ctypes / any FFI) binds.  Every entry point names
 * the reference interface it replaces, as file:line relative to
 * propagation/SWALS/src/shallow_water/.
 *
 * Conventions
 *  - Plain C types only; status is an int (SWALS_OK == 0).  The Fortran shim
 *    maps a nonzero status to generic_stop (util/stop_mod.f90:7-33), which
 *    keeps the reference's fatal-error semantics.
 *  - Host arrays use the reference's Fortran column-major layout: U(i,j,k),
 *    i fastest, leading dimensions nx then ny; k = STG(1), UH(2), VH(3), ELV(4)
 *    (domain_mod.f90:79).  Element type is double, or float when the domain
 *    was created with real_bytes = 4 (the -DREALFLOAT build).
 *  - A handle owns one CUDA stream; calls on one handle are not thread-safe.
 *    Stepping calls are stream-ordered and return without waiting; calls
 *    that hand data back to the host synchronise the handle's stream.
 *  - There is no CPU fallback: without a CUDA device, creation fails with
 *    SWALS_ERR_NO_DEVICE.
 */
#ifndef SWALS_GPU_H
#define SWALS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define SWALS_OK                        0
#define SWALS_ERR_INVALID_ARGUMENT      1
#define SWALS_ERR_UNKNOWN_METHOD        2  /* timestepping_method string not one of SWALS's 8 */
#define SWALS_ERR_UNSUPPORTED           3  /* valid SWALS option that this GPU path does not implement */
#define SWALS_ERR_CUDA                  4
#define SWALS_ERR_NONFINITE             5  /* NaN/Inf found by a stability check */
#define SWALS_ERR_UNSUPPORTED_CALLBACK  6  /* host boundary/forcing procedure pointer given */
#define SWALS_ERR_TIMESTEP_REQUIRED     7  /* staggered methods need an explicit timestep */
#define SWALS_ERR_OUT_OF_MEMORY         8
#define SWALS_ERR_NO_DEVICE             9
#define SWALS_ERR_CAPACITY             10  /* a fixed-size buffer (e.g. gauge records) is full */

/* ---- boundary conditions (boundary_mod.f90) ------------------------------ */
#define SWALS_BC_NONE                              0 /* walls via high elevation, no routine */
#define SWALS_BC_TRANSMISSIVE                      1 /* transmissive_boundary, boundary_mod.f90:21-75 */
#define SWALS_BC_STAGE_TRANSMISSIVE_NORMAL_MOMENTUM 2 /* boundary_mod.f90:78-163 */
#define SWALS_BC_FLATHER                           3 /* flather_boundary, boundary_mod.f90:502-730; the
                                                        'outside' state from boundary_function_kind,
                                                        or stage max(msl_linear, elev) at rest (SWALS_BF_NONE) */

/* Device-native boundary_function kinds (domain_mod.f90:594-633 interface). */
#define SWALS_BF_NONE                   0
#define SWALS_BF_SOLITARY_WEST_WALLS    1 /* params: H, depth, x0. West edge: stage = H sech^2(k(x-x0-ct)), elev = -depth;
                                             other edges: stage = elev = wall_elevation. */

/* friction_type (domain_mod.f90:178) */
#define SWALS_FRICTION_MANNING 0
#define SWALS_FRICTION_CHEZY   1

typedef struct swals_domain_desc {
    int32_t nx[2];                  /* domain%nx */
    double  lw[2];                  /* domain%lw */
    double  lower_left[2];          /* domain%lower_left */
    char    timestepping_method[64];/* domain%timestepping_method, NUL-terminated */
    double  cfl;                    /* domain%cfl; -DBL_MAX = method default */
    double  theta;                  /* domain%theta; -DBL_MAX = method default */
    double  msl_linear;             /* domain%msl_linear */
    double  linear_friction_coeff;  /* domain%linear_friction_coeff */
    double  maximum_timestep;       /* domain%maximum_timestep (default 1e20) */
    int32_t linear_solver_is_truely_linear;
    int32_t friction_type;          /* SWALS_FRICTION_* */
    int32_t spherical;              /* compile-time -DSPHERICAL in the reference */
    int32_t coriolis;               /* CORIOLIS: spherical and not -DNOCORIOLIS */
    int32_t nofriction;             /* -DNOFRICTION */
    int32_t real_bytes;             /* 8: FP64 state (default); 4: FP32 state (-DREALFLOAT) */
    int32_t xL, xU, yL, yU;         /* domain%xL.. (1-based); 0 = 1/nx/1/ny */
    int32_t boundary_exterior[4];   /* domain%boundary_exterior, order N,E,S,W */
    int32_t boundary_kind;          /* SWALS_BC_* (domain%boundary_subroutine) */
    int32_t boundary_function_kind; /* SWALS_BF_* (domain%boundary_function) */
    double  boundary_function_params[8];
    int32_t record_max_stage;       /* 'max_stage' in nontemporal_grids_to_store (default 1) */
    int32_t exterior_cells_width;   /* domain%exterior_cells_width (default 2) */
    int32_t has_host_boundary_subroutine; /* nonzero: a host callback was set -> rejected */
    int32_t has_host_forcing_subroutine;  /* nonzero: a host callback was set -> rejected */
    int32_t device;                 /* CUDA device ordinal; -1 = the calling thread's current device */
    char    compute_fluxes_inner_method[64]; /* domain%compute_fluxes_inner_method (default
                                        'DE1_low_fr_diffusion'; also 'DE1', 'DE1_upwind_transverse',
                                        'DE1_low_fr_diffusion_upwind_transverse',
                                        compute_fluxes_alternatives_include.f90:11-64) */
} swals_domain_desc;

typedef struct swals_domain_state {
    double  time;                   /* domain%time */
    double  max_dt;                 /* domain%max_dt */
    double  dt_last_update;         /* domain%dt_last_update */
    double  evolve_step_dt;         /* domain%evolve_step_dt */
    int64_t nsteps_advanced;        /* domain%nsteps_advanced */
    int64_t negative_depth_fix_counter; /* domain%negative_depth_fix_counter */
    double  boundary_flux_store[4];         /* N,E,S,W of the last flux evaluation */
    double  boundary_flux_evolve_integral;  /* last evolve_one_step */
    double  boundary_flux_time_integral;    /* running total */
} swals_domain_state;

typedef struct swals_domain swals_domain;  /* opaque */

/* Fills *desc with domain_type's initial values (domain_mod.f90:142-220). */
int swals_gpu_desc_init(swals_domain_desc *desc);

/* domain%allocate_quantities (domain_mod.f90:852-1358) on the device. */
int swals_gpu_domain_create(const swals_domain_desc *desc, swals_domain **out);
int swals_gpu_domain_destroy(swals_domain *d);

/* domain%U = host U (column-major nx*ny*4), and the reverse. */
int swals_gpu_upload_U(swals_domain *d, const void *U_host);
int swals_gpu_download_U(swals_domain *d, void *U_host);
/* One variable (k = 1..4) as an (nx,ny) column-major host array. */
int swals_gpu_upload_var(swals_domain *d, int32_t k, const void *host);
int swals_gpu_download_var(swals_domain *d, int32_t k, void *host);
/* domain%manning_squared (domain_mod.f90:1179-1188), (nx,ny) column-major. */
int swals_gpu_upload_manning_squared(swals_domain *d, const void *host);

/* Geometry arrays of allocate_quantities (domain_mod.f90:925-1014), computed
 * on the host at creation.  Lengths: x nx, y ny, dxb ny+1, dyl nx+1, area ny,
 * coriolis ny, coriolis_bottom_edge ny+1, tanlat_on_radius_earth ny.
 * upload_metrics lets a Fortran caller pass its own arrays instead. */
int swals_gpu_get_metrics(swals_domain *d, double *x, double *y, double *dxb, double *dyl,
                          double *area, double *coriolis, double *coriolis_bottom_edge,
                          double *tanlat_on_radius_earth);
int swals_gpu_upload_metrics(swals_domain *d, const double *dxb, const double *dyl,
                             const double *area, const double *coriolis,
                             const double *coriolis_bottom_edge, const double *tanlat_on_radius_earth);

/* domain%evolve_one_step([timestep]) (domain_mod.f90:1679-1813).
 * has_timestep == 0 selects adaptive (CFL) stepping for the FV methods. */
int swals_gpu_evolve_one_step(swals_domain *d, double timestep, int32_t has_timestep);
/* nsteps repeated evolve_one_step calls, launched back to back (no host sync). */
int swals_gpu_evolve_steps(swals_domain *d, int32_t nsteps, double timestep, int32_t has_timestep);

int swals_gpu_get_state(swals_domain *d, swals_domain_state *st);
int swals_gpu_set_time(swals_domain *d, double time);      /* domain%time = time */
/* Waits for the domain's stream.  Also SWALS_ERR_CUDA when bounded waits of
 * the bulk-copy linear kernel (SWALS_LINEAR_KERNEL=bulk) ran out since the
 * last check, i.e. rows of a step were not updated (the count is cleared). */
int swals_gpu_synchronize(swals_domain *d);

/* domain%max_U(:,:,1) ('max_stage'), column-major (nx,ny). */
int swals_gpu_download_max_stage(swals_domain *d, void *host);

/* domain%linear_timestep_max / nonlinear_stationary_timestep_max /
 * stationary_timestep_max (domain_mod.f90:1906-2022). */
int swals_gpu_linear_timestep_max(swals_domain *d, double *out);
int swals_gpu_nonlinear_stationary_timestep_max(swals_domain *d, double *out);
int swals_gpu_stationary_timestep_max(swals_domain *d, double *out);

/* domain%volume_interior (domain_mod.f90:1815-1849), FP64, row order fixed. */
int swals_gpu_volume_interior(swals_domain *d, double *out);

/* Point gauges (point_gauge_mod.f90:208-245,336-340).  xy is (2,n)
 * column-major (x1,y1,x2,y2,...).  After setup, every evolve_one_step appends
 * [STG,UH,VH] at each site to a device buffer of `capacity` records;
 * read returns records * n * 3 values (record-major, then gauge, then var). */
int swals_gpu_gauges_setup(swals_domain *d, const double *xy, int32_t n, int32_t capacity);
int swals_gpu_gauges_site_index(swals_domain *d, int32_t *site_index_1based);
int swals_gpu_gauges_read(swals_domain *d, double *out, int32_t max_records, int32_t *n_records);
int swals_gpu_gauges_reset(swals_domain *d);

/* Per-kernel CUDA-event timers, the device analogue of the reference's
 * EVOLVE_TIMER sections (domain_mod.f90:10-17).  While enabled, every kernel
 * launch of a step is bracketed by events on the handle's stream.
 * timers_read synchronises and writes, for each category c < n/2,
 * ms_out[2c] = total milliseconds and ms_out[2c+1] = number of launches;
 * categories: 0 CFL pre-pass, 1 FV stage 1, 2 boundary after stage 1,
 * 3 FV stage 2 (+rk2 average), 4 boundary after stage 2, 5 step finalise,
 * 6 leapfrog edge/boundary, 7 leapfrog fused step, 8 gauges, 9 max_stage. */
#define SWALS_TIMER_CATEGORIES 10
int swals_gpu_timers_enable(swals_domain *d, int32_t enable);
int swals_gpu_timers_read(swals_domain *d, double *ms_out, int32_t n, int32_t *n_written);
/* Number of kernels this handle has launched since creation. */
int swals_gpu_launch_count(swals_domain *d, int64_t *count);

/* The handle's CUDA stream (cudaStream_t) and device pointers, for callers
 * that keep data on the device (the PyTorch harness). */
int swals_gpu_stream(swals_domain *d, void **stream_out);
int swals_gpu_device_planes(swals_domain *d, void **stg, void **uh, void **vh, void **elv,
                            int64_t *pitch_elems);

/* Allocation-free volume_interior.  This entry point has no counterpart in
 * the reference.  It serves callers that cannot call cudaMalloc: code that
 * runs while a CUDA graph is being captured, hosts whose device memory
 * belongs to another allocator, loops that cannot take cudaMalloc's implicit
 * device synchronisation.  The caller passes device pointers to its own STG
 * and ELV planes (ny rows of pitch_elems elements, real_bytes 8 or 4), to
 * area_cell_y (ny values, same type) and to one output double; the sum is
 * written there, stream-ordered on `stream` (a cudaStream_t, NULL = legacy
 * default stream), without synchronising.  Per-row scratch lives in a fixed
 * device array of SWALS_NOALLOC_MAX_ROWS doubles that every GPU loading the
 * library holds until exit; larger ny is rejected with SWALS_ERR_CAPACITY.
 * The first call on each device looks up the array's device address (with
 * that device current), so make that first call before any stream capture.
 * All calls on a device share the scratch: calls that overlap on the GPU
 * race.  Nothing is allocated or freed. */
#define SWALS_NOALLOC_MAX_ROWS 65536
int swals_gpu_volume_interior_noalloc(const void *stg, const void *elv, const void *area, int32_t nx, int32_t ny,
                                      int64_t pitch_elems, int32_t real_bytes, int32_t exterior_cells_width,
                                      double *out_device, void *stream);

/* ---- batched linear leapfrog --------------------------------------------
 * B independent initial conditions on one grid.  The reference has no
 * batched form; a batch is B independent sequences of
 * domain%evolve_one_step(dt) with timestepping_method='linear'
 * (domain_mod_linear_solver_include.f90:58-571) that share geometry, ELV
 * and options of `grid` (a 'linear' domain without a boundary routine, which
 * must outlive the batch).  Each step is one kernel launch over all
 * instances; evolve() replays steps from a CUDA graph. */
typedef struct swals_batch swals_batch;  /* opaque */
int swals_gpu_batch_create(swals_domain *grid, int32_t nbatch, int32_t record_max_stage, swals_batch **out);
int swals_gpu_batch_destroy(swals_batch *b);
/* count instances from `first`, each (nx,ny,3) column-major [STG,UH,VH]. */
int swals_gpu_batch_upload_U(swals_batch *b, int32_t first, int32_t count, const void *U3);
int swals_gpu_batch_download_U(swals_batch *b, int32_t first, int32_t count, void *U3);
int swals_gpu_batch_download_max_stage(swals_batch *b, int32_t first, int32_t count, void *host);
/* Device layout for callers that fill or read instances in place:
 * instance b, variable v (0 STG, 1 UH, 2 VH), row j, column i is element
 * b*instance_stride + v*plane + j*pitch + i of *stg0 (current buffer). */
int swals_gpu_batch_device_state(swals_batch *b, void **stg0, int64_t *pitch_elems, int64_t *plane_elems,
                                 int64_t *instance_stride_elems);
/* Stage at gauge sites of every instance after every step; read returns
 * records * nbatch * n values ordered [record][instance][gauge]. */
int swals_gpu_batch_gauges_setup(swals_batch *b, const double *xy, int32_t n, int32_t capacity);
int swals_gpu_batch_gauges_read(swals_batch *b, double *out, int32_t max_records, int32_t *n_records);
int swals_gpu_batch_evolve(swals_batch *b, int32_t nsteps, double dt);
int swals_gpu_batch_time(swals_batch *b, double *time, int64_t *nsteps);
/* Autotuner: times every tile shape on this batch with state-preserving
 * dt = 0 steps and keeps the fastest. */
int swals_gpu_batch_tune(swals_batch *b, int32_t *cfg_out, double *ms_per_step_out);
int swals_gpu_batch_set_tile_config(swals_batch *b, int32_t cfg);
/* Number of kernel configurations the autotuner chooses from (valid cfg
 * values of swals_gpu_batch_set_tile_config are 0 .. n-1). */
int swals_gpu_batch_tile_config_count(int32_t *n);

/* ---- discrete adjoint of the truly linear leapfrog -------------------------
 * The reference has no adjoint.  For a 'linear' domain with
 * linear_solver_is_truely_linear and no boundary routine, one step is a
 * linear map x' = M x on x = (STG, UH, VH) with fixed dt.  With gauges set
 * up (swals_gpu_gauges_setup), y_n = stage at the gauges after step n.
 *
 * adjoint_linear: given gauge_adjoint[n][g] = dL/dy_{n+1,g} for n < nsteps
 * (nsteps x n_gauges, host, may be NULL) and an optional lambda_seed
 * (dL/dx_nsteps as (nx,ny,3) column-major host array, may be NULL), writes
 * dL/dx_0 into grad_U0 ((nx,ny,3) column-major host array).  The domain's
 * state is not used or changed.
 *
 * misfit_gradient_linear: L = 1/2 sum_n sum_g (y_{n,g} - target[n][g])^2
 * for n = 1..nsteps starting from the domain's current state (unchanged on
 * return); forward keeping a checkpoint every `checkpoint_every` steps, then
 * per segment recomputation and the adjoint sweep.  Writes L and
 * dL/d(STG,UH,VH)_0. */
int swals_gpu_adjoint_linear(swals_domain *d, int32_t nsteps, double timestep, const double *gauge_adjoint,
                             const void *lambda_seed, void *grad_U0);
int swals_gpu_misfit_gradient_linear(swals_domain *d, int32_t nsteps, double timestep, const double *target,
                                     int32_t checkpoint_every, double *loss, void *grad_U0);

/* ---- Multidomain nesting on one GPU -------------------------------------
 * Replaces multidomain_type's evolve_one_step and halo exchange
 * (multidomain_mod.f90:1081-1212, send_halos/recv_halos :2449-2565) for
 * domains that share a device.  The tables are what the reference's setup
 * (setup_multidomain_domains, multidomain_mod.f90:2781-3553) produces; the
 * Python mirror ptha_b200/nesting.py builds them the same way. */
typedef struct swals_multidomain swals_multidomain;

/* A matched pair of a receive box of `receiver` and the send box of
 * `sender` that feeds it (a recv_metadata row and its send_metadata row,
 * multidomain_mod.f90:3170-3330).  Boxes are 1-based and inclusive:
 * iL, iU, jL, jU.  All four variables STG..ELV are exchanged. */
typedef struct swals_nest_exchange {
    int32_t sender, receiver;   /* indices into the domain array */
    int32_t send_box[4];
    int32_t recv_box[4];
} swals_nest_exchange;

/* The nesting metadata builder: setup_multidomain + setup_multidomain_domains
 * for one image (multidomain_mod.f90:2663-3553), natively.  In: each
 * domain's interior extent, method, refinement factor, minimum nesting layer
 * thickness, use_eddy_viscosity and interior bounding box (all zero: the
 * extent's rectangle, create_all_bbox_and_dx :960-1060).  Out, written into
 * the same structs: the widened extent (lower_left, lw, nx grow by
 * nest_layer_width on each nesting boundary, :2860-2895), nest_layer_width,
 * is_nesting_boundary (N, E, S, W) and max_parent_dx_ratio; and a metadata
 * object with every domain's priority_domain_index / image and recv_metadata
 * rows, and the exchanges in the reference's receive order. */
typedef struct swals_nest_domain_desc {
    double  lower_left[2];
    double  lw[2];
    int32_t nx[2];
    int32_t timestepping_refinement_factor;
    int32_t minimum_nesting_layer_thickness;
    int32_t use_eddy_viscosity;
    int32_t nest_layer_width;          /* out */
    int32_t is_nesting_boundary[4];    /* out: N, E, S, W */
    double  max_parent_dx_ratio;       /* out */
    double  interior_bounding_box[8];  /* ll, lr, ur, ul (x, y); in/out */
    char    timestepping_method[64];
} swals_nest_domain_desc;

typedef struct swals_md_exchange {
    int32_t sender, receiver;
    int32_t send_box[4];
    int32_t recv_box[4];
    int32_t recv_row, send_row;        /* 0-based rows of recv_metadata / send_metadata */
} swals_md_exchange;

typedef struct swals_md_metadata swals_md_metadata;

/* periodic_xs / periodic_ys: the periodic extent (NULL: none). */
int swals_md_build_metadata(swals_nest_domain_desc *domains, int32_t n, int32_t extra_halo_buffer,
                            int32_t extra_cells_in_halo, const double periodic_xs[2], const double periodic_ys[2],
                            swals_md_metadata **out);
/* count = number of exchanges; out (capacity entries, or NULL to query). */
int swals_md_metadata_exchanges(const swals_md_metadata *m, swals_md_exchange *out, int32_t capacity, int32_t *count);
/* priority_domain_index / image of a domain (nx*ny of its widened extent, column-major). */
int swals_md_metadata_priority(const swals_md_metadata *m, int32_t domain, int32_t *index_out, int32_t *image_out);
/* recv_metadata rows (ind, img, iL, iU, jL, jU) of a domain. */
int swals_md_metadata_recv_boxes(const swals_md_metadata *m, int32_t domain, int64_t *rows_out, int32_t capacity,
                                 int32_t *count);
void swals_md_metadata_free(swals_md_metadata *m);

/* Create a multidomain over `ndomains` (<= 16) domains on one device, with
 * all_dx (2 per domain: the cell sizes setup recorded before widening the
 * domains, all_dx_md of multidomain_mod.f90:960-1060; NULL: lw/nx of each
 * domain), each domain's timestepping_refinement_factor (NULL: all 1), the exchange
 * table, and, when flux_correction is nonzero, each domain's
 * priority_domain_index (nx*ny, column-major, 1-based domain indices;
 * multidomain_mod.f90:2935-2960).  use_wetdry_limiting mirrors
 * use_wetdry_limiting_nesting (:2663).  While the multidomain exists every
 * domain launches on the first domain's stream; destroy it before its
 * domains. */
int swals_gpu_md_create(swals_domain *const *domains, int32_t ndomains, const double *all_dx,
                        const int32_t *timestepping_refinement_factor, const swals_nest_exchange *exchanges,
                        int32_t nexchanges, const int32_t *const *priority_domain_index,
                        int32_t use_wetdry_limiting, int32_t flux_correction, swals_multidomain **out);
int swals_gpu_md_destroy(swals_multidomain *md);
/* evolve_multidomain_one_step_shallow_water (multidomain_mod.f90:1093-1212):
 * every domain takes its refinement factor of sub-steps of dt/nt (fixed
 * steps), then all halos are packed, unpacked and flux-corrected. */
int swals_gpu_md_evolve_one_step(swals_multidomain *md, double dt);
/* process_data_to_send for every exchange (nested_grid_comms_mod.f90:1387-2046). */
int swals_gpu_md_send_halos(swals_multidomain *md);
/* process_received_data for every exchange, then the staggered-grid fix-ups
 * (nested_grid_comms_mod.f90:2048-2249; domain_mod.f90:3712-3893). */
int swals_gpu_md_recv_halos(swals_multidomain *md);
/* nesting_flux_correction_everywhere on every domain (domain_mod.f90:2766-3610). */
int swals_gpu_md_flux_correction(swals_multidomain *md);
/* Length of an exchange's buffer, and a copy of it (send_buffer). */
int swals_gpu_md_buffer_size(swals_multidomain *md, int32_t exchange, int64_t *n);
int swals_gpu_md_download_buffer(swals_multidomain *md, int32_t exchange, double *out, int64_t n);
/* Flux integrals of an exchange: which = 0 send box, 1 receive box,
 * 2 receive-box flux error; laid out edge by edge (N, S, E, W), then
 * variable by variable (STG..ELV). */
int swals_gpu_md_download_flux(swals_multidomain *md, int32_t exchange, int32_t which, double *out, int64_t n);
/* Capture nsteps md steps of a fixed dt into a CUDA graph (nsteps must bring
 * every domain back to its state buffer: a multiple of 3 always does), and
 * replay it: every domain, sub-step and exchange of nsteps md steps in one
 * graph launch.  The host time and step counts advance on replay. */
int swals_gpu_md_capture_graph(swals_multidomain *md, int32_t nsteps, double dt);
int swals_gpu_md_replay(swals_multidomain *md, int32_t nreplays);
/* Many multidomains advanced together (for example B sources on the same
 * nest: the batched form of the nested configuration; the reference steps
 * each multidomain_type on its own, multidomain_mod.f90:1093-1212).  The
 * group captures nsteps md steps of fixed dt of every member into one CUDA
 * graph, each member on its own branch, so one replay advances all of them
 * with their kernels running concurrently.  The members stay usable on
 * their own (a replay is ordered after work already issued on their
 * streams, and work issued later after the replay); every member's domains
 * must be in the state buffers they were captured in (steps in multiples of
 * 3 keep them there).  Destroy the group before its members. */
typedef struct swals_md_group swals_md_group;
int swals_gpu_md_group_create(swals_multidomain *const *mds, int32_t n, int32_t nsteps, double dt,
                              swals_md_group **out);
int swals_gpu_md_group_replay(swals_md_group *g, int32_t nreplays);
int swals_gpu_md_group_stream(swals_md_group *g, void **stream);
int swals_gpu_md_group_destroy(swals_md_group *g);
int swals_gpu_md_time(swals_multidomain *md, double *time);
int swals_gpu_md_synchronize(swals_multidomain *md);
int swals_gpu_md_launch_count(swals_multidomain *md, int64_t *n);

/* ---- Domain diagnostics ------------------------------------------------ */
typedef struct swals_domain_stats {
    double maxstage, maxspeed, minstage, minspeed;
    double energy_potential_on_rho, energy_kinetic_on_rho, energy_total_on_rho;
} swals_domain_stats;
/* The cells a nested domain owns (is_priority_domain_not_periodic,
 * multidomain_mod.f90:2960-2966): mask[i + nx*j] != 0, 0-based; NULL: all
 * cells.  Used by swals_gpu_domain_statistics. */
int swals_gpu_set_priority_mask(swals_domain *d, const uint8_t *mask);
/* compute_domain_statistics_new (domain_mod.f90:683-849): over the cells
 * exterior_cells_width+1 .. n-exterior_cells_width that the priority mask
 * keeps, the max/min stage and speed of wet cells and the potential and
 * kinetic energy per unit density (row sums reduced by warps, rows added in
 * order). */
int swals_gpu_domain_statistics(swals_domain *d, swals_domain_stats *out);
/* ---- forcing patches (forcing_mod.f90:23-339) ----------------------------
 * forcing_patch%setup + forcing_work, applied with apply_forcing_patch_array
 * (:241-262) as the domain's forcing_subroutine: forcing_work (doubles,
 * column-major over i0:i1, j0:j1, k0:k1, 1-based, k in STG=1..ELV=4) is
 * added to U(i0:i1, j0:j1, k0:k1) at a constant rate between start_time and
 * end_time (add_forcing_work_to_U_over_time, :80-156, with the default
 * forcing_time_function; host time functions are not supported).  Patches
 * are applied in the order added, after every update_U and boundary update
 * of the finite-volume steppers and after the stage sweep and boundary
 * update of the leapfrog solvers (domain_mod.f90:1564-1582,
 * linear_solver_include.f90:123).  Elevation forcing follows
 * support_elevation_forcing: 'euler' and the leapfrog solvers only.
 * Leapfrog patches stay off the boundary ring (and, when they force UH or
 * VH, keep exterior_cells_width + 1 cells from the edges).
 * Adding or clearing patches drops a captured evolve_steps graph; capture
 * multidomain graphs after the patches are in place. */
int swals_gpu_forcing_patch_add(swals_domain *d, int32_t i0, int32_t i1, int32_t j0, int32_t j1, int32_t k0,
                                int32_t k1, double start_time, double end_time, const double *forcing_work,
                                int32_t *index_out);
int swals_gpu_forcing_clear(swals_domain *d);
/* domain%apply_forcing(dt) (domain_mod.f90:1600-1646) on the current state
 * at domain%time, outside a step. */
int swals_gpu_apply_forcing(swals_domain *d, double dt);

/* domain%use_eddy_viscosity and domain%eddy_visc_constants = [constant,
 * shiono_knight] (domain_mod.f90:233-243, 890-898): the finite-volume
 * fluxes take the *_eddyvisc form of their compute_fluxes_inner_method
 * (compute_fluxes_alternatives_include.f90, domain_mod.f90:1448-1484), with
 * the viscosity of get_eddy_viscosity (compute_fluxes_DE1_inner_include.f90:
 * 864-1017; constant when shiono_knight is 0, else constant + Shiono-Knight).
 * 'rk2', 'rk2n', 'midpoint' and 'euler' only (SWALS_ERR_UNSUPPORTED
 * otherwise, as the reference's error stop).  use_eddy_viscosity = 0 turns it
 * off.  Drops a captured evolve_steps graph. */
int swals_gpu_set_eddy_viscosity(swals_domain *d, int32_t use_eddy_viscosity, double constant, double shiono_knight);

/* domain%static_before_time (domain_mod.f90:185, 1706-1716): a step that
 * starts before it only advances the clock by the given timestep (and
 * counts itself).  The host reads the clock once per step until the time
 * has passed; such steps are not captured in graphs. */
int swals_gpu_set_static_before_time(swals_domain *d, double static_before_time);
/* domain%max_U_update_frequency (domain_mod.f90:431, 1794-1798): max_stage
 * is updated after steps whose count before the step is a multiple of it. */
int swals_gpu_set_max_U_update_frequency(swals_domain *d, int32_t every);
/* The optional max_U_variables after max_stage (domain_mod.f90:1038-1117,
 * 2243-2404), as a mask: 1 time_of_max_stage, 2 max_speed, 4 max_flux,
 * 8 arrival_time, 16 min_stage; with stage_extrema_include_dry_cells and
 * arrival_stage_threshold_above_msl_linear (defaults 1 and 0.01).  Needs
 * record_max_stage; set before the first step (initialises the planes). */
int swals_gpu_set_max_U_variables(swals_domain *d, int32_t mask, int32_t stage_extrema_include_dry_cells,
                                  double arrival_stage_threshold_above_msl_linear);
/* One recorded variable (a single mask bit) as nx*ny doubles, column-major. */
int swals_gpu_download_max_U(swals_domain *d, int32_t bit, double *host);

/* ---- REAL4 output staging ------------------------------------------------
 * What SWALS's netCDF writers store, converted to REAL4 (round to nearest)
 * on the device and copied to host_out in one transfer; the call returns
 * when host_out is filled.
 * Grids (write_grids, util/netcdf_util_mod.f90:437-510; static max_stage,
 * :store_static_variable): the variables of var_mask (1 STG, 2 UH, 4 VH,
 * 8 ELV, 16 max_stage), each U(start:nx:stride, start:ny:stride) with
 * start = stride/2 + 1, x fastest, one after another; count_xy receives the
 * strided extents. */
int swals_gpu_stage_grids_real4(swals_domain *d, int32_t var_mask, int32_t spatial_stride, float *host_out,
                                int64_t capacity_floats, int32_t *count_xy);
/* Gauges (point_gauge_mod.f90:411-638): the recorded STG, UH and VH series
 * as three (station, time) blocks, station fastest. */
int swals_gpu_gauges_read_real4(swals_domain *d, float *out, int32_t max_records, int32_t *n_records);

/* volume_in_priority_domain (domain_mod.f90:1851-1889): volume_interior over
 * the cells the priority mask keeps (all cells without a mask). */
int swals_gpu_volume_in_priority_domain(swals_domain *d, double *out);

/* Last error message of this thread (util/stop_mod.f90 prints before stopping). */
int swals_gpu_last_error(char *buf, size_t len);
/* Library version string. */
const char *swals_gpu_version(void);

#ifdef __cplusplus
}
#endif
#endif
