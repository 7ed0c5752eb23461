/*
 * swals_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, IEEE-strict restatement of the SWALS shallow-water time-step
 * hot path (GeoscienceAustralia/ptha, propagation/SWALS/src/shallow_water).
 * It is the checker for the CUDA implementation: only tests/, the smoke
 * check and the CPU-baseline leg of the benchmark may load it.  Nothing in
 * the product (ptha_b200/) links or calls it.
 *
 * Arrays follow the reference's Fortran column-major layout: U(i,j,k) with
 * i fastest, 1-based indices in the code below; k = STG,UH,VH,ELV (1..4).
 *
 * Parity pinning: the reference cannot be compiled here (no Fortran
 * compiler).  The restatement is pinned against the reference's own unit
 * test known answers (MC limiter cases, spherical area values, point-gauge
 * indexing, nested-comms linear-field exactness) and against conservation
 * properties; see tests/test_oracle_golden.py.
 *
 * REAL is double unless compiled with -DORACLE_REAL32, mirroring the
 * reference's -DREALFLOAT switch (global_mod.f90:16-34).  Variables that the
 * reference declares real(force_double) stay double in both builds.
 */
#ifndef SWALS_ORACLE_H
#define SWALS_ORACLE_H

#include <stdint.h>

#ifdef ORACLE_REAL32
typedef float REAL;
#define ORACLE_FN(name) oracle32_##name
#else
typedef double REAL;
#define ORACLE_FN(name) oracle64_##name
#endif

enum { OR_STG = 1, OR_UH = 2, OR_VH = 3, OR_ELV = 4 };

/* timestepping_method codes (timestepping_metadata_mod.f90:135-232). */
enum {
    OR_METHOD_RK2 = 1,
    OR_METHOD_RK2N = 2,
    OR_METHOD_MIDPOINT = 3,
    OR_METHOD_EULER = 4,
    OR_METHOD_LINEAR = 5,
    OR_METHOD_LEAPFROG_LINEAR_PLUS_NONLINEAR_FRICTION = 6,
    OR_METHOD_CLIFFS = 7,
    OR_METHOD_LEAPFROG_NONLINEAR = 8
};

/* Boundary condition kinds supported by the oracle (boundary_mod.f90). */
enum {
    OR_BC_NONE = 0,                               /* walls via elevation */
    OR_BC_TRANSMISSIVE = 1,                       /* boundary_mod.f90:21-75 */
    OR_BC_STAGE_TRANSMISSIVE_NORMAL_MOMENTUM = 2, /* boundary_mod.f90:78-163 */
    OR_BC_FLATHER = 3                             /* boundary_mod.f90:502-730 */
};

/* compute_fluxes_inner_method (compute_fluxes_alternatives_include.f90:11-64):
 * 'DE1_low_fr_diffusion' = 0, 'DE1' = PLAIN_DIFFUSION,
 * 'DE1_upwind_transverse' = PLAIN_DIFFUSION | UPWIND_TRANSVERSE,
 * 'DE1_low_fr_diffusion_upwind_transverse' = UPWIND_TRANSVERSE. */
enum {
    OR_FLUX_PLAIN_DIFFUSION = 1,   /* reduced_momentum_diffusion = .false. */
    OR_FLUX_UPWIND_TRANSVERSE = 2  /* upwind_transverse_momentum = .true. */
};

/* Analytic boundary functions (domain%boundary_function) for
 * OR_BC_STAGE_TRANSMISSIVE_NORMAL_MOMENTUM and OR_BC_FLATHER. */
enum {
    OR_BF_NONE = 0,                /* not associated */
    OR_BF_SOLITARY_WEST_WALLS = 1  /* solitary wave on the west edge, walls elsewhere */
};

typedef struct oracle_domain {
    /* geometry (domain_mod.f90:137-160) */
    int32_t nx, ny;
    double lw[2];
    double lower_left[2];
    /* solver */
    int32_t method;
    int32_t spherical;           /* -DSPHERICAL */
    int32_t coriolis;            /* CORIOLIS (spherical and not -DNOCORIOLIS) */
    int32_t nofriction;          /* -DNOFRICTION */
    int32_t truely_linear;       /* linear_solver_is_truely_linear */
    int32_t friction_chezy;      /* friction_type == 'chezy' */
    int32_t xL, xU, yL, yU;      /* 1-based active region */
    int32_t exterior_cells_width;
    int32_t boundary_exterior[4];/* N, E, S, W */
    int32_t bc_kind;
    int32_t bf_kind;
    int32_t record_max_stage;
    int32_t flux_variant;        /* compute_fluxes_inner_method: OR_FLUX_* bits, 0 = 'DE1_low_fr_diffusion' */
    double theta, cfl, msl_linear, linear_friction_coeff, maximum_timestep;
    double bf_params[8];
    /* state */
    double time, max_dt, dt_last_update, evolve_step_dt;
    int64_t nsteps_advanced;
    int64_t negative_depth_fix_counter;
    double boundary_flux_store[4];
    double boundary_flux_evolve_integral;
    double boundary_flux_time_integral;
    /* arrays, owned by the caller (sizes in comments) */
    REAL *U;            /* nx*ny*4 */
    REAL *max_stage;    /* nx*ny */
    REAL *manning_squared; /* nx*ny (rk2 family) */
    REAL *x, *y;        /* nx, ny */
    REAL *dxb;          /* distance_bottom_edge, ny+1 */
    REAL *dyl;          /* distance_left_edge, nx+1 */
    REAL *area;         /* area_cell_y, ny */
    REAL *coriolis_c;   /* coriolis, ny */
    REAL *coriolis_be;  /* coriolis_bottom_edge, ny+1 */
    REAL *tanlat_on_R;  /* tanlat_on_radius_earth, ny */
    /* rk2 work arrays */
    REAL *depth;        /* nx*ny */
    REAL *velocity;     /* nx*ny*2 (UH, VH slots) */
    REAL *flux_NS;      /* nx*(ny+1)*3 */
    REAL *flux_EW;      /* (nx+1)*ny*3 */
    double *explicit_source;      /* nx*ny*2 (UH, VH) */
    double *explicit_source_VH_j_minus_1; /* nx*(ny+1) */
    REAL *backup_U;     /* nx*ny*3 */
    /* Nesting flux integrals (nested_grid_comms_mod.f90:2300-2469) of the
     * boxes of this domain's send and recv comms.  Box b is (iL,iU,jL,jU),
     * 1-based, at nest_boxes[4b..4b+3]; its integrals are the doubles at
     * nest_integral + nest_offset[b], edge by edge (N, S, E, W) and within
     * an edge variable by variable (STG..ELV), each of length iU-iL+1 (N, S)
     * or jU-jL+1 (E, W). */
    int32_t nest_nbox;
    int32_t friction_work_is_setup;
    const int32_t *nest_boxes;
    const int64_t *nest_offset;
    double *nest_integral;
    /* leapfrog_linear_plus_nonlinear_friction: g n^2 depth^p at the UH and
     * VH points (nx*ny*2, domain%friction_work) */
    REAL *friction_work;
    /* forcing_patch_array_type (forcing_mod.f90:55-60), applied in order */
    int32_t n_forcing;
    int32_t pad2;
    const struct oracle_forcing_patch *forcing;
    /* leapfrog_nonlinear: advection_work (nx*ny*5: DEPTH_LAG, UUH, UVH, VUH, VVH) */
    REAL *advection_work;
    /* eddy viscosity (domain_mod.f90:233-243): flag, constants (constant,
     * Shiono-Knight), and an nx*ny work plane */
    int32_t use_eddy_viscosity;
    int32_t pad3;
    double eddy_visc_constants[2];
    REAL *eddy_visc;
    /* domain%static_before_time (-HUGE: never static) and
     * domain%max_U_update_frequency (domain_mod.f90:185, 431) */
    double static_before_time;
    int32_t max_U_update_frequency;
    /* the optional max_U_variables (domain_mod.f90:2243-2404) as bits:
     * 1 time_of_max_stage, 2 max_speed, 4 max_flux, 8 arrival_time,
     * 16 min_stage; one nx*ny plane each in max_U_extra, in bit order */
    int32_t max_U_extra;
    int32_t stage_extrema_include_dry_cells;
    int32_t pad5;
    double arrival_stage_threshold_above_msl_linear;
    REAL *max_U_extra_planes;
} oracle_domain;

/* forcing_patch_type (forcing_mod.f90:23-53) with the default (identity)
 * forcing_time_function: work (i fastest, then j, then k, over
 * i0..i1 x j0..j1 x k0..k1, 1-based, k in STG..ELV) is added to
 * U(i0:i1, j0:j1, k0:k1) at a constant rate between start_time and
 * end_time. */
typedef struct oracle_forcing_patch {
    int32_t i0, i1, j0, j1, k0, k1;
    double start_time, end_time;
    const REAL *work;
} oracle_forcing_patch;

/* add_forcing_work_to_U_over_time (forcing_mod.f90:80-156) on an array U of
 * n values with the matching forcing_work, for the time step
 * (time - dt, time). */
void ORACLE_FN(add_forcing_work_to_U_over_time)(REAL *U, const REAL *work, int64_t n, REAL time, REAL dt,
                                                REAL start_time, REAL end_time);

/* One side of a two_way_nesting_comms_type (nested_grid_comms_mod.f90:
 * 120-255), as set up by initialise_two_way_nesting_comms (:257-658). */
typedef struct oracle_nest_comm {
    int32_t send_active, recv_active;
    int32_t send_inds[6];        /* iL,iU,jL,jU,kL,kU */
    int32_t recv_inds[6];
    double cell_ratios[2];       /* my_dx / neighbour_dx */
    int32_t my_domain_is_finer, equal_cell_ratios;
    int32_t my_domain_staggered_grid, neighbour_domain_staggered_grid;
    int32_t use_wetdry_limiting;
    int32_t pad;
    int64_t nsend, nsend_interior, send_flux_start, send_timeind;   /* 1-based indices */
    int64_t nrecv, nrecv_interior, recv_flux_start, recv_timeind;
} oracle_nest_comm;

#ifdef __cplusplus
extern "C" {
#endif

/* Defaults that allocate_quantities takes from timestepping metadata. */
void ORACLE_FN(apply_method_defaults)(oracle_domain *d);
/* Geometry arrays (domain_mod.f90:925-1014). */
void ORACLE_FN(setup_geometry)(oracle_domain *d);
/* domain%evolve_one_step(timestep) (domain_mod.f90:1679-1813). has_dt=0 means adaptive. */
int  ORACLE_FN(evolve_one_step)(oracle_domain *d, double dt, int has_dt);
/* Pieces used by tests directly. */
void ORACLE_FN(update_max_quantities)(oracle_domain *d);
double ORACLE_FN(linear_timestep_max)(const oracle_domain *d);
double ORACLE_FN(nonlinear_stationary_timestep_max)(const oracle_domain *d);
double ORACLE_FN(volume_interior)(const oracle_domain *d);
double ORACLE_FN(volume_in_priority_domain)(const oracle_domain *d, const uint8_t *mask);
void ORACLE_FN(compute_depth_and_velocity)(oracle_domain *d);
double ORACLE_FN(compute_fluxes_DE1_low_fr_diffusion)(oracle_domain *d);
void ORACLE_FN(limited_gradient_dx_vectorized)(const REAL *U_local, const REAL *U_lower,
        const REAL *U_upper, const REAL *theta, REAL *gradient_dx, int32_t n);
double ORACLE_FN(area_lonlat_rectangle)(double lon1, double lat1, double dlon, double dlat, int flat);
void ORACLE_FN(gauge_site_index)(const double *xy, int32_t n, const double *ll,
        const double *dx, const int32_t *nxy, int32_t *site_index);
double ORACLE_FN(pow_friction)(double x, int32_t chezy);
double ORACLE_FN(pow_eddy)(double x);
double ORACLE_FN(cosh_cr)(double a);
void ORACLE_FN(boundary_function)(const oracle_domain *d, double t, int32_t i, int32_t j, REAL *out4);

void ORACLE_FN(domain_statistics)(const oracle_domain *d, const uint8_t *mask, double *out);

/* Nesting (swals_nesting_oracle.c). */
int  ORACLE_FN(nest_comm_init)(oracle_nest_comm *c, const double my_dx[2], const double neighbour_dx[2],
                               const int32_t send_inds[6], const int32_t recv_inds[6], int32_t send_only,
                               int32_t recv_only, int32_t use_wetdry_limiting, int32_t my_staggered,
                               int32_t neighbour_staggered);
void ORACLE_FN(nest_pack)(const oracle_nest_comm *c, const REAL *U, int32_t nx, int32_t ny,
                          const double *send_integral, double time, int32_t has_time, REAL *send_buffer);
void ORACLE_FN(nest_unpack)(const oracle_nest_comm *c, const REAL *recv_buffer, REAL *U, int32_t nx, int32_t ny,
                            const double *recv_integral, double *recv_error, double *time_received);
void ORACLE_FN(nest_recv_fixup)(oracle_domain *d, const int32_t recv_inds[4]);
void ORACLE_FN(nest_flux_correction)(oracle_domain *d, int32_t ncomm, const int32_t *recv_boxes,
                                     const int32_t *my_index, const int32_t *nbr_index, const double *recv_error,
                                     const int64_t *error_offset, const int32_t *priority_index,
                                     const double *all_dx, const int32_t *all_methods, double fraction_of);

#ifdef __cplusplus
}
#endif

#endif
