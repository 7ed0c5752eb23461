// rk2_common.cuh -- device pieces shared by the finite-volume stage kernels
// (rk2.cu: shared-memory tiles; rk2_stream.cu: register streaming).
#pragma once
#include "swals_kernels.h"

namespace swals {
namespace fv {

// MODE_FLUX: the CFL pass of an adaptive step that also stores every
// cell's dt-independent update terms (CellSums) for the stage-1 update.
enum { MODE_CFL = 0, MODE_STAGE1 = 1, MODE_STAGE2 = 2, MODE_FLUX = 3 };

// Stored per-cell results of a flux pass, everything of update_U that does
// not depend on dt: the flux sums (N - S) + (E - W) of STG, UH, VH (fluxes
// already multiplied by the edge lengths) and the explicit-source sums of
// UH and VH.
template <typename R>
struct CellSums {
    R *d[3];
    double *eu, *ev;
};
enum { FRIC_MANNING = 0, FRIC_CHEZY = 1, FRIC_NONE = 2 };

template <typename R>
struct Rk2Args {
    int nx, ny;
    int64_t P;
    const R *stg, *uh, *vh;        // stage input (U0 for stage 1, U1 for stage 2)
    const R *stg0, *uh0, *vh0;     // backup U0 (stage 2 average)
    R *stg_o, *uh_o, *vh_o;        // stage output
    const R *elv;
    const R *nsq;                  // manning_squared
    R *max_stage;
    Metrics<R> m;
    R theta, half_cfl;
    R lin_fric;                    // linear_friction_coeff
    double dt_fixed;               // used when dt_from_cfl == 0
    int dt_from_cfl;               // stage dt = 1/max(1/maximum_timestep, CFL max) (adaptive)
    double max_dt_inv_init;        // 1/maximum_timestep, rounded to R
    int write_cfl;                 // accumulate the CFL max into sc
    int n_ext;
    int bc_ring;                   // a boundary routine rewrites the outer ring after this stage
    int bext[4];
    R *side;                       // stage-2 pre-average values of the outer two rings
    double *lines;                 // flux_STG on the 4 boundary-flux lines: N[nx], E[ny], S[nx], W[ny]
    DevScalars *sc;
    CellSums<R> cs;                // MODE_FLUX output / stage-1 update input
    int flux_variant;              // FLUX_* bits (compute_fluxes_inner_method)
    R dt_scale;                    // the stage's dt times this (midpoint half step, rk2n last step; else 1)
    int base0;                     // stage 1 updates U0 (stg0..) with this state's fluxes (midpoint)
    R *ev;                         // per-cell eddy viscosity of the stage input (FLUX_EDDY), else null
    R ev_c1, ev_c2;                // eddy_visc_constants
    int pre_bf;                    // stage-1 update: store sc->bf_col0 for the step's two stage boundaries
    BoundaryFn bf;                 // ... of this boundary function, cell-centre x coordinates bf_x
    const R *bf_x;
};

template <typename R> struct Cell { R stg, dep, u, v, elv; };

__device__ __forceinline__ void atomic_max_pos_double(unsigned long long *addr, double v)
{
    atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// MC limiter, extrapolation_limiting_mod.f90:63-79 (sign(1,a) == copysign),
// returning HALF the limited gradient: the reconstruction's 1/2 (U -+ 1/2
// grad at the two edges) is applied here, once per gradient, instead of in
// each of the two edges that use it (the same product, so the same bits).
// (A branch form without the sign products measured 3 % slower.)
template <typename R>
__device__ __forceinline__ R mc_half_gradient(R local, R lower, R upper, R th)
{
    const R a = upper - local;
    const R b = local - lower;
    const R sa = copysign(R(1), a);
    const R sb = copysign(R(1), b);
    const R half_sasb = R(0.5) * (sa + sb);
    const R d = rmin(R(fabs(a)), R(fabs(b))) * half_sasb * th;
    const R e = R(0.5) * (a + b);
    const R c = (d == R(0)) ? R(0) : e;
    return R(0.5) * ((d > R(0)) ? rmin(c, d) : rmax(c, d));
}

// theta_wd of DE1_inner_include.f90:751-757 / :813-819.
template <typename R>
__device__ __forceinline__ R theta_wd(R d0, R d1, R d2, R theta)
{
    const R coef4 = R(1) / (K<R>::limiter_coef2() - K<R>::limiter_coef1());
    const R mindep = rmin(rmin(d0, d1), d2) - K<R>::min_depth();
    const R maxdep = rmax(rmax(d0, d1), d2) + K<R>::limiter_coef3() * K<R>::min_depth();
    const R theta_local = coef4 * (mindep / maxdep - K<R>::limiter_coef1());
    return rmax(theta * rmin(R(1), theta_local), R(0));
}

// Half the limited gradients of stage, depth, u, v (mc_half_gradient).
template <typename R> struct Grad { R ds, dd, du, dv; };

template <typename R>
struct EdgeRes {
    R f[3];          // STG, UH, VH flux (already multiplied by edge length)
    double es_pos;   // explicit-source contribution to the cell on the + side
    double es_neg;   // contribution to the cell on the - side
};

// A momentum flux of the *_eddyvisc variants (DE1_inner_include.f90:
// 289-358, 551-620): the advective part plus the HLL and turbulent
// diffusions, summed unless both have the same sign
// (reduced_numerical_diffusion), when the larger magnitude is taken.
template <typename R>
__device__ __forceinline__ R eddy_momentum_flux(R adv, R hll, R turb)
{
    const R dmax = rmax(R(fabs(turb)), R(fabs(hll)));
    const R tot = (turb * hll > R(0)) ? R(copysign(dmax, turb)) : turb + hll;
    return adv + tot;
}

// One Audusse/HLL edge of DE1_inner_include.f90 (:187-430 NS, :456-716 EW).
// NS=true: normal velocity v, edge between (i,j-1) and (i,j).
// variant: compute_fluxes_inner_method as FLUX_* bits (swals_kernels.h);
// 0 is the default 'DE1_low_fr_diffusion'.  EDDY (FLUX_EDDY): ev_n / ev_p are
// the eddy viscosities of the two cells and vel_div the distance the
// velocity difference is taken over (distance_left_edge(i) for NS edges,
// the mean of distance_bottom_edge(j), (j+1) for EW edges).
template <typename R, bool NS, bool EDDY = false>
__device__ __forceinline__ void edge_flux(const Cell<R> &cn, const Grad<R> &gn, const Cell<R> &cp, const Grad<R> &gp,
                                          R edge_len, R dx_cfl_half_inv, EdgeRes<R> &out, double &cfl_cand,
                                          int variant = 0, R ev_n = R(0), R ev_p = R(0), R vel_div = R(1))
{
    const R half = R(0.5);
    const double half_gravity = (double)(half * K<R>::gravity());
    const R EPS = R(1.0e-12);
    // sqrt(gravity * minimum_allowed_depth) in the state precision (the
    // correctly rounded root of the rounded product, as written out here)
    const R EPS_gs = sizeof(R) == 8 ? R(0x1.4462fb7ff5035p-7) : R(0x1.4462fcp-7f);
    const R beta = R(1.0);

    // (gn, gp hold half gradients: DE1_inner_include.f90's U +- 1/2 grad)
    R stage_neg = cn.stg + gn.ds;
    R stage_pos = cp.stg - gp.ds;
    double depth_neg = (double)(cn.dep + gn.dd);
    double depth_pos = (double)(cp.dep - gp.dd);
    R u_neg = cn.u + gn.du;
    R u_pos = cp.u - gp.du;
    R v_neg = cn.v + gn.dv;
    R v_pos = cp.v - gp.dv;
    double depth_neg_c = (double)cn.dep;
    double depth_pos_c = (double)cp.dep;

    R z_neg = R((double)stage_neg - depth_neg);
    R z_pos = R((double)stage_pos - depth_pos);
    R z_half = rmax(z_neg, z_pos);

    R stage_neg_star = rmax(stage_neg, z_half);
    double depth_neg_star = (double)(stage_neg_star - z_half);
    if (depth_neg_star == 0.0) { u_neg = R(0); v_neg = R(0); }
    R ud_neg = R((double)u_neg * depth_neg_star);
    R vd_neg = R((double)v_neg * depth_neg_star);
    R gs_neg = R(sqrt((double)K<R>::gravity() * depth_neg_star));

    R stage_pos_star = rmax(stage_pos, z_half);
    double depth_pos_star = (double)(stage_pos_star - z_half);
    if (depth_pos_star == 0.0) { u_pos = R(0); v_pos = R(0); }
    R ud_pos = R((double)u_pos * depth_pos_star);
    R vd_pos = R((double)v_pos * depth_pos_star);
    R gs_pos = R(sqrt((double)K<R>::gravity() * depth_pos_star));

    const R vel_beta_neg = (NS ? v_neg : u_neg) * beta;
    const R vel_beta_pos = (NS ? v_pos : u_pos) * beta;

    const R s_max = rmax(rmax(vel_beta_neg + gs_neg, vel_beta_pos + gs_pos), R(0));
    const R s_min = rmin(rmin(vel_beta_neg - gs_neg, vel_beta_pos - gs_pos), R(0));
    const double denom = (double)(s_max - s_min);
    double inv_denom;
    if (denom > (double)EPS && (gs_pos > EPS_gs || gs_neg > EPS_gs))
        inv_denom = (double)edge_len / denom;
    else
        inv_denom = 0.0;
    const R sminsmax = s_min * s_max * R(1);
    const R fr2num = ((v_neg * v_neg + v_pos * v_pos) + u_neg * u_neg) + u_pos * u_pos;
    const R fr2den = (gs_neg * gs_neg + gs_pos * gs_pos) + R(1.0e-10);
    // reduced_momentum_diffusion (the low_fr_diffusion variants), else 1
    const R fr2 = (variant & FLUX_PLAIN_DIFFUSION) ? R(1) : beta * R(sqrt(rmax(R(0.001), rmin(R(1), fr2num / fr2den))));

    const R qn_neg = NS ? vd_neg : ud_neg, qn_pos = NS ? vd_pos : ud_pos;
    const R qt_neg = NS ? ud_neg : vd_neg, qt_pos = NS ? ud_pos : vd_pos;
    const R f_mass = R((double)((s_max * qn_neg - s_min * qn_pos) + sminsmax * (stage_pos_star - stage_neg_star)) *
                       inv_denom);
    R f_norm, f_tran;
    if (!EDDY) {
        f_norm = R((double)((s_max * qn_neg * vel_beta_neg - s_min * qn_pos * vel_beta_pos) +
                            fr2 * sminsmax * (qn_pos - qn_neg)) * inv_denom);
        if (variant & FLUX_UPWIND_TRANSVERSE)   // upwind_transverse_momentum: the transverse velocity upwind of the mass flux
            f_tran = beta * ((f_mass > R(0)) ? (NS ? u_neg : v_neg) : (NS ? u_pos : v_pos)) * f_mass;
        else
            f_tran = R((double)((s_max * qt_neg * vel_beta_neg - s_min * qt_pos * vel_beta_pos) +
                                fr2 * sminsmax * (qt_pos - qt_neg)) * inv_denom);
    } else {
        // turbulent diffusion: eddy_visc * depth * edge length * velocity gradient,
        // with the geometric mean of the edge depths
        const R evh = half * (ev_p + ev_n);
        const R gdep = R(sqrt(depth_neg_star * depth_pos_star));
        R adv = R((double)(s_max * qn_neg * vel_beta_neg - s_min * qn_pos * vel_beta_pos) * inv_denom);
        R hll = R((double)(fr2 * sminsmax * (qn_pos - qn_neg)) * inv_denom);
        R turb = -(evh * gdep * edge_len * ((NS ? (cp.v - cn.v) : (cp.u - cn.u)) / vel_div));
        f_norm = eddy_momentum_flux<R>(adv, hll, turb);
        if (variant & FLUX_UPWIND_TRANSVERSE) {
            adv = beta * ((f_mass > R(0)) ? (NS ? u_neg : v_neg) : (NS ? u_pos : v_pos)) * f_mass;
            hll = R(0);
        } else {
            adv = R((double)(s_max * qt_neg * vel_beta_neg - s_min * qt_pos * vel_beta_pos) * inv_denom);
            hll = R((double)(fr2 * sminsmax * (qt_pos - qt_neg)) * inv_denom);
        }
        turb = -(evh * gdep * edge_len * ((NS ? (cp.u - cn.u) : (cp.v - cn.v)) / vel_div));
        f_tran = eddy_momentum_flux<R>(adv, hll, turb);
    }
    out.f[0] = f_mass;
    out.f[1] = NS ? f_tran : f_norm;
    out.f[2] = NS ? f_norm : f_tran;

    const double half_g_hh_edge = inv_denom * half_gravity *
        ((double)s_max * depth_neg_star * depth_neg_star - (double)s_min * depth_pos_star * depth_pos_star);
    const double bs_neg = half_gravity * ((depth_neg_star - depth_neg) * (depth_neg_star + depth_neg) -
                                          (depth_neg + depth_neg_c) * (double)(z_neg - cn.elv));
    out.es_neg = bs_neg * (double)edge_len - half_g_hh_edge;
    const double bs_pos = half_gravity * ((depth_pos_star - depth_pos) * (depth_pos_star + depth_pos) -
                                          (depth_pos + depth_pos_c) * (double)(z_pos - cp.elv));
    out.es_pos = (0.0 - bs_pos * (double)edge_len) + half_g_hh_edge;

    const double max_speed = (double)rmax(s_max, -s_min);
    cfl_cand = (max_speed > (double)EPS) ? max_speed * (double)dx_cfl_half_inv : 0.0;
}



// Timestep of a stage: fixed, or domain%max_dt of the first stage
// 1/max(1/maximum_timestep, max speed/(dx cfl/2)) for adaptive stepping.
template <typename R>
__device__ __forceinline__ R stage_dt(const Rk2Args<R> &a)
{
    if (a.dt_from_cfl) {
        const double bits_max = __longlong_as_double((long long)a.sc->max_dt_inv_bits);
        const R inv = R(fmax(a.max_dt_inv_init, bits_max));
        return (R(1) / inv) * a.dt_scale;
    }
    return R(a.dt_fixed) * a.dt_scale;
}

// The dt-independent part of update_U for cell (i, r)
// (update_U_DE1_inner_include.f90:38-96) from its four edges: the flux sums
// (n_hi - n_lo) + (w_hi - w_lo) and the explicit sources of UH and VH,
// accumulated in the reference's order.  Um_uh / Um_vh are U(i,j,UH/VH)
// after compute_depth_and_velocity (zero where depth <= minimum_allowed_depth);
// only the spherical terms read them.
template <typename R> struct CellFlux {
    R d[3];
    double eu, ev;
};
template <typename R, bool SPH, bool COR>
__device__ __forceinline__ CellFlux<R> cell_flux(const Rk2Args<R> &a, int i, int r, const Cell<R> &c, R Um_uh,
                                                 R Um_vh, const EdgeRes<R> &n_lo, const EdgeRes<R> &n_hi,
                                                 const EdgeRes<R> &w_lo, const EdgeRes<R> &w_hi)
{
    const int nx = a.nx, ny = a.ny;
    CellFlux<R> f;
    f.d[0] = (n_hi.f[0] - n_lo.f[0]) + (w_hi.f[0] - w_lo.f[0]);
    f.d[1] = (n_hi.f[1] - n_lo.f[1]) + (w_hi.f[1] - w_lo.f[1]);
    f.d[2] = (n_hi.f[2] - n_lo.f[2]) + (w_hi.f[2] - w_lo.f[2]);
    double es_uh = 0.0, es_vh = 0.0, es_jm1 = 0.0;
    if (r >= 1) {
        if (i >= 1) {
            es_vh = n_lo.es_pos;   // NS loop (:403-409)
            es_uh = w_lo.es_pos;   // EW loop (:649-654)
            if (SPH) {
                const double dep = (double)c.dep;
                const double hg = (double)(R(0.5) * K<R>::gravity());
                es_vh = es_vh + hg * dep * dep * (double)(a.m.dxb[r + 1] - a.m.dxb[r]);
                if (COR) {
                    const R cm = a.m.area[r] * a.m.cor[r];
                    es_uh = es_uh + (double)(cm * Um_vh);
                    es_vh = es_vh - (double)(cm * Um_uh);
                }
                const R cm2 = a.m.area[r] * a.m.tanlat[r] * c.u;
                es_uh = es_uh + (double)(cm2 * Um_vh);
                es_vh = es_vh - (double)(cm2 * Um_uh);
            }
        }
        es_uh = es_uh + ((i + 1 <= nx - 1) ? w_hi.es_neg : 0.0);  // explicit_source_im1_work (:721)
    }
    if (r + 1 <= ny - 1 && i >= 1) es_jm1 = n_hi.es_neg;          // explicit_source_VH_j_minus_1(i, j+1)
    f.eu = es_uh;
    f.ev = es_vh + es_jm1;
    return f;
}

// U(i,j,UH/VH) after compute_depth_and_velocity: the stage input where the
// fixed-up depth exceeds minimum_allowed_depth, else zero.
template <typename R>
__device__ __forceinline__ void fixed_momenta(const Rk2Args<R> &a, int64_t o, const Cell<R> &c, R &Um_uh, R &Um_vh)
{
    if (c.dep > K<R>::min_depth()) { Um_uh = a.uh[o]; Um_vh = a.vh[o]; }
    else { Um_uh = R(0); Um_vh = R(0); }
}

// The rest of update_U for cell (i, r) with the stage's dt: the flux
// update, the wet/dry test, the semi-implicit friction and the explicit
// sources; stage 2 also forms the rk2 average and max_stage.
// inv_cell_area_dt is the row's dt / area_cell_y(r) (a row constant the
// callers may evaluate once per row).
template <typename R, int MODE, int FRIC>
__device__ __forceinline__ void fv_apply(const Rk2Args<R> &a, int i, int r, const Cell<R> &c, R Um_uh, R Um_vh,
                                         const CellFlux<R> &f, R dt, R inv_cell_area_dt)
{
    const int nx = a.nx, ny = a.ny;
    const int64_t P = a.P;
    const R mad = K<R>::min_depth();
    const int64_t o = (int64_t)r * P + i;
    R U_stg = c.stg;
    R U_uh = Um_uh, U_vh = Um_vh;
    if (MODE == MODE_STAGE1 && a.base0) {
        // one_midpoint_step's full step: U was reset to the backup, and
        // update_U applies the midpoint's fluxes to it.
        U_stg = a.stg0[o]; U_uh = a.uh0[o]; U_vh = a.vh0[o];
    }

    U_stg = U_stg - inv_cell_area_dt * f.d[0];
    U_uh = U_uh - inv_cell_area_dt * f.d[1];
    U_vh = U_vh - inv_cell_area_dt * f.d[2];

    if (U_stg <= c.elv + mad) {
        U_uh = R(0);
        U_vh = R(0);
    } else {
        R implicit_factor;
        if (FRIC == FRIC_NONE) {
            implicit_factor = R(1);
        } else {
            const R depth = c.dep;
            const R fs = a.nsq[o] * R(sqrt(c.u * c.u + c.v * c.v)) *
                         R(pow_friction<FRIC == FRIC_CHEZY>((double)rmax(depth, mad)));
            implicit_factor = R(1) / ((R(1) + dt * K<R>::gravity() * rmax(depth, R(0)) * fs) + dt * a.lin_fric);
        }
        U_uh = R((double)U_uh + (double)inv_cell_area_dt * f.eu);
        U_uh = U_uh * implicit_factor;
        U_vh = R((double)U_vh + (double)inv_cell_area_dt * f.ev);
        U_vh = U_vh * implicit_factor;
    }

    if (MODE == MODE_STAGE2) {
        const bool outer2 = (i <= 1 || i >= nx - 2 || r <= 1 || r >= ny - 2);   // the outer two rings
        if (a.bc_ring && outer2) {
            // Keep the pre-average outer two rings for the boundary kernel.
            R *side = a.side;
            const int cols[4] = {0, 1, nx - 2, nx - 1};
            const int rows[4] = {0, 1, ny - 2, ny - 1};
            for (int k = 0; k < 4; k++) {
                if (i == cols[k]) {
                    R *d = side + ((int64_t)k * ny + r) * 3;
                    d[0] = U_stg; d[1] = U_uh; d[2] = U_vh;
                }
                if (r == rows[k]) {
                    R *d = side + (int64_t)4 * ny * 3 + ((int64_t)k * nx + i) * 3;
                    d[0] = U_stg; d[1] = U_uh; d[2] = U_vh;
                }
            }
        }
        U_stg = R(0.5) * (U_stg + a.stg0[o]);
        U_uh = R(0.5) * (U_uh + a.uh0[o]);
        U_vh = R(0.5) * (U_vh + a.vh0[o]);
        if (a.max_stage) {
            const bool ring = a.bc_ring && outer2 && ((i == 0 && a.bext[3]) || (i == nx - 1 && a.bext[1]) ||
                                                      (r == 0 && a.bext[2]) || (r == ny - 1 && a.bext[0]));
            if (!ring) {
                R mx = a.max_stage[o];
                a.max_stage[o] = (U_stg > mx) ? U_stg : mx;
            }
        }
    }
    a.stg_o[o] = U_stg;
    a.uh_o[o] = U_uh;
    a.vh_o[o] = U_vh;
}

// update_U for cell (i, r) (update_U_DE1_inner_include.f90:38-96) from its
// fixed-up centre values and its four edges.
template <typename R, int MODE, bool SPH, bool COR, int FRIC>
__device__ __forceinline__ void fv_update(const Rk2Args<R> &a, int i, int r, const Cell<R> &c, const EdgeRes<R> &n_lo,
                                          const EdgeRes<R> &n_hi, const EdgeRes<R> &w_lo, const EdgeRes<R> &w_hi,
                                          R dt, R inv_cell_area_dt)
{
    R Um_uh, Um_vh;
    fixed_momenta<R>(a, (int64_t)r * a.P + i, c, Um_uh, Um_vh);
    const CellFlux<R> f = cell_flux<R, SPH, COR>(a, i, r, c, Um_uh, Um_vh, n_lo, n_hi, w_lo, w_hi);
    fv_apply<R, MODE, FRIC>(a, i, r, c, Um_uh, Um_vh, f, dt, inv_cell_area_dt);
}
}  // namespace fv
}  // namespace swals
