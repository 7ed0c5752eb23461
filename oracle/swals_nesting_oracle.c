/*
 * swals_nesting_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of SWALS's two-way nesting exchange between domains
 * (GeoscienceAustralia/ptha, propagation/SWALS/src/shallow_water):
 *   - comms setup: initialise_two_way_nesting_comms
 *     (nested_grid_comms_mod.f90:257-658)
 *   - pack: process_data_to_send_2022Feb (:1387-2046)
 *   - unpack: process_received_data (:2048-2249)
 *   - staggered-grid receive fix-ups: receive_halos (domain_mod.f90:3712-3893)
 *   - flux integrals: boundary_flux_integral_tstep (:2300-2469), called from
 *     the time steppers (see swals_oracle.c)
 *   - flux correction: nesting_flux_correction_everywhere and
 *     compute_offset_inside_or_out (domain_mod.f90:2766-3610)
 * Loops follow the reference's order so that every floating-point result is
 * the same.  It is the checker for the CUDA nesting kernels; nothing in the
 * product links it.
 */
#include "swals_oracle.h"

#include <float.h>
#include <math.h>
#include <stddef.h>
#include <string.h>

#define NEST_EPS 1.0e-06          /* nested_grid_comms_mod.f90:39 */
#define NGRAD 4                   /* number_of_gradients_coarse_to_fine (:45) */
#define MIN_DEPTH ((REAL)1.0e-05) /* minimum_allowed_depth (global_mod.f90) */

#ifdef ORACLE_REAL32
#define MISSING_TIME (-FLT_MAX)  /* missing_time_value = -HUGE(1.0_dp) (:40) */
#else
#define MISSING_TIME (-DBL_MAX)
#endif

#define UX(U, nx, ny, i, j, k) (U)[((size_t)((k) - 1) * (size_t)(ny) + (size_t)((j) - 1)) * (size_t)(nx) + (size_t)((i) - 1)]

static int64_t f_nint(double v) { return (int64_t)lround(v); }
static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }
static REAL rmaxr(REAL a, REAL b) { return (b > a) ? b : a; }
static REAL rminr(REAL a, REAL b) { return (b < a) ? b : a; }

/* Edge layout of one box's integrals (N, S, E, W; 4 variables each). */
static void edge_layout(const int32_t *inds, int64_t off[4], int64_t len[4])
{
    const int64_t bl = inds[1] - inds[0] + 1, bw = inds[3] - inds[2] + 1;
    len[0] = bl; len[1] = bl; len[2] = bw; len[3] = bw;
    off[0] = 0; off[1] = 4 * bl; off[2] = 8 * bl; off[3] = 8 * bl + 4 * bw;
}

/* initialise_two_way_nesting_comms (nested_grid_comms_mod.f90:257-658).
 * Returns 0, or 1 for the reference's generic_stop conditions. */
int ORACLE_FN(nest_comm_init)(oracle_nest_comm *c, const double my_dx[2], const double neighbour_dx[2],
                              const int32_t send_inds[6], const int32_t recv_inds[6], int32_t send_only,
                              int32_t recv_only, int32_t use_wetdry_limiting, int32_t my_staggered,
                              int32_t neighbour_staggered)
{
    memset(c, 0, sizeof(*c));
    c->send_active = 1;
    c->recv_active = 1;
    if (send_only && recv_only) return 1;
    if (send_only) c->recv_active = 0;
    if (recv_only) c->send_active = 0;
    c->use_wetdry_limiting = use_wetdry_limiting;
    c->my_domain_staggered_grid = my_staggered;
    c->neighbour_domain_staggered_grid = neighbour_staggered;
    REAL cr[2] = {(REAL)my_dx[0] / (REAL)neighbour_dx[0], (REAL)my_dx[1] / (REAL)neighbour_dx[1]};
    const int equal = (fabs(cr[0] - 1.0) < NEST_EPS) && (fabs(cr[1] - 1.0) < NEST_EPS);
    const REAL prod = cr[0] * cr[1];
    if (prod >= (REAL)1.0 || equal) {
        c->my_domain_is_finer = 0;
        for (int k = 0; k < 2; k++) {
            if (cr[k] < 1.0 - NEST_EPS) return 1;
            if (fabs(cr[k] - (double)f_nint(cr[k])) > NEST_EPS) return 1;
        }
    } else {
        c->my_domain_is_finer = 1;
        for (int k = 0; k < 2; k++)
            if (cr[k] > 1.0 + NEST_EPS) return 1;
        double mx = fmax(1.0 / cr[0], 1.0 / cr[1]);
        double tol = fmin(0.499, fmax(NEST_EPS, 100.0 * (nextafter(mx, INFINITY) - mx)));
        for (int k = 0; k < 2; k++)
            if (fabs(1.0 / cr[k] - (double)f_nint(1.0 / cr[k])) > tol) return 1;
    }
    c->cell_ratios[0] = cr[0];
    c->cell_ratios[1] = cr[1];
    c->equal_cell_ratios = equal;
    memcpy(c->send_inds, send_inds, 6 * sizeof(int32_t));
    memcpy(c->recv_inds, recv_inds, 6 * sizeof(int32_t));
    if (c->send_active) {
        const int iL = send_inds[0], iU = send_inds[1], jL = send_inds[2], jU = send_inds[3];
        const int kL = send_inds[4], kU = send_inds[5];
        if (c->my_domain_is_finer) {
            if ((iU - iL + 1) % f_nint(1.0 / cr[0]) != 0) return 1;
            if ((jU - jL + 1) % f_nint(1.0 / cr[1]) != 0) return 1;
        }
        if (iL > iU || jL > jU || kL > kU) return 1;
        const int64_t bl = iU - iL + 1, bw = jU - jL + 1, bd = kU - kL + 1;
        const int64_t fsz = f_nint((double)(bl * bd) * cr[0]) + f_nint((double)(bl * bd) * cr[0]) +
                            f_nint((double)(bw * bd) * cr[1]) + f_nint((double)(bw * bd) * cr[1]);
        int64_t sbs;
        if (c->my_domain_is_finer || equal)
            sbs = bl * bw * bd / f_nint((1.0 / cr[0]) * (1.0 / cr[1]));
        else
            sbs = bl * bw * bd * (1 + NGRAD);
        c->nsend_interior = sbs;
        c->send_flux_start = sbs + 1;
        sbs += fsz;
        sbs += 1;
        c->send_timeind = sbs;
        c->nsend = sbs;
    }
    if (c->recv_active) {
        const int64_t bl = recv_inds[1] - recv_inds[0] + 1, bw = recv_inds[3] - recv_inds[2] + 1;
        const int64_t bd = recv_inds[5] - recv_inds[4] + 1;
        const int64_t fsz = (bl + bl + bw + bw) * bd;
        int64_t rbs;
        if (c->my_domain_is_finer && !equal)
            rbs = f_nint(((double)(bl * bw * bd) * (cr[0] * cr[1])) * (1 + NGRAD));
        else
            rbs = bl * bw * bd;
        c->nrecv_interior = rbs;
        c->recv_flux_start = rbs + 1;
        rbs += fsz;
        rbs += 1;
        c->recv_timeind = rbs;
        c->nrecv = rbs;
    }
    return 0;
}

/* process_data_to_send_2022Feb (nested_grid_comms_mod.f90:1387-2046). */
void ORACLE_FN(nest_pack)(const oracle_nest_comm *c, const REAL *U, int32_t nx, int32_t ny,
                          const double *send_integral, double time, int32_t has_time, REAL *buf)
{
    if (!c->send_active) return;
    const int imn = 1, jmn = 1, imx = nx, jmx = ny;
    const int iL = c->send_inds[0], iU = c->send_inds[1], jL = c->send_inds[2], jU = c->send_inds[3];
    const int kL = c->send_inds[4], kU = c->send_inds[5];
    const REAL cell_ratios[2] = {(REAL)c->cell_ratios[0], (REAL)c->cell_ratios[1]};
    const int equal = c->equal_cell_ratios;
    const int mys = c->my_domain_staggered_grid, nbs = c->neighbour_domain_staggered_grid;
    REAL inv_cr[2];
    int inv_ip[2], cr_ip[2], iR, jR;
    if (equal) {
        inv_cr[0] = inv_cr[1] = (REAL)1.0;
        inv_ip[0] = inv_ip[1] = 1;
        cr_ip[0] = cr_ip[1] = 1;
        iR = iU - iL + 1;
        jR = jU - jL + 1;
    } else {
        inv_cr[0] = (REAL)1.0 / cell_ratios[0];
        inv_cr[1] = (REAL)1.0 / cell_ratios[1];
        inv_ip[0] = (int)f_nint(inv_cr[0]);
        inv_ip[1] = (int)f_nint(inv_cr[1]);
        cr_ip[0] = (int)f_nint(cell_ratios[0]);
        cr_ip[1] = (int)f_nint(cell_ratios[1]);
        iR = (int)f_nint((iU - iL + 1) * cell_ratios[0]);
        jR = (int)f_nint((jU - jL + 1) * cell_ratios[1]);
    }
    for (int64_t q = 0; q < c->nsend; q++) buf[q] = (REAL)0.0;

    if (c->my_domain_is_finer || equal) {
        for (int k = kL; k <= kU; k++) {
            for (int jouter = jL; jouter <= jU; jouter += inv_ip[1]) {
                for (int jinner = 0; jinner <= inv_ip[1] - 1; jinner++) {
                    const int j = jouter + jinner;
                    const int kC = (k - kL) + 1;
                    if (equal && mys == nbs) {
                        const int jC = (j - jL) + 1;
                        const int64_t off = ((int64_t)(jC - 1) + (int64_t)(kC - 1) * jR) * iR;
                        for (int i = iL; i <= iU; i++) buf[off + (i - iL)] = UX(U, nx, ny, i, j, k);
                        continue;
                    }
                    const int jC = (j - jL) / inv_ip[1] + 1;
                    const int64_t off = ((int64_t)(jC - 1) + (int64_t)(kC - 1) * jR) * iR;
                    for (int i = iL; i <= iU; i++) {
                        const int iC = (i - iL) / inv_ip[0] + 1;
                        REAL *b = &buf[iC + off - 1];
                        const int ci = (i - iL) % inv_ip[0];
                        const int cj = (j - jL) % inv_ip[1];
                        const int centre = (ci == inv_ip[0] / 2) && (cj == inv_ip[1] / 2);
                        if (mys == 1 && nbs == 1) {
                            if (k == OR_STG || k == OR_ELV) {
                                if (centre) *b = UX(U, nx, ny, i, j, k);
                            } else if (k == OR_UH) {
                                if (ci == inv_ip[0] - 1) *b = *b + UX(U, nx, ny, i, j, k) * cell_ratios[1];
                            } else if (k == OR_VH) {
                                if (cj == inv_ip[1] - 1) *b = *b + UX(U, nx, ny, i, j, k) * cell_ratios[0];
                            }
                        } else if (mys == 0 && nbs == 0) {
                            if (centre) *b = UX(U, nx, ny, i, j, k);
                        } else if (mys == 0 && nbs == 1) {
                            if (k == OR_STG || k == OR_ELV) {
                                if (centre) *b = UX(U, nx, ny, i, j, k);
                            } else if (k == OR_UH) {
                                if (ci == inv_ip[0] - 1 && cj == inv_ip[1] / 2) {
                                    const int ip1 = imin(i + 1, nx);
                                    *b = (REAL)0.5 * (UX(U, nx, ny, i, j, k) + UX(U, nx, ny, ip1, j, k));
                                }
                            } else if (k == OR_VH) {
                                if (ci == inv_ip[0] / 2 && cj == inv_ip[1] - 1) {
                                    const int jp1 = imin(j + 1, ny);
                                    *b = (REAL)0.5 * (UX(U, nx, ny, i, j, k) + UX(U, nx, ny, i, jp1, k));
                                }
                            }
                        } else {  /* staggered sender, non-staggered receiver */
                            if (k == OR_STG || k == OR_ELV) {
                                if (centre) *b = UX(U, nx, ny, i, j, k);
                            } else if (k == OR_UH) {
                                if (ci == inv_ip[0] / 2) {
                                    const int im1 = imax(i - 1, 1);
                                    *b = *b + ((REAL)0.5 * UX(U, nx, ny, i, j, k) + (REAL)0.5 * UX(U, nx, ny, im1, j, k)) *
                                                  cell_ratios[1];
                                }
                            } else if (k == OR_VH) {
                                if (cj == inv_ip[1] / 2) {
                                    const int jm1 = imax(j - 1, 1);
                                    *b = *b + ((REAL)0.5 * UX(U, nx, ny, i, j, k) + (REAL)0.5 * UX(U, nx, ny, i, jm1, k)) *
                                                  cell_ratios[0];
                                }
                            }
                        }
                    }
                }
            }
        }
    } else {
        /* Coarse-to-fine: value and one-sided gradients per coarse cell. */
        const REAL upper = (REAL)0.25, lower = (REAL)0.05;
        for (int j = jL; j <= jU; j++) {
            for (int i = iL; i <= iU; i++) {
                const int iim1 = imax(imn, i - 1), iip1 = imin(imx, i + 1);
                const int jjm1 = imax(jmn, j - 1), jjp1 = imin(jmx, j + 1);
                REAL gsx = (REAL)1.0, gsy = (REAL)1.0;
                if (c->use_wetdry_limiting) {
                    REAL dmx = -HUGE_VAL, dmn = HUGE_VAL;
                    for (int ii = iim1; ii <= iip1; ii++) {
                        const REAL dep = UX(U, nx, ny, ii, j, OR_STG) - UX(U, nx, ny, ii, j, OR_ELV);
                        dmx = (ii == iim1) ? dep : rmaxr(dmx, dep);
                        dmn = (ii == iim1) ? dep : rminr(dmn, dep);
                    }
                    if (dmn < upper * dmx) gsx = rmaxr(dmn / dmx - lower, (REAL)0.0) / (upper - lower);
                    if (dmx < (REAL)0.0 || dmn < (REAL)0.0) gsx = (REAL)0.0;
                    for (int jj = jjm1; jj <= jjp1; jj++) {
                        const REAL dep = UX(U, nx, ny, i, jj, OR_STG) - UX(U, nx, ny, i, jj, OR_ELV);
                        dmx = (jj == jjm1) ? dep : rmaxr(dmx, dep);
                        dmn = (jj == jjm1) ? dep : rminr(dmn, dep);
                    }
                    if (dmn < upper * dmx) gsy = rmaxr(dmn / dmx - lower, (REAL)0.0) / (upper - lower);
                    if (dmx < (REAL)0.0 || dmn < (REAL)0.0) gsy = (REAL)0.0;
                }
                for (int k = kL; k <= kU; k++) {
                    REAL dip = 0, dim = 0, djp = 0, djm = 0;
                    if (i > iim1 && i < iip1) {
                        dip = UX(U, nx, ny, i + 1, j, k) - UX(U, nx, ny, i, j, k);
                        dim = UX(U, nx, ny, i, j, k) - UX(U, nx, ny, i - 1, j, k);
                    } else {
                        if (i == iim1) dip = UX(U, nx, ny, i + 1, j, k) - UX(U, nx, ny, i, j, k);
                        else if (i == iip1) dip = UX(U, nx, ny, i, j, k) - UX(U, nx, ny, i - 1, j, k);
                        dim = dip;
                    }
                    if (j > jjm1 && j < jjp1) {
                        djp = UX(U, nx, ny, i, j + 1, k) - UX(U, nx, ny, i, j, k);
                        djm = UX(U, nx, ny, i, j, k) - UX(U, nx, ny, i, j - 1, k);
                    } else {
                        if (j == jjm1) djp = UX(U, nx, ny, i, j + 1, k) - UX(U, nx, ny, i, j, k);
                        else if (j == jjp1) djp = UX(U, nx, ny, i, j, k) - UX(U, nx, ny, i, j - 1, k);
                        djm = djp;
                    }
                    REAL uc = UX(U, nx, ny, i, j, k);
                    if (mys == 1) {
                        if (k == OR_UH) {
                            const REAL del = (nbs == 1) ? (REAL)0.5 - inv_cr[0] * (REAL)0.5 : (REAL)0.5;
                            uc = uc - dim * del;
                            dip = dim;
                            djp = (REAL)0.5 * (UX(U, nx, ny, i, jjp1, k) - UX(U, nx, ny, i, j, k)) +
                                  (REAL)0.5 * (UX(U, nx, ny, iim1, jjp1, k) - UX(U, nx, ny, iim1, j, k));
                            djm = (REAL)0.5 * (UX(U, nx, ny, i, j, k) - UX(U, nx, ny, i, jjm1, k)) +
                                  (REAL)0.5 * (UX(U, nx, ny, iim1, j, k) - UX(U, nx, ny, iim1, jjm1, k));
                        } else if (k == OR_VH) {
                            const REAL del = (nbs == 1) ? (REAL)0.5 - inv_cr[1] * (REAL)0.5 : (REAL)0.5;
                            uc = uc - djm * del;
                            djp = djm;
                            dip = (REAL)0.5 * (UX(U, nx, ny, iip1, j, k) - UX(U, nx, ny, i, j, k)) +
                                  (REAL)0.5 * (UX(U, nx, ny, iip1, jjm1, k) - UX(U, nx, ny, i, jjm1, k));
                            dim = (REAL)0.5 * (UX(U, nx, ny, i, j, k) - UX(U, nx, ny, iim1, j, k)) +
                                  (REAL)0.5 * (UX(U, nx, ny, i, jjm1, k) - UX(U, nx, ny, iim1, jjm1, k));
                        }
                    }
                    if (mys == 0 && nbs == 1) {
                        if (k == OR_UH) uc = uc + (REAL)0.5 * inv_cr[0] * dip;
                        else if (k == OR_VH) uc = uc + (REAL)0.5 * inv_cr[1] * djp;
                    }
                    dip = dip * gsx;
                    djp = djp * gsy;
                    dim = dim * gsx;
                    djm = djm * gsy;
                    const int64_t off = (int64_t)(iU - iL + 1) * (jU - jL + 1) * (k - kL) * (1 + NGRAD) +
                                        (int64_t)(iU - iL + 1) * (j - jL) * (1 + NGRAD) + (int64_t)(i - iL) * (1 + NGRAD);
                    buf[off + 0] = uc;
                    buf[off + 1] = dip;
                    buf[off + 2] = dim;
                    buf[off + 3] = djp;
                    buf[off + 4] = djm;
                }
            }
        }
    }

    /* Boundary flux integrals (:1940-2033). */
    if (send_integral) {
        int64_t eoff[4], elen[4];
        edge_layout(c->send_inds, eoff, elen);
        const int nvar = kU - kL + 1;
        int64_t already = c->send_flux_start - 1;
        if (equal) {
            for (int nb = 0; nb < 4; nb++)
                for (int k = 0; k < nvar; k++)
                    for (int64_t m = 0; m < elen[nb]; m++)
                        buf[already++] = (REAL)send_integral[eoff[nb] + k * elen[nb] + m];
        } else if (c->my_domain_is_finer) {
            const int stride[4] = {inv_ip[0], inv_ip[0], inv_ip[1], inv_ip[1]};
            for (int nb = 0; nb < 4; nb++)
                for (int k = 0; k < nvar; k++)
                    for (int64_t m = 1; m <= elen[nb]; m++) {
                        buf[already] = buf[already] + (REAL)send_integral[eoff[nb] + k * elen[nb] + (m - 1)];
                        if (m % stride[nb] == 0) already++;
                    }
        } else {
            const int stride[4] = {cr_ip[0], cr_ip[0], cr_ip[1], cr_ip[1]};
            for (int nb = 0; nb < 4; nb++) {
                const REAL inv_stride = (REAL)1.0 / (REAL)stride[nb];
                for (int k = 0; k < nvar; k++)
                    for (int64_t m = 0; m < elen[nb]; m++) {
                        const REAL v = (REAL)send_integral[eoff[nb] + k * elen[nb] + m] * inv_stride;
                        for (int q = 0; q < stride[nb]; q++) buf[already + q] = buf[already + q] + v;
                        already += stride[nb];
                    }
            }
        }
    }
    buf[c->send_timeind - 1] = has_time ? (REAL)time : MISSING_TIME;
}

/* process_received_data (nested_grid_comms_mod.f90:2048-2249). */
void ORACLE_FN(nest_unpack)(const oracle_nest_comm *c, const REAL *buf, REAL *U, int32_t nx, int32_t ny,
                            const double *recv_integral, double *recv_error, double *time_received)
{
    if (!c->recv_active) return;
    const int iL = c->recv_inds[0], iU = c->recv_inds[1], jL = c->recv_inds[2], jU = c->recv_inds[3];
    const int kL = c->recv_inds[4], kU = c->recv_inds[5];
    if (time_received) *time_received = (double)buf[c->recv_timeind - 1];
    int64_t n1;
    if (c->my_domain_is_finer) {
        const REAL cr[2] = {(REAL)c->cell_ratios[0], (REAL)c->cell_ratios[1]};
        n1 = f_nint((double)((int64_t)(iU - iL + 1) * (jU - jL + 1) * (kU - kL + 1)) * (cr[0] * cr[1]) * (1 + NGRAD));
        const int inv_ip[2] = {(int)f_nint(1.0 / cr[0]), (int)f_nint(1.0 / cr[1])};
        const REAL mid[2] = {(REAL)0.5 * (REAL)(inv_ip[0] + 1), (REAL)0.5 * (REAL)(inv_ip[1] + 1)};
        const int niC = (iU - iL + 1) / inv_ip[0], njC = (jU - jL + 1) / inv_ip[1];
        const int nC = niC * njC;
        for (int64_t i = 1; i <= n1 - (1 + NGRAD) + 1; i += (1 + NGRAD)) {
            const REAL uc = buf[i - 1], dip = buf[i], dim = buf[i + 1], djp = buf[i + 2], djm = buf[i + 3];
            const int64_t cnt = (i - 1) / (1 + NGRAD);
            const int ck = (int)(cnt / nC);
            const int cj = (int)((cnt - (int64_t)ck * nC) / niC);
            const int ci = (int)(cnt - ((int64_t)ck * nC + (int64_t)cj * niC));
            const int iL1 = iL + ci * inv_ip[0], iU1 = iL1 + inv_ip[0] - 1;
            const int jL1 = jL + cj * inv_ip[1], jU1 = jL1 + inv_ip[1] - 1;
            const int k1 = kL + ck;
            for (int j1 = jL1; j1 <= jU1; j1++) {
                const REAL dUdj = ((REAL)(j1 - jL1 + 1) < mid[1]) ? djm : djp;
                const REAL dUj = ((REAL)(j1 - jL1 + 1) - mid[1]) * cr[1] * dUdj;
                for (int i1 = iL1; i1 <= iU1; i1++) {
                    const REAL dUdi = ((REAL)(i1 - iL1 + 1) < mid[0]) ? dim : dip;
                    const REAL dUi = ((REAL)(i1 - iL1 + 1) - mid[0]) * cr[0] * dUdi;
                    UX(U, nx, ny, i1, j1, k1) = (uc + dUj + dUi);
                }
            }
        }
    } else {
        n1 = (int64_t)(iU - iL + 1) * (jU - jL + 1) * (kU - kL + 1);
        int64_t q = 0;
        for (int k = kL; k <= kU; k++)
            for (int j = jL; j <= jU; j++)
                for (int i = iL; i <= iU; i++) UX(U, nx, ny, i, j, k) = buf[q++];
    }
    if (recv_integral && recv_error) {
        int64_t eoff[4], elen[4];
        edge_layout(c->recv_inds, eoff, elen);
        const int nvar = kU - kL + 1;
        for (int nb = 0; nb < 4; nb++)
            for (int k = 0; k < nvar; k++) {
                const int64_t n0 = n1 + 1;
                n1 = n1 + elen[nb];
                for (int64_t m = 0; m < elen[nb]; m++)
                    recv_error[eoff[nb] + k * elen[nb] + m] =
                        (double)recv_integral[eoff[nb] + k * elen[nb] + m] - (double)buf[n0 - 1 + m];
            }
    }
}

/* Staggered-grid receive fix-ups (domain_mod.f90:3744-3887). */
void ORACLE_FN(nest_recv_fixup)(oracle_domain *d, const int32_t ri[4])
{
    const int nx = d->nx, ny = d->ny;
    REAL *U = d->U;
    const int staggered = (d->method == OR_METHOD_LINEAR || d->method == OR_METHOD_LEAPFROG_LINEAR_PLUS_NONLINEAR_FRICTION ||
                           d->method == OR_METHOD_LEAPFROG_NONLINEAR);
    if (!staggered) return;
    const int iL = ri[0], iU = ri[1], jL = ri[2], jU = ri[3];
    if ((d->method == OR_METHOD_LINEAR || d->method == OR_METHOD_LEAPFROG_LINEAR_PLUS_NONLINEAR_FRICTION) &&
        d->truely_linear) {
        const REAL elev_lim = (REAL)d->msl_linear - MIN_DEPTH;
        for (int jj = jL; jj <= jU; jj++) {
            const int jp1 = imin(jj + 1, ny);
            for (int ii = iL; ii <= iU; ii++) {
                const int ip1 = imin(ii + 1, nx);
                if (UX(U, nx, ny, ii, jj, OR_ELV) >= elev_lim || UX(U, nx, ny, ip1, jj, OR_ELV) >= elev_lim)
                    UX(U, nx, ny, ii, jj, OR_UH) = (REAL)0.0;
                if (UX(U, nx, ny, ii, jj, OR_ELV) >= elev_lim || UX(U, nx, ny, ii, jp1, OR_ELV) >= elev_lim)
                    UX(U, nx, ny, ii, jj, OR_VH) = (REAL)0.0;
            }
        }
    } else if (d->method != OR_METHOD_LEAPFROG_NONLINEAR) {
        for (int jj = jL; jj <= jU; jj++) {
            const int jp1 = imin(jj + 1, ny);
            for (int ii = iL; ii <= iU; ii++) {
                const int ip1 = imin(ii + 1, nx);
                const REAL d0 = UX(U, nx, ny, ii, jj, OR_STG) - UX(U, nx, ny, ii, jj, OR_ELV);
                if (d0 <= MIN_DEPTH || UX(U, nx, ny, ip1, jj, OR_STG) - UX(U, nx, ny, ip1, jj, OR_ELV) <= MIN_DEPTH)
                    UX(U, nx, ny, ii, jj, OR_UH) = (REAL)0.0;
                if (d0 <= MIN_DEPTH || UX(U, nx, ny, ii, jp1, OR_STG) - UX(U, nx, ny, ii, jp1, OR_ELV) <= MIN_DEPTH)
                    UX(U, nx, ny, ii, jj, OR_VH) = (REAL)0.0;
            }
        }
    }
}

/* timestepping_metadata_mod.f90:60-160 */
static int method_mass_only(int m)
{
    return m == OR_METHOD_LINEAR || m == OR_METHOD_LEAPFROG_LINEAR_PLUS_NONLINEAR_FRICTION ||
           m == OR_METHOD_LEAPFROG_NONLINEAR;
}
static int method_unsupported(int m) { return m == OR_METHOD_CLIFFS; }

/* compute_offset_inside_or_out (domain_mod.f90:3486-3608); indices 1-based. */
static void offset_inside_or_out(int *dm, int dm_outside, int out_index, int nbr_index, int my_index, int is_ew,
                                 int *dx_ratio, int *var1, int *varN, const double *all_dx, const int32_t *all_methods)
{
    const int i1 = is_ew ? 0 : 1;
#define ADX(c, d) all_dx[2 * ((d) - 1) + (c)]
    const REAL area_out = (REAL)ADX(0, out_index) * (REAL)ADX(1, out_index);
    const REAL area_nbr = (REAL)ADX(0, nbr_index) * (REAL)ADX(1, nbr_index);
    if (area_out > (REAL)1.25 * area_nbr) *dm = dm_outside;
    else if (area_out < (REAL)0.8 * area_nbr) *dm = 0;
    else *dm = (dm_outside > 0) ? 0 : dm_outside;
    int cor, notcor;
    if (*dm == dm_outside) { cor = out_index; notcor = nbr_index; }
    else { cor = nbr_index; notcor = out_index; }
    if ((REAL)ADX(i1, cor) > (REAL)0.8 * (REAL)ADX(i1, my_index))
        *dx_ratio = (int)f_nint((REAL)ADX(i1, cor) / (REAL)ADX(i1, my_index));
    else
        *dx_ratio = 0;
    const int ct = all_methods[cor - 1], nt = all_methods[notcor - 1];
    if (method_unsupported(ct) || method_unsupported(nt)) { *var1 = -1; *varN = -2; }
    else if (method_mass_only(ct)) { *var1 = OR_STG; *varN = OR_STG; }
    else { *var1 = OR_STG; *varN = OR_VH; }
#undef ADX
}

/* nesting_flux_correction_everywhere (domain_mod.f90:2766-3485), with the
 * default flux_correct_dry_cells_outside_priority_domain = .true.
 * recv_boxes: 4 ints per comm; errors of comm c at recv_error +
 * error_offset[c] in the edge layout above; priority_index: (nx, ny)
 * column-major 1-based domain indices; all_dx: 2 per domain. */
void ORACLE_FN(nest_flux_correction)(oracle_domain *d, int32_t ncomm, const int32_t *recv_boxes,
                                     const int32_t *my_index, const int32_t *nbr_index, const double *recv_error,
                                     const int64_t *error_offset, const int32_t *pind, const double *all_dx,
                                     const int32_t *all_methods, double fraction_of)
{
    const int nx = d->nx, ny = d->ny;
    REAL *U = d->U;
    const REAL frac = (REAL)fraction_of;
#define PIND(i, j) pind[(size_t)((j) - 1) * (size_t)nx + (size_t)((i) - 1)]
    for (int pass = 0; pass < 4; pass++) {  /* NORTH, SOUTH, EAST, WEST */
        for (int c = 0; c < ncomm; c++) {
            const int myi = my_index[c], nbi = nbr_index[c];
            const int n0 = recv_boxes[4 * c], n1 = recv_boxes[4 * c + 1];
            const int m0 = recv_boxes[4 * c + 2], m1 = recv_boxes[4 * c + 3];
            int64_t eoff[4], elen[4];
            edge_layout(&recv_boxes[4 * c], eoff, elen);
            const double *err = recv_error + error_offset[c] + eoff[pass];
            const int64_t len = elen[pass];
            if (pass == 0 || pass == 1) {
                const int north = (pass == 0);
                const int dm_outside = north ? 1 : -1;
                if (north ? !(m1 < ny) : !(m0 > 1)) continue;
                const int medge = north ? m1 : m0;
                for (int ni = n0; ni <= n1; ni++) {
                    const int out_index = PIND(ni, medge + dm_outside);
                    if (out_index == nbi) continue;
                    int dm, dx_ratio, var1, varN;
                    offset_inside_or_out(&dm, dm_outside, out_index, nbi, myi, 0, &dx_ratio, &var1, &varN, all_dx,
                                         all_methods);
                    if (dx_ratio <= 0) continue;
                    int p0, p1, sg;
                    if (north ? (dm > 0) : (dm < 0)) {
                        p0 = north ? medge + dm : medge + dm - dx_ratio + 1;
                        p1 = north ? medge + dm + dx_ratio - 1 : medge + dm;
                        sg = 1;
                    } else {
                        p0 = north ? medge + dm - dx_ratio + 1 : medge + dm;
                        p1 = north ? medge + dm : medge + dm + dx_ratio - 1;
                        sg = -1;
                    }
                    if (!(out_index == myi))
                        if (dm != 0) sg = -sg;
                    if (myi != PIND(ni, p0)) sg = -sg;
                    REAL area_scale = (REAL)0.0;
                    for (int p = p0; p <= p1; p++) area_scale = area_scale + d->area[p - 1];
                    for (int p = p0; p <= p1; p++)
                        for (int k = var1; k <= varN; k++) {
                            const REAL q = (REAL)(err[(int64_t)(k - 1) * len + (ni - n0)] / (double)area_scale);
                            if (north)
                                UX(U, nx, ny, ni, p, k) = UX(U, nx, ny, ni, p, k) - (REAL)sg * q * frac;
                            else
                                UX(U, nx, ny, ni, p, k) = UX(U, nx, ny, ni, p, k) + (REAL)sg * q * frac;
                        }
                }
            } else {
                const int east = (pass == 2);
                const int dn_outside = east ? 1 : -1;
                if (east ? !(n1 < nx) : !(n0 > 1)) continue;
                const int nedge = east ? n1 : n0;
                for (int mi = m0; mi <= m1; mi++) {
                    const int out_index = PIND(nedge + dn_outside, mi);
                    if (out_index == nbi) continue;
                    int dn, dx_ratio, var1, varN;
                    offset_inside_or_out(&dn, dn_outside, out_index, nbi, myi, 1, &dx_ratio, &var1, &varN, all_dx,
                                         all_methods);
                    if (dx_ratio <= 0) continue;
                    int p0, p1, sg;
                    if (east ? (dn > 0) : (dn < 0)) {
                        p0 = east ? nedge + dn : nedge + dn - dx_ratio + 1;
                        p1 = east ? nedge + dn + dx_ratio - 1 : nedge + dn;
                        sg = 1;
                    } else {
                        p0 = east ? nedge + dn - dx_ratio + 1 : nedge + dn;
                        p1 = east ? nedge + dn : nedge + dn + dx_ratio - 1;
                        sg = -1;
                    }
                    if (!(out_index == myi))
                        if (dn != 0) sg = -sg;
                    if (myi != PIND(p0, mi)) sg = -sg;
                    const REAL area_scale = d->area[mi - 1] * (REAL)dx_ratio;
                    for (int p = p0; p <= p1; p++)
                        for (int k = var1; k <= varN; k++) {
                            const REAL q = (REAL)(err[(int64_t)(k - 1) * len + (mi - m0)] / (double)area_scale);
                            if (east)
                                UX(U, nx, ny, p, mi, k) = UX(U, nx, ny, p, mi, k) - (REAL)sg * q * frac;
                            else
                                UX(U, nx, ny, p, mi, k) = UX(U, nx, ny, p, mi, k) + (REAL)sg * q * frac;
                        }
                }
            }
        }
    }
#undef PIND
}
