// nesting.cu -- two-way nesting between domains that live on one GPU: the
// multidomain step of SWALS (multidomain_mod.f90:1093-1212) with its pack /
// unpack exchange (nested_grid_comms_mod.f90:1387-2249), staggered-grid
// receive fix-ups (domain_mod.f90:3712-3893), nesting flux integrals
// (nested_grid_comms_mod.f90:2300-2469) and flux correction
// (domain_mod.f90:2766-3610).
//
// Device layout.  One pool per multidomain holds, per exchange, the
// reference's send buffer (interior values, flux integrals, time; identical
// length on both sides so one buffer serves as the send and the receive
// buffer), the flux integrals of its send box (sender) and receive box
// (receiver), and the receiver's flux errors.  Integrals are laid out edge by
// edge (N, S, E, W) and variable by variable (STG..ELV).  All buffers are
// double; a value is rounded to the precision of the domain that computes
// with it, so the arithmetic of an all-FP64 (or all-FP32) multidomain is the
// reference's.
//
// Kernels: one pack launch and one unpack launch cover every exchange
// (blockIdx.y = exchange); a fix-up launch zeroes staggered-grid fluxes on
// dry faces of received regions; flux correction applies a static, ordered
// list of per-cell corrections built once on the host from the priority
// metadata (the reference's four passes evaluate to the same list every
// step); flux integrals are accumulated per domain after each sub-step
// (recomputing the rk2 stage fluxes along the box edges from the two stage
// inputs, which the step leaves intact).
#include <algorithm>
#include <cfloat>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "domain_internal.h"
#include "rk2_common.cuh"

namespace swals {
namespace nest {

constexpr int MAX_DOMAINS = 16;
constexpr int NG = 5;  // 1 + number_of_gradients_coarse_to_fine
enum { MODE_COPY = 0, MODE_FINE_TO_COARSE = 1, MODE_COARSE_TO_FINE = 2 };

// The state planes of one domain at the time of a launch.
struct DomPtr {
    void *stg, *uh, *vh, *elv;
    int nx, ny;
    int64_t P;
    int fp64;
    int staggered;
    int truely_linear;
    double msl_linear;
};
struct DomTab { DomPtr d[MAX_DOMAINS]; };

// One exchange (a matched send / receive box pair).
struct Ex {
    int sdom, rdom;
    int s[4], r[4];          // iL, iU, jL, jU (1-based, inclusive)
    int mode;                // MODE_* from the sender's point of view
    int equal;               // equal cell sizes (fluxes are copied)
    int s_stag, r_stag, wetdry;
    int inv_ip[2], cr_ip[2]; // sender: nint(1/cell_ratios), nint(cell_ratios)
    double s_cr[2];          // sender's cell_ratios (dx_sender / dx_receiver)
    double r_cr[2];          // receiver's cell_ratios
    int r_finer;
    int r_inv_ip[2];
    int64_t buf;             // offset of the buffer
    int64_t n_interior, flux_start, n_flux, time_index;   // 0-based positions in the buffer
    int64_t s_int, r_int, r_err;   // offsets of the integrals / errors
    int64_t s_len[4], r_len[4];    // edge lengths (N, S, E, W)
    int64_t pack_items, unpack_items;
};

// A flux-integral box of one domain (a send or a receive box).
struct IBox {
    int b[4];
    int64_t off;      // integral offset
    int64_t first;    // first item (edge position) of this box
};

// One flux-correction update (domain_mod.f90:2800-3480 evaluate these).
struct Corr {
    int64_t err;      // index of the flux error (variable STG)
    int64_t err_stride;  // distance between the error of variable k and k+1
    double area_scale;   // in the domain's precision
    int sg_op;        // sg * (+1 subtract, -1 add)
    int var1, varN;
};

__device__ __forceinline__ int64_t cell_off(const DomPtr &d, int i, int j) { return (int64_t)(j - 1) * d.P + (i - 1); }

template <typename R>
__device__ __forceinline__ R ld(const DomPtr &d, int k, int i, int j)
{
    const R *p = (const R *)((k == 1) ? d.stg : (k == 2) ? d.uh : (k == 3) ? d.vh : d.elv);
    return p[cell_off(d, i, j)];
}
template <typename R>
__device__ __forceinline__ void st(const DomPtr &d, int k, int i, int j, R v)
{
    R *p = (R *)((k == 1) ? d.stg : (k == 2) ? d.uh : (k == 3) ? d.vh : d.elv);
    p[cell_off(d, i, j)] = v;
}

// ---------------------------------------------------------------------------
// Pack (process_data_to_send_2022Feb).

template <typename R>
__device__ void pack_f2c(const Ex &e, const DomPtr &s, int64_t q, double *buf)
{
    const int iL = e.s[0], iU = e.s[1], jL = e.s[2], jU = e.s[3];
    const int r0 = e.inv_ip[0], r1 = e.inv_ip[1];
    const int iR = (iU - iL + 1) / r0, jR = (jU - jL + 1) / r1;
    const int ic = (int)(q % iR);
    const int jc = (int)((q / iR) % jR);
    const int k = 1 + (int)(q / ((int64_t)iR * jR));
    const R cr0 = R(e.s_cr[0]), cr1 = R(e.s_cr[1]);
    const int mys = e.s_stag, nbs = e.r_stag;
    R acc = R(0);
    for (int jinner = 0; jinner < r1; jinner++) {
        const int j = jL + jc * r1 + jinner;
        const int cj = jinner;
        for (int ii = 0; ii < r0; ii++) {
            const int i = iL + ic * r0 + ii;
            const int ci = ii;
            const bool centre = (ci == r0 / 2) && (cj == r1 / 2);
            if (mys == 1 && nbs == 1) {
                if (k == 1 || k == 4) { if (centre) acc = ld<R>(s, k, i, j); }
                else if (k == 2) { if (ci == r0 - 1) acc = acc + ld<R>(s, k, i, j) * cr1; }
                else { if (cj == r1 - 1) acc = acc + ld<R>(s, k, i, j) * cr0; }
            } else if (mys == 0 && nbs == 0) {
                if (centre) acc = ld<R>(s, k, i, j);
            } else if (mys == 0 && nbs == 1) {
                if (k == 1 || k == 4) { if (centre) acc = ld<R>(s, k, i, j); }
                else if (k == 2) {
                    if (ci == r0 - 1 && cj == r1 / 2) {
                        const int ip1 = min(i + 1, s.nx);
                        acc = R(0.5) * (ld<R>(s, k, i, j) + ld<R>(s, k, ip1, j));
                    }
                } else {
                    if (ci == r0 / 2 && cj == r1 - 1) {
                        const int jp1 = min(j + 1, s.ny);
                        acc = R(0.5) * (ld<R>(s, k, i, j) + ld<R>(s, k, i, jp1));
                    }
                }
            } else {
                if (k == 1 || k == 4) { if (centre) acc = ld<R>(s, k, i, j); }
                else if (k == 2) {
                    if (ci == r0 / 2) {
                        const int im1 = max(i - 1, 1);
                        acc = acc + (R(0.5) * ld<R>(s, k, i, j) + R(0.5) * ld<R>(s, k, im1, j)) * cr1;
                    }
                } else {
                    if (cj == r1 / 2) {
                        const int jm1 = max(j - 1, 1);
                        acc = acc + (R(0.5) * ld<R>(s, k, i, j) + R(0.5) * ld<R>(s, k, i, jm1)) * cr0;
                    }
                }
            }
        }
    }
    buf[q] = (double)acc;
}

template <typename R>
__device__ __forceinline__ R gscale(R dmn, R dmx)
{
    R g = R(1);
    if (dmn < R(0.25) * dmx) g = rmax(dmn / dmx - R(0.05), R(0)) / (R(0.25) - R(0.05));
    if (dmx < R(0) || dmn < R(0)) g = R(0);
    return g;
}

template <typename R>
__device__ void pack_c2f(const Ex &e, const DomPtr &s, int64_t q, double *buf)
{
    const int iL = e.s[0], iU = e.s[1], jL = e.s[2], jU = e.s[3];
    const int nI = iU - iL + 1, nJ = jU - jL + 1;
    const int i = iL + (int)(q % nI);
    const int j = jL + (int)(q / nI);
    const int iim1 = max(1, i - 1), iip1 = min(s.nx, i + 1);
    const int jjm1 = max(1, j - 1), jjp1 = min(s.ny, j + 1);
    R gsx = R(1), gsy = R(1);
    if (e.wetdry) {
        R dmx = R(0), dmn = R(0);
        for (int ii = iim1; ii <= iip1; ii++) {
            const R dep = ld<R>(s, 1, ii, j) - ld<R>(s, 4, ii, j);
            dmx = (ii == iim1) ? dep : rmax(dmx, dep);
            dmn = (ii == iim1) ? dep : rmin(dmn, dep);
        }
        gsx = gscale<R>(dmn, dmx);
        for (int jj = jjm1; jj <= jjp1; jj++) {
            const R dep = ld<R>(s, 1, i, jj) - ld<R>(s, 4, i, jj);
            dmx = (jj == jjm1) ? dep : rmax(dmx, dep);
            dmn = (jj == jjm1) ? dep : rmin(dmn, dep);
        }
        gsy = gscale<R>(dmn, dmx);
    }
    const R inv_cr0 = R(1) / R(e.s_cr[0]), inv_cr1 = R(1) / R(e.s_cr[1]);
    const int mys = e.s_stag, nbs = e.r_stag;
    for (int k = 1; k <= 4; k++) {
        const R u = ld<R>(s, k, i, j);
        R dip, dim, djp, djm;
        if (i > iim1 && i < iip1) {
            dip = ld<R>(s, k, i + 1, j) - u;
            dim = u - ld<R>(s, k, i - 1, j);
        } else {
            dip = R(0);
            if (i == iim1) dip = ld<R>(s, k, i + 1, j) - u;
            else if (i == iip1) dip = u - ld<R>(s, k, i - 1, j);
            dim = dip;
        }
        if (j > jjm1 && j < jjp1) {
            djp = ld<R>(s, k, i, j + 1) - u;
            djm = u - ld<R>(s, k, i, j - 1);
        } else {
            djp = R(0);
            if (j == jjm1) djp = ld<R>(s, k, i, j + 1) - u;
            else if (j == jjp1) djp = u - ld<R>(s, k, i, j - 1);
            djm = djp;
        }
        R uc = u;
        if (mys == 1) {
            if (k == 2) {
                const R del = (nbs == 1) ? R(0.5) - inv_cr0 * R(0.5) : R(0.5);
                uc = uc - dim * del;
                dip = dim;
                djp = R(0.5) * (ld<R>(s, k, i, jjp1) - u) + R(0.5) * (ld<R>(s, k, iim1, jjp1) - ld<R>(s, k, iim1, j));
                djm = R(0.5) * (u - ld<R>(s, k, i, jjm1)) + R(0.5) * (ld<R>(s, k, iim1, j) - ld<R>(s, k, iim1, jjm1));
            } else if (k == 3) {
                const R del = (nbs == 1) ? R(0.5) - inv_cr1 * R(0.5) : R(0.5);
                uc = uc - djm * del;
                djp = djm;
                dip = R(0.5) * (ld<R>(s, k, iip1, j) - u) + R(0.5) * (ld<R>(s, k, iip1, jjm1) - ld<R>(s, k, i, jjm1));
                dim = R(0.5) * (u - ld<R>(s, k, iim1, j)) + R(0.5) * (ld<R>(s, k, i, jjm1) - ld<R>(s, k, iim1, jjm1));
            }
        }
        if (mys == 0 && nbs == 1) {
            if (k == 2) uc = uc + R(0.5) * inv_cr0 * dip;
            else if (k == 3) uc = uc + R(0.5) * inv_cr1 * djp;
        }
        dip = dip * gsx;
        djp = djp * gsy;
        dim = dim * gsx;
        djm = djm * gsy;
        double *o = buf + (((int64_t)(k - 1) * nJ + (j - jL)) * nI + (i - iL)) * NG;
        o[0] = (double)uc; o[1] = (double)dip; o[2] = (double)dim; o[3] = (double)djp; o[4] = (double)djm;
    }
}

// Entry q of the packed flux integrals (nested_grid_comms_mod.f90:1940-2033).
template <typename R>
__device__ void pack_flux(const Ex &e, int64_t q, const double *sint, double *buf)
{
    // Locate edge nb and variable k of buffer entry q.
    int64_t base_in = 0, pos = q;
    for (int nb = 0; nb < 4; nb++) {
        const int stride = (!e.equal && e.mode == MODE_FINE_TO_COARSE) ? ((nb < 2) ? e.inv_ip[0] : e.inv_ip[1]) : 1;
        const int spread = (e.mode == MODE_COARSE_TO_FINE) ? ((nb < 2) ? e.cr_ip[0] : e.cr_ip[1]) : 1;
        const int64_t len_in = e.s_len[nb];
        const int64_t len_out = (len_in / stride) * spread;
        if (pos < 4 * len_out) {
            const int k = (int)(pos / len_out);
            const int64_t m = pos % len_out;
            const double *x = sint + base_in + (int64_t)k * len_in;
            R v;
            if (e.equal) {
                v = R(x[m]);
            } else if (e.mode == MODE_FINE_TO_COARSE) {
                R acc = R(0);
                for (int t = 0; t < stride; t++) acc = acc + R(x[m * stride + t]);
                v = acc;
            } else {
                const R inv_stride = R(1) / R(spread);
                v = R(0) + R(x[m / spread]) * inv_stride;
            }
            buf[q] = (double)v;
            return;
        }
        pos -= 4 * len_out;
        base_in += 4 * len_in;
    }
}

template <typename R>
__device__ void pack_item(const Ex &e, const DomPtr &s, int64_t q, double *buf, const double *sint)
{
    if (q < e.n_interior) {
        if (e.mode == MODE_COPY) {
            const int nI = e.s[1] - e.s[0] + 1, nJ = e.s[3] - e.s[2] + 1;
            const int i = e.s[0] + (int)(q % nI);
            const int j = e.s[2] + (int)((q / nI) % nJ);
            const int k = 1 + (int)(q / ((int64_t)nI * nJ));
            buf[q] = (double)ld<R>(s, k, i, j);
        } else if (e.mode == MODE_FINE_TO_COARSE) {
            pack_f2c<R>(e, s, q, buf);
        } else {
            pack_c2f<R>(e, s, q, buf);  // q indexes sender cells here
        }
    } else if (q < e.n_interior + e.n_flux) {
        pack_flux<R>(e, q - e.n_interior, sint + e.s_int, buf + e.flux_start);
    } else {
        buf[e.time_index] = s.fp64 ? -DBL_MAX : (double)(-FLT_MAX);  // missing_time_value
    }
}

__global__ void pack_kernel(const Ex *ex, DomTab tab, double *buffers, const double *ints)
{
    const Ex &e = ex[blockIdx.y];
    const DomPtr &s = tab.d[e.sdom];
    double *buf = buffers + e.buf;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < e.pack_items;
         q += (int64_t)gridDim.x * blockDim.x) {
        // Coarse-to-fine packs one item per sender cell (all 4 variables).
        int64_t qq = q;
        if (e.mode == MODE_COARSE_TO_FINE) {
            const int64_t ncell = (int64_t)(e.s[1] - e.s[0] + 1) * (e.s[3] - e.s[2] + 1);
            if (q >= ncell) qq = e.n_interior + (q - ncell);
        }
        if (s.fp64) pack_item<double>(e, s, qq, buf, ints);
        else pack_item<float>(e, s, qq, buf, ints);
    }
}

// ---------------------------------------------------------------------------
// Unpack (process_received_data).

template <typename R>
__device__ void unpack_item(const Ex &e, const DomPtr &d, int64_t q, const double *buf, const double *rint,
                            double *rerr)
{
    const int iL = e.r[0], iU = e.r[1], jL = e.r[2], jU = e.r[3];
    const int nI = iU - iL + 1, nJ = jU - jL + 1;
    const int64_t ncell = (int64_t)nI * nJ * 4;
    if (q < ncell) {
        const int i1 = iL + (int)(q % nI);
        const int j1 = jL + (int)((q / nI) % nJ);
        const int k1 = 1 + (int)(q / ((int64_t)nI * nJ));
        if (e.r_finer) {
            const int r0 = e.r_inv_ip[0], r1 = e.r_inv_ip[1];
            const int niC = nI / r0, njC = nJ / r1;
            const int ci = (i1 - iL) / r0, cj = (j1 - jL) / r1;
            const int64_t cnt = ((int64_t)(k1 - 1) * njC + cj) * niC + ci;
            const double *b = buf + cnt * NG;
            const R uc = R(b[0]), dip = R(b[1]), dim = R(b[2]), djp = R(b[3]), djm = R(b[4]);
            const R mid0 = R(0.5) * R(r0 + 1), mid1 = R(0.5) * R(r1 + 1);
            const int iL1 = iL + ci * r0, jL1 = jL + cj * r1;
            const R cr0 = R(e.r_cr[0]), cr1 = R(e.r_cr[1]);
            const R dUdj = (R(j1 - jL1 + 1) < mid1) ? djm : djp;
            const R dUj = (R(j1 - jL1 + 1) - mid1) * cr1 * dUdj;
            const R dUdi = (R(i1 - iL1 + 1) < mid0) ? dim : dip;
            const R dUi = (R(i1 - iL1 + 1) - mid0) * cr0 * dUdi;
            st<R>(d, k1, i1, j1, (uc + dUj + dUi));
        } else {
            st<R>(d, k1, i1, j1, R(buf[q]));
        }
        return;
    }
    q -= ncell;
    if (q < e.n_flux) {
        // recv_box_flux_error = own integral - received (force_double).
        rerr[e.r_err + q] = rint[e.r_int + q] - (double)R(buf[e.flux_start + q]);
    }
}

__global__ void unpack_kernel(const Ex *ex, DomTab tab, const double *buffers, const double *ints, double *errs)
{
    const Ex &e = ex[blockIdx.y];
    const DomPtr &d = tab.d[e.rdom];
    const double *buf = buffers + e.buf;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < e.unpack_items;
         q += (int64_t)gridDim.x * blockDim.x) {
        if (d.fp64) unpack_item<double>(e, d, q, buf, ints, errs);
        else unpack_item<float>(e, d, q, buf, ints, errs);
    }
}

// Staggered-grid receive fix-ups (domain_mod.f90:3744-3815).
template <typename R>
__device__ void fixup_cell(const DomPtr &d, int ii, int jj)
{
    const int ip1 = min(ii + 1, d.nx), jp1 = min(jj + 1, d.ny);
    if (d.truely_linear) {
        const R lim = R(d.msl_linear) - K<R>::min_depth();
        const R e0 = ld<R>(d, 4, ii, jj);
        if (e0 >= lim || ld<R>(d, 4, ip1, jj) >= lim) st<R>(d, 2, ii, jj, R(0));
        if (e0 >= lim || ld<R>(d, 4, ii, jp1) >= lim) st<R>(d, 3, ii, jj, R(0));
    } else {
        const R md = K<R>::min_depth();
        const R d0 = ld<R>(d, 1, ii, jj) - ld<R>(d, 4, ii, jj);
        if (d0 <= md || ld<R>(d, 1, ip1, jj) - ld<R>(d, 4, ip1, jj) <= md) st<R>(d, 2, ii, jj, R(0));
        if (d0 <= md || ld<R>(d, 1, ii, jp1) - ld<R>(d, 4, ii, jp1) <= md) st<R>(d, 3, ii, jj, R(0));
    }
}

__global__ void fixup_kernel(const Ex *ex, DomTab tab)
{
    const Ex &e = ex[blockIdx.y];
    const DomPtr &d = tab.d[e.rdom];
    if (!d.staggered) return;
    const int nI = e.r[1] - e.r[0] + 1, nJ = e.r[3] - e.r[2] + 1;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < (int64_t)nI * nJ;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int ii = e.r[0] + (int)(q % nI), jj = e.r[2] + (int)(q / nI);
        if (d.fp64) fixup_cell<double>(d, ii, jj);
        else fixup_cell<float>(d, ii, jj);
    }
}

// Flux correction: cell c owns corrections [start[c], start[c+1]) in order.
template <typename R>
__device__ void correct_cell(const DomPtr &d, int i, int j, const Corr *cs, int64_t a, int64_t b, const double *errs,
                             double frac)
{
    for (int64_t t = a; t < b; t++) {
        const Corr &c = cs[t];
        const int sgn = c.sg_op >= 0 ? 1 : -1;         // +1: U - sg*q, -1: U + sg*q
        const R sg = R(c.sg_op >= 0 ? c.sg_op : -c.sg_op);
        for (int k = c.var1; k <= c.varN; k++) {
            const R q = R(errs[c.err + (int64_t)(k - 1) * c.err_stride] / c.area_scale);
            const R u = ld<R>(d, k, i, j);
            const R t2 = sg * q * R(frac);
            st<R>(d, k, i, j, (sgn > 0) ? u - t2 : u + t2);
        }
    }
}

__global__ void correction_kernel(DomPtr d, const int *cells, const int64_t *start, int64_t ncell, const Corr *cs,
                                  const double *errs, double frac)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < ncell; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = cells[2 * q], j = cells[2 * q + 1];
        if (d.fp64) correct_cell<double>(d, i, j, cs, start[q], start[q + 1], errs, frac);
        else correct_cell<float>(d, i, j, cs, start[q], start[q + 1], errs, frac);
    }
}

// ---------------------------------------------------------------------------
// Nesting flux integrals.

// Multidomain time on the device, so that a captured graph of md steps
// replays correctly: t[1] = t[0] + dt at the start of a step (tend,
// multidomain_mod.f90:1108), each domain's time = tend after its sub-steps
// (:1152), t[0] = tend at the end.
__global__ void md_time_begin_kernel(double *t, double dt) { t[1] = t[0] + dt; }
__global__ void md_time_set_kernel(DevScalars *sc, const double *t) { sc->time = t[1]; }
__global__ void md_time_end_kernel(double *t) { t[0] = t[1]; }

__global__ void scale_kernel(double *x, int64_t n, double c)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        x[q] = c * x[q];
}

// Decode item q of a domain's box table into (box, edge, position).
__device__ __forceinline__ int find_box(const IBox *bx, int nbox, int64_t q)
{
    int lo = 0, hi = nbox - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (bx[mid].first <= q) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Linear leapfrog: fluxes are UH / VH before the update, lower index 2,
// STG only, multiplied by the edge length (domain_mod_linear_solver_include.f90:71-77).
template <typename R>
__global__ void integral_leapfrog_kernel(DomPtr d, const R *dxb, const R *dyl, const IBox *bx, int nbox,
                                         int64_t nitems, double *ints, R dt)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nitems; q += (int64_t)gridDim.x * blockDim.x) {
        const int b = find_box(bx, nbox, q);
        const IBox &B = bx[b];
        const int64_t bl = B.b[1] - B.b[0] + 1, bw = B.b[3] - B.b[2] + 1;
        int64_t p = q - B.first;
        double *x = ints + B.off;
        if (p < 2 * bl) {
            const int e = (int)(p / bl);             // 0 north, 1 south
            const int m = B.b[0] + (int)(p % bl);
            const int ns = (e == 0) ? B.b[3] + 1 : B.b[2];
            if (!(ns - 1 >= 1 && ns - 1 <= d.ny)) continue;
            const R f = ld<R>(d, 3, m, ns - 1);
            double *xe = x + e * 4 * bl + (m - B.b[0]);
            *xe = (double)(R(*xe) + (dt * f) * dxb[ns - 1]);
        } else {
            p -= 2 * bl;
            const int e = (int)(p / bw);             // 0 east, 1 west
            const int m = B.b[2] + (int)(p % bw);
            const int ns = (e == 0) ? B.b[1] + 1 : B.b[0];
            if (!(ns - 1 >= 1 && ns - 1 <= d.nx)) continue;
            const R f = ld<R>(d, 2, ns - 1, m);
            double *xe = x + 8 * bl + e * 4 * bw + (m - B.b[2]);
            *xe = (double)(R(*xe) + (dt * f) * dyl[ns - 1]);
        }
    }
}

template <typename R>
__device__ __forceinline__ fv::Cell<R> fv_cell(const R *stg, const R *uh, const R *vh, const R *elv, int64_t P, int i0,
                                               int r0)
{
    // compute_depth_and_velocity (domain_mod.f90:1387-1412) for one cell.
    fv::Cell<R> c;
    const int64_t o = (int64_t)r0 * P + i0;
    R s = stg[o];
    const R e = elv[o];
    R dep = s - e;
    c.u = R(0); c.v = R(0);
    if (dep > K<R>::min_depth()) {
        const R inv = R(1) / dep;
        c.u = uh[o] * inv;
        c.v = vh[o] * inv;
    } else if (dep < R(0)) {
        dep = R(0);
        s = e;
    }
    c.stg = s; c.dep = dep; c.elv = e;
    return c;
}

template <typename R>
__device__ __forceinline__ fv::Grad<R> fv_grad(const fv::Cell<R> &lo, const fv::Cell<R> &c, const fv::Cell<R> &up, R theta)
{
    fv::Grad<R> g;
    const R th = fv::theta_wd<R>(lo.dep, c.dep, up.dep, theta);
    g.ds = fv::mc_half_gradient<R>(c.stg, lo.stg, up.stg, th);
    g.dd = fv::mc_half_gradient<R>(c.dep, lo.dep, up.dep, th);
    g.du = fv::mc_half_gradient<R>(c.u, lo.u, up.u, th);
    g.dv = fv::mc_half_gradient<R>(c.v, lo.v, up.v, th);
    return g;
}

// flux_NS(i, e+1, 1:3) (1-based edge e+1 = bottom edge of 0-based row e) or
// flux_EW; zero where the reference never computes an edge.
template <typename R, bool NS>
__device__ void fv_edge(const R *stg, const R *uh, const R *vh, const R *elv, int64_t P, int nx, int ny,
                        const Metrics<R> &m, R theta, int variant, int i0, int e0, R out[3])
{
    out[0] = out[1] = out[2] = R(0);
    fv::Cell<R> c[4];
    for (int t = 0; t < 4; t++) { c[t].stg = c[t].dep = c[t].u = c[t].v = c[t].elv = R(0); }
    fv::Grad<R> gl, gh;
    const fv::Grad<R> zero = {R(0), R(0), R(0), R(0)};
    if (NS) {
        if (!(e0 >= 1 && e0 <= ny - 1 && i0 >= 1 && i0 <= nx - 1)) return;
        for (int t = 0; t < 4; t++) {
            const int r = e0 - 2 + t;
            if (r >= 0 && r < ny) c[t] = fv_cell<R>(stg, uh, vh, elv, P, i0, r);
        }
        gl = (e0 - 1 > 0 && e0 - 1 < ny - 1) ? fv_grad<R>(c[0], c[1], c[2], theta) : zero;
        gh = (e0 > 0 && e0 < ny - 1) ? fv_grad<R>(c[1], c[2], c[3], theta) : zero;
        fv::EdgeRes<R> res;
        double cand;
        fv::edge_flux<R, true>(c[1], gl, c[2], gh, m.dxb[e0], R(1), res, cand, variant);
        out[0] = res.f[0]; out[1] = res.f[1]; out[2] = res.f[2];
    } else {
        // EW edge at 0-based column e0 (west face of column e0), row i0.
        if (!(e0 >= 1 && e0 <= nx - 1 && i0 >= 1 && i0 <= ny - 1)) return;
        for (int t = 0; t < 4; t++) {
            const int col = e0 - 2 + t;
            if (col >= 0 && col < nx) c[t] = fv_cell<R>(stg, uh, vh, elv, P, col, i0);
        }
        gl = (e0 - 1 > 0 && e0 - 1 < nx - 1) ? fv_grad<R>(c[0], c[1], c[2], theta) : zero;
        gh = (e0 > 0 && e0 < nx - 1) ? fv_grad<R>(c[1], c[2], c[3], theta) : zero;
        fv::EdgeRes<R> res;
        double cand;
        fv::edge_flux<R, false>(c[1], gl, c[2], gh, m.dyl[e0], R(1), res, cand, variant);
        out[0] = res.f[0]; out[1] = res.f[1]; out[2] = res.f[2];
    }
}

// Finite-volume step: for each stage input S (U0, then U1 for rk2), add
// dts * flux(S) to STG..VH (timestepping_alternatives_include.f90:50-59, 95-118).
template <typename R>
__global__ void integral_fv_kernel(DomPtr d, Metrics<R> m, R theta, int variant, const R *s1, const R *u1, const R *v1, const R *s2,
                                   const R *u2, const R *v2, const IBox *bx, int nbox, int64_t nitems, double *ints,
                                   R dts, int nstage)
{
    const R *elv = (const R *)d.elv;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nitems; q += (int64_t)gridDim.x * blockDim.x) {
        const int b = find_box(bx, nbox, q);
        const IBox &B = bx[b];
        const int64_t bl = B.b[1] - B.b[0] + 1, bw = B.b[3] - B.b[2] + 1;
        int64_t p = q - B.first;
        double *x = ints + B.off;
        double *xe;
        int64_t len;
        R f[2][3];
        if (p < 2 * bl) {
            const int e = (int)(p / bl);
            const int mcol = B.b[0] + (int)(p % bl);
            const int ns = (e == 0) ? B.b[3] + 1 : B.b[2];
            if (!(ns >= 1 && ns <= d.ny + 1)) continue;
            fv_edge<R, true>(s1, u1, v1, elv, d.P, d.nx, d.ny, m, theta, variant, mcol - 1, ns - 1, f[0]);
            if (nstage > 1) fv_edge<R, true>(s2, u2, v2, elv, d.P, d.nx, d.ny, m, theta, variant, mcol - 1, ns - 1, f[1]);
            xe = x + e * 4 * bl + (mcol - B.b[0]);
            len = bl;
        } else {
            p -= 2 * bl;
            const int e = (int)(p / bw);
            const int mrow = B.b[2] + (int)(p % bw);
            const int ns = (e == 0) ? B.b[1] + 1 : B.b[0];
            if (!(ns >= 1 && ns <= d.nx + 1)) continue;
            fv_edge<R, false>(s1, u1, v1, elv, d.P, d.nx, d.ny, m, theta, variant, mrow - 1, ns - 1, f[0]);
            if (nstage > 1) fv_edge<R, false>(s2, u2, v2, elv, d.P, d.nx, d.ny, m, theta, variant, mrow - 1, ns - 1, f[1]);
            xe = x + 8 * bl + e * 4 * bw + (mrow - B.b[2]);
            len = bw;
        }
        for (int k = 0; k < 3; k++) {
            R v = R(xe[k * len]);
            for (int s = 0; s < nstage; s++) v = v + (dts * f[s][k]) * R(1);
            xe[k * len] = (double)v;
        }
    }
}

}  // namespace nest
}  // namespace swals

using namespace swals;
using namespace swals::nest;

struct swals_multidomain {
    std::vector<swals_domain *> doms;
    std::vector<cudaStream_t> own_streams;
    std::vector<int> nt;
    std::vector<double> dx;   // all_dx_md: each domain's cell size as the setup computed it
    std::vector<Ex> ex;
    cudaStream_t stream = nullptr;
    int device = 0;
    void *pool = nullptr;
    Ex *d_ex = nullptr;
    double *d_buf = nullptr, *d_int = nullptr, *d_err = nullptr;
    int64_t n_buf = 0, n_int = 0, n_err = 0;
    int64_t max_pack = 0, max_unpack = 0, max_fix = 0;
    // per-domain flux-integral boxes and corrections
    struct PerDom {
        IBox *d_box = nullptr;
        int nbox = 0;
        int64_t nitems = 0;
        int *d_cells = nullptr;
        int64_t *d_start = nullptr;
        Corr *d_corr = nullptr;
        int64_t ncell = 0, ncorr = 0;
    };
    std::vector<PerDom> per;
    bool flux_correction = true;
    double time = 0.0;       // host copy (advanced as steps are issued)
    double *d_time = nullptr; // device copy: [0] md time, [1] tend of the step in flight
    int64_t launches = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_steps = 0;
    double graph_dt = 0.0;
    std::vector<int> graph_cur;   // each domain's state buffer at the capture
};

namespace {

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return api_fail(code, buf);
}

#define MDCK(x)                                                        \
    do {                                                               \
        cudaError_t e_ = (x);                                          \
        if (e_ != cudaSuccess) return api_cuda_fail(e_, #x);           \
    } while (0)

int64_t nint64(double v) { return (int64_t)llround(v); }

DomTab make_tab(const swals_multidomain *md)
{
    DomTab t;
    memset(&t, 0, sizeof(t));
    for (size_t k = 0; k < md->doms.size(); k++) {
        const swals_domain *d = md->doms[k];
        DomPtr &p = t.d[k];
        p.stg = d->planes[d->cur][0];
        p.uh = d->planes[d->cur][1];
        p.vh = d->planes[d->cur][2];
        p.elv = d->elv;
        p.nx = d->nx; p.ny = d->ny; p.P = d->pitch;
        p.fp64 = d->fp64 ? 1 : 0;
        p.staggered = is_linear_leapfrog(d->method) ? 1 : 0;
        p.truely_linear = d->desc.linear_solver_is_truely_linear ? 1 : 0;
        p.msl_linear = d->desc.msl_linear;
    }
    return t;
}

int grid_for(int64_t items)
{
    int64_t b = (items + 255) / 256;
    if (b < 1) b = 1;
    if (b > 4 * 148) b = 4 * 148;
    return (int)b;
}

// The list of flux corrections of one domain, in the reference's order
// (nesting_flux_correction_everywhere, domain_mod.f90:2766-3485, with the
// default flux_correct_dry_cells_outside_priority_domain = .true.).
struct HostCorr { int i, j; Corr c; };

template <typename R>
int build_corrections(const swals_multidomain *md, int dj, const int32_t *pind, std::vector<HostCorr> &out)
{
    const swals_domain *d = md->doms[dj];
    const int nx = d->nx, ny = d->ny;
    auto P = [&](int i, int j) { return pind[(size_t)(j - 1) * nx + (i - 1)]; };
    auto dxof = [&](int idx, int c) -> R { return R(md->dx[2 * (idx - 1) + c]); };  // all_dx_md(c, idx)
    auto mass_only = [&](int idx) { return is_linear_leapfrog(md->doms[idx - 1]->method); };
    const std::vector<double> &area = d->h_metric[2];
    const int myi = dj + 1;
    for (int pass = 0; pass < 4; pass++) {
        for (size_t x = 0; x < md->ex.size(); x++) {
            const Ex &e = md->ex[x];
            if (e.rdom != dj) continue;
            const int nbi = e.sdom + 1;
            const int n0 = e.r[0], n1 = e.r[1], m0 = e.r[2], m1 = e.r[3];
            const int is_ew = pass >= 2;
            const int outside = (pass == 0 || pass == 2) ? 1 : -1;
            const int64_t len = e.r_len[pass];
            int64_t eoff = 0;
            for (int t = 0; t < pass; t++) eoff += 4 * e.r_len[t];
            if (!is_ew) {
                if (pass == 0 ? !(m1 < ny) : !(m0 > 1)) continue;
            } else {
                if (pass == 2 ? !(n1 < nx) : !(n0 > 1)) continue;
            }
            const int a0 = is_ew ? m0 : n0, a1 = is_ew ? m1 : n1;
            const int edge = is_ew ? (pass == 2 ? n1 : n0) : (pass == 0 ? m1 : m0);
            for (int a = a0; a <= a1; a++) {
                const int out_index = is_ew ? P(edge + outside, a) : P(a, edge + outside);
                if (out_index == nbi) continue;
                // compute_offset_inside_or_out (domain_mod.f90:3486-3608)
                const R area_out = dxof(out_index, 0) * dxof(out_index, 1);
                const R area_nbr = dxof(nbi, 0) * dxof(nbi, 1);
                int dm;
                if (area_out > R(1.25) * area_nbr) dm = outside;
                else if (area_out < R(0.8) * area_nbr) dm = 0;
                else dm = (outside > 0) ? 0 : outside;
                const int cor = (dm == outside) ? out_index : nbi;
                const int i1 = is_ew ? 0 : 1;
                int dx_ratio = 0;
                if (dxof(cor, i1) > R(0.8) * dxof(myi, i1)) dx_ratio = (int)nint64(dxof(cor, i1) / dxof(myi, i1));
                if (dx_ratio <= 0) continue;
                const int var1 = 1, varN = mass_only(cor) ? 1 : 3;
                int p0, p1, sg;
                const bool fwd = (outside > 0) ? (dm > 0) : (dm < 0);
                if (fwd) {
                    p0 = (outside > 0) ? edge + dm : edge + dm - dx_ratio + 1;
                    p1 = (outside > 0) ? edge + dm + dx_ratio - 1 : edge + dm;
                    sg = 1;
                } else {
                    p0 = (outside > 0) ? edge + dm - dx_ratio + 1 : edge + dm;
                    p1 = (outside > 0) ? edge + dm : edge + dm + dx_ratio - 1;
                    sg = -1;
                }
                if (!(out_index == myi))
                    if (dm != 0) sg = -sg;
                const int lim = is_ew ? nx : ny;
                if (p0 < 1 || p1 > lim)
                    return fail(SWALS_ERR_INVALID_ARGUMENT,
                                "domain %d: flux correction of receive box %zu reaches outside the domain", dj, x);
                const int pp = is_ew ? P(p0, a) : P(a, p0);
                if (myi != pp) sg = -sg;
                R area_scale;
                if (!is_ew) {
                    area_scale = R(0);
                    for (int p = p0; p <= p1; p++) area_scale = area_scale + R(area[p - 1]);
                } else {
                    area_scale = R(area[a - 1]) * R(dx_ratio);
                }
                const int op = (pass == 0 || pass == 2) ? 1 : -1;  // N, E subtract; S, W add
                for (int p = p0; p <= p1; p++) {
                    HostCorr h;
                    h.i = is_ew ? p : a;
                    h.j = is_ew ? a : p;
                    h.c.err = e.r_err + eoff + (a - a0);
                    h.c.err_stride = len;
                    h.c.area_scale = (double)area_scale;
                    h.c.sg_op = sg * op;
                    h.c.var1 = var1;
                    h.c.varN = varN;
                    out.push_back(h);
                }
            }
        }
    }
    return SWALS_OK;
}

static int integrals_scale(swals_multidomain *md, int k, double c)
{
    // nesting_boundary_flux_integral_multiply: every send and recv box of domain k.
    for (const Ex &e : md->ex) {
        if (e.sdom == k) {
            const int64_t n = 4 * (2 * e.s_len[0] + 2 * e.s_len[2]);
            scale_kernel<<<grid_for(n), 256, 0, md->stream>>>(md->d_int + e.s_int, n, c);
            md->launches++;
        }
        if (e.rdom == k) {
            const int64_t n = 4 * (2 * e.r_len[0] + 2 * e.r_len[2]);
            scale_kernel<<<grid_for(n), 256, 0, md->stream>>>(md->d_int + e.r_int, n, c);
            md->launches++;
        }
    }
    MDCK(cudaGetLastError());
    return SWALS_OK;
}

template <typename R>
static int integral_step(swals_multidomain *md, int k, int phase, int A, double dt_local)
{
    swals_domain *d = md->doms[k];
    const auto &pd = md->per[k];
    if (pd.nitems == 0) return SWALS_OK;
    DomPtr p = make_tab(md).d[k];
    const Metrics<R> m = metrics_of<R>(d);
    if (is_linear_leapfrog(d->method)) {
        if (phase != 0) return SWALS_OK;
        integral_leapfrog_kernel<R><<<grid_for(pd.nitems), 256, 0, md->stream>>>(
            p, m.dxb, m.dyl, pd.d_box, pd.nbox, pd.nitems, md->d_int, R(dt_local));
    } else {
        if (phase != 1) return SWALS_OK;
        const int B = (A + 1) % 3;
        const bool euler = (d->method == M_EULER);
        const R dts = euler ? R(dt_local) : R(R(dt_local) * R(0.5));
        integral_fv_kernel<R><<<grid_for(pd.nitems), 256, 0, md->stream>>>(
            p, m, R(d->cfg.theta), d->cfg.flux_variant, (const R *)d->planes[A][0], (const R *)d->planes[A][1], (const R *)d->planes[A][2],
            (const R *)d->planes[B][0], (const R *)d->planes[B][1], (const R *)d->planes[B][2], pd.d_box, pd.nbox,
            pd.nitems, md->d_int, dts, euler ? 1 : 2);
    }
    md->launches++;
    MDCK(cudaGetLastError());
    return SWALS_OK;
}

}  // namespace

extern "C" {

int swals_gpu_md_create(swals_domain *const *domains, int32_t ndomains, const double *all_dx,
                        const int32_t *refinement, const swals_nest_exchange *exchanges, int32_t nex,
                        const int32_t *const *priority_index, int32_t use_wetdry_limiting, int32_t flux_correction,
                        swals_multidomain **out)
{
    if (!out) return fail(SWALS_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!domains || ndomains < 1 || ndomains > MAX_DOMAINS)
        return fail(SWALS_ERR_INVALID_ARGUMENT, "ndomains must be 1..%d", MAX_DOMAINS);
    if (nex < 0 || (nex > 0 && !exchanges)) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad exchange table");
    for (int k = 0; k < ndomains; k++) {
        const swals_domain *d = domains[k];
        if (!d) return fail(SWALS_ERR_INVALID_ARGUMENT, "domain %d is NULL", k);
        if (d->device != domains[0]->device) return fail(SWALS_ERR_UNSUPPORTED, "all domains must be on one device");
        if (!is_linear_leapfrog(d->method) && d->method != M_RK2 && d->method != M_EULER)
            return fail(SWALS_ERR_UNSUPPORTED, "domain %d: method '%s' is not supported in a multidomain", k,
                        d->desc.timestepping_method);
        if (refinement && refinement[k] < 1) return fail(SWALS_ERR_INVALID_ARGUMENT, "refinement factor < 1");
        if (all_dx && !(all_dx[2 * k] > 0.0 && all_dx[2 * k + 1] > 0.0))
            return fail(SWALS_ERR_INVALID_ARGUMENT, "all_dx of domain %d must be > 0", k);
    }
    if (flux_correction && !priority_index)
        return fail(SWALS_ERR_INVALID_ARGUMENT, "flux correction needs the priority_domain_index arrays");

    auto *md = new swals_multidomain();
    md->device = domains[0]->device;
    md->flux_correction = flux_correction != 0;
    for (int k = 0; k < ndomains; k++) {
        md->doms.push_back(domains[k]);
        md->nt.push_back(refinement ? refinement[k] : 1);
        for (int c = 0; c < 2; c++)
            md->dx.push_back(all_dx ? all_dx[2 * k + c] : domains[k]->desc.lw[c] / (1.0 * domains[k]->desc.nx[c]));
    }
    auto cleanup = [&](int rc) {
        if (md->pool) cudaFree(md->pool);
        delete md;
        return rc;
    };

    // Exchanges: geometry, modes and buffer layout (initialise_two_way_nesting_comms).
    int64_t off_buf = 0, off_int = 0, off_err = 0;
    for (int x = 0; x < nex; x++) {
        const swals_nest_exchange &h = exchanges[x];
        // sender == receiver is a periodic self-exchange (check_periodic boxes).
        if (h.sender < 0 || h.sender >= ndomains || h.receiver < 0 || h.receiver >= ndomains)
            return cleanup(fail(SWALS_ERR_INVALID_ARGUMENT, "exchange %d: bad domain index", x));
        const swals_domain *S = domains[h.sender], *Rd = domains[h.receiver];
        Ex e;
        memset(&e, 0, sizeof(e));
        e.sdom = h.sender; e.rdom = h.receiver;
        for (int t = 0; t < 4; t++) { e.s[t] = h.send_box[t]; e.r[t] = h.recv_box[t]; }
        if (e.s[0] < 1 || e.s[1] > S->nx || e.s[2] < 1 || e.s[3] > S->ny || e.s[0] > e.s[1] || e.s[2] > e.s[3] ||
            e.r[0] < 1 || e.r[1] > Rd->nx || e.r[2] < 1 || e.r[3] > Rd->ny || e.r[0] > e.r[1] || e.r[2] > e.r[3])
            return cleanup(fail(SWALS_ERR_INVALID_ARGUMENT, "exchange %d: box outside its domain", x));
        double sdx[2], rdx[2];
        for (int c = 0; c < 2; c++) {
            sdx[c] = md->dx[2 * h.sender + c];
            rdx[c] = md->dx[2 * h.receiver + c];
        }
        e.s_stag = is_linear_leapfrog(S->method) ? 1 : 0;
        e.r_stag = is_linear_leapfrog(Rd->method) ? 1 : 0;
        e.wetdry = use_wetdry_limiting ? 1 : 0;
        for (int c = 0; c < 2; c++) { e.s_cr[c] = sdx[c] / rdx[c]; e.r_cr[c] = rdx[c] / sdx[c]; }
        const bool equal = fabs(e.s_cr[0] - 1.0) < 1e-6 && fabs(e.s_cr[1] - 1.0) < 1e-6;
        const bool s_finer = !(e.s_cr[0] * e.s_cr[1] >= 1.0 || equal);
        e.r_finer = (!equal && e.r_cr[0] * e.r_cr[1] < 1.0) ? 1 : 0;
        for (int c = 0; c < 2; c++) {
            e.inv_ip[c] = equal ? 1 : (int)nint64(1.0 / e.s_cr[c]);
            e.cr_ip[c] = equal ? 1 : (int)nint64(e.s_cr[c]);
            e.r_inv_ip[c] = (int)nint64(1.0 / e.r_cr[c]);
            const double ratio = std::max(e.s_cr[c], e.r_cr[c]);
            if (fabs(ratio - (double)nint64(ratio)) > std::min(0.499, std::max(1e-6, 100 * (nextafter(ratio, INFINITY) - ratio))))
                return cleanup(fail(SWALS_ERR_INVALID_ARGUMENT, "exchange %d: non-integer cell ratio %g", x, ratio));
        }
        e.equal = equal ? 1 : 0;
        if (equal && e.s_stag == e.r_stag) e.mode = MODE_COPY;
        else if (equal || s_finer) e.mode = MODE_FINE_TO_COARSE;
        else e.mode = MODE_COARSE_TO_FINE;
        const int64_t snI = e.s[1] - e.s[0] + 1, snJ = e.s[3] - e.s[2] + 1;
        const int64_t rnI = e.r[1] - e.r[0] + 1, rnJ = e.r[3] - e.r[2] + 1;
        // Box shapes must correspond through the cell ratio.
        if (e.mode == MODE_COARSE_TO_FINE) {
            if (snI * e.cr_ip[0] != rnI || snJ * e.cr_ip[1] != rnJ)
                return cleanup(fail(SWALS_ERR_INVALID_ARGUMENT, "exchange %d: send/recv boxes do not match", x));
        } else {
            if (snI % e.inv_ip[0] || snJ % e.inv_ip[1] || snI / e.inv_ip[0] != rnI || snJ / e.inv_ip[1] != rnJ)
                return cleanup(fail(SWALS_ERR_INVALID_ARGUMENT, "exchange %d: send/recv boxes do not match", x));
        }
        e.s_len[0] = e.s_len[1] = snI; e.s_len[2] = e.s_len[3] = snJ;
        e.r_len[0] = e.r_len[1] = rnI; e.r_len[2] = e.r_len[3] = rnJ;
        e.n_interior = (e.mode == MODE_COARSE_TO_FINE) ? snI * snJ * 4 * NG : rnI * rnJ * 4;
        e.n_flux = 4 * (2 * rnI + 2 * rnJ);
        e.flux_start = e.n_interior;
        e.time_index = e.n_interior + e.n_flux;
        e.buf = off_buf;
        off_buf += e.time_index + 1;
        e.s_int = off_int; off_int += 4 * (2 * snI + 2 * snJ);
        e.r_int = off_int; off_int += 4 * (2 * rnI + 2 * rnJ);
        e.r_err = off_err; off_err += 4 * (2 * rnI + 2 * rnJ);
        e.pack_items = ((e.mode == MODE_COARSE_TO_FINE) ? snI * snJ : e.n_interior) + e.n_flux + 1;
        e.unpack_items = rnI * rnJ * 4 + e.n_flux;
        md->max_pack = std::max(md->max_pack, e.pack_items);
        md->max_unpack = std::max(md->max_unpack, e.unpack_items);
        md->max_fix = std::max(md->max_fix, rnI * rnJ);
        md->ex.push_back(e);
    }
    md->n_buf = off_buf; md->n_int = off_int; md->n_err = off_err;

    // Per-domain flux-integral boxes (send boxes, then receive boxes).
    std::vector<std::vector<IBox>> boxes(ndomains);
    for (const Ex &e : md->ex) {
        IBox b;
        for (int t = 0; t < 4; t++) b.b[t] = e.s[t];
        b.off = e.s_int;
        boxes[e.sdom].push_back(b);
    }
    for (const Ex &e : md->ex) {
        IBox b;
        for (int t = 0; t < 4; t++) b.b[t] = e.r[t];
        b.off = e.r_int;
        boxes[e.rdom].push_back(b);
    }
    md->per.resize(ndomains);
    std::vector<std::vector<HostCorr>> corr(ndomains);
    int64_t pool_bytes = 0;
    auto al = [](int64_t b) { return (b + 255) / 256 * 256; };
    pool_bytes += al((int64_t)sizeof(Ex) * std::max<int64_t>(1, nex)) + al(2 * sizeof(double));
    pool_bytes += al(8 * std::max<int64_t>(1, md->n_buf)) + al(8 * std::max<int64_t>(1, md->n_int)) +
                  al(8 * std::max<int64_t>(1, md->n_err));
    for (int k = 0; k < ndomains; k++) {
        int64_t first = 0;
        for (IBox &b : boxes[k]) {
            b.first = first;
            first += 2 * (b.b[1] - b.b[0] + 1) + 2 * (b.b[3] - b.b[2] + 1);
        }
        md->per[k].nbox = (int)boxes[k].size();
        md->per[k].nitems = first;
        pool_bytes += al((int64_t)sizeof(IBox) * std::max<size_t>(1, boxes[k].size()));
        if (md->flux_correction) {
            if (!priority_index[k]) return cleanup(fail(SWALS_ERR_INVALID_ARGUMENT, "priority index %d is NULL", k));
            const int rc = domains[k]->fp64 ? build_corrections<double>(md, k, priority_index[k], corr[k])
                                            : build_corrections<float>(md, k, priority_index[k], corr[k]);
            if (rc) return cleanup(rc);
            // Group by cell, keeping each cell's corrections in order.
            std::stable_sort(corr[k].begin(), corr[k].end(), [](const HostCorr &a, const HostCorr &b) {
                return a.j != b.j ? a.j < b.j : a.i < b.i;
            });
            int64_t ncell = 0;
            for (size_t t = 0; t < corr[k].size(); t++)
                if (t == 0 || corr[k][t].i != corr[k][t - 1].i || corr[k][t].j != corr[k][t - 1].j) ncell++;
            md->per[k].ncell = ncell;
            md->per[k].ncorr = (int64_t)corr[k].size();
            pool_bytes += al((int64_t)sizeof(int) * 2 * (ncell + 1)) + al(8 * (ncell + 1)) +
                          al((int64_t)sizeof(Corr) * std::max<int64_t>(1, md->per[k].ncorr));
        }
    }

    cudaError_t ce = cudaSetDevice(md->device);
    if (ce != cudaSuccess) return cleanup(api_cuda_fail(ce, "cudaSetDevice"));
    ce = cudaMalloc(&md->pool, (size_t)pool_bytes);
    if (ce != cudaSuccess) return cleanup(fail(SWALS_ERR_OUT_OF_MEMORY, "multidomain pool of %lld bytes", (long long)pool_bytes));
    char *p = (char *)md->pool;
    md->d_ex = (Ex *)p; p += al((int64_t)sizeof(Ex) * std::max<int64_t>(1, nex));
    md->d_time = (double *)p; p += al(2 * sizeof(double));
    md->d_buf = (double *)p; p += al(8 * std::max<int64_t>(1, md->n_buf));
    md->d_int = (double *)p; p += al(8 * std::max<int64_t>(1, md->n_int));
    md->d_err = (double *)p; p += al(8 * std::max<int64_t>(1, md->n_err));
    md->stream = domains[0]->stream;
    std::vector<char> zeros;
    auto up = [&](void *dst, const void *src, size_t n) {
        return cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice);
    };
    if (nex && (ce = up(md->d_ex, md->ex.data(), sizeof(Ex) * nex)) != cudaSuccess) return cleanup(api_cuda_fail(ce, "upload"));
    if ((ce = cudaMemset(md->d_buf, 0, 8 * std::max<int64_t>(1, md->n_buf))) != cudaSuccess ||
        (ce = cudaMemset(md->d_int, 0, 8 * std::max<int64_t>(1, md->n_int))) != cudaSuccess ||
        (ce = cudaMemset(md->d_err, 0, 8 * std::max<int64_t>(1, md->n_err))) != cudaSuccess)
        return cleanup(api_cuda_fail(ce, "memset"));
    for (int k = 0; k < ndomains; k++) {
        auto &pd = md->per[k];
        pd.d_box = (IBox *)p; p += al((int64_t)sizeof(IBox) * std::max<size_t>(1, boxes[k].size()));
        if (!boxes[k].empty() && (ce = up(pd.d_box, boxes[k].data(), sizeof(IBox) * boxes[k].size())) != cudaSuccess)
            return cleanup(api_cuda_fail(ce, "upload"));
        if (md->flux_correction) {
            std::vector<int> cells;
            std::vector<int64_t> start;
            std::vector<Corr> cs;
            for (size_t t = 0; t < corr[k].size(); t++) {
                if (t == 0 || corr[k][t].i != corr[k][t - 1].i || corr[k][t].j != corr[k][t - 1].j) {
                    cells.push_back(corr[k][t].i);
                    cells.push_back(corr[k][t].j);
                    start.push_back((int64_t)t);
                }
                cs.push_back(corr[k][t].c);
            }
            start.push_back((int64_t)cs.size());
            pd.d_cells = (int *)p; p += al((int64_t)sizeof(int) * 2 * (pd.ncell + 1));
            pd.d_start = (int64_t *)p; p += al(8 * (pd.ncell + 1));
            pd.d_corr = (Corr *)p; p += al((int64_t)sizeof(Corr) * std::max<int64_t>(1, pd.ncorr));
            if (!cells.empty() && (ce = up(pd.d_cells, cells.data(), sizeof(int) * cells.size())) != cudaSuccess)
                return cleanup(api_cuda_fail(ce, "upload"));
            if ((ce = up(pd.d_start, start.data(), sizeof(int64_t) * start.size())) != cudaSuccess)
                return cleanup(api_cuda_fail(ce, "upload"));
            if (!cs.empty() && (ce = up(pd.d_corr, cs.data(), sizeof(Corr) * cs.size())) != cudaSuccess)
                return cleanup(api_cuda_fail(ce, "upload"));
        }
    }
    // All domains run on one stream while they belong to the multidomain.
    for (int k = 0; k < ndomains; k++) {
        md->own_streams.push_back(domains[k]->stream);
        domains[k]->stream = md->stream;
    }
    swals_domain_state st;
    swals_gpu_get_state(domains[0], &st);
    md->time = st.time;
    const double t2[2] = {st.time, st.time};
    if ((ce = cudaMemcpy(md->d_time, t2, sizeof(t2), cudaMemcpyHostToDevice)) != cudaSuccess)
        return cleanup(api_cuda_fail(ce, "upload time"));
    *out = md;
    return SWALS_OK;
}

int swals_gpu_md_destroy(swals_multidomain *md)
{
    if (!md) return SWALS_OK;
    cudaStreamSynchronize(md->stream);
    if (md->graph_exec) cudaGraphExecDestroy(md->graph_exec);
    if (md->graph) cudaGraphDestroy(md->graph);
    for (size_t k = 0; k < md->doms.size(); k++) md->doms[k]->stream = md->own_streams[k];
    if (md->pool) cudaFree(md->pool);
    delete md;
    return SWALS_OK;
}

int swals_gpu_md_send_halos(swals_multidomain *md)
{
    if (!md) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL multidomain");
    if (md->ex.empty()) return SWALS_OK;
    MDCK(cudaSetDevice(md->device));
    dim3 grid(grid_for(md->max_pack), (unsigned)md->ex.size());
    pack_kernel<<<grid, 256, 0, md->stream>>>(md->d_ex, make_tab(md), md->d_buf, md->d_int);
    md->launches++;
    MDCK(cudaGetLastError());
    return SWALS_OK;
}

int swals_gpu_md_recv_halos(swals_multidomain *md)
{
    if (!md) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL multidomain");
    if (md->ex.empty()) return SWALS_OK;
    MDCK(cudaSetDevice(md->device));
    const DomTab tab = make_tab(md);
    dim3 grid(grid_for(md->max_unpack), (unsigned)md->ex.size());
    unpack_kernel<<<grid, 256, 0, md->stream>>>(md->d_ex, tab, md->d_buf, md->d_int, md->d_err);
    md->launches++;
    MDCK(cudaGetLastError());
    bool any_stag = false;
    for (const Ex &e : md->ex) any_stag |= (e.r_stag != 0);
    if (any_stag) {
        dim3 g2(grid_for(md->max_fix), (unsigned)md->ex.size());
        fixup_kernel<<<g2, 256, 0, md->stream>>>(md->d_ex, tab);
        md->launches++;
        MDCK(cudaGetLastError());
    }
    return SWALS_OK;
}

int swals_gpu_md_flux_correction(swals_multidomain *md)
{
    if (!md) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL multidomain");
    if (!md->flux_correction) return SWALS_OK;
    MDCK(cudaSetDevice(md->device));
    const DomTab tab = make_tab(md);
    for (size_t k = 0; k < md->doms.size(); k++) {
        const auto &pd = md->per[k];
        if (pd.ncell == 0) continue;
        correction_kernel<<<grid_for(pd.ncell), 256, 0, md->stream>>>(tab.d[k], pd.d_cells, pd.d_start, pd.ncell,
                                                                     pd.d_corr, md->d_err, 1.0);
        md->launches++;
        MDCK(cudaGetLastError());
    }
    return SWALS_OK;
}

int swals_gpu_md_evolve_one_step(swals_multidomain *md, double dt)
{
    if (!md) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL multidomain");
    if (!(dt > 0.0)) return fail(SWALS_ERR_INVALID_ARGUMENT, "dt must be > 0");
    MDCK(cudaSetDevice(md->device));
    const double tend = md->time + dt;
    md_time_begin_kernel<<<1, 1, 0, md->stream>>>(md->d_time, dt);
    md->launches++;
    for (size_t k = 0; k < md->doms.size(); k++) {
        swals_domain *d = md->doms[k];
        int rc = integrals_scale(md, (int)k, 0.0);
        if (rc) return rc;
        const int nt = md->nt[k];
        const double dt_local = dt / (1.0 * nt);
        for (int s = 0; s < nt; s++) {
            rc = d->fp64 ? integral_step<double>(md, (int)k, 0, d->cur, dt_local)
                         : integral_step<float>(md, (int)k, 0, d->cur, dt_local);
            if (rc) return rc;
            const int A = d->cur;
            rc = swals_gpu_evolve_one_step(d, dt_local, 1);
            if (rc) return rc;
            rc = d->fp64 ? integral_step<double>(md, (int)k, 1, A, dt_local)
                         : integral_step<float>(md, (int)k, 1, A, dt_local);
            if (rc) return rc;
        }
        // domains(j)%time = tend (multidomain_mod.f90:1152)
        md_time_set_kernel<<<1, 1, 0, md->stream>>>(d->sc, md->d_time);
        md->launches++;
        MDCK(cudaGetLastError());
    }
    int rc = swals_gpu_md_send_halos(md);
    if (rc) return rc;
    rc = swals_gpu_md_recv_halos(md);
    if (rc) return rc;
    rc = swals_gpu_md_flux_correction(md);
    if (rc) return rc;
    md_time_end_kernel<<<1, 1, 0, md->stream>>>(md->d_time);
    md->launches++;
    MDCK(cudaGetLastError());
    md->time = tend;
    return SWALS_OK;
}

int swals_gpu_md_capture_graph(swals_multidomain *md, int32_t nsteps, double dt)
{
    if (!md || nsteps < 1 || !(dt > 0.0)) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    MDCK(cudaSetDevice(md->device));
    // Every domain must come back to the same state buffer after the
    // captured steps, so that the graph can be replayed as often as wanted.
    std::vector<int> cur0;
    for (swals_domain *d : md->doms) cur0.push_back(d->cur);
    if (md->graph_exec) { cudaGraphExecDestroy(md->graph_exec); md->graph_exec = nullptr; }
    if (md->graph) { cudaGraphDestroy(md->graph); md->graph = nullptr; }
    MDCK(cudaStreamSynchronize(md->stream));
    const double time0 = md->time;
    const int64_t l0 = md->launches;
    std::vector<int64_t> dl0;
    for (swals_domain *d : md->doms) dl0.push_back(d->launches);
    std::vector<int64_t> ns0;
    for (swals_domain *d : md->doms) ns0.push_back(d->nsteps);
    MDCK(cudaStreamBeginCapture(md->stream, cudaStreamCaptureModeThreadLocal));
    int rc = SWALS_OK;
    for (int s = 0; s < nsteps && rc == SWALS_OK; s++) rc = swals_gpu_md_evolve_one_step(md, dt);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(md->stream, &g);
    // Capture records work without running it: restore the host bookkeeping.
    md->time = time0;
    md->launches = l0;
    bool same = true;
    for (size_t k = 0; k < md->doms.size(); k++) {
        same &= (md->doms[k]->cur == cur0[k]);
        md->doms[k]->cur = cur0[k];
        md->doms[k]->launches = dl0[k];
        md->doms[k]->nsteps = ns0[k];
    }
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (ce != cudaSuccess) { if (g) cudaGraphDestroy(g); return api_cuda_fail(ce, "cudaStreamEndCapture"); }
    if (!same) {
        cudaGraphDestroy(g);
        return fail(SWALS_ERR_INVALID_ARGUMENT,
                    "%d md steps do not return every domain to its state buffer; capture a multiple of 3 steps",
                    nsteps);
    }
    ce = cudaGraphInstantiate(&md->graph_exec, g, 0);
    if (ce != cudaSuccess) { cudaGraphDestroy(g); return api_cuda_fail(ce, "cudaGraphInstantiate"); }
    md->graph = g;
    md->graph_steps = nsteps;
    md->graph_dt = dt;
    md->graph_cur = cur0;
    return SWALS_OK;
}

int swals_gpu_md_replay(swals_multidomain *md, int32_t nreplays)
{
    if (!md || nreplays < 0) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    if (!md->graph_exec) return fail(SWALS_ERR_INVALID_ARGUMENT, "no captured graph");
    for (size_t k = 0; k < md->doms.size(); k++)
        if (md->doms[k]->cur != md->graph_cur[k])
            return fail(SWALS_ERR_INVALID_ARGUMENT,
                        "domain %d has moved to another state buffer since the graph was captured (md steps taken "
                        "in between that are not a multiple of 3); capture the graph again", (int)k);
    MDCK(cudaSetDevice(md->device));
    for (int r = 0; r < nreplays; r++) {
        MDCK(cudaGraphLaunch(md->graph_exec, md->stream));
        md->launches++;
        md->time += md->graph_steps * md->graph_dt;
        for (swals_domain *d : md->doms) d->nsteps += (int64_t)md->graph_steps;
    }
    return SWALS_OK;
}

// A group of multidomains (independent instances: many sources on the same
// nest, or different nests) advanced together: nsteps md steps of every
// member captured into one CUDA graph, each member on its own branch (its
// own stream, forked from and joined back to the group's stream), so one
// launch advances all of them and the kernels of different members run
// concurrently: the small exchange kernels and the partial last waves of
// each domain's step kernels are overlapped with other members' work.
struct swals_md_group {
    std::vector<swals_multidomain *> mds;
    std::vector<std::vector<int>> cur;   // each member's domains' state buffers at the capture
    cudaStream_t stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;
    int steps = 0;
    double dt = 0.0;
};

int swals_gpu_md_group_create(swals_multidomain *const *mds, int32_t n, int32_t nsteps, double dt,
                              swals_md_group **out)
{
    if (!mds || n < 1 || nsteps < 1 || !(dt > 0.0) || !out) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    *out = nullptr;
    for (int q = 0; q < n; q++) {
        if (!mds[q]) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL multidomain %d", q);
        if (mds[q]->device != mds[0]->device) return fail(SWALS_ERR_INVALID_ARGUMENT, "members on different devices");
        for (int r = 0; r < q; r++)
            if (mds[r] == mds[q]) return fail(SWALS_ERR_INVALID_ARGUMENT, "multidomain %d appears twice", q);
    }
    MDCK(cudaSetDevice(mds[0]->device));
    swals_md_group *g = new swals_md_group();
    g->mds.assign(mds, mds + n);
    g->device = mds[0]->device;
    g->steps = nsteps;
    g->dt = dt;
    cudaError_t ce = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) { delete g; return api_cuda_fail(ce, "group stream"); }
    // Host bookkeeping of every member, restored after the capture.
    struct Saved { double time; int64_t launches; std::vector<int> cur; std::vector<int64_t> dl, ns; };
    std::vector<Saved> saved(n);
    for (int q = 0; q < n; q++) {
        swals_multidomain *md = g->mds[q];
        MDCK(cudaStreamSynchronize(md->stream));
        saved[q].time = md->time;
        saved[q].launches = md->launches;
        for (swals_domain *d : md->doms) {
            saved[q].cur.push_back(d->cur);
            saved[q].dl.push_back(d->launches);
            saved[q].ns.push_back(d->nsteps);
        }
    }
    std::vector<cudaEvent_t> evs(n + 1, nullptr);
    int rc = SWALS_OK;
    for (auto &e : evs)
        if (rc == SWALS_OK && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            rc = fail(SWALS_ERR_CUDA, "event creation");
    cudaGraph_t graph = nullptr;
    if (rc == SWALS_OK) {
        ce = cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal);
        if (ce != cudaSuccess) rc = api_cuda_fail(ce, "cudaStreamBeginCapture");
    }
    if (rc == SWALS_OK) {
        bool capturing = true;
        ce = cudaEventRecord(evs[n], g->stream);   // fork
        for (int q = 0; q < n && ce == cudaSuccess; q++) ce = cudaStreamWaitEvent(g->mds[q]->stream, evs[n], 0);
        if (ce != cudaSuccess) rc = api_cuda_fail(ce, "fork");
        for (int q = 0; q < n && rc == SWALS_OK; q++)
            for (int s = 0; s < nsteps && rc == SWALS_OK; s++) rc = swals_gpu_md_evolve_one_step(g->mds[q], dt);
        for (int q = 0; q < n && rc == SWALS_OK; q++) {   // join
            ce = cudaEventRecord(evs[q], g->mds[q]->stream);
            if (ce == cudaSuccess) ce = cudaStreamWaitEvent(g->stream, evs[q], 0);
            if (ce != cudaSuccess) rc = api_cuda_fail(ce, "join");
        }
        ce = cudaStreamEndCapture(g->stream, &graph);
        capturing = false;
        (void)capturing;
        if (rc == SWALS_OK && ce != cudaSuccess) rc = api_cuda_fail(ce, "cudaStreamEndCapture");
    }
    // Capture records work without running it: restore the bookkeeping, and
    // require every domain back in its state buffer after nsteps.
    bool same = true;
    for (int q = 0; q < n; q++) {
        swals_multidomain *md = g->mds[q];
        md->time = saved[q].time;
        md->launches = saved[q].launches;
        for (size_t k = 0; k < md->doms.size(); k++) {
            same &= (md->doms[k]->cur == saved[q].cur[k]);
            md->doms[k]->cur = saved[q].cur[k];
            md->doms[k]->launches = saved[q].dl[k];
            md->doms[k]->nsteps = saved[q].ns[k];
        }
        g->cur.push_back(saved[q].cur);
    }
    for (auto &e : evs)
        if (e) cudaEventDestroy(e);
    if (rc == SWALS_OK && !same)
        rc = fail(SWALS_ERR_INVALID_ARGUMENT,
                  "%d md steps do not return every domain to its state buffer; capture a multiple of 3 steps", nsteps);
    if (rc == SWALS_OK) {
        ce = cudaGraphInstantiate(&g->exec, graph, 0);
        if (ce != cudaSuccess) rc = api_cuda_fail(ce, "cudaGraphInstantiate");
    }
    if (graph) cudaGraphDestroy(graph);
    if (rc != SWALS_OK) {
        if (g->exec) cudaGraphExecDestroy(g->exec);
        cudaStreamDestroy(g->stream);
        delete g;
        return rc;
    }
    *out = g;
    return SWALS_OK;
}

int swals_gpu_md_group_replay(swals_md_group *g, int32_t nreplays)
{
    if (!g || nreplays < 0) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    for (size_t q = 0; q < g->mds.size(); q++)
        for (size_t k = 0; k < g->mds[q]->doms.size(); k++)
            if (g->mds[q]->doms[k]->cur != g->cur[q][k])
                return fail(SWALS_ERR_INVALID_ARGUMENT,
                            "member %d, domain %d has moved to another state buffer since the group was captured",
                            (int)q, (int)k);
    MDCK(cudaSetDevice(g->device));
    // the members' own streams may hold work issued before: the graph
    // starts after it
    cudaEvent_t ev = nullptr;
    MDCK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    for (swals_multidomain *md : g->mds) {
        MDCK(cudaEventRecord(ev, md->stream));
        MDCK(cudaStreamWaitEvent(g->stream, ev, 0));
    }
    for (int r = 0; r < nreplays; r++) MDCK(cudaGraphLaunch(g->exec, g->stream));
    // and work issued on a member's stream afterwards follows the replays
    MDCK(cudaEventRecord(ev, g->stream));
    for (swals_multidomain *md : g->mds) MDCK(cudaStreamWaitEvent(md->stream, ev, 0));
    cudaEventDestroy(ev);
    for (swals_multidomain *md : g->mds) {
        md->launches += nreplays;
        md->time += (double)nreplays * g->steps * g->dt;
        for (swals_domain *d : md->doms) d->nsteps += (int64_t)nreplays * g->steps;
    }
    return SWALS_OK;
}

int swals_gpu_md_group_stream(swals_md_group *g, void **stream)
{
    if (!g || !stream) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    *stream = (void *)g->stream;
    return SWALS_OK;
}

int swals_gpu_md_group_destroy(swals_md_group *g)
{
    if (!g) return SWALS_OK;
    cudaSetDevice(g->device);
    cudaStreamSynchronize(g->stream);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    cudaStreamDestroy(g->stream);
    delete g;
    return SWALS_OK;
}

int swals_gpu_md_buffer_size(swals_multidomain *md, int32_t x, int64_t *n)
{
    if (!md || !n || x < 0 || x >= (int32_t)md->ex.size()) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    *n = md->ex[x].time_index + 1;
    return SWALS_OK;
}

int swals_gpu_md_download_buffer(swals_multidomain *md, int32_t x, double *out, int64_t n)
{
    if (!md || !out || x < 0 || x >= (int32_t)md->ex.size()) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    const Ex &e = md->ex[x];
    if (n != e.time_index + 1) return fail(SWALS_ERR_INVALID_ARGUMENT, "buffer of exchange %d has %lld values", x,
                                           (long long)(e.time_index + 1));
    MDCK(cudaSetDevice(md->device));
    MDCK(cudaMemcpyAsync(out, md->d_buf + e.buf, sizeof(double) * n, cudaMemcpyDeviceToHost, md->stream));
    MDCK(cudaStreamSynchronize(md->stream));
    return SWALS_OK;
}

int swals_gpu_md_download_flux(swals_multidomain *md, int32_t x, int32_t which, double *out, int64_t n)
{
    if (!md || !out || x < 0 || x >= (int32_t)md->ex.size() || which < 0 || which > 2)
        return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    const Ex &e = md->ex[x];
    const int64_t len = (which == 0) ? 4 * (2 * e.s_len[0] + 2 * e.s_len[2]) : 4 * (2 * e.r_len[0] + 2 * e.r_len[2]);
    if (n != len) return fail(SWALS_ERR_INVALID_ARGUMENT, "expected %lld values", (long long)len);
    const double *src = (which == 0) ? md->d_int + e.s_int : (which == 1) ? md->d_int + e.r_int : md->d_err + e.r_err;
    MDCK(cudaSetDevice(md->device));
    MDCK(cudaMemcpyAsync(out, src, sizeof(double) * n, cudaMemcpyDeviceToHost, md->stream));
    MDCK(cudaStreamSynchronize(md->stream));
    return SWALS_OK;
}

int swals_gpu_md_time(swals_multidomain *md, double *time)
{
    if (!md || !time) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    *time = md->time;
    return SWALS_OK;
}

int swals_gpu_md_synchronize(swals_multidomain *md)
{
    if (!md) return fail(SWALS_ERR_INVALID_ARGUMENT, "NULL multidomain");
    MDCK(cudaSetDevice(md->device));
    MDCK(cudaStreamSynchronize(md->stream));
    return swals::api_check_bulk_waits(md->stream);
}

int swals_gpu_md_launch_count(swals_multidomain *md, int64_t *n)
{
    if (!md || !n) return fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    int64_t t = md->launches;
    for (swals_domain *d : md->doms) t += d->launches;
    *n = t;
    return SWALS_OK;
}

}  // extern "C"
