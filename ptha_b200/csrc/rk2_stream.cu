// rk2_stream.cu -- finite-volume stage kernels, streaming forms: the
// register form (rk2_stream_kernel) and the shared-memory-rows form
// (rk2_srow_kernel, below), whose strips are one warp wide or, by default
// for every stage, as wide as the CTA (four warps, 124 output columns).
//
// Same computation as the shared-memory tile kernel in rk2.cu (and the same
// device functions: edge_flux, mc_half_gradient, theta_wd, fv_update), organised
// for sm_100a's FP64 pipes instead of for shared memory:
//   - each warp owns a strip of 28 columns (lanes 2..29; lanes 0,1,30,31
//     carry the 2-cell x-halo) and marches down SH rows plus a 2-row halo at
//     each end;
//   - the three rows the north-south limiter needs (j-2, j-1, j), the
//     north-south gradients of two rows and the south edge of the row being
//     updated live in registers; east-west neighbours come from warp
//     shuffles;
//   - each cell's north-south edge, gradient and fix-ups are computed once
//     (the tile kernel computes ~2.2 edges and ~2.3 gradients per cell) and
//     there is no __syncthreads at all;
//   - the next row's loads are issued before the current row is processed;
//   - registers are capped for 4 CTAs (16 warps) per SM: the FP64 chains are
//     latency-bound, and 16 warps beat 12 unspilled ones (measured 12% faster
//     on the 2048x2048 beach, a few spilled values included).
#include "rk2_common.cuh"

#include <cmath>
#include <cstdlib>
#include <cstring>

namespace swals {
namespace {
using namespace fv;

constexpr int SLANES = 32;
constexpr int SOUT = 28;    // output columns per warp
#ifndef SWALS_STREAM_WARPS
#define SWALS_STREAM_WARPS 4
#endif
constexpr int SWARPS = SWALS_STREAM_WARPS;   // warps per CTA
#ifndef SWALS_STREAM_MIN_CTAS
#define SWALS_STREAM_MIN_CTAS 4  // CTAs per SM the register cap is sized for
#endif
// Rows per strip segment (fv_rows, below): on the 2048^2 rk2 step (B200)
// 12 rows beat 32 by 4 % (and 24 by 2 %) despite the larger share of the
// two lead-in rows, as the more numerous, shorter strips balance better
// over the SMs; with the shared-memory-rows update stages, 8 / 10 / 12 / 16
// / 20 rows give 0.789 / 0.783 / 0.786 / 0.796 / 0.811 ms a step, and with
// the CTA-wide strips 8 / 10 / 12 / 14 / 16 / 20 rows 0.757 / 0.747 / 0.743
// / 0.760 / 0.748 / 0.744 ms; more CTAs per SM (a lower register cap) spill
// and lose 15-25 %.
// Also measured and dropped: a persistent one-wave launch with equal
// contiguous runs per warp (fewer recomputed halo rows, 8 % slower), the
// same grid looping over 12-row strips (15 % slower), the row constants
// dt/area and 1/(dx cfl/2) evaluated once per 32 rows and shuffled (2 %
// slower: the extra live registers spill), 3 CTAs per SM without spills
// (9 % slower than 4) or 5 CTAs (13 % slower), FMA contraction (2 %
// faster, but no longer bit-exact with the IEEE-strict oracle, and 2e-9
// relative after 600 steps), and a two-phase software pipeline of the
// shared-memory-rows march (the update of row r-3 and the north-south work
// of row r between the same two barriers, one barrier fewer a row, 52 KB of
// shared memory per CTA: flux pass 0.268 -> 0.278 ms, stage 2 0.362 ->
// 0.366).
constexpr unsigned FULL = 0xffffffffu;

template <typename R> struct Raw { R s, uh, vh, e; };

template <typename R>
__device__ __forceinline__ Raw<R> load_raw(const Rk2Args<R> &a, int i, int r)
{
    Raw<R> x;
    if (i >= 0 && i < a.nx && r >= 0 && r < a.ny) {
        const int64_t o = (int64_t)r * a.P + i;
        x.s = a.stg[o]; x.uh = a.uh[o]; x.vh = a.vh[o]; x.e = a.elv[o];
    } else {
        x.s = R(0); x.uh = R(0); x.vh = R(0); x.e = R(0);
    }
    return x;
}

// compute_depth_and_velocity for one cell (domain_mod.f90:1387-1412).
template <typename R>
__device__ __forceinline__ Cell<R> fix_up(const Raw<R> &x, bool valid, long long &negfix, bool count)
{
    Cell<R> c;
    c.stg = R(0); c.dep = R(0); c.u = R(0); c.v = R(0); c.elv = R(0);
    if (valid) {
        R s = x.s;
        const R e = x.e;
        R dep = s - e;
        if (dep > K<R>::min_depth()) {
            const R depth_inv = R(1) / dep;
            c.u = x.uh * depth_inv;
            c.v = x.vh * depth_inv;
        } else if (dep < R(0)) {
            dep = R(0);
            s = e;
            if (count) negfix += 1;
        }
        c.stg = s; c.dep = dep; c.elv = e;
    }
    return c;
}

// Bring a line into L2 ahead of its use (no register is written).
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

template <typename R> __device__ __forceinline__ R up1(R v) { return __shfl_up_sync(FULL, v, 1); }
template <typename R> __device__ __forceinline__ R dn1(R v) { return __shfl_down_sync(FULL, v, 1); }

template <typename R>
__device__ __forceinline__ Cell<R> up1(const Cell<R> &c)
{
    Cell<R> x; x.stg = up1(c.stg); x.dep = up1(c.dep); x.u = up1(c.u); x.v = up1(c.v); x.elv = up1(c.elv); return x;
}
template <typename R>
__device__ __forceinline__ Cell<R> dn1(const Cell<R> &c)
{
    Cell<R> x; x.stg = dn1(c.stg); x.dep = dn1(c.dep); x.u = dn1(c.u); x.v = dn1(c.v); x.elv = dn1(c.elv); return x;
}

template <typename R>
__device__ __forceinline__ Grad<R> limited(const Cell<R> &lo, const Cell<R> &c, const Cell<R> &up, R theta)
{
    Grad<R> g;
    const R th = theta_wd<R>(lo.dep, c.dep, up.dep, theta);
    g.ds = mc_half_gradient<R>(c.stg, lo.stg, up.stg, th);
    g.dd = mc_half_gradient<R>(c.dep, lo.dep, up.dep, th);
    g.du = mc_half_gradient<R>(c.u, lo.u, up.u, th);
    g.dv = mc_half_gradient<R>(c.v, lo.v, up.v, th);
    return g;
}

template <typename R>
__device__ __forceinline__ void zero_edge(EdgeRes<R> &e)
{
    e.f[0] = R(0); e.f[1] = R(0); e.f[2] = R(0); e.es_pos = 0.0; e.es_neg = 0.0;
}

// The flux pass's output for cell (i, r): its dt-independent update terms
// (cell_flux) from its four edges, for the stage-1 update once dt is known.
template <typename R, bool SPH, bool COR>
__device__ __forceinline__ void store_cell_flux(const Rk2Args<R> &a, int i, int r, const Cell<R> &c,
                                                const EdgeRes<R> &n_lo, const EdgeRes<R> &n_hi,
                                                const EdgeRes<R> &w_lo, const EdgeRes<R> &w_hi)
{
    const int64_t o = (int64_t)r * a.P + i;
    R Um_uh = R(0), Um_vh = R(0);
    if (SPH) fixed_momenta<R>(a, o, c, Um_uh, Um_vh);   // only the spherical terms read them
    const CellFlux<R> f = cell_flux<R, SPH, COR>(a, i, r, c, Um_uh, Um_vh, n_lo, n_hi, w_lo, w_hi);
    a.cs.d[0][o] = f.d[0]; a.cs.d[1][o] = f.d[1]; a.cs.d[2][o] = f.d[2];
    a.cs.eu[o] = f.eu; a.cs.ev[o] = f.ev;
}

template <typename R, int MODE, bool SPH, bool COR, int FRIC, bool EDDY>
__global__ void __launch_bounds__(SLANES *SWARPS, SWALS_STREAM_MIN_CTAS) rk2_stream_kernel(const Rk2Args<R> a, int SH)
{
    const int lane = threadIdx.x & 31;
    const int wid = blockIdx.x * SWARPS + (threadIdx.x >> 5);
    const int nx = a.nx, ny = a.ny;
    const int strips_x = (nx + SOUT - 1) / SOUT;
    const int sx = wid % strips_x, sy = wid / strips_x;
    const int ra = sy * SH;
    if (ra >= ny) return;  // whole warp
    const int rb = min(ra + SH, ny);
    const int i = sx * SOUT - 2 + lane;
    const bool col_valid = (i >= 0 && i < nx);
    const bool out_lane = (lane >= 2 && lane <= 29 && i < nx);
    const bool ew_lane = (lane >= 2 && lane <= 30);   // lanes whose west edge is fully determined

    R dt = R(0);
    if (MODE == MODE_STAGE1 || MODE == MODE_STAGE2) dt = stage_dt<R>(a);
    const R inv2 = R(1) / (a.m.dyl[0] * a.half_cfl);  // dx_cfl_half_inv(2): NS edges
    double cfl = 0.0;
    long long negfix = 0;

    Cell<R> c0, c1, c2;
    c0.stg = c0.dep = c0.u = c0.v = c0.elv = R(0);
    c1 = c0; c2 = c0;
    Grad<R> g1, g2;
    g1.ds = g1.dd = g1.du = g1.dv = R(0);
    g2 = g1;
    EdgeRes<R> e_s;  // south edge of the row being updated
    zero_edge(e_s);

    Raw<R> nxt = load_raw<R>(a, i, ra - 2);
    for (int r = ra - 2, k = 0; r <= rb + 1; r++, k++) {
        const Raw<R> cur = nxt;
        if (r + 1 <= rb + 1) nxt = load_raw<R>(a, i, r + 1);
        // Inputs that only the update reads (friction coefficient, stage-2
        // U0 and max_stage): start them towards L2 three rows early.
        if ((MODE == MODE_STAGE1 || MODE == MODE_STAGE2) && out_lane && r + 1 >= ra && r + 1 < rb) {
            const int64_t o = (int64_t)(r + 1) * a.P + i;
            if (FRIC != FRIC_NONE) prefetch_l2(a.nsq + o);
            if (MODE == MODE_STAGE2) {
                prefetch_l2(a.stg0 + o);
                prefetch_l2(a.uh0 + o);
                prefetch_l2(a.vh0 + o);
                if (a.max_stage) prefetch_l2(a.max_stage + o);
            }
        }
        c2 = c1;
        c1 = c0;
        c0 = fix_up<R>(cur, col_valid && r >= 0 && r < ny, negfix,
                       (MODE == MODE_STAGE1 || MODE == MODE_STAGE2) && out_lane && r >= ra && r < rb);
        if (k < 2) continue;

        // North-south gradient of row r-1 (DE1_inner_include.f90:746-781).
        g2 = g1;
        {
            const int rg = r - 1;
            if (col_valid && rg > 0 && rg < ny - 1) g1 = limited<R>(c2, c1, c0, a.theta);
            else { g1.ds = R(0); g1.dd = R(0); g1.du = R(0); g1.dv = R(0); }
        }
        if (k < 3) continue;

        // North-south edge between rows r-2 and r-1 (edge index r-1).
        EdgeRes<R> e_n;
        zero_edge(e_n);
        {
            const int e = r - 1;
            if (e >= 1 && e <= ny - 1 && i >= 1 && i <= nx - 1) {
                double cand;
                edge_flux<R, true, EDDY>(c2, g2, c1, g1, a.m.dxb[e], inv2, e_n, cand, a.flux_variant,
                                         EDDY ? a.ev[(int64_t)(e - 1) * a.P + i] : R(0),
                                         EDDY ? a.ev[(int64_t)e * a.P + i] : R(0), EDDY ? a.m.dyl[i] : R(1));
                if (MODE != MODE_STAGE2) cfl = fmax(cfl, cand);   // stage 2 writes no CFL
                if (MODE != MODE_CFL && a.lines && i >= a.n_ext && i <= nx - a.n_ext - 1) {
                    if (e == ny - a.n_ext) a.lines[i] = (double)e_n.f[0];
                    if (e == a.n_ext) a.lines[nx + ny + i] = (double)e_n.f[0];
                }
            }
        }
        if (k < 4) { e_s = e_n; continue; }

        // Row R = r-2: east-west gradient and west edge, then the update.
        const int R_ = r - 2;
        const Cell<R> cl = up1(c2), cr = dn1(c2);
        Grad<R> gew;
        if (col_valid && i > 0 && i < nx - 1) gew = limited<R>(cl, c2, cr, a.theta);
        else { gew.ds = R(0); gew.dd = R(0); gew.du = R(0); gew.dv = R(0); }
        Grad<R> gw;
        gw.ds = up1(gew.ds); gw.dd = up1(gew.dd); gw.du = up1(gew.du); gw.dv = up1(gew.dv);
        EdgeRes<R> e_w;
        zero_edge(e_w);
        if (ew_lane && i >= 1 && i <= nx - 1 && R_ >= 1 && R_ <= ny - 1) {
            const R inv1 = R(1) / (a.m.dxb[R_] * a.half_cfl);  // dx_cfl_half_inv(1): EW edges
            double cand;
            const int64_t oe = (int64_t)R_ * a.P + i;
            edge_flux<R, false, EDDY>(cl, gw, c2, gew, a.m.dyl[i], inv1, e_w, cand, a.flux_variant,
                                      EDDY ? a.ev[oe - 1] : R(0), EDDY ? a.ev[oe] : R(0),
                                      EDDY ? R(0.5) * (a.m.dxb[R_] + a.m.dxb[R_ + 1]) : R(1));
            if (MODE != MODE_STAGE2) cfl = fmax(cfl, cand);
            if (MODE != MODE_CFL && a.lines && R_ >= a.n_ext && R_ <= ny - a.n_ext - 1) {
                if (i == nx - a.n_ext) a.lines[nx + R_] = (double)e_w.f[0];
                if (i == a.n_ext) a.lines[2 * nx + ny + R_] = (double)e_w.f[0];
            }
        }
        if (MODE == MODE_STAGE1 || MODE == MODE_STAGE2 || MODE == MODE_FLUX) {
            EdgeRes<R> e_e;
            e_e.f[0] = dn1(e_w.f[0]); e_e.f[1] = dn1(e_w.f[1]); e_e.f[2] = dn1(e_w.f[2]);
            e_e.es_neg = dn1(e_w.es_neg);
            e_e.es_pos = 0.0;
            if (MODE == MODE_FLUX) {
                if (out_lane) store_cell_flux<R, SPH, COR>(a, i, R_, c2, e_s, e_n, e_w, e_e);
            } else if (out_lane) {
                fv_update<R, MODE, SPH, COR, FRIC>(a, i, R_, c2, e_s, e_n, e_w, e_e, dt, dt / a.m.area[R_]);
            }
        }
        e_s = e_n;
    }

    // Warp reductions: CFL max and the negative-depth count.
    if (MODE != MODE_STAGE2 && (a.write_cfl || MODE == MODE_CFL || MODE == MODE_FLUX)) {
        for (int o = 16; o > 0; o >>= 1) cfl = fmax(cfl, __shfl_down_sync(FULL, cfl, o));
        if (lane == 0 && cfl > 0.0) atomicMax(&a.sc->max_dt_inv_bits, (unsigned long long)__double_as_longlong(cfl));
    }
    if (MODE == MODE_STAGE1 || MODE == MODE_STAGE2) {
        for (int o = 16; o > 0; o >>= 1) negfix += __shfl_down_sync(FULL, negfix, o);
        if (lane == 0 && negfix) atomicAdd((unsigned long long *)&a.sc->negative_depth_fix_counter,
                                           (unsigned long long)negfix);
    }
}

// The same march with the rows it carries kept in shared memory instead of
// registers: per warp a ring of the last three fixed-up rows, the
// north-south gradients of two rows, the south edge of the row being
// updated, and the east-west gradient and west edge of that row (read by
// the neighbouring lanes, in place of shuffles).  Fewer registers per
// thread, so more warps per SM hide the FP64 latency.  Lanes touch other
// lanes' entries only after a __syncwarp.
#ifndef SWALS_SROW_MIN_CTAS
// Measured on the 2048^2 step with warp-wide strips: with 4 CTAs per SM
// stage 2 takes 0.391 ms against the register form's 0.412, the flux pass
// 0.280 against 0.275; with 5 CTAs (spills) 0.412 and 0.299.
#define SWALS_SROW_MIN_CTAS 4
#endif
//
// SW is the width of a strip in threads: 32 (one warp per strip, 28 output
// columns, __syncwarp) or 128 (the CTA's four warps side by side on one
// strip of 124 output columns, __syncthreads): the wider strip spends its
// two-column halos on 4 of 128 threads instead of 4 of 32.
constexpr int SROW_RC = 64;   // segments of up to this many rows keep their row constants in shared memory
// CTAs per SM the register cap of the shared-memory-rows kernel is sized
// for: 5 (96 registers, 20 warps) for stage 2 of CTA-wide strips, whose
// shared memory (43 KB FP64) leaves room for five; 4 for the other passes
// (the flux pass and the fused stage 1 spill at 96 registers), the
// eddy-viscosity forms (spills of 100-200 bytes) and warp-wide strips
// (46 KB a CTA).  Measured on the 2048^2 step: stage 2 0.334 -> 0.313 ms
// with 5, FP32 0.277 -> 0.252; the flux pass at 5 loses 1 %, the fused
// stage 1 at 1280^2 7 %; 3 CTAs lose 20 %.  FP32 state fits every pass of
// the CTA-wide strips in 96 registers: 5 CTAs for all of them (flux pass
// 0.208 -> 0.195 ms).
constexpr int srow_min_ctas(int mode, int sw, bool eddy, int real_bytes)
{
    if (sw == 128 && !eddy && (mode == MODE_STAGE2 || real_bytes == 4)) return 5;
    return SWALS_SROW_MIN_CTAS;
}
template <typename R, int SW>
struct SRows {
    Cell<R> c[3][SW];     // rows r % 3
    Grad<R> g[2][SW];     // north-south gradients, rows r % 2
    EdgeRes<R> es[SW];    // south edge of the row being updated
    Grad<R> gew[2][SW];   // east-west gradients, rows r % 2
    EdgeRes<R> ew[SW];    // west edges of the row being updated
    R rc[2][SROW_RC];     // the segment's row constants: 1 / (dx cfl/2) of its east-west edges, dt / area
};

template <int SW> __device__ __forceinline__ void strip_sync()
{
    if (SW == 32) __syncwarp();
    else __syncthreads();
}

template <typename R, int MODE, bool SPH, bool COR, int FRIC, bool EDDY, int SW>
__global__ void __launch_bounds__(SLANES *SWARPS, srow_min_ctas(MODE, SW, EDDY, (int)sizeof(R))) rk2_srow_kernel(const Rk2Args<R> a, int SH)
{
    static_assert(SW == 32 || SW == SLANES * SWARPS, "a strip is one warp or the whole CTA");
    constexpr int SO = SW - 4;   // output columns of a strip
    extern __shared__ __align__(16) unsigned char srow_smem[];
    const int lane = threadIdx.x % SW;   // the thread's place in its strip
    SRows<R, SW> &sm = reinterpret_cast<SRows<R, SW> *>(srow_smem)[threadIdx.x / SW];
    const int wid = blockIdx.x * (SLANES * SWARPS / SW) + threadIdx.x / SW;
    const int nx = a.nx, ny = a.ny;
    const int strips_x = (nx + SO - 1) / SO;
    const int sx = wid % strips_x, sy = wid / strips_x;
    const int ra = sy * SH;
    if (ra >= ny) return;  // the whole strip
    const int rb = min(ra + SH, ny);
    const int i = sx * SO - 2 + lane;
    const bool col_valid = (i >= 0 && i < nx);
    const bool out_lane = (lane >= 2 && lane <= SW - 3 && i < nx);
    const bool ew_lane = (lane >= 2 && lane <= SW - 2);
    const int lw = max(lane - 1, 0), le = min(lane + 1, SW - 1);   // the shuffles' edge behaviour

    R dt = R(0);
    if (MODE == MODE_STAGE1 || MODE == MODE_STAGE2) dt = stage_dt<R>(a);
    const R inv2 = R(1) / (a.m.dyl[0] * a.half_cfl);
    double cfl = 0.0;
    long long negfix = 0;
    // The row constants of the segment's rows, one division each by the
    // strip's threads instead of one per cell (the same expressions; read
    // after the loop's first barrier).
    const bool rc_sm = (rb - ra) <= SROW_RC;
    if (rc_sm)
        for (int t = lane; t < rb - ra; t += SW) {
            const int rr = ra + t;
            sm.rc[0][t] = R(1) / (a.m.dxb[rr] * a.half_cfl);
            if (MODE == MODE_STAGE1 || MODE == MODE_STAGE2) sm.rc[1][t] = dt / a.m.area[rr];
        }

    Raw<R> nxt = load_raw<R>(a, i, ra - 2);
    // ring slots of rows r, r-1, r-2, rotated each row (the first row's
    // slot is (ra - 2 + 3) % 3 == (ra + 1) % 3)
    int s0 = (ra + 1) % 3, s1 = (s0 + 2) % 3, s2 = (s0 + 1) % 3;
    for (int r = ra - 2, k = 0; r <= rb + 1; r++, k++, s2 = s1, s1 = s0, s0 = (s0 == 2) ? 0 : s0 + 1) {
        strip_sync<SW>();   // every lane is done with the entries this iteration rewrites
        const Raw<R> cur = nxt;
        if (r + 1 <= rb + 1) nxt = load_raw<R>(a, i, r + 1);
        if ((MODE == MODE_STAGE1 || MODE == MODE_STAGE2) && out_lane && r + 1 >= ra && r + 1 < rb) {
            const int64_t o = (int64_t)(r + 1) * a.P + i;
            if (FRIC != FRIC_NONE) prefetch_l2(a.nsq + o);
            if (MODE == MODE_STAGE2) {
                prefetch_l2(a.stg0 + o);
                prefetch_l2(a.uh0 + o);
                prefetch_l2(a.vh0 + o);
                if (a.max_stage) prefetch_l2(a.max_stage + o);
            }
        }
        const Cell<R> c0 = fix_up<R>(cur, col_valid && r >= 0 && r < ny, negfix,
                                     (MODE == MODE_STAGE1 || MODE == MODE_STAGE2) && out_lane && r >= ra && r < rb);
        sm.c[s0][lane] = c0;
        if (k < 2) continue;

        // North-south gradient of row r-1.
        {
            const int rg = r - 1;
            Grad<R> g1;
            if (col_valid && rg > 0 && rg < ny - 1) g1 = limited<R>(sm.c[s2][lane], sm.c[s1][lane], c0, a.theta);
            else { g1.ds = R(0); g1.dd = R(0); g1.du = R(0); g1.dv = R(0); }
            sm.g[(r + 1) & 1][lane] = g1;
        }
        if (k < 3) continue;

        // East-west gradient of row r-1 (its neighbours' fixed-up values were
        // written before this row's barrier), for the west edges of row r-1
        // in the next row's pass.
        if (r <= rb) {
            Grad<R> gew;
            if (col_valid && i > 0 && i < nx - 1) gew = limited<R>(sm.c[s1][lw], sm.c[s1][lane], sm.c[s1][le], a.theta);
            else { gew.ds = R(0); gew.dd = R(0); gew.du = R(0); gew.dv = R(0); }
            sm.gew[(r + 1) & 1][lane] = gew;
        }

        // North-south edge between rows r-2 and r-1.
        EdgeRes<R> e_n;
        zero_edge(e_n);
        {
            const int e = r - 1;
            if (e >= 1 && e <= ny - 1 && i >= 1 && i <= nx - 1) {
                double cand;
                edge_flux<R, true, EDDY>(sm.c[s2][lane], sm.g[r & 1][lane], sm.c[s1][lane], sm.g[(r + 1) & 1][lane],
                                         a.m.dxb[e], inv2, e_n, cand, a.flux_variant,
                                         EDDY ? a.ev[(int64_t)(e - 1) * a.P + i] : R(0),
                                         EDDY ? a.ev[(int64_t)e * a.P + i] : R(0), EDDY ? a.m.dyl[i] : R(1));
                if (MODE != MODE_STAGE2) cfl = fmax(cfl, cand);   // stage 2 writes no CFL
                // the boundary-flux lines (rows n_ext and ny - n_ext): tested
                // on the row first, the same for the whole strip
                if (MODE != MODE_CFL && (e == ny - a.n_ext || e == a.n_ext) && a.lines && i >= a.n_ext &&
                    i <= nx - a.n_ext - 1) {
                    if (e == ny - a.n_ext) a.lines[i] = (double)e_n.f[0];
                    if (e == a.n_ext) a.lines[nx + ny + i] = (double)e_n.f[0];
                }
            }
        }
        if (k < 4) { sm.es[lane] = e_n; continue; }

        // Row R = r-2: its west edges (between the same barriers as the
        // north-south work of row r-1, which they do not depend on), then,
        // after the barrier, the update.
        const int R_ = r - 2;
        EdgeRes<R> e_w;
        zero_edge(e_w);
        if (ew_lane && i >= 1 && i <= nx - 1 && R_ >= 1 && R_ <= ny - 1) {
            const R inv1 = rc_sm ? sm.rc[0][R_ - ra] : R(1) / (a.m.dxb[R_] * a.half_cfl);
            double cand;
            const int64_t oe = (int64_t)R_ * a.P + i;
            const Grad<R> *gw = sm.gew[r & 1];
            edge_flux<R, false, EDDY>(sm.c[s2][lw], gw[lw], sm.c[s2][lane], gw[lane], a.m.dyl[i], inv1, e_w,
                                      cand, a.flux_variant, EDDY ? a.ev[oe - 1] : R(0), EDDY ? a.ev[oe] : R(0),
                                      EDDY ? R(0.5) * (a.m.dxb[R_] + a.m.dxb[R_ + 1]) : R(1));
            if (MODE != MODE_STAGE2) cfl = fmax(cfl, cand);
            if (MODE != MODE_CFL && (i == nx - a.n_ext || i == a.n_ext) && a.lines && R_ >= a.n_ext &&
                R_ <= ny - a.n_ext - 1) {
                if (i == nx - a.n_ext) a.lines[nx + R_] = (double)e_w.f[0];
                if (i == a.n_ext) a.lines[2 * nx + ny + R_] = (double)e_w.f[0];
            }
        }
        if (MODE == MODE_STAGE1 || MODE == MODE_STAGE2 || MODE == MODE_FLUX) {
            sm.ew[lane] = e_w;
            strip_sync<SW>();
            EdgeRes<R> e_e;
            const EdgeRes<R> &en = sm.ew[le];
            e_e.f[0] = en.f[0]; e_e.f[1] = en.f[1]; e_e.f[2] = en.f[2];
            e_e.es_neg = en.es_neg;
            e_e.es_pos = 0.0;
            if (MODE == MODE_FLUX) {
                if (out_lane) store_cell_flux<R, SPH, COR>(a, i, R_, sm.c[s2][lane], sm.es[lane], e_n, e_w, e_e);
            } else if (out_lane) {
                fv_update<R, MODE, SPH, COR, FRIC>(a, i, R_, sm.c[s2][lane], sm.es[lane], e_n, e_w, e_e, dt,
                                                   rc_sm ? sm.rc[1][R_ - ra] : dt / a.m.area[R_]);
            }
        }
        sm.es[lane] = e_n;
    }

    if (MODE != MODE_STAGE2 && (a.write_cfl || MODE == MODE_CFL || MODE == MODE_FLUX)) {
        for (int o = 16; o > 0; o >>= 1) cfl = fmax(cfl, __shfl_down_sync(FULL, cfl, o));
        if ((threadIdx.x & 31) == 0 && cfl > 0.0)
            atomicMax(&a.sc->max_dt_inv_bits, (unsigned long long)__double_as_longlong(cfl));
    }
    if (MODE == MODE_STAGE1 || MODE == MODE_STAGE2) {
        for (int o = 16; o > 0; o >>= 1) negfix += __shfl_down_sync(FULL, negfix, o);
        if ((threadIdx.x & 31) == 0 && negfix) atomicAdd((unsigned long long *)&a.sc->negative_depth_fix_counter,
                                           (unsigned long long)negfix);
    }
}

// The shared-memory-rows form for the FP64 update stages and the register
// form for the flux pass and for FP32 state (the faster of the two for each:
// FP32 stage 2 0.311 ms in registers, 0.330 in shared-memory rows), unless
// SWALS_FV_STREAM=stream or =srow picks one form for all.
// 0: register form; 1: shared-memory rows, one warp per strip; 2: shared-
// memory rows, the CTA's four warps on one strip.  Grids of 1.5 M cells and
// more take the CTA-wide strips (2048^2 rk2 step: FP64 flux pass 0.268 ms
// against 0.283 for the register form, stage 2 0.362 against 0.390 for
// one-warp strips, the step 0.732 against 0.777 ms; 1536^2 0.460 against
// 0.465; FP32 2048^2 0.624 against 0.640).  Smaller grids, L2-resident
// and short of CTAs, keep one-warp strips (1024^2: 0.261 against 0.266 ms
// at a fixed dt; the nested configuration's 0.9-1.1 M-cell rk2 domains
// 5.23 against 5.56 ms per md step): shared-memory rows for the FP64
// update stages, registers for the rest.
int fv_stream_form(int mode, int real_bytes, int64_t cells)
{
    // read at every launch, so that a process can switch forms between steps
    const char *e = getenv("SWALS_FV_STREAM");
    if (e && strcmp(e, "stream") == 0) return 0;
    if (e && strcmp(e, "srow") == 0) return 1;
    if (e && strcmp(e, "crow") == 0) return 2;
    if (cells >= 1500000) return 2;
    return (real_bytes == 8 && (mode == MODE_STAGE1 || mode == MODE_STAGE2)) ? 1 : 0;
}

// CTAs of a launch of the given form with sh rows per strip segment.
int64_t fv_ctas(int form, int nx, int ny, int sh)
{
    const int64_t segs = (ny + sh - 1) / sh;
    if (form == 2) return (int64_t)((nx + SLANES * SWARPS - 5) / (SLANES * SWARPS - 4)) * segs;
    const int64_t warps = (int64_t)((nx + SOUT - 1) / SOUT) * segs;
    return (warps + SWARPS - 1) / SWARPS;
}

// Rows per strip segment for a grid: 12 (the best on large grids, where
// every choice fills its waves about as well) unless another of 8, 16 and
// 24 rows is at least 2 % cheaper by the estimate
//   (rows + 4) / rows x ceil(waves) / waves,   waves = CTAs / resident CTAs,
// the rows marched per output row times the share of the last wave left
// idle.  Measured (rk2 beach, ms a step, rows 8 / 12 / 16 / 24): 768^2
// 0.180 / 0.160 / 0.190 / 0.240 (estimate picks 12); 1024^2 0.234 / 0.274 /
// 0.229 / 0.282 (picks 16); 1536^2 0.467 / 0.458 / 0.498 / 0.524 and
// 2048^2 0.744 / 0.731 / 0.736 / 0.772 (picks 12).  SWALS_FV_ROWS sets it.
int fv_rows(int form, int ctas_per_sm, int nx, int ny)
{
    const char *e = getenv("SWALS_FV_ROWS");
    if (e && atoi(e) > 0) return atoi(e);
    static int sms = 0;
    if (sms == 0) {
        int dev = 0, n = 148;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        sms = n;
    }
    const int slots = ctas_per_sm * sms;   // resident CTAs
    const int cand[] = {12, 16, 8, 24};
    int best = 0;
    double best_cost = 0.0;
    for (int sh : cand) {
        const double w = (double)fv_ctas(form, nx, ny, sh) / slots;
        const double cost = (sh + 4.0) / sh * std::ceil(w) / w;
        if (best == 0 || cost < 0.98 * best_cost) {
            best = sh;
            best_cost = cost;
        }
    }
    return best;
}

}  // namespace

template <typename R, int MODE, bool SPH, bool COR, int FRIC>
cudaError_t launch_stage_stream(const Rk2Args<R> &a, cudaStream_t s)
{
    // Stage 2 takes the first stage's dt and accumulates no CFL maximum: its
    // kernels leave the edges' wave-speed candidates out.
    if (MODE == MODE_STAGE2 && a.write_cfl) return cudaErrorInvalidValue;
    const int form = fv_stream_form(MODE, (int)sizeof(R), (int64_t)a.nx * a.ny);
    // (the wave estimate counts 4 resident CTAs per SM for every form: with
    // stage 2's 5 it would pick 24 rows at 2048^2, 2 % slower than 12)
    const int SH = fv_rows(form, 4, a.nx, a.ny);
    const int blocks = (int)fv_ctas(form, a.nx, a.ny, SH);
    if (form == 1 || form == 2) {
        constexpr int SW = SLANES * SWARPS;
        const size_t smem = form == 1 ? sizeof(SRows<R, 32>) * SWARPS : sizeof(SRows<R, SW>);   // 41 KB (FP64)
        auto go = [&](auto kernel) -> cudaError_t {
            kernel<<<blocks, SLANES * SWARPS, smem, s>>>(a, SH);
            return cudaGetLastError();
        };
        if (form == 1) {
            if constexpr (MODE != MODE_CFL) {
                if (a.flux_variant & FLUX_EDDY) return go(rk2_srow_kernel<R, MODE, SPH, COR, FRIC, true, 32>);
            }
            return go(rk2_srow_kernel<R, MODE, SPH, COR, FRIC, false, 32>);
        }
        if constexpr (MODE != MODE_CFL) {
            if (a.flux_variant & FLUX_EDDY) return go(rk2_srow_kernel<R, MODE, SPH, COR, FRIC, true, SW>);
        }
        return go(rk2_srow_kernel<R, MODE, SPH, COR, FRIC, false, SW>);
    }
    if constexpr (MODE != MODE_CFL) {
        if (a.flux_variant & FLUX_EDDY) {
            rk2_stream_kernel<R, MODE, SPH, COR, FRIC, true><<<blocks, SLANES * SWARPS, 0, s>>>(a, SH);
            return cudaGetLastError();
        }
    }
    rk2_stream_kernel<R, MODE, SPH, COR, FRIC, false><<<blocks, SLANES * SWARPS, 0, s>>>(a, SH);
    return cudaGetLastError();
}

#define SWALS_INST(R, MODE, SPH, COR, FRIC) \
    template cudaError_t launch_stage_stream<R, MODE, SPH, COR, FRIC>(const fv::Rk2Args<R> &, cudaStream_t);
#define SWALS_INST_F(R, MODE, SPH, COR) \
    SWALS_INST(R, MODE, SPH, COR, fv::FRIC_MANNING) SWALS_INST(R, MODE, SPH, COR, fv::FRIC_CHEZY) \
    SWALS_INST(R, MODE, SPH, COR, fv::FRIC_NONE)
#define SWALS_INST_M(R, SPH, COR) \
    SWALS_INST_F(R, fv::MODE_CFL, SPH, COR) SWALS_INST_F(R, fv::MODE_STAGE1, SPH, COR) \
    SWALS_INST_F(R, fv::MODE_FLUX, SPH, COR) \
    SWALS_INST_F(R, fv::MODE_STAGE2, SPH, COR)
SWALS_INST_M(double, false, false)
SWALS_INST_M(double, true, false)
SWALS_INST_M(double, true, true)
SWALS_INST_M(float, false, false)
SWALS_INST_M(float, true, false)
SWALS_INST_M(float, true, true)

}  // namespace swals
