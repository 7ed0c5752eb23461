// linear.cu -- truly-linear / not-truly-linear leapfrog step on sm_100a.
//
// Restates domain_mod_linear_solver_include.f90:58-571 (one_truely_linear_
// leapfrog_step / one_not_truely_linear_leapfrog_step,
// domain_mod_timestepping_alternatives_include.f90:339-387).
//
// The reference makes two sweeps over the grid (stage, then UH/VH) and uses
// hand-made OpenMP chunking with thread-boundary snapshots so the Coriolis
// averages see pre-update UH/VH without copying.  Here one fused pass reads
// the old state once and writes the new state to a second buffer:
//   - each CTA stages a tile of old UH/VH/ELV (plus a one-cell halo) in shared
//     memory, recomputes the new stage on the tile plus its east/north halo,
//     then applies the momentum update and writes STG/UH/VH and max_stage;
//   - the ping-pong buffers make every old value available to the Coriolis
//     averages, so no snapshots are needed.
// Algorithmic traffic: read STG,UH,VH,ELV + write STG,UH,VH (7 planes), plus
// max_stage read+write when recorded.  Halo re-reads hit L2.
// A one-block edge kernel runs first: it applies the device boundary
// function to the stage/elevation ring at time+dt/2 (boundary_mod.f90:78-163
// staggered branch), forms the boundary flux sums (:126-205) and advances
// domain%time.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "swals_kernels.h"

namespace swals {
namespace {

constexpr int LBX = 32;   // tile columns (one warp wide)

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

template <typename R>
struct LinArgs {
    StepPlanes<R> p;        // planes of instance 0
    Metrics<R> m;
    int xl, xu, yl, yu;
    int bc_stage;           // the ring stage is in stg_o before the step kernel runs
    int bc_fn_ring;         // the edge kernel writes it from the boundary function
    int bext[4];
    R dt;
    R msl;
    int lin_fric;
    R lin_fric_mult;
    R lin_fric_dt;          // dt * linear_friction_coeff
    // leapfrog_linear_plus_nonlinear_friction: friction_work at the UH points,
    // then (fw_plane elements on) the VH points; null for the other solvers.
    const R *fw;
    int64_t fw_plane;
    int nbatch;             // instances sharing ELV and the metrics (1 for a plain domain)
    int64_t inst_stride;    // elements between consecutive instances' planes
    int64_t max_stride;     // elements between consecutive instances' max_stage planes
    // Optional gauge sampling fused into the streaming kernel: rec[g] = new
    // stage at site g (0-based i, j pairs).
    const int *sites;
    int n_sites;
    double *rec;
    // Bulk-copy rows (linear_wide_kernel<..., BULK>): SM clock cycles a ring
    // slot may take to arrive before the warp gives up, and bytes added to
    // every slot's expected count (0; a positive value makes no slot ever
    // complete, which exercises the give-up path).
    long long wait_cycles;
    unsigned bulk_extra_tx;
    // The step's point gauges recorded by the tile kernel (plain steps whose
    // last kernel it is): g_n sites, records[rec][g][STG, UH, VH].
    const int *g_sites;
    int g_n;
    double *g_records;
    int g_capacity;
    DevScalars *g_sc;
};

__device__ __forceinline__ bool on_bc_ring(int i, int r, int nx, int ny, const int bext[4])
{
    return (i == 0 && bext[3]) || (i == nx - 1 && bext[1]) || (r == 0 && bext[2]) || (r == ny - 1 && bext[0]);
}

// leapfrog_linear_plus_nonlinear_friction (linear_solver_include.f90:
// 458-505): the semi-implicit friction multipliers of cell o from its old
// momenta uh0, vh0 and the old two-point averages; linear friction is folded
// in.  Applied after the pressure-gradient (and Coriolis) update, by
// linear_nlfric_kernel after the step kernel (which then skips the linear
// friction), so the plain solvers' step kernels carry none of it.
template <typename R>
__device__ __forceinline__ void nl_friction(const LinArgs<R> &a, int64_t o, R uh0, R vh0, R vh_iph_jmh, R vh_iph_jph,
                                            R uh_i_j, R uh_i_jp1, R &uh_new, R &vh_new)
{
    const R half = K<R>::half(), one = K<R>::one();
    const R tv = half * (vh_iph_jmh + vh_iph_jph);
    const R tu = half * (uh_i_j + uh_i_jp1);
    const R fm_uh = one / ((one + a.lin_fric_dt) + a.dt * a.fw[o] * R(sqrt(uh0 * uh0 + tv * tv)));
    const R fm_vh = one / ((one + a.lin_fric_dt) + a.dt * a.fw[a.fw_plane + o] * R(sqrt(vh0 * vh0 + tu * tu)));
    uh_new = fm_uh * uh_new;
    vh_new = fm_vh * vh_new;
}

// One CTA: a 32 x BY tile (TYT thread rows, BY/TYT cells per thread) for IB
// instances in turn.  ELV (and, for the truly linear solver, the face depths
// that depend only on ELV) are staged once and reused by every instance.
template <typename R, bool CORIOLIS, bool TRUELY_LINEAR, int BY, int TYT, int IB>
__global__ void __launch_bounds__(LBX *TYT) linear_step_kernel(const LinArgs<R> a)
{
    constexpr int CPT = BY / TYT;
    constexpr int NT = LBX * TYT;
    __shared__ R s_uh[BY + 1][LBX + 2];  // old UH: rows r0..r0+BY, cols i0-1..i0+LBX (clamped)
    __shared__ R s_vh[BY + 2][LBX + 1];  // old VH: rows r0-1..r0+BY, cols i0..i0+LBX (clamped)
    __shared__ R s_sn[BY + 1][LBX + 1];  // new STG: rows r0..r0+BY, cols i0..i0+LBX
    __shared__ R s_el[BY + 1][LBX + 1];  // ELV on the same window as s_sn

    const int nx = a.p.nx, ny = a.p.ny;
    const int64_t P = a.p.pitch;
    const int i0 = blockIdx.x * LBX, r0 = blockIdx.y * BY;
    const int tid = threadIdx.y * LBX + threadIdx.x;
    const R g = K<R>::gravity();
    const R half = K<R>::half();
    const R one = K<R>::one();
    const R zero = K<R>::zero();
    const R mad = K<R>::min_depth();

    for (int q = tid; q < (BY + 1) * (LBX + 1); q += NT) {
        int rr = q / (LBX + 1), cc = q - rr * (LBX + 1);
        int r = clampi(r0 + rr, 0, ny - 1), i = clampi(i0 + cc, 0, nx - 1);
        s_el[rr][cc] = a.p.elv[r * P + i];
    }
    __syncthreads();

    // Truly linear face depths h_{i+1/2}, h_{j+1/2} depend on ELV only (:353-370).
    R h_iph_c[CPT], h_jph_c[CPT];
#pragma unroll
    for (int k = 0; k < CPT; k++) {
        const int rr = threadIdx.y + k * TYT, cc = threadIdx.x;
        h_iph_c[k] = zero;
        h_jph_c[k] = zero;
        if (TRUELY_LINEAR) {
            const R e0 = s_el[rr][cc], e_e = s_el[rr][cc + 1], e_n = s_el[rr + 1][cc];
            bool wi = (e0 < -mad + a.msl) && (e_e < -mad + a.msl);
            h_iph_c[k] = wi ? (a.msl - half * (e_e + e0)) : zero;
            bool wj = (e_n < -mad + a.msl) && (e0 < -mad + a.msl);
            h_jph_c[k] = wj ? (a.msl - half * (e_n + e0)) : zero;
        }
    }

    for (int ib = 0; ib < IB; ib++) {
        const int b = blockIdx.z * IB + ib;
        if (b >= a.nbatch) break;  // uniform across the CTA
        const int64_t io = (int64_t)b * a.inst_stride;
        const R *stg = a.p.stg + io, *uhp = a.p.uh + io, *vhp = a.p.vh + io;
        R *stg_o = a.p.stg_o + io, *uh_o = a.p.uh_o + io, *vh_o = a.p.vh_o + io;
        R *max_stage = a.p.max_stage ? a.p.max_stage + (int64_t)b * a.max_stride : nullptr;
        if (ib > 0) __syncthreads();  // the previous instance is done with the tiles

        for (int q = tid; q < (BY + 1) * (LBX + 2); q += NT) {
            int rr = q / (LBX + 2), cc = q - rr * (LBX + 2);
            int r = clampi(r0 + rr, 0, ny - 1), i = clampi(i0 - 1 + cc, 0, nx - 1);
            s_uh[rr][cc] = uhp[r * P + i];
        }
        for (int q = tid; q < (BY + 2) * (LBX + 1); q += NT) {
            int rr = q / (LBX + 1), cc = q - rr * (LBX + 1);
            int r = clampi(r0 - 1 + rr, 0, ny - 1), i = clampi(i0 + cc, 0, nx - 1);
            s_vh[rr][cc] = vhp[r * P + i];
        }
        __syncthreads();

        // New stage on the tile plus east/north halo (:92-115).
        for (int q = tid; q < (BY + 1) * (LBX + 1); q += NT) {
            int rr = q / (LBX + 1), cc = q - rr * (LBX + 1);
            int r = r0 + rr, i = i0 + cc;
            R sn = R(0);
            if (r < ny && i < nx) {
                R s_old = stg[r * P + i];
                bool interior = (i >= a.xl + 1) && (i <= a.xu - 1) && (r >= a.yl + 1) && (r <= a.yu - 1);
                if (interior) {
                    R inv_cell_area_dt = a.dt / a.m.area[r];
                    R t1 = (s_uh[rr][cc + 1] - s_uh[rr][cc]) * a.m.dyl[i];
                    R t2 = s_vh[rr + 1][cc] * a.m.dxb[r + 1] - s_vh[rr][cc] * a.m.dxb[r];
                    sn = s_old - inv_cell_area_dt * (t1 + t2);
                } else if (a.bc_stage && on_bc_ring(i, r, nx, ny, a.bext)) {
                    sn = stg_o[r * P + i];  // set by the edge kernel at time+dt/2
                } else {
                    sn = s_old;
                }
            }
            s_sn[rr][cc] = sn;
        }
        __syncthreads();

#pragma unroll
        for (int k = 0; k < CPT; k++) {
            const int rr = threadIdx.y + k * TYT, cc = threadIdx.x;
            const int r = r0 + rr, i = i0 + cc;
            if (r >= ny || i >= nx) continue;
            const int64_t o = r * P + i;
            const R sn = s_sn[rr][cc];
            stg_o[o] = sn;
            if (max_stage && i >= a.xl && i <= a.xu && r >= a.yl && r <= a.yu) {
                R mx = max_stage[o];
                max_stage[o] = (sn > mx) ? sn : mx;
            }
            R uh = s_uh[rr][cc + 1];
            R vh = s_vh[rr + 1][cc];
            if (i >= a.xl && i <= a.xu - 1 && r >= a.yl && r <= a.yu - 1) {
                const R inv_cell_area_dt_g = g * a.dt / a.m.area[r];
                const R inv_cell_area_dt_vh_g = g * a.dt / (half * (a.m.area[r] + a.m.area[r + 1]));
                const R e0 = s_el[rr][cc], e_e = s_el[rr][cc + 1], e_n = s_el[rr + 1][cc];
                const R s_e = s_sn[rr][cc + 1], s_n = s_sn[rr + 1][cc];
                R h_iph, h_jph, wet_iph, wet_jph;
                if (TRUELY_LINEAR) {
                    h_iph = h_iph_c[k];
                    h_jph = h_jph_c[k];
                    wet_iph = one;
                    wet_jph = one;
                } else {
                    bool wi = (sn - e0 > mad) && (s_e - e_e > mad);
                    h_iph = wi ? (half * ((s_e + sn) - (e_e + e0))) : zero;
                    bool wj = (s_n - e_n > mad) && (sn - e0 > mad);
                    h_jph = wj ? (half * ((s_n + sn) - (e_n + e0))) : zero;
                    wet_iph = (h_iph > zero) ? one : zero;
                    wet_jph = (h_jph > zero) ? one : zero;
                }
                const R dw_j = s_n - sn;
                R uh_n = uh * wet_iph - inv_cell_area_dt_g * h_iph * (s_e - sn) * a.m.dyl[i + 1];
                R vh_n = vh * wet_jph - inv_cell_area_dt_vh_g * h_jph * dw_j * a.m.dxb[r + 1];
                if (CORIOLIS) {
                    // Pre-update 2-point averages (:409-428); rows/cols clamp like
                    // the reference's j=1 and max(xL-1,1) special cases.
                    const R vh_iph_jmh = half * (s_vh[rr][cc] + s_vh[rr][cc + 1]);
                    const R vh_iph_jph = half * (s_vh[rr + 1][cc] + s_vh[rr + 1][cc + 1]);
                    const R uh_i_j = half * (s_uh[rr][cc + 1] + s_uh[rr][cc]);
                    const R uh_i_jp1 = half * (s_uh[rr + 1][cc + 1] + s_uh[rr + 1][cc]);
                    const R dt_half_coriolis = a.dt * a.m.cor[r] * half * ((h_iph > zero) ? one : zero);
                    const R dt_half_coriolis_jph = a.dt * a.m.cor_be[r + 1] * half * ((h_jph > zero) ? one : zero);
                    uh_n = uh_n + dt_half_coriolis * (vh_iph_jmh + vh_iph_jph);
                    vh_n = vh_n - dt_half_coriolis_jph * (uh_i_j + uh_i_jp1);
                }
                if (a.lin_fric) {
                    uh_n = a.lin_fric_mult * uh_n;
                    vh_n = a.lin_fric_mult * vh_n;
                }
                uh = uh_n;
                vh = vh_n;
            }
            uh_o[o] = uh;
            vh_o[o] = vh;
        }
    }

    if (a.g_n > 0) {
        // The step's gauges inside this tile (a plain step: one instance).
        // This CTA wrote the tile's new values; they are visible to all its
        // threads after the barrier.  Every CTA reads the record index before
        // it counts itself done; the last one advances it.
        const int rec = a.g_sc->gauge_records;
        __syncthreads();
        if (rec < a.g_capacity)
            for (int q = tid; q < a.g_n; q += NT) {
                const int gi = a.g_sites[2 * q], gr = a.g_sites[2 * q + 1];
                if (gi >= i0 && gi < i0 + LBX && gr >= r0 && gr < r0 + BY) {
                    const int64_t o = (int64_t)gr * P + gi;
                    double *dst = a.g_records + ((int64_t)rec * a.g_n + q) * 3;
                    dst[0] = (double)a.p.stg_o[o];
                    dst[1] = (double)a.p.uh_o[o];
                    dst[2] = (double)a.p.vh_o[o];
                }
            }
        if (tid == 0) {
            __threadfence();
            const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
            if (atomicAdd(reinterpret_cast<unsigned *>(&a.g_sc->blocks_done), 1u) == nblk - 1) {
                a.g_sc->gauge_records = rec + 1;
                a.g_sc->blocks_done = 0;
            }
        }
    }
}

// Streaming form of the same step, for HBM-bound grids: a warp owns a strip
// of 30 columns (lanes 1..30; lanes 0 and 31 carry the west and east
// neighbour columns, clamped at the domain edge like the tile's halo) and
// marches down SH rows.  Per row it loads STG, UH, VH and ELV once (the next
// row's loads are in flight while the current row is computed), forms the
// new stage of the next row and the momentum of the current row from
// registers and shuffles, and writes the row: no shared memory, no block
// barriers, and the three row-constant divisions are done once per row per
// warp.  Every value is the same expression, in the same order, as in
// linear_step_kernel.
constexpr int SOUT = 30;
#ifndef LIN_MINB
#define LIN_MINB 8
#endif

template <typename R, bool CORIOLIS, bool TRUELY_LINEAR, bool GAUGES = false>
__global__ void __launch_bounds__(128, LIN_MINB) linear_stream_kernel(const LinArgs<R> a, int SH, int nstrips, int total)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.x;  // instance: consecutive CTAs share ELV rows in L2
    if (b >= a.nbatch) return;
    const int nx = a.p.nx, ny = a.p.ny;
    const int64_t P = a.p.pitch;
    const int64_t io = (int64_t)b * a.inst_stride;
    const R *stg = a.p.stg + io, *uhp = a.p.uh + io, *vhp = a.p.vh + io;
    R *stg_o = a.p.stg_o + io, *uh_o = a.p.uh_o + io, *vh_o = a.p.vh_o + io;
    R *max_stage = a.p.max_stage ? a.p.max_stage + (int64_t)b * a.max_stride : nullptr;
    const R *elv = a.p.elv;
    const R g = K<R>::gravity();
    const R half = K<R>::half();
    const R one = K<R>::one();
    const R zero = K<R>::zero();
    const R mad = K<R>::min_depth();

    for (int w = blockIdx.y * 4 + (threadIdx.x >> 5); w < total; w += gridDim.y * 4) {
        const int sx = w % nstrips, sy = w / nstrips;
        const int ra = sy * SH;
        const int rb = min(ra + SH, ny);
        const int i = sx * SOUT - 1 + lane;
        const int ic = clampi(i, 0, nx - 1);
        const bool in_x = (i >= 0 && i < nx);
        const bool out = (lane >= 1 && lane <= SOUT && i < nx);
        const R dyl_i = a.m.dyl[ic];
        const R dyl_ip1 = a.m.dyl[min(ic + 1, nx)];
        const unsigned long long gmask =
            GAUGES ? gauges_in(a.sites, a.n_sites, sx * SOUT, sx * SOUT + SOUT - 1, ra, rb - 1) : 0ull;

        // New stage of cell (i, r) from its row's loads (domain_mod_linear_solver_include.f90:92-115).
        auto stage_new = [&](int r, R s_old, R uh_r, R uh_w, R vh_r, R vh_s) -> R {
            R sn = R(0);
            if (r < ny && in_x) {
                const bool interior = (i >= a.xl + 1) && (i <= a.xu - 1) && (r >= a.yl + 1) && (r <= a.yu - 1);
                if (interior) {
                    const R inv_cell_area_dt = a.dt / a.m.area[r];
                    const R t1 = (uh_r - uh_w) * dyl_i;
                    const R t2 = vh_r * a.m.dxb[r + 1] - vh_s * a.m.dxb[r];
                    sn = s_old - inv_cell_area_dt * (t1 + t2);
                } else if (a.bc_stage && on_bc_ring(i, r, nx, ny, a.bext)) {
                    sn = stg_o[(int64_t)r * P + i];
                } else {
                    sn = s_old;
                }
            }
            return sn;
        };
        auto ld = [&](const R *p, int r) -> R { return p[(int64_t)clampi(r, 0, ny - 1) * P + ic]; };

        // Prologue: VH of row ra-1, row ra, then row ra+1 in flight.
        R vh_jm1 = ld(vhp, ra - 1);
        R uh_j = ld(uhp, ra), vh_j = ld(vhp, ra), e_j = ld(elv, ra);
        R st_j = (ra < ny && in_x) ? stg[(int64_t)ra * P + i] : R(0);
        R sn_j;
        {
            const R uh_w = __shfl_up_sync(FULL, uh_j, 1);
            sn_j = stage_new(ra, st_j, uh_j, uh_w, vh_j, vh_jm1);
        }
        R uh_n = ld(uhp, ra + 1), vh_n = ld(vhp, ra + 1), e_n = ld(elv, ra + 1);
        R st_n = (ra + 1 < ny && in_x) ? stg[(int64_t)(ra + 1) * P + i] : R(0);

        for (int j = ra; j < rb; j++) {
            // Loads of row j+2 go out first.
            const R uh_f = ld(uhp, j + 2), vh_f = ld(vhp, j + 2), e_f = ld(elv, j + 2);
            const R st_f = (j + 2 < ny && in_x) ? stg[(int64_t)(j + 2) * P + i] : R(0);
            R mx = R(0);
            const bool in_ms = max_stage && out && i >= a.xl && i <= a.xu && j >= a.yl && j <= a.yu;
            if (in_ms) mx = max_stage[(int64_t)j * P + i];

            // New stage of row j+1.
            const R uh_nw = __shfl_up_sync(FULL, uh_n, 1);
            const R sn_n = stage_new(j + 1, st_n, uh_n, uh_nw, vh_n, vh_j);

            // Momentum of row j (:225-567).
            const R s_e = __shfl_down_sync(FULL, sn_j, 1);
            const R e_e = __shfl_down_sync(FULL, e_j, 1);
            const R uh_w = __shfl_up_sync(FULL, uh_j, 1);
            const R vh_e = __shfl_down_sync(FULL, vh_j, 1);
            const R vh_se = __shfl_down_sync(FULL, vh_jm1, 1);
            if (out) {
                const int64_t o = (int64_t)j * P + i;
                stg_o[o] = sn_j;
                if (GAUGES && gmask) {
                    if (a.n_sites > 64) {
                        for (int q = 0; q < a.n_sites; q++)
                            if (a.sites[2 * q] == i && a.sites[2 * q + 1] == j) a.rec[q] = (double)sn_j;
                    } else {
                        for (unsigned long long m = gmask; m; m &= m - 1) {
                            const int q = __ffsll((long long)m) - 1;
                            if (a.sites[2 * q] == i && a.sites[2 * q + 1] == j) a.rec[q] = (double)sn_j;
                        }
                    }
                }
                if (in_ms) max_stage[o] = (sn_j > mx) ? sn_j : mx;
                R uh = uh_j, vh = vh_j;
                if (i >= a.xl && i <= a.xu - 1 && j >= a.yl && j <= a.yu - 1) {
                    const R inv_cell_area_dt_g = g * a.dt / a.m.area[j];
                    const R inv_cell_area_dt_vh_g = g * a.dt / (half * (a.m.area[j] + a.m.area[j + 1]));
                    const R e0 = e_j;
                    const R sn = sn_j, s_n = sn_n;
                    R h_iph, h_jph, wet_iph, wet_jph;
                    if (TRUELY_LINEAR) {
                        const bool wi = (e0 < -mad + a.msl) && (e_e < -mad + a.msl);
                        h_iph = wi ? (a.msl - half * (e_e + e0)) : zero;
                        const bool wj = (e_n < -mad + a.msl) && (e0 < -mad + a.msl);
                        h_jph = wj ? (a.msl - half * (e_n + e0)) : zero;
                        wet_iph = one;
                        wet_jph = one;
                    } else {
                        const bool wi = (sn - e0 > mad) && (s_e - e_e > mad);
                        h_iph = wi ? (half * ((s_e + sn) - (e_e + e0))) : zero;
                        const bool wj = (s_n - e_n > mad) && (sn - e0 > mad);
                        h_jph = wj ? (half * ((s_n + sn) - (e_n + e0))) : zero;
                        wet_iph = (h_iph > zero) ? one : zero;
                        wet_jph = (h_jph > zero) ? one : zero;
                    }
                    const R dw_j = s_n - sn;
                    R uh_new = uh * wet_iph - inv_cell_area_dt_g * h_iph * (s_e - sn) * dyl_ip1;
                    R vh_new = vh * wet_jph - inv_cell_area_dt_vh_g * h_jph * dw_j * a.m.dxb[j + 1];
                    if (CORIOLIS) {
                        const R vh_iph_jmh = half * (vh_jm1 + vh_se);
                        const R vh_iph_jph = half * (vh_j + vh_e);
                        const R uh_i_j = half * (uh_j + uh_w);
                        const R uh_i_jp1 = half * (uh_n + uh_nw);
                        const R dt_half_coriolis = a.dt * a.m.cor[j] * half * ((h_iph > zero) ? one : zero);
                        const R dt_half_coriolis_jph = a.dt * a.m.cor_be[j + 1] * half * ((h_jph > zero) ? one : zero);
                        uh_new = uh_new + dt_half_coriolis * (vh_iph_jmh + vh_iph_jph);
                        vh_new = vh_new - dt_half_coriolis_jph * (uh_i_j + uh_i_jp1);
                    }
                    if (a.lin_fric) {
                        uh_new = a.lin_fric_mult * uh_new;
                        vh_new = a.lin_fric_mult * vh_new;
                    }
                    uh = uh_new;
                    vh = vh_new;
                }
                uh_o[o] = uh;
                vh_o[o] = vh;
            }
            vh_jm1 = vh_j;
            uh_j = uh_n; vh_j = vh_n; e_j = e_n; sn_j = sn_n;
            uh_n = uh_f; vh_n = vh_f; e_n = e_f; st_n = st_f;
        }
    }
}

// The streaming step with its row loads staged through shared memory by
// asynchronous copies (cp.async), so that AD rows per warp are in flight
// without holding them in registers: each lane copies its own element of
// UH, VH, STG, ELV and max_stage for a row into a per-warp ring of AD slots
// and reads it back when the row is consumed; no other lane touches it, so
// only the per-thread group waits are needed.  The arithmetic is
// linear_stream_kernel's.
constexpr int AD = 4;   // ring slots per warp (AD-1 rows in flight)

__device__ __forceinline__ void cp_async_elem(void *smem, const void *gmem, int bytes, bool valid)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    const int src = valid ? bytes : 0;   // 0: zero-fill, nothing read
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(src));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gmem), "r"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <typename R, bool CORIOLIS, bool TRUELY_LINEAR, bool GAUGES = false>
__global__ void __launch_bounds__(128, LIN_MINB) linear_async_kernel(const LinArgs<R> a, int SH, int nstrips, int total)
{
    __shared__ R ring[4][AD][5][32];   // [warp][slot][UH, VH, STG, ELV, max_stage][lane]
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int b = blockIdx.x;
    if (b >= a.nbatch) return;
    const int nx = a.p.nx, ny = a.p.ny;
    const int64_t P = a.p.pitch;
    const int64_t io = (int64_t)b * a.inst_stride;
    const R *stg = a.p.stg + io, *uhp = a.p.uh + io, *vhp = a.p.vh + io;
    R *stg_o = a.p.stg_o + io, *uh_o = a.p.uh_o + io, *vh_o = a.p.vh_o + io;
    R *max_stage = a.p.max_stage ? a.p.max_stage + (int64_t)b * a.max_stride : nullptr;
    const R *elv = a.p.elv;
    const R g = K<R>::gravity();
    const R half = K<R>::half();
    const R one = K<R>::one();
    const R zero = K<R>::zero();
    const R mad = K<R>::min_depth();
    R (*rg)[5][32] = ring[wib];

    for (int w = blockIdx.y * 4 + wib; w < total; w += gridDim.y * 4) {
        const int sx = w % nstrips, sy = w / nstrips;
        const int ra = sy * SH;
        const int rb = min(ra + SH, ny);
        const int i = sx * SOUT - 1 + lane;
        const int ic = clampi(i, 0, nx - 1);
        const bool in_x = (i >= 0 && i < nx);
        const bool out = (lane >= 1 && lane <= SOUT && i < nx);
        const R dyl_i = a.m.dyl[ic];
        const R dyl_ip1 = a.m.dyl[min(ic + 1, nx)];
        const unsigned long long gmask =
            GAUGES ? gauges_in(a.sites, a.n_sites, sx * SOUT, sx * SOUT + SOUT - 1, ra, rb - 1) : 0ull;
        // Row k of the segment's sequence is row ra - 1 + k, k = 0 .. rb - ra + 1.
        const int nrow = rb - ra + 2;
        auto issue = [&](int k) {
            if (k < nrow) {
                const int q = ra - 1 + k;
                const int qc = clampi(q, 0, ny - 1);
                const int slot = k % AD;
                const int64_t oc = (int64_t)qc * P + ic;
                cp_async_elem(&rg[slot][0][lane], uhp + oc, sizeof(R), true);
                cp_async_elem(&rg[slot][1][lane], vhp + oc, sizeof(R), true);
                const bool sv = (q >= 0 && q < ny && in_x);
                cp_async_elem(&rg[slot][2][lane], stg + oc, sizeof(R), sv);
                cp_async_elem(&rg[slot][3][lane], elv + oc, sizeof(R), true);
                const bool mv = max_stage && out && i >= a.xl && i <= a.xu && q >= a.yl && q <= a.yu && q >= ra && q < rb;
                cp_async_elem(&rg[slot][4][lane], (max_stage ? max_stage : stg) + oc, sizeof(R), mv);
            }
            cp_async_commit();
        };
        auto stage_new = [&](int r, R s_old, R uh_r, R uh_w, R vh_r, R vh_s, R inv_cell_area_dt) -> R {
            R sn = R(0);
            if (r < ny && in_x) {
                const bool interior = (i >= a.xl + 1) && (i <= a.xu - 1) && (r >= a.yl + 1) && (r <= a.yu - 1);
                if (interior) {
                    const R t1 = (uh_r - uh_w) * dyl_i;
                    const R t2 = vh_r * a.m.dxb[r + 1] - vh_s * a.m.dxb[r];
                    sn = s_old - inv_cell_area_dt * (t1 + t2);
                } else if (a.bc_stage && on_bc_ring(i, r, nx, ny, a.bext)) {
                    sn = stg_o[(int64_t)r * P + i];
                } else {
                    sn = s_old;
                }
            }
            return sn;
        };

        __syncwarp();  // the previous segment's reads of the ring are done
        for (int k = 0; k < AD - 1; k++) issue(k);
        // k = 0: row ra-1 (VH only)
        cp_async_wait<AD - 2>();
        R vh_jm1 = rg[0][1][lane];
        issue(AD - 1);
        // k = 1: row ra
        cp_async_wait<AD - 2>();
        R uh_j = rg[1][0][lane], vh_j = rg[1][1][lane], st_j = rg[1][2][lane], e_j = rg[1][3][lane];
        R mx = rg[1][4][lane];
        issue(AD);
        R sn_j;
        {
            const R uh_w = __shfl_up_sync(FULL, uh_j, 1);
            sn_j = stage_new(ra, st_j, uh_j, uh_w, vh_j, vh_jm1, a.dt / a.m.area[ra]);
        }
        // The row factors dt/area (the new stage, row j+1) and g dt/area,
        // g dt/mean area (the momenta, row j) are the same in every lane:
        // lane L evaluates them for row jb + L of each 32-row chunk and the
        // rows take them by shuffle, one division per chunk instead of three
        // per row.
        R rc_s = R(0), rc_u = R(0), rc_v = R(0);
        for (int j = ra; j < rb; j++) {
            const int k = j - ra + 2;  // row j+1
            if (((j - ra) & 31) == 0) {
                const int rr = min(j + lane, ny - 1);
                const int rs = min(j + 1 + lane, ny - 1);
                rc_s = a.dt / a.m.area[rs];
                rc_u = g * a.dt / a.m.area[rr];
                rc_v = g * a.dt / (half * (a.m.area[rr] + a.m.area[min(rr + 1, ny - 1)]));
            }
            const int rl = (j - ra) & 31;
            const R inv_cell_area_dt_n = __shfl_sync(FULL, rc_s, rl);
            const R inv_cell_area_dt_g = __shfl_sync(FULL, rc_u, rl);
            const R inv_cell_area_dt_vh_g = __shfl_sync(FULL, rc_v, rl);
            cp_async_wait<AD - 2>();
            const int slot = k % AD;
            const R uh_n = rg[slot][0][lane], vh_n = rg[slot][1][lane], st_n = rg[slot][2][lane];
            const R e_n = rg[slot][3][lane], mx_n = rg[slot][4][lane];
            issue(k + AD - 1);
            const bool in_ms = max_stage && out && i >= a.xl && i <= a.xu && j >= a.yl && j <= a.yu;

            const R uh_nw = __shfl_up_sync(FULL, uh_n, 1);
            const R sn_n = stage_new(j + 1, st_n, uh_n, uh_nw, vh_n, vh_j, inv_cell_area_dt_n);

            const R s_e = __shfl_down_sync(FULL, sn_j, 1);
            const R e_e = __shfl_down_sync(FULL, e_j, 1);
            const R uh_w = __shfl_up_sync(FULL, uh_j, 1);
            const R vh_e = __shfl_down_sync(FULL, vh_j, 1);
            const R vh_se = __shfl_down_sync(FULL, vh_jm1, 1);
            if (out) {
                const int64_t o = (int64_t)j * P + i;
                stg_o[o] = sn_j;
                if (GAUGES && gmask) {
                    if (a.n_sites > 64) {
                        for (int q = 0; q < a.n_sites; q++)
                            if (a.sites[2 * q] == i && a.sites[2 * q + 1] == j) a.rec[q] = (double)sn_j;
                    } else {
                        for (unsigned long long m = gmask; m; m &= m - 1) {
                            const int q = __ffsll((long long)m) - 1;
                            if (a.sites[2 * q] == i && a.sites[2 * q + 1] == j) a.rec[q] = (double)sn_j;
                        }
                    }
                }
                if (in_ms) max_stage[o] = (sn_j > mx) ? sn_j : mx;
                R uh = uh_j, vh = vh_j;
                if (i >= a.xl && i <= a.xu - 1 && j >= a.yl && j <= a.yu - 1) {
                    const R e0 = e_j;
                    const R sn = sn_j, s_n = sn_n;
                    R h_iph, h_jph, wet_iph, wet_jph;
                    if (TRUELY_LINEAR) {
                        const bool wi = (e0 < -mad + a.msl) && (e_e < -mad + a.msl);
                        h_iph = wi ? (a.msl - half * (e_e + e0)) : zero;
                        const bool wj = (e_n < -mad + a.msl) && (e0 < -mad + a.msl);
                        h_jph = wj ? (a.msl - half * (e_n + e0)) : zero;
                        wet_iph = one;
                        wet_jph = one;
                    } else {
                        const bool wi = (sn - e0 > mad) && (s_e - e_e > mad);
                        h_iph = wi ? (half * ((s_e + sn) - (e_e + e0))) : zero;
                        const bool wj = (s_n - e_n > mad) && (sn - e0 > mad);
                        h_jph = wj ? (half * ((s_n + sn) - (e_n + e0))) : zero;
                        wet_iph = (h_iph > zero) ? one : zero;
                        wet_jph = (h_jph > zero) ? one : zero;
                    }
                    const R dw_j = s_n - sn;
                    R uh_new = uh * wet_iph - inv_cell_area_dt_g * h_iph * (s_e - sn) * dyl_ip1;
                    R vh_new = vh * wet_jph - inv_cell_area_dt_vh_g * h_jph * dw_j * a.m.dxb[j + 1];
                    if (CORIOLIS) {
                        const R vh_iph_jmh = half * (vh_jm1 + vh_se);
                        const R vh_iph_jph = half * (vh_j + vh_e);
                        const R uh_i_j = half * (uh_j + uh_w);
                        const R uh_i_jp1 = half * (uh_n + uh_nw);
                        const R dt_half_coriolis = a.dt * a.m.cor[j] * half * ((h_iph > zero) ? one : zero);
                        const R dt_half_coriolis_jph = a.dt * a.m.cor_be[j + 1] * half * ((h_jph > zero) ? one : zero);
                        uh_new = uh_new + dt_half_coriolis * (vh_iph_jmh + vh_iph_jph);
                        vh_new = vh_new - dt_half_coriolis_jph * (uh_i_j + uh_i_jp1);
                    }
                    if (a.lin_fric) {
                        uh_new = a.lin_fric_mult * uh_new;
                        vh_new = a.lin_fric_mult * vh_new;
                    }
                    uh = uh_new;
                    vh = vh_new;
                }
                uh_o[o] = uh;
                vh_o[o] = vh;
            }
            vh_jm1 = vh_j;
            uh_j = uh_n; vh_j = vh_n; e_j = e_n; sn_j = sn_n; mx = mx_n;
        }
        cp_async_wait<0>();
    }
}

// The streaming step with aligned, wide row segments: a warp owns W = 32 CPL
// columns (lane L holds columns base + L CPL .. + CPL - 1, one 4/8/16-byte
// cp.async per plane and row), so every strip starts on a 128- or 256-byte
// boundary and each row of each plane is read and written as whole sectors
// (the 30-column strips of linear_async_kernel start mid-sector, and two
// warps write the sector their strips share).  The two neighbour columns
// the stencil needs outside the strip are single-element copies into a
// per-warp halo ring: UH of column base - 1 (clamped at the west edge, like
// the reference's UH(max(xL-1, 1))) and STG, UH, VH, ELV of column base + W,
// whose new stage every lane evaluates (the same expression).  Lanes read
// only their own ring entries; lanes 0 and 31 hand the halo values on by
// shuffle.  The arithmetic is linear_stream_kernel's, column by column.
#ifndef LIN_WIDE_MINB
#define LIN_WIDE_MINB 4
#endif
#ifndef LIN_WIDE_AD
// Ring slots per warp (LIN_WIDE_AD - 1 rows in flight).  Measured at
// 4096^2 / 8192^2: 3 slots 0.86 / 0.95 of HBM in FP64 and 0.78 / 0.90 in
// FP32 (batched 0.74), against 0.84 / 0.93, 0.73 / 0.87 (0.71) with 4; a
// register cap for 3 CTAs per SM loses 6-9 %, for 5 or 6 CTAs about half.
#define LIN_WIDE_AD 3
#endif

__device__ __forceinline__ void cp_async_vec(void *smem, const void *gmem, int bytes, int src_bytes)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    if (bytes == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes));
    else if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes));
}

template <typename R, int CPL> struct VecOf { typedef R T; };
template <> struct VecOf<double, 2> { typedef double2 T; };
template <> struct VecOf<float, 2> { typedef float2 T; };
template <> struct VecOf<float, 4> { typedef float4 T; };
template <typename R, int CPL>
__device__ __forceinline__ void store_vec(R *p, const R (&v)[CPL])
{
    typename VecOf<R, CPL>::T x;
    R *xs = reinterpret_cast<R *>(&x);
#pragma unroll
    for (int c = 0; c < CPL; c++) xs[c] = v[c];
    *reinterpret_cast<typename VecOf<R, CPL>::T *>(p) = x;
}

template <typename R, int CPL> struct WideRing {
    R v[LIN_WIDE_AD][5][32 * CPL];   // [slot][UH, VH, STG, ELV, max_stage][column]
    R h[LIN_WIDE_AD][2][4];          // [slot][lane 0: UH west | lane 31: STG, UH, VH, ELV east][]
};

// Ring of the bulk-copy form: per slot, UH, VH, STG and ELV of the strip's
// row with one 16-byte granule either side (which hold the halo columns),
// and max_stage of the strip.
template <typename R> struct BulkRing {
    R v[LIN_WIDE_AD][4][32 * (16 / (int)sizeof(R)) + 2 * (16 / (int)sizeof(R))];
    R m[LIN_WIDE_AD][32 * (16 / (int)sizeof(R))];
};
#ifndef LIN_BULK_FENCE
#define LIN_BULK_FENCE 1
#endif

// Bounded waits of the bulk-copy rows that gave up, on this device.
__device__ unsigned int g_linear_wait_expired;
// Set on the host when a bulk-copy step is first launched.
std::atomic<bool> g_bulk_launched{false};

// mbarrier and bulk-copy primitives (PTX ISA: mbarrier.*, cp.async.bulk).
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes)
{
    unsigned long long state;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;\n"
                 : "=l"(state)
                 : "r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    (void)state;
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}
// Wait until the phase of the given parity has completed, for at most
// `limit` SM clock cycles; false when the bound ran out first.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity, long long limit)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (clock64() - t0 < limit)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// `bytes` (a multiple of 16, both addresses 16-byte aligned) from global to
// this CTA's shared memory, completing on mbarrier `bar`.  No multicast.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

template <typename R, bool CORIOLIS, bool TRUELY_LINEAR, bool GAUGES, int CPL, bool BULK>
__global__ void __launch_bounds__(128, LIN_WIDE_MINB) linear_wide_kernel(const LinArgs<R> a, int SH, int nstrips,
                                                                         int total)
{
    constexpr int W = 32 * CPL;
    constexpr int VB = CPL * (int)sizeof(R);
    static_assert(!BULK || VB == 16, "bulk-copy rows use 16-byte lanes");
    typedef typename std::conditional<BULK, BulkRing<R>, WideRing<R, CPL>>::type Ring;
    __shared__ __align__(128) Ring rings[4];
    __shared__ __align__(8) unsigned long long bars[4][LIN_WIDE_AD];   // bulk form: one mbarrier per slot
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int b = blockIdx.x;
    if (b >= a.nbatch) return;
    if constexpr (BULK) {
        if (threadIdx.x < 4 * LIN_WIDE_AD) {
            mbar_init(&bars[0][0] + threadIdx.x, 1);
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
        __syncthreads();
    }
    const int nx = a.p.nx, ny = a.p.ny;
    const int64_t P = a.p.pitch;
    const int64_t io = (int64_t)b * a.inst_stride;
    const R *stg = a.p.stg + io, *uhp = a.p.uh + io, *vhp = a.p.vh + io;
    R *stg_o = a.p.stg_o + io, *uh_o = a.p.uh_o + io, *vh_o = a.p.vh_o + io;
    R *max_stage = a.p.max_stage ? a.p.max_stage + (int64_t)b * a.max_stride : nullptr;
    const R *elv = a.p.elv;
    const R g = K<R>::gravity();
    const R half = K<R>::half();
    const R one = K<R>::one();
    const R zero = K<R>::zero();
    const R mad = K<R>::min_depth();
    Ring &rg = rings[wib];
    unsigned long long *bar = bars[wib];
    unsigned phase = 0u;   // bulk form, per slot: parity of the slot's next completion
    unsigned pend = 0u;    // bulk form, per slot: copies issued and not yet waited for
    // Bulk form: wait for ring slot s, in every lane, for at most
    // a.wait_cycles; false in every lane when one lane's bound ran out.
    auto wait_slot = [&](int s) -> bool {
        const bool ok = __all_sync(FULL, mbar_wait_bounded(&bar[s], (phase >> s) & 1u, a.wait_cycles));
        if (ok) {
            phase ^= 1u << s;
            pend &= ~(1u << s);
        }
        return ok;
    };
    // Bulk form, after a wait that ran out: count it, give the warp's other
    // copies in flight (with the same bound) time to land, and leave.
    auto give_up = [&]() {
        if (lane == 0) atomicAdd(&g_linear_wait_expired, 1u);
        for (int s = 0; s < LIN_WIDE_AD; s++)
            if (pend & (1u << s)) (void)mbar_wait_bounded(&bar[s], (phase >> s) & 1u, a.wait_cycles);
    };

    for (int w = blockIdx.y * 4 + wib; w < total; w += gridDim.y * 4) {
        const int sx = w % nstrips, sy = w / nstrips;
        const int ra = sy * SH;
        const int rb = min(ra + SH, ny);
        const int base = sx * W;
        const int c0 = base + lane * CPL;                 // this lane's first column
        const int iw = max(base - 1, 0);                  // west neighbour column (clamped)
        const int ie = base + W;                          // east neighbour column
        const int iec = min(ie, nx - 1);
        const bool e_in = ie < nx;
        const int src_bytes = clampi(nx - c0, 0, CPL) * (int)sizeof(R);
        R dyl_i[CPL], dyl_ip1[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            const int ic = min(c0 + c, nx - 1);
            dyl_i[c] = a.m.dyl[ic];
            dyl_ip1[c] = a.m.dyl[min(ic + 1, nx)];
        }
        const R dyl_e = a.m.dyl[iec];
        // The lane's columns against the active region (xL..xU), once per
        // segment: bit c for column c0 + c.
        unsigned in_xm = 0u, int_xm = 0u, mom_xm = 0u, ms_xm = 0u;
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            const int col = c0 + c;
            in_xm |= (unsigned)(col < nx) << c;
            int_xm |= (unsigned)(col >= a.xl + 1 && col <= a.xu - 1) << c;
            mom_xm |= (unsigned)(col >= a.xl && col <= a.xu - 1) << c;
            ms_xm |= (unsigned)(col >= a.xl && col <= a.xu) << c;
        }
        const bool e_int = (ie >= a.xl + 1) && (ie <= a.xu - 1);
        const unsigned long long gmask =
            GAUGES ? gauges_in(a.sites, a.n_sites, base, base + W - 1, ra, rb - 1) : 0ull;
        // the gauges of the segment in this lane's own columns
        unsigned long long lmask = 0ull;
        if (GAUGES && gmask && a.n_sites <= 64)
            for (unsigned long long m = gmask; m; m &= m - 1) {
                const int q = __ffsll((long long)m) - 1;
                if (a.sites[2 * q] >= c0 && a.sites[2 * q] < c0 + CPL) lmask |= 1ull << q;
            }
        const int nrow = rb - ra + 2;   // rows ra-1 .. rb
        // Bulk form: the columns [lo, hi) copied per plane row -- the strip
        // and one granule either side, cut to the row (nx rounded up to a
        // granule, inside the pitch) -- which hold the clamped west and east
        // halo columns; max_stage takes the strip's nb bytes alone.
        const int nxg = (nx + CPL - 1) / CPL * CPL;
        const unsigned nb = (unsigned)(min(W, nxg - base) * (int)sizeof(R));
        const int lo = max(base - CPL, 0), hi = min(base + W + CPL, nxg);
        const unsigned hb = (unsigned)((hi - lo) * (int)sizeof(R));
        const int iwo = CPL + iw - base, ieo = CPL + iec - base;   // halo columns in a plane row
        auto issue_bulk = [&](int k) {
            if constexpr (BULK) {
                if (k >= nrow) return;
                const int q = ra - 1 + k;
                const int qc = clampi(q, 0, ny - 1);
                const int slot = k % LIN_WIDE_AD;
                const int64_t orow = (int64_t)qc * P;
                const bool mv = max_stage && q >= ra && q < rb;
                if (lane == 0) mbar_arrive_expect_tx(&bar[slot], 4u * hb + (mv ? nb : 0u) + a.bulk_extra_tx);
                // the slot's last reads (all lanes) and the expected count come
                // before the copies that overwrite it
                __syncwarp();
                if (lane < 5) {
                    const int64_t o = orow + (lane < 4 ? lo : base);
                    const R *src = lane == 0 ? uhp + o : lane == 1 ? vhp + o : lane == 2 ? stg + o
                                 : lane == 3 ? elv + o : (mv ? max_stage + o : nullptr);
                    R *dst = lane < 4 ? &rg.v[slot][lane][lo - (base - CPL)] : rg.m[slot];
                    if (src) {
                        if (LIN_BULK_FENCE) asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                        bulk_copy_g2s(dst, src, lane < 4 ? hb : nb, &bar[slot]);
                    }
                }
                pend |= 1u << (unsigned)slot;
            }
        };
        auto issue = [&](int k) {
            if constexpr (BULK) {
                issue_bulk(k);
            } else {
                if (k < nrow) {
                    const int q = ra - 1 + k;
                    const int qc = clampi(q, 0, ny - 1);
                    const int slot = k % LIN_WIDE_AD;
                    const int64_t orow = (int64_t)qc * P;
                    const bool qv = (q >= 0 && q < ny);
                    cp_async_vec(&rg.v[slot][0][lane * CPL], uhp + orow + (src_bytes ? c0 : 0), VB, src_bytes);
                    cp_async_vec(&rg.v[slot][1][lane * CPL], vhp + orow + (src_bytes ? c0 : 0), VB, src_bytes);
                    cp_async_vec(&rg.v[slot][2][lane * CPL], stg + orow + (src_bytes ? c0 : 0), VB,
                                 qv ? src_bytes : 0);
                    cp_async_vec(&rg.v[slot][3][lane * CPL], elv + orow + (src_bytes ? c0 : 0), VB, src_bytes);
                    const bool mv = max_stage && q >= ra && q < rb;
                    cp_async_vec(&rg.v[slot][4][lane * CPL], (max_stage ? max_stage : stg) + orow + (src_bytes ? c0 : 0),
                                 VB, mv ? src_bytes : 0);
                    if (lane == 0) {
                        cp_async_vec(&rg.h[slot][0][0], uhp + orow + iw, (int)sizeof(R), (int)sizeof(R));
                    } else if (lane == 31) {
                        cp_async_vec(&rg.h[slot][1][0], stg + orow + iec, (int)sizeof(R), (qv && e_in) ? (int)sizeof(R) : 0);
                        cp_async_vec(&rg.h[slot][1][1], uhp + orow + iec, (int)sizeof(R), (int)sizeof(R));
                        cp_async_vec(&rg.h[slot][1][2], vhp + orow + iec, (int)sizeof(R), (int)sizeof(R));
                        cp_async_vec(&rg.h[slot][1][3], elv + orow + iec, (int)sizeof(R), (int)sizeof(R));
                    }
                }
                cp_async_commit();
            }
        };
        // New stage of cell (col, r) (domain_mod_linear_solver_include.f90:92-115).
        // (interior: the cell is inside xL+1..xU-1, yL+1..yU-1; dxb_r1, dxb_r:
        // distance_bottom_edge of rows r+1 and r)
        auto stage_new = [&](int col, bool in_x, bool interior, R dyl, int r, R dxb_r1, R dxb_r, R s_old, R uh_r,
                             R uh_w, R vh_r, R vh_s, R inv_cell_area_dt) -> R {
            R sn = R(0);
            if (r < ny && in_x) {
                if (interior) {
                    const R t1 = (uh_r - uh_w) * dyl;
                    const R t2 = vh_r * dxb_r1 - vh_s * dxb_r;
                    sn = s_old - inv_cell_area_dt * (t1 + t2);
                } else if (a.bc_stage && on_bc_ring(col, r, nx, ny, a.bext)) {
                    sn = stg_o[(int64_t)r * P + col];
                } else {
                    sn = s_old;
                }
            }
            return sn;
        };
        // Neighbour values across lanes: west (the previous column) and east.
        auto west = [&](const R (&v)[CPL], R halo_w, int c) -> R {
            const R up = __shfl_up_sync(FULL, v[CPL - 1], 1);
            return c > 0 ? v[c > 0 ? c - 1 : 0] : (lane > 0 ? up : halo_w);
        };

        // Halo values of a ring slot: 0 UH west; 1-4 STG, UH, VH, ELV east.
        auto halo = [&](int slot, int which) -> R {
            if constexpr (BULK)
                return which == 0 ? rg.v[slot][0][iwo] : rg.v[slot][which == 1 ? 2 : which == 4 ? 3 : which - 2][ieo];
            else
                return which == 0 ? __shfl_sync(FULL, lane == 0 ? rg.h[slot][0][0] : R(0), 0)
                                  : __shfl_sync(FULL, lane == 31 ? rg.h[slot][1][which - 1] : R(0), 31);
        };
        // Value of plane p (UH, VH, STG, ELV, max_stage) at strip column idx
        // of a ring slot.
        auto cell = [&](int slot, int p, int idx) -> R {
            if constexpr (BULK)
                return p < 4 ? rg.v[slot][p][CPL + idx] : rg.m[slot][idx];
            else
                return rg.v[slot][p][idx];
        };
        // Row k of the segment is in its ring slot (false: a bounded wait ran out).
        auto wait_row = [&](int k) -> bool {
            if constexpr (BULK) {
                return wait_slot(k % LIN_WIDE_AD);
            } else {
                cp_async_wait<LIN_WIDE_AD - 2>();
                return true;
            }
        };

        __syncwarp();  // the previous segment's reads of the ring are done
        for (int k = 0; k < LIN_WIDE_AD - 1; k++) issue(k);
        // k = 0: row ra-1 (VH only)
        if (!wait_row(0)) {
            give_up();
            return;
        }
        R vh_jm1[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) vh_jm1[c] = cell(0, 1, lane * CPL + c);
        R vhE_jm1 = halo(0, 3);
        issue(LIN_WIDE_AD - 1);
        // k = 1: row ra
        if (!wait_row(1)) {
            give_up();
            return;
        }
        R uh_j[CPL], vh_j[CPL], e_j[CPL], sn_j[CPL], mx[CPL];
        R st_j[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            uh_j[c] = cell(1, 0, lane * CPL + c);
            vh_j[c] = cell(1, 1, lane * CPL + c);
            st_j[c] = cell(1, 2, lane * CPL + c);
            e_j[c] = cell(1, 3, lane * CPL + c);
            mx[c] = cell(1, 4, lane * CPL + c);
        }
        R uhW_j = halo(1, 0);
        const R stE_j = halo(1, 1);
        const R uhE_j0 = halo(1, 2);
        R vhE_j = halo(1, 3);
        R eE_j = halo(1, 4);
        issue(LIN_WIDE_AD);
        R snE_j;
        {
            const R dta = a.dt / a.m.area[ra];
            const bool int_y = (ra >= a.yl + 1) && (ra <= a.yu - 1);
            const R dxb1 = a.m.dxb[ra + 1], dxb0 = a.m.dxb[ra];
            R uw[CPL];
#pragma unroll
            for (int c = 0; c < CPL; c++) uw[c] = west(uh_j, uhW_j, c);
#pragma unroll
            for (int c = 0; c < CPL; c++)
                sn_j[c] = stage_new(c0 + c, (in_xm >> c) & 1u, int_y && ((int_xm >> c) & 1u), dyl_i[c], ra, dxb1, dxb0,
                                    st_j[c], uh_j[c], uw[c], vh_j[c], vh_jm1[c], dta);
            const R uh_last = __shfl_sync(FULL, uh_j[CPL - 1], 31);
            snE_j = stage_new(ie, e_in, int_y && e_int, dyl_e, ra, dxb1, dxb0, stE_j, uhE_j0, uh_last, vhE_j,
                              vhE_jm1, dta);
        }
        // Row factors dt/area (the new stage, row j+1) and g dt/area,
        // g dt/mean area (the momenta, row j): lane L evaluates them for row
        // jb + L of each 32-row chunk and the rows take them by shuffle.
        R rc_s = R(0), rc_u = R(0), rc_v = R(0);
        for (int j = ra; j < rb; j++) {
            const int k = j - ra + 2;  // row j+1
            if (((j - ra) & 31) == 0) {
                const int rr = min(j + lane, ny - 1);
                const int rs = min(j + 1 + lane, ny - 1);
                rc_s = a.dt / a.m.area[rs];
                rc_u = g * a.dt / a.m.area[rr];
                rc_v = g * a.dt / (half * (a.m.area[rr] + a.m.area[min(rr + 1, ny - 1)]));
            }
            const int rl = (j - ra) & 31;
            const R inv_cell_area_dt_n = __shfl_sync(FULL, rc_s, rl);
            const R inv_cell_area_dt_g = __shfl_sync(FULL, rc_u, rl);
            const R inv_cell_area_dt_vh_g = __shfl_sync(FULL, rc_v, rl);
            if (!wait_row(k)) {
                give_up();
                return;
            }
            const int slot = k % LIN_WIDE_AD;
            R uh_n[CPL], vh_n[CPL], st_n[CPL], e_n[CPL], mx_n[CPL];
#pragma unroll
            for (int c = 0; c < CPL; c++) {
                uh_n[c] = cell(slot, 0, lane * CPL + c);
                vh_n[c] = cell(slot, 1, lane * CPL + c);
                st_n[c] = cell(slot, 2, lane * CPL + c);
                e_n[c] = cell(slot, 3, lane * CPL + c);
                mx_n[c] = cell(slot, 4, lane * CPL + c);
            }
            const R uhW_n = halo(slot, 0);
            const R stE_n = halo(slot, 1);
            const R uhE_n = halo(slot, 2);
            const R vhE_n = halo(slot, 3);
            const R eE_n = halo(slot, 4);
            issue(k + LIN_WIDE_AD - 1);

            // Row constants: distance_bottom_edge of rows j+1 and j+2 (dxb has
            // ny + 1 entries; row ny is never updated), the region tests.
            const R dxb_j1 = a.m.dxb[j + 1], dxb_j2 = a.m.dxb[min(j + 2, ny)];
            const bool int_y = (j + 1 >= a.yl + 1) && (j + 1 <= a.yu - 1);
            const bool mom_y = (j >= a.yl) && (j <= a.yu - 1);
            const bool ms_y = (j >= a.yl) && (j <= a.yu);
            // dt cor / 2 of row j and of its north face: (dt * cor) * half, the
            // reference's product order, before the wet factor
            R dtc_j = zero, dtc_jph = zero;
            if (CORIOLIS) {
                dtc_j = a.dt * a.m.cor[j] * half;
                dtc_jph = a.dt * a.m.cor_be[j + 1] * half;
            }

            // New stage of row j+1: own columns and the east neighbour column.
            R uh_nw[CPL], sn_n[CPL];
#pragma unroll
            for (int c = 0; c < CPL; c++) uh_nw[c] = west(uh_n, uhW_n, c);
#pragma unroll
            for (int c = 0; c < CPL; c++)
                sn_n[c] = stage_new(c0 + c, (in_xm >> c) & 1u, int_y && ((int_xm >> c) & 1u), dyl_i[c], j + 1, dxb_j2,
                                    dxb_j1, st_n[c], uh_n[c], uh_nw[c], vh_n[c], vh_j[c], inv_cell_area_dt_n);
            const R uh_n_last = __shfl_sync(FULL, uh_n[CPL - 1], 31);
            const R snE_n = stage_new(ie, e_in, int_y && e_int, dyl_e, j + 1, dxb_j2, dxb_j1, stE_n, uhE_n, uh_n_last,
                                      vhE_n, vhE_j, inv_cell_area_dt_n);

            // Momentum of row j (:225-567), column by column.
            const R sn_dn = __shfl_down_sync(FULL, sn_j[0], 1);
            const R e_dn = __shfl_down_sync(FULL, e_j[0], 1);
            const R vh_dn = __shfl_down_sync(FULL, vh_j[0], 1);
            const R vhm_dn = __shfl_down_sync(FULL, vh_jm1[0], 1);
            R uh_w[CPL];
#pragma unroll
            for (int c = 0; c < CPL; c++) uh_w[c] = west(uh_j, uhW_j, c);
            const int jrow = j;
            R o_uh[CPL], o_vh[CPL], o_mx[CPL];
            bool ms_all = true;
#pragma unroll
            for (int c = 0; c < CPL; c++) {
                const int i = c0 + c;
                const bool last = (c == CPL - 1);
                const R s_e = !last ? sn_j[c + 1 < CPL ? c + 1 : c] : (lane < 31 ? sn_dn : snE_j);
                const R e_e = !last ? e_j[c + 1 < CPL ? c + 1 : c] : (lane < 31 ? e_dn : eE_j);
                const R vh_e = !last ? vh_j[c + 1 < CPL ? c + 1 : c] : (lane < 31 ? vh_dn : vhE_j);
                const R vh_se = !last ? vh_jm1[c + 1 < CPL ? c + 1 : c] : (lane < 31 ? vhm_dn : vhE_jm1);
                const R snc = sn_j[c];
                const bool in_ms = max_stage && ms_y && ((ms_xm >> c) & 1u);
                ms_all = ms_all && in_ms;
                o_mx[c] = (snc > mx[c]) ? snc : mx[c];
                R uh = uh_j[c], vh = vh_j[c];
                if (mom_y && ((mom_xm >> c) & 1u)) {
                    const R e0 = e_j[c];
                    const R sn = snc, s_n = sn_n[c];
                    R h_iph, h_jph, wet_iph, wet_jph;
                    if (TRUELY_LINEAR) {
                        const bool wi = (e0 < -mad + a.msl) && (e_e < -mad + a.msl);
                        h_iph = wi ? (a.msl - half * (e_e + e0)) : zero;
                        const bool wj = (e_n[c] < -mad + a.msl) && (e0 < -mad + a.msl);
                        h_jph = wj ? (a.msl - half * (e_n[c] + e0)) : zero;
                        wet_iph = one;
                        wet_jph = one;
                    } else {
                        const bool wi = (sn - e0 > mad) && (s_e - e_e > mad);
                        h_iph = wi ? (half * ((s_e + sn) - (e_e + e0))) : zero;
                        const bool wj = (s_n - e_n[c] > mad) && (sn - e0 > mad);
                        h_jph = wj ? (half * ((s_n + sn) - (e_n[c] + e0))) : zero;
                        wet_iph = (h_iph > zero) ? one : zero;
                        wet_jph = (h_jph > zero) ? one : zero;
                    }
                    const R dw_j = s_n - sn;
                    R uh_new = uh * wet_iph - inv_cell_area_dt_g * h_iph * (s_e - sn) * dyl_ip1[c];
                    R vh_new = vh * wet_jph - inv_cell_area_dt_vh_g * h_jph * dw_j * dxb_j1;
                    if (CORIOLIS) {
                        const R vh_iph_jmh = half * (vh_jm1[c] + vh_se);
                        const R vh_iph_jph = half * (vh_j[c] + vh_e);
                        const R uh_i_j = half * (uh_j[c] + uh_w[c]);
                        const R uh_i_jp1 = half * (uh_n[c] + uh_nw[c]);
                        const R dt_half_coriolis = dtc_j * ((h_iph > zero) ? one : zero);
                        const R dt_half_coriolis_jph = dtc_jph * ((h_jph > zero) ? one : zero);
                        uh_new = uh_new + dt_half_coriolis * (vh_iph_jmh + vh_iph_jph);
                        vh_new = vh_new - dt_half_coriolis_jph * (uh_i_j + uh_i_jp1);
                    }
                    if (a.lin_fric) {
                        uh_new = a.lin_fric_mult * uh_new;
                        vh_new = a.lin_fric_mult * vh_new;
                    }
                    uh = uh_new;
                    vh = vh_new;
                }
                o_uh[c] = uh;
                o_vh[c] = vh;
                if (GAUGES && gmask && i < nx) {
                    if (a.n_sites > 64) {
                        for (int q = 0; q < a.n_sites; q++)
                            if (a.sites[2 * q] == i && a.sites[2 * q + 1] == jrow) a.rec[q] = (double)snc;
                    } else {
                        for (unsigned long long m = lmask; m; m &= m - 1) {
                            const int q = __ffsll((long long)m) - 1;
                            if (a.sites[2 * q] == i && a.sites[2 * q + 1] == jrow) a.rec[q] = (double)snc;
                        }
                    }
                }
            }
            {
                const int64_t o = (int64_t)jrow * P + c0;
                if (src_bytes == VB) {   // the lane's whole vector is inside the row
                    store_vec<R, CPL>(stg_o + o, sn_j);
                    store_vec<R, CPL>(uh_o + o, o_uh);
                    store_vec<R, CPL>(vh_o + o, o_vh);
                    if (ms_all) store_vec<R, CPL>(max_stage + o, o_mx);
                }
                if (src_bytes != VB || (max_stage && !ms_all)) {
#pragma unroll
                    for (int c = 0; c < CPL; c++) {
                        const int i = c0 + c;
                        if (i >= nx) continue;
                        if (src_bytes != VB) {
                            stg_o[o + c] = sn_j[c];
                            uh_o[o + c] = o_uh[c];
                            vh_o[o + c] = o_vh[c];
                        }
                        if (max_stage && i >= a.xl && i <= a.xu && jrow >= a.yl && jrow <= a.yu)
                            max_stage[o + c] = o_mx[c];
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < CPL; c++) {
                vh_jm1[c] = vh_j[c];
                uh_j[c] = uh_n[c]; vh_j[c] = vh_n[c]; e_j[c] = e_n[c]; sn_j[c] = sn_n[c]; mx[c] = mx_n[c];
            }
            vhE_jm1 = vhE_j;
            vhE_j = vhE_n; eE_j = eE_n; snE_j = snE_n; uhW_j = uhW_n;
        }
        if constexpr (!BULK) cp_async_wait<0>();
    }
}

// One block: boundary stage/elevation at time+dt/2, boundary flux sums,
// time bookkeeping (:117-205, :571).
template <typename R>
__global__ void __launch_bounds__(512) linear_edge_kernel(const LinArgs<R> a, DevScalars *sc, int n_ext,
                                                          BoundaryFn bf)
{
    const int nx = a.p.nx, ny = a.p.ny;
    const int64_t P = a.p.pitch;
    const double time0 = sc->time;
    const double t_half = time0 + (double)(a.dt * K<R>::half());
    if (a.bc_fn_ring) {
        const int nring = 2 * nx + 2 * ny;
        for (int q = threadIdx.x; q < nring; q += blockDim.x) {
            int i, r, side;
            if (q < ny) { i = 0; r = q; side = 3; }
            else if (q < 2 * ny) { i = nx - 1; r = q - ny; side = 1; }
            else if (q < 2 * ny + nx) { i = q - 2 * ny; r = 0; side = 2; }
            else { i = q - 2 * ny - nx; r = ny - 1; side = 0; }
            if (!a.bext[side]) continue;
            R stg, elv;
            boundary_function<R>(bf, a.m.x, t_half, i, r, stg, elv);
            a.p.stg_o[r * P + i] = stg;
            a.p.elv[r * P + i] = elv;
        }
    }
    // Boundary flux sums of the interior lines, using pre-update UH/VH.
    __shared__ double red[4][32];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = n_ext + threadIdx.x; i <= nx - n_ext - 1; i += blockDim.x) {
        acc[0] += (double)a.p.vh[(int64_t)(ny - n_ext - 1) * P + i];
        acc[2] += (double)a.p.vh[(int64_t)(n_ext - 1) * P + i];
    }
    for (int r = n_ext + threadIdx.x; r <= ny - n_ext - 1; r += blockDim.x) {
        acc[1] += (double)a.p.uh[(int64_t)r * P + (nx - n_ext - 1)];
        acc[3] += (double)a.p.uh[(int64_t)r * P + (n_ext - 1)];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < 4; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s[4];
        const int nw = blockDim.x >> 5;
        for (int k = 0; k < 4; k++) {
            double v = 0.0;
            for (int w = 0; w < nw; w++) v += red[k][w];
            s[k] = v;
        }
        sc->boundary_flux_store[0] = s[0] * (double)a.m.dxb[ny - n_ext];
        sc->boundary_flux_store[1] = s[1] * (double)a.m.dyl[nx - n_ext];
        sc->boundary_flux_store[2] = -(s[2] * (double)a.m.dxb[n_ext]);
        sc->boundary_flux_store[3] = -(s[3] * (double)a.m.dyl[n_ext]);
        double tot = 0.0;
        for (int k = 0; k < 4; k++) tot += sc->boundary_flux_store[k];
        sc->boundary_flux_evolve_integral = tot * (double)a.dt;
        sc->boundary_flux_time_integral += sc->boundary_flux_evolve_integral;
        sc->time0 = time0;
        sc->time = t_half + (double)(K<R>::half() * a.dt);
        sc->dt = (double)a.dt;
        sc->dt_last_update = (double)a.dt;
        sc->evolve_step_dt = sc->time - time0;
        sc->nsteps_advanced += 1;
    }
}

// ---------------------------------------------------------------------------
// flather_boundary on the staggered grid (boundary_mod.f90:502-730, called
// between the stage and the momentum sweep, linear_solver_include.f90:122).
// The fused step kernels read the old momenta once for both sweeps, but the
// momentum sweep has to see the ring's momenta as the boundary routine left
// them.  So with Flather a step is three launches:
//   1. linear_flather_ring_kernel: the ring values from the inner cells'
//      swept stage (recomputed with the sweep's own expression) and old
//      momenta; the ring stage goes to the output stage plane, where the step
//      kernel keeps it as it does for a stage boundary, and the ring momenta
//      to a ring buffer;
//   2. the step kernel, unchanged;
//   3. linear_flather_fix_kernel: the momentum update of the outer two rings
//      -- the only cells whose update reads a ring momentum (own value or a
//      Coriolis average) -- again, from the new stage and the ring buffer.
// Ring cell q: rows 0 and ny-1 in full (q < 2 nx), then columns 0 and nx-1 of
// rows 1 .. ny-2.
__device__ __forceinline__ int ring_index(int i, int r, int nx, int ny)
{
    if (r == 0) return i;
    if (r == ny - 1) return nx + i;
    return 2 * nx + ((i == 0) ? (r - 1) : (ny - 2) + (r - 1));
}

// Stage of cell (i, r) after the stage sweep (:92-115).
template <typename R>
__device__ __forceinline__ R swept_stage(const LinArgs<R> &a, int i, int r)
{
    const int64_t P = a.p.pitch;
    const int64_t o = (int64_t)r * P + i;
    const R s_old = a.p.stg[o];
    const bool interior = (i >= a.xl + 1) && (i <= a.xu - 1) && (r >= a.yl + 1) && (r <= a.yu - 1);
    if (!interior) return s_old;
    const R inv_cell_area_dt = a.dt / a.m.area[r];
    const R t1 = (a.p.uh[o] - a.p.uh[o - 1]) * a.m.dyl[i];
    const R t2 = a.p.vh[o] * a.m.dxb[r + 1] - a.p.vh[o - P] * a.m.dxb[r];
    return s_old - inv_cell_area_dt * (t1 + t2);
}

template <typename R> struct LinRing { R s, uh, vh; };

// West/east pass value of ring cell (i, r), i in {0, nx-1}.
template <typename R>
__device__ __forceinline__ LinRing<R> flather_we(const LinArgs<R> &a, const BoundaryFn &bf, double t, int i, int r)
{
    const int in = (i == 0) ? 1 : a.p.nx - 2;
    const int64_t ro = (int64_t)r * a.p.pitch;
    LinRing<R> v;
    flather_cell<R>(bf, a.m.x, t, i, r, a.msl, i == 0, swept_stage(a, in, r), a.p.uh[ro + in], a.p.vh[ro + in],
                    a.p.elv[ro + in], a.p.elv[ro + i], v.s, v.uh, v.vh);
    return v;
}

template <typename R>
__global__ void __launch_bounds__(256) linear_flather_ring_kernel(const LinArgs<R> a, const DevScalars *sc,
                                                                  BoundaryFn bf, R *ring)
{
    const int nx = a.p.nx, ny = a.p.ny;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    int i, r;
    if (q < 2 * nx) { i = q % nx; r = (q < nx) ? 0 : ny - 1; }
    else if (q < 2 * nx + 2 * (ny - 2)) { const int p = q - 2 * nx; r = 1 + p % (ny - 2); i = (p < ny - 2) ? 0 : nx - 1; }
    else return;
    const bool sn = (r == 0 && a.bext[2]) || (r == ny - 1 && a.bext[0]);
    const bool we = (i == 0 && a.bext[3]) || (i == nx - 1 && a.bext[1]);
    if (!sn && !we) return;
    // domain%time after the stage sweep, as linear_edge_kernel forms it.
    const double t = sc->time + (double)(a.dt * K<R>::half());
    const int64_t P = a.p.pitch;
    LinRing<R> v;
    if (sn) {
        // South/north pass: reads the column neighbour after the west/east pass.
        const int rn = (r == 0) ? 1 : ny - 2;
        LinRing<R> nb;
        if (we) {
            nb = flather_we<R>(a, bf, t, i, rn);
        } else {
            nb.s = swept_stage(a, i, rn);
            nb.uh = a.p.uh[(int64_t)rn * P + i];
            nb.vh = a.p.vh[(int64_t)rn * P + i];
        }
        flather_cell<R>(bf, a.m.x, t, i, r, a.msl, r == 0, nb.s, nb.vh, nb.uh, a.p.elv[(int64_t)rn * P + i],
                        a.p.elv[(int64_t)r * P + i], v.s, v.vh, v.uh);
    } else {
        v = flather_we<R>(a, bf, t, i, r);
    }
    a.p.stg_o[(int64_t)r * P + i] = v.s;
    ring[2 * q] = v.uh;
    ring[2 * q + 1] = v.vh;
}

// The momentum update (:225-567) of one cell (i, r), redone after the step
// kernel from the stage in stg_o, the elevation and the old momenta as the
// boundary routine (ring buffer) and any forcing left them.  Cells outside
// the update range get their old momenta when write_outside.
template <typename R, bool CORIOLIS, bool TRUELY_LINEAR>
__device__ __forceinline__ void momentum_recompute(const LinArgs<R> &a, const R *ring, int i, int r, bool write_outside)
{
    const int nx = a.p.nx, ny = a.p.ny;
    const int64_t P = a.p.pitch;
    const R g = K<R>::gravity(), half = K<R>::half(), one = K<R>::one(), zero = K<R>::zero();
    const R mad = K<R>::min_depth();
    // Momenta as the boundary routine (and any forcing) left them.
    auto uhb = [&](int ii, int rr) -> R {
        return (ring && on_bc_ring(ii, rr, nx, ny, a.bext)) ? ring[2 * ring_index(ii, rr, nx, ny)]
                                                            : a.p.uh[(int64_t)rr * P + ii];
    };
    auto vhb = [&](int ii, int rr) -> R {
        return (ring && on_bc_ring(ii, rr, nx, ny, a.bext)) ? ring[2 * ring_index(ii, rr, nx, ny) + 1]
                                                            : a.p.vh[(int64_t)rr * P + ii];
    };
    const int64_t o = (int64_t)r * P + i;
    R uh = uhb(i, r), vh = vhb(i, r);
    const bool updated = (i >= a.xl && i <= a.xu - 1 && r >= a.yl && r <= a.yu - 1);
    if (!updated && !write_outside) return;
    if (updated) {
        const R inv_cell_area_dt_g = g * a.dt / a.m.area[r];
        const R inv_cell_area_dt_vh_g = g * a.dt / (half * (a.m.area[r] + a.m.area[r + 1]));
        const R e0 = a.p.elv[o], e_e = a.p.elv[o + 1], e_n = a.p.elv[o + P];
        const R sn = a.p.stg_o[o], s_e = a.p.stg_o[o + 1], s_n = a.p.stg_o[o + P];
        R h_iph, h_jph, wet_iph, wet_jph;
        if (TRUELY_LINEAR) {
            const bool wi = (e0 < -mad + a.msl) && (e_e < -mad + a.msl);
            h_iph = wi ? (a.msl - half * (e_e + e0)) : zero;
            const bool wj = (e_n < -mad + a.msl) && (e0 < -mad + a.msl);
            h_jph = wj ? (a.msl - half * (e_n + e0)) : zero;
            wet_iph = one;
            wet_jph = one;
        } else {
            const bool wi = (sn - e0 > mad) && (s_e - e_e > mad);
            h_iph = wi ? (half * ((s_e + sn) - (e_e + e0))) : zero;
            const bool wj = (s_n - e_n > mad) && (sn - e0 > mad);
            h_jph = wj ? (half * ((s_n + sn) - (e_n + e0))) : zero;
            wet_iph = (h_iph > zero) ? one : zero;
            wet_jph = (h_jph > zero) ? one : zero;
        }
        const R dw_j = s_n - sn;
        R uh_new = uh * wet_iph - inv_cell_area_dt_g * h_iph * (s_e - sn) * a.m.dyl[i + 1];
        R vh_new = vh * wet_jph - inv_cell_area_dt_vh_g * h_jph * dw_j * a.m.dxb[r + 1];
        if (CORIOLIS) {
            const int rm = (r > 0) ? r - 1 : 0, im = (i > 0) ? i - 1 : 0;
            const R vh_iph_jmh = half * (vhb(i, rm) + vhb(i + 1, rm));
            const R vh_iph_jph = half * (vh + vhb(i + 1, r));
            const R uh_i_j = half * (uh + uhb(im, r));
            const R uh_i_jp1 = half * (uhb(i, r + 1) + uhb(im, r + 1));
            const R dt_half_coriolis = a.dt * a.m.cor[r] * half * ((h_iph > zero) ? one : zero);
            const R dt_half_coriolis_jph = a.dt * a.m.cor_be[r + 1] * half * ((h_jph > zero) ? one : zero);
            uh_new = uh_new + dt_half_coriolis * (vh_iph_jmh + vh_iph_jph);
            vh_new = vh_new - dt_half_coriolis_jph * (uh_i_j + uh_i_jp1);
        }
        if (a.lin_fric) {
            uh_new = a.lin_fric_mult * uh_new;
            vh_new = a.lin_fric_mult * vh_new;
        }
        uh = uh_new;
        vh = vh_new;
    }
    a.p.uh_o[o] = uh;
    a.p.vh_o[o] = vh;
}

template <typename R, bool CORIOLIS, bool TRUELY_LINEAR>
__global__ void __launch_bounds__(256) linear_flather_fix_kernel(const LinArgs<R> a, const R *ring)
{
    const int nx = a.p.nx, ny = a.p.ny;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    // Rows 0, 1, ny-2, ny-1 in full, then columns 0, 1, nx-2, nx-1 of rows 2 .. ny-3.
    int i, r;
    if (q < 4 * nx) {
        const int k = q / nx;
        i = q - k * nx;
        r = (k < 2) ? k : ny - 4 + k;
    } else if (q < 4 * nx + 4 * (ny - 4)) {
        const int p = q - 4 * nx;
        const int k = p / (ny - 4);
        r = 2 + (p - k * (ny - 4));
        i = (k < 2) ? k : nx - 4 + k;
    } else {
        return;
    }
    momentum_recompute<R, CORIOLIS, TRUELY_LINEAR>(a, ring, i, r, true);
}

// The momentum of the cells within one cell of a forcing patch box
// (0-based inclusive [i0, i1] x [r0, r1], already widened), after the forcing.
template <typename R, bool CORIOLIS, bool TRUELY_LINEAR>
__global__ void __launch_bounds__(256) linear_box_fix_kernel(const LinArgs<R> a, int i0, int i1, int r0, int r1)
{
    const int w = i1 - i0 + 1;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= w * (r1 - r0 + 1)) return;
    const int r = r0 + q / w, i = i0 + q % w;
    momentum_recompute<R, CORIOLIS, TRUELY_LINEAR>(a, nullptr, i, r, false);
}

// precompute_friction_work (linear_solver_include.f90:590-618,
// leapfrog_solver_friction_include.f90): g n^2 depth^p at the UH and VH
// points with p = -7/3 (Manning) or -2 (Chezy), correctly rounded.  The
// depth is from msl_linear when truely linear (done once), else from the
// stage after the stage sweep and the boundary (every step; the ring stage
// of a stage boundary is already in stg_o).
// With from_out the stage is read from stg_o (final, after a forcing) over
// the sub-box [i_lo, i_hi] x [r_lo, r_hi] only.
template <typename R, bool CHEZY>
__global__ void __launch_bounds__(256) friction_work_kernel(const LinArgs<R> a, const R *nsq, R *fw, int truely_linear,
                                                            int from_out, int i_lo, int i_hi, int r_lo, int r_hi)
{
    const int nx = a.p.nx, ny = a.p.ny;
    const int i = i_lo + blockIdx.x * 32 + threadIdx.x, r = r_lo + blockIdx.y * 8 + threadIdx.y;
    if (i > i_hi || r > r_hi) return;
    const int64_t P = a.p.pitch;
    const int ip1 = min(i + 1, nx - 1), jp1 = min(r + 1, ny - 1);
    const int64_t o = (int64_t)r * P + i, oe = (int64_t)r * P + ip1, on = (int64_t)jp1 * P + i;
    const R half = K<R>::half(), mad = K<R>::min_depth(), g = K<R>::gravity();
    const R e0 = a.p.elv[o], e_e = a.p.elv[oe], e_n = a.p.elv[on];
    R depth_iph, depth_jph;
    if (truely_linear) {
        depth_iph = half * (((a.msl - e0) + a.msl) - e_e);
        depth_jph = half * (((a.msl - e0) + a.msl) - e_n);
    } else {
        auto stage = [&](int ii, int rr) -> R {
            if (from_out) return a.p.stg_o[(int64_t)rr * P + ii];
            if (a.bc_stage && on_bc_ring(ii, rr, nx, ny, a.bext) &&
                !((ii >= a.xl + 1) && (ii <= a.xu - 1) && (rr >= a.yl + 1) && (rr <= a.yu - 1)))
                return a.p.stg_o[(int64_t)rr * P + ii];
            return swept_stage(a, ii, rr);
        };
        const R s0 = stage(i, r);
        depth_iph = half * (((s0 - e0) + stage(ip1, r)) - e_e);
        depth_jph = half * (((s0 - e0) + stage(i, jp1)) - e_n);
    }
    depth_iph = (depth_iph > mad) ? depth_iph : mad;
    depth_jph = (depth_jph > mad) ? depth_jph : mad;
    const R nsq_iph = half * (nsq[o] + nsq[oe]);
    const R nsq_jph = half * (nsq[o] + nsq[on]);
    fw[o] = g * nsq_iph * R(pow_friction<CHEZY>((double)depth_iph));
    fw[(int64_t)ny * P + o] = g * nsq_jph * R(pow_friction<CHEZY>((double)depth_jph));
}

// The friction multipliers of leapfrog_linear_plus_nonlinear_friction on the
// momenta the step kernel (and a Flather fix-up) wrote.  The old momenta are
// those after the boundary routine: the ring buffer on a Flather ring.
template <typename R>
__global__ void __launch_bounds__(256) linear_nlfric_kernel(const LinArgs<R> a, const R *ring)
{
    const int nx = a.p.nx, ny = a.p.ny;
    const int i = blockIdx.x * 32 + threadIdx.x, r = blockIdx.y * 8 + threadIdx.y;
    if (i >= nx || r >= ny) return;
    if (!(i >= a.xl && i <= a.xu - 1 && r >= a.yl && r <= a.yu - 1)) return;
    const int64_t P = a.p.pitch;
    const R half = K<R>::half();
    auto uhb = [&](int ii, int rr) -> R {
        return (ring && on_bc_ring(ii, rr, nx, ny, a.bext)) ? ring[2 * ring_index(ii, rr, nx, ny)]
                                                            : a.p.uh[(int64_t)rr * P + ii];
    };
    auto vhb = [&](int ii, int rr) -> R {
        return (ring && on_bc_ring(ii, rr, nx, ny, a.bext)) ? ring[2 * ring_index(ii, rr, nx, ny) + 1]
                                                            : a.p.vh[(int64_t)rr * P + ii];
    };
    const int64_t o = (int64_t)r * P + i;
    const int rm = (r > 0) ? r - 1 : 0, im = (i > 0) ? i - 1 : 0;
    const R uh0 = uhb(i, r), vh0 = vhb(i, r);
    const R vh_iph_jmh = half * (vhb(i, rm) + vhb(i + 1, rm));
    const R vh_iph_jph = half * (vh0 + vhb(i + 1, r));
    const R uh_i_j = half * (uh0 + uhb(im, r));
    const R uh_i_jp1 = half * (uhb(i, r + 1) + uhb(im, r + 1));
    R u = a.p.uh_o[o], v = a.p.vh_o[o];
    nl_friction<R>(a, o, uh0, vh0, vh_iph_jmh, vh_iph_jph, uh_i_j, uh_i_jp1, u, v);
    a.p.uh_o[o] = u;
    a.p.vh_o[o] = v;
}

template <typename R>
__global__ void max_stage_kernel(int nx, int ny, int64_t P, const R *stg, R *mx, int xl, int xu, int yl, int yu,
                                 const DevScalars *sc, int every)
{
    // every > 1: max_U_update_frequency (domain_mod.f90:1794-1798), after a
    // step that has already counted itself in nsteps_advanced; every == 0:
    // the update before the first step (:1719), which a replayed graph
    // repeats as a launch but only the first replay carries out
    if (every > 1 && (sc->nsteps_advanced - 1) % every != 0) return;
    if (every == 0 && sc->nsteps_advanced != 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (i < xl || i > xu || r < yl || r > yu || i >= nx || r >= ny) return;
    int64_t o = r * P + i;
    R s = stg[o], m = mx[o];
    mx[o] = (s > m) ? s : m;
}

template <typename R>
__global__ void gauge_kernel(int64_t P, const R *stg, const R *uh, const R *vh, const int *site_ij, int n,
                             double *records, int capacity, DevScalars *sc)
{
    const int rec = sc->gauge_records;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
        if (rec < capacity) {
            int i = site_ij[2 * g], r = site_ij[2 * g + 1];
            int64_t o = (int64_t)r * P + i;
            double *dst = records + ((int64_t)rec * n + g) * 3;
            dst[0] = (double)stg[o];
            dst[1] = (double)uh[o];
            dst[2] = (double)vh[o];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) sc->gauge_records = rec + 1;
}

template <typename R>
__global__ void batch_gauge_kernel(int64_t P, const R *stg0, int64_t inst_stride, int nbatch, const int *site_ij,
                                   int n, double *records, int rec)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n * nbatch) return;
    const int b = q / n, gi = q - b * n;
    const int i = site_ij[2 * gi], r = site_ij[2 * gi + 1];
    records[((int64_t)rec * nbatch + b) * n + gi] = (double)stg0[(int64_t)b * inst_stride + (int64_t)r * P + i];
}

}  // namespace

template <typename R>
cudaError_t launch_batch_gauges(int64_t pitch, const R *stg0, int64_t inst_stride, int nbatch, const int *site_ij,
                                int n, double *records, int rec, int capacity, cudaStream_t s)
{
    if (rec >= capacity || n <= 0) return cudaSuccess;
    const int tot = n * nbatch;
    batch_gauge_kernel<R><<<(tot + 255) / 256, 256, 0, s>>>(pitch, stg0, inst_stride, nbatch, site_ij, n, records,
                                                            rec);
    return cudaGetLastError();
}
template cudaError_t launch_batch_gauges<double>(int64_t, const double *, int64_t, int, const int *, int, double *,
                                                 int, int, cudaStream_t);
template cudaError_t launch_batch_gauges<float>(int64_t, const float *, int64_t, int, const int *, int, double *, int,
                                                int, cudaStream_t);

// Tile configurations (rows per tile, thread rows, instances per CTA); the
// batched form's autotuner times each on the real problem.
// Configurations 0-4: shared-memory tiles (rows per CTA, thread rows,
// instances per CTA); 5-7: streaming warps with 32, 64 or 128 rows per
// segment; 8: streaming with the segment height chosen from the grid size;
// 9-10: cp.async-pipelined streaming, 64 rows or chosen; 11-12: aligned
// wide strips (8- or 16-byte lanes); 13: aligned wide strips whose rows
// arrive by bulk copies.  Plain domains use PLAIN_DEFAULT.
struct TileCfg { int by, tyt, ib; };
constexpr TileCfg kTileCfgs[] = {{16, 8, 1}, {16, 8, 2}, {16, 8, 4}, {32, 8, 2}, {8, 8, 4}};
constexpr int kStreamSH[] = {32, 64, 128, 0};
constexpr int kAsyncSH[] = {64, 0};
// 11-13: aligned wide strips (linear_wide_kernel) with 8- and 16-byte lanes,
// rows through per-lane cp.async, and with 16-byte lanes, rows through bulk
// copies completing on an mbarrier.
struct WideCfg { int lane_bytes; bool bulk; };
constexpr WideCfg kWideCfgs[] = {{8, false}, {16, false}, {16, true}};
constexpr int kNumTileCfgs = sizeof(kTileCfgs) / sizeof(kTileCfgs[0]) + sizeof(kStreamSH) / sizeof(kStreamSH[0]) +
                             sizeof(kAsyncSH) / sizeof(kAsyncSH[0]) + sizeof(kWideCfgs) / sizeof(kWideCfgs[0]);
constexpr int STREAM_DEFAULT = 8;
constexpr int ASYNC_DEFAULT = 10;
constexpr int WIDE8_CFG = 11;
constexpr int WIDE16_CFG = 12;
constexpr int BULK_CFG = 13;
// Plain steps use the aligned wide strips with 16-byte lanes: measured on
// the 4096^2 / 8192^2 Gaussian basin (whole step against the measured copy
// bandwidth) 0.84 / 0.93 in FP64 and 0.74 / 0.86 in FP32, against 0.72 /
// 0.76 and 0.63 / 0.66 for the 30-column cp.async strips and 0.67 / 0.71
// and 0.59 / 0.66 for wide strips with 8-byte lanes.
constexpr int PLAIN_DEFAULT = WIDE16_CFG;

// Rows per segment: the longest segment (up to 128 rows, which amortises the
// two rows a segment reloads) that still gives every SM about 24 warps.
inline int stream_rows(int nx, int ny, int nbatch, int strip_cols = SOUT, int min_rows = 16)
{
    // At least four waves of 20 warps per SM (so the last, partial wave is a
    // small part of the launch), but no segment under min_rows rows.
    const int64_t nstrips = (nx + strip_cols - 1) / strip_cols;
    const int64_t want = 148 * 20 * 4;
    int sh = 128;
    while (sh > min_rows && (int64_t)nbatch * nstrips * ((ny + sh - 1) / sh) < want) sh /= 2;
    return sh;
}

template <typename R, bool COR, bool TL>
void launch_stream(const LinArgs<R> &a, int sh, cudaStream_t s)
{
    if (sh <= 0) sh = stream_rows(a.p.nx, a.p.ny, a.nbatch);
    const int nstrips = (a.p.nx + SOUT - 1) / SOUT;
    const int nseg = (a.p.ny + sh - 1) / sh;
    const int total = nstrips * nseg;
    const int gy = std::min((total + 3) / 4, 65535);
    dim3 grid(a.nbatch, gy);
    if (a.rec && a.n_sites > 0)
        linear_stream_kernel<R, COR, TL, true><<<grid, 128, 0, s>>>(a, sh, nstrips, total);
    else
        linear_stream_kernel<R, COR, TL, false><<<grid, 128, 0, s>>>(a, sh, nstrips, total);
}

template <typename R, bool COR, bool TL, int BY, int TYT, int IB>
void launch_cfg(const LinArgs<R> &a, cudaStream_t s)
{
    dim3 block(LBX, TYT);
    dim3 grid((a.p.nx + LBX - 1) / LBX, (a.p.ny + BY - 1) / BY, (a.nbatch + IB - 1) / IB);
    linear_step_kernel<R, COR, TL, BY, TYT, IB><<<grid, block, 0, s>>>(a);
}

template <typename R, bool COR, bool TL>
void launch_async(const LinArgs<R> &a, int sh, cudaStream_t s)
{
    if (sh <= 0) sh = stream_rows(a.p.nx, a.p.ny, a.nbatch);
    const int nstrips = (a.p.nx + SOUT - 1) / SOUT;
    const int nseg = (a.p.ny + sh - 1) / sh;
    const int total = nstrips * nseg;
    const int gy = std::min((total + 3) / 4, 65535);
    dim3 grid(a.nbatch, gy);
    if (a.rec && a.n_sites > 0)
        linear_async_kernel<R, COR, TL, true><<<grid, 128, 0, s>>>(a, sh, nstrips, total);
    else
        linear_async_kernel<R, COR, TL, false><<<grid, 128, 0, s>>>(a, sh, nstrips, total);
}

template <typename R, bool COR, bool TL, int CPL, bool BULK = false>
void launch_wide(const LinArgs<R> &a, cudaStream_t s)
{
    constexpr int W = 32 * CPL;
    // Every lane vector (and bulk-copied row) starts on a VB-byte boundary
    // when the planes and strides are VB-aligned, as the library allocates
    // them (256-byte planes, pitch a multiple of 32 elements); anything else
    // takes the register-streaming kernel, which has no alignment needs.
    constexpr uintptr_t VB = CPL * sizeof(R);
    const uintptr_t mis = (uintptr_t)a.p.stg | (uintptr_t)a.p.uh | (uintptr_t)a.p.vh | (uintptr_t)a.p.stg_o |
                          (uintptr_t)a.p.uh_o | (uintptr_t)a.p.vh_o | (uintptr_t)a.p.elv |
                          (uintptr_t)a.p.max_stage | (uintptr_t)(a.p.pitch * sizeof(R)) |
                          (uintptr_t)(a.inst_stride * sizeof(R)) | (uintptr_t)(a.max_stride * sizeof(R));
    if (mis % VB) {
        launch_stream<R, COR, TL>(a, 0, s);
        return;
    }
    // The wide strips are few on small grids: FP64 segments down to 8 rows;
    // FP32 ones, twice as wide, down to 16 (4096^2 FP32: 8 / 16 / 32 rows
    // 0.742 / 0.770 / 0.776 of HBM; FP64 4096^2 takes 16 rows, 0.86, and
    // 8192^2 64 rows, 0.95, within 1 % of the best).  SWALS_LINEAR_ROWS sets
    // the segment height.
    const char *env_rows = getenv("SWALS_LINEAR_ROWS");
    const int sh = (env_rows && atoi(env_rows) > 0) ? atoi(env_rows)
                                                    : stream_rows(a.p.nx, a.p.ny, a.nbatch, W, sizeof(R) == 4 ? 16 : 8);
    const int nstrips = (a.p.nx + W - 1) / W;
    const int nseg = (a.p.ny + sh - 1) / sh;
    const int total = nstrips * nseg;
    const int gy = std::min((total + 3) / 4, 65535);
    dim3 grid(a.nbatch, gy);
    if (BULK) g_bulk_launched.store(true, std::memory_order_relaxed);
    if (a.rec && a.n_sites > 0)
        linear_wide_kernel<R, COR, TL, true, CPL, BULK><<<grid, 128, 0, s>>>(a, sh, nstrips, total);
    else
        linear_wide_kernel<R, COR, TL, false, CPL, BULK><<<grid, 128, 0, s>>>(a, sh, nstrips, total);
}

template <typename R, bool COR, bool TL>
void launch_tile(const LinArgs<R> &a, int cfg, cudaStream_t s)
{
    const int ntile = (int)(sizeof(kTileCfgs) / sizeof(kTileCfgs[0]));
    const int nstream = (int)(sizeof(kStreamSH) / sizeof(kStreamSH[0]));
    const int nasync = (int)(sizeof(kAsyncSH) / sizeof(kAsyncSH[0]));
    if (cfg >= ntile + nstream + nasync) {
        const WideCfg &wc = kWideCfgs[cfg - ntile - nstream - nasync];
        if (wc.lane_bytes == 8)
            launch_wide<R, COR, TL, 8 / (int)sizeof(R)>(a, s);
        else if (!wc.bulk)
            launch_wide<R, COR, TL, 16 / (int)sizeof(R)>(a, s);
        else
            launch_wide<R, COR, TL, 16 / (int)sizeof(R), true>(a, s);
        return;
    }
    if (cfg >= ntile + nstream) {
        launch_async<R, COR, TL>(a, kAsyncSH[cfg - ntile - nstream], s);
        return;
    }
    if (cfg >= ntile) {
        launch_stream<R, COR, TL>(a, kStreamSH[cfg - ntile], s);
        return;
    }
    switch (cfg) {
    case 1: launch_cfg<R, COR, TL, 16, 8, 2>(a, s); break;
    case 2: launch_cfg<R, COR, TL, 16, 8, 4>(a, s); break;
    case 3: launch_cfg<R, COR, TL, 32, 8, 2>(a, s); break;
    case 4: launch_cfg<R, COR, TL, 8, 8, 4>(a, s); break;
    default: launch_cfg<R, COR, TL, 16, 8, 1>(a, s); break;
    }
}

template <typename R>
void launch_main(const LinArgs<R> &a, const StepConfig &c, int cfg, cudaStream_t s)
{
    const bool cor = c.coriolis != 0, tl = c.truely_linear != 0;
    if (cor && tl) launch_tile<R, true, true>(a, cfg, s);
    else if (cor && !tl) launch_tile<R, true, false>(a, cfg, s);
    else if (!cor && tl) launch_tile<R, false, true>(a, cfg, s);
    else launch_tile<R, false, false>(a, cfg, s);
}

// Kernel of a plain (unbatched) step: the default streaming form unless
// SWALS_LINEAR_KERNEL selects "tile", "stream" (registers only), "async"
// (30-column strips through cp.async), "wide8" / "wide16" (aligned wide
// strips, 8- or 16-byte lanes) or "bulk" (wide strips, rows by bulk copy).
// Read at every launch (not cached), so a process can switch kernels between
// steps.
int linear_kernel_config()
{
    const char *e = getenv("SWALS_LINEAR_KERNEL");
    if (!e) return PLAIN_DEFAULT;
    if (strcmp(e, "tile") == 0) return 0;
    if (strcmp(e, "stream") == 0) return STREAM_DEFAULT;
    if (strcmp(e, "async") == 0) return ASYNC_DEFAULT;
    if (strcmp(e, "wide8") == 0) return WIDE8_CFG;
    if (strcmp(e, "wide16") == 0) return WIDE16_CFG;
    if (strcmp(e, "bulk") == 0) return BULK_CFG;
    return PLAIN_DEFAULT;
}

// Plain-step kernel for a grid: small grids (up to 0.7 M cells; L2-resident,
// a few hundred warp strips) run faster as shared-memory tiles, whose rows
// are all loaded at once, than as streaming warps that march down their rows
// (measured crossover between 800^2 and 1200^2 FP64).  An explicit
// SWALS_LINEAR_KERNEL choice wins.
int plain_config(int nx, int ny)
{
    const char *e = getenv("SWALS_LINEAR_KERNEL");
    if (e && *e) return linear_kernel_config();
    if ((int64_t)nx * ny <= 700000) return 0;
    return linear_kernel_config();
}

// A plain linear step whose last kernel is the tile kernel records its
// gauges there (one launch fewer a step on the small, launch-bound grids).
bool fuses_gauges(const StepConfig &c, int nx, int ny)
{
    return c.g_n > 0 && c.bc_kind != 3 && c.n_forcing == 0 && !c.fw && plain_config(nx, ny) == 0;
}

// Bound on a bulk-copy ring slot's wait: 2^31 SM clock cycles (about 1.1 s
// at 1965 MHz) unless SWALS_BULK_WAIT_CYCLES gives another (positive) bound.
long long bulk_wait_cycles()
{
    static long long v = -1;
    if (v < 0) {
        const char *e = getenv("SWALS_BULK_WAIT_CYCLES");
        const long long x = e ? atoll(e) : 0;
        v = x > 0 ? x : (1ll << 31);
    }
    return v;
}

// Bytes added to every bulk-copy slot's expected count: 0 unless
// SWALS_TEST_BULK_EXTRA_TX sets it, in which case no slot ever completes and
// every warp takes the bounded give-up path (the copies themselves land
// normally).  Only the give-up test sets it.
unsigned bulk_extra_tx()
{
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("SWALS_TEST_BULK_EXTRA_TX");
        const int x = e ? atoi(e) : 0;
        v = (x > 0 && x < (1 << 16)) ? x : 0;
    }
    return (unsigned)v;
}

template <typename R>
LinArgs<R> make_args(const StepPlanes<R> &p, const Metrics<R> &m, const StepConfig &c, R dt)
{
    LinArgs<R> a;
    a.p = p;
    a.m = m;
    a.xl = c.xl; a.xu = c.xu; a.yl = c.yl; a.yu = c.yu;
    // Ring stage set before the step kernel: from the boundary function by
    // the edge kernel (SWALS_BC_STAGE_TRANSMISSIVE_NORMAL_MOMENTUM), or by the
    // Flather ring kernel.
    a.bc_stage = (c.bc_kind == 2 || c.bc_kind == 3) ? 1 : 0;
    a.bc_fn_ring = (c.bc_kind == 2) ? 1 : 0;
    for (int k = 0; k < 4; k++) a.bext[k] = c.bext[k];
    a.dt = dt;
    a.msl = R(c.msl_linear);
    R lfc = R(c.linear_friction_coeff);
    a.lin_fric = (lfc != R(0)) ? 1 : 0;
    a.lin_fric_mult = a.lin_fric ? (R(1) / (R(1) + dt * lfc)) : R(0);
    a.lin_fric_dt = dt * lfc;
    a.fw = nullptr;
    a.fw_plane = 0;
    a.nbatch = 1;
    a.inst_stride = 0;
    a.max_stride = 0;
    a.sites = nullptr;
    a.n_sites = 0;
    a.rec = nullptr;
    a.wait_cycles = bulk_wait_cycles();
    a.bulk_extra_tx = bulk_extra_tx();
    a.g_sites = nullptr;
    a.g_n = 0;
    a.g_records = nullptr;
    a.g_capacity = 0;
    a.g_sc = nullptr;
    return a;
}

// leapfrog_linear_plus_nonlinear_friction: the friction work, before the
// step kernel (and after any ring-stage kernel).
template <typename R>
void launch_friction_work(LinArgs<R> &a, const StepPlanes<R> &p, const StepConfig &c, cudaStream_t s,
                          const LaunchHook &hook)
{
    a.fw = (const R *)c.fw;
    a.fw_plane = p.pitch * (int64_t)p.ny;
    a.lin_fric = 0;   // folded into the friction multipliers
    if (c.truely_linear && c.fw_ready) return;
    hook(CAT_LINEAR_EDGE, 0);
    dim3 block(32, 8), grid((p.nx + 31) / 32, (p.ny + 7) / 8);
    if (c.chezy)
        friction_work_kernel<R, true><<<grid, block, 0, s>>>(a, p.manning_sq, (R *)c.fw, c.truely_linear, 0, 0,
                                                             p.nx - 1, 0, p.ny - 1);
    else
        friction_work_kernel<R, false><<<grid, block, 0, s>>>(a, p.manning_sq, (R *)c.fw, c.truely_linear, 0, 0,
                                                              p.nx - 1, 0, p.ny - 1);
    hook(CAT_LINEAR_EDGE, 1);
}

// apply_forcing between the stage sweep and the momentum sweep
// (linear_solver_include.f90:123), after the step kernel: the patches are
// added to the new stage and to the old momenta and elevation (in place:
// the step kernel has read them), max_stage is redone over the patches, and
// the momentum of every cell within one cell of a patch is recomputed.
// Patches stay off the boundary ring, and patches that force momenta keep
// n_ext + 1 cells from the edges, clear of the boundary-flux lines (checked
// when added).
template <typename R>
void launch_leapfrog_forcing(const LinArgs<R> &a, const StepPlanes<R> &p, const StepConfig &c, const DevScalars *sc,
                             cudaStream_t s, const LaunchHook &hook)
{
    ForcingClock clk{};
    clk.mode = FORCE_LEAPFROG;
    clk.dt = (double)a.dt;
    launch_forcing<R>(c, clk, p.pitch, p.stg_o, const_cast<R *>(p.uh), const_cast<R *>(p.vh), p.elv, sc, s, hook,
                      CAT_LINEAR_EDGE);
    if (p.max_stage) launch_forcing_restore_max<R>(c, p.pitch, p.stg_o, p.max_stage, s, hook, CAT_LINEAR_EDGE);
    const bool cor = c.coriolis != 0, tl = c.truely_linear != 0;
    for (int k = 0; k < c.n_forcing; k++) {
        const ForcingPatch &f = c.forcing[k];
        const int i0 = max(f.i0 - 1, 0), i1 = min(f.i1 + 1, p.nx - 1);
        const int r0 = max(f.j0 - 1, 0), r1 = min(f.j1 + 1, p.ny - 1);
        const int n = (i1 - i0 + 1) * (r1 - r0 + 1), blocks = (n + 255) / 256;
        hook(CAT_LINEAR_EDGE, 0);
        if (cor && tl) linear_box_fix_kernel<R, true, true><<<blocks, 256, 0, s>>>(a, i0, i1, r0, r1);
        else if (cor && !tl) linear_box_fix_kernel<R, true, false><<<blocks, 256, 0, s>>>(a, i0, i1, r0, r1);
        else if (!cor && tl) linear_box_fix_kernel<R, false, true><<<blocks, 256, 0, s>>>(a, i0, i1, r0, r1);
        else linear_box_fix_kernel<R, false, false><<<blocks, 256, 0, s>>>(a, i0, i1, r0, r1);
        hook(CAT_LINEAR_EDGE, 1);
        if (c.fw && !c.truely_linear) {
            // precompute_friction_work runs after apply_forcing: redo it where
            // the forced stage enters (the patch widened by one cell west and
            // south)
            const int fi0 = max(f.i0 - 1, 0), fr0 = max(f.j0 - 1, 0);
            dim3 block(32, 8), grid((f.i1 - fi0 + 32) / 32, (f.j1 - fr0 + 8) / 8);
            hook(CAT_LINEAR_EDGE, 0);
            if (c.chezy)
                friction_work_kernel<R, true><<<grid, block, 0, s>>>(a, p.manning_sq, (R *)c.fw, 0, 1, fi0, f.i1, fr0,
                                                                     f.j1);
            else
                friction_work_kernel<R, false><<<grid, block, 0, s>>>(a, p.manning_sq, (R *)c.fw, 0, 1, fi0, f.i1, fr0,
                                                                      f.j1);
            hook(CAT_LINEAR_EDGE, 1);
        }
    }
}

template <typename R>
void launch_nlfric(const LinArgs<R> &a, const StepPlanes<R> &p, const R *ring, cudaStream_t s, const LaunchHook &hook)
{
    hook(CAT_LINEAR_EDGE, 0);
    dim3 block(32, 8), grid((p.nx + 31) / 32, (p.ny + 7) / 8);
    linear_nlfric_kernel<R><<<grid, block, 0, s>>>(a, ring);
    hook(CAT_LINEAR_EDGE, 1);
}

template <typename R>
cudaError_t launch_linear_step(const StepPlanes<R> &p, const Metrics<R> &m, const StepConfig &c, R dt,
                               DevScalars *sc, cudaStream_t s, const LaunchHook &hook, const AuxStream *aux)
{
    LinArgs<R> a = make_args<R>(p, m, c, dt);
    if (fuses_gauges(c, p.nx, p.ny)) {
        a.g_sites = c.g_sites;
        a.g_n = c.g_n;
        a.g_records = c.g_records;
        a.g_capacity = c.g_capacity;
        a.g_sc = sc;
    }
    // Forcing patches read domain%time from the edge kernel and change the
    // old momenta in place, so the edge kernel then runs in line.
    const bool side = aux && aux->stream && !a.bc_stage && !c.n_forcing;
    if (side) {
        // Bookkeeping beside the main kernel: it reads the input planes and
        // writes only the scalars; the main stream waits for it at the end.
        // (The caller passes `aux` only when the per-launch timers are off;
        // the hook then only counts launches.)
        cudaEventRecord(aux->fork, s);
        cudaStreamWaitEvent(aux->stream, aux->fork, 0);
        hook(CAT_LINEAR_EDGE, 0);
        linear_edge_kernel<R><<<1, 512, 0, aux->stream>>>(a, sc, c.exterior_cells_width, c.bf);
        hook(CAT_LINEAR_EDGE, 1);
        cudaEventRecord(aux->join, aux->stream);
        if (c.fw) launch_friction_work<R>(a, p, c, s, hook);
        hook(CAT_LINEAR_MAIN, 0);
        launch_main<R>(a, c, plain_config(p.nx, p.ny), s);
        hook(CAT_LINEAR_MAIN, 1);
        if (c.fw) launch_nlfric<R>(a, p, nullptr, s, hook);
        cudaStreamWaitEvent(s, aux->join, 0);
        return cudaGetLastError();
    }
    const bool flather = (c.bc_kind == 3);
    R *ring = (R *)c.ring;
    if (flather) {
        // Before the edge kernel: it reads domain%time before the step.
        hook(CAT_LINEAR_EDGE, 0);
        const int n = 2 * p.nx + 2 * (p.ny - 2);
        linear_flather_ring_kernel<R><<<(n + 255) / 256, 256, 0, s>>>(a, sc, c.bf, ring);
        hook(CAT_LINEAR_EDGE, 1);
    }
    hook(CAT_LINEAR_EDGE, 0);
    linear_edge_kernel<R><<<1, 512, 0, s>>>(a, sc, c.exterior_cells_width, c.bf);
    hook(CAT_LINEAR_EDGE, 1);
    if (c.fw) launch_friction_work<R>(a, p, c, s, hook);
    if (c.n_forcing && p.max_stage) launch_forcing_save_max<R>(c, p.pitch, p.max_stage, s, hook, CAT_LINEAR_EDGE);
    hook(CAT_LINEAR_MAIN, 0);
    launch_main<R>(a, c, plain_config(p.nx, p.ny), s);
    hook(CAT_LINEAR_MAIN, 1);
    if (flather) {
        hook(CAT_LINEAR_EDGE, 0);
        const int n = 4 * p.nx + 4 * (p.ny - 4);
        const int blocks = (n + 255) / 256;
        const bool cor = c.coriolis != 0, tl = c.truely_linear != 0;
        if (cor && tl) linear_flather_fix_kernel<R, true, true><<<blocks, 256, 0, s>>>(a, ring);
        else if (cor && !tl) linear_flather_fix_kernel<R, true, false><<<blocks, 256, 0, s>>>(a, ring);
        else if (!cor && tl) linear_flather_fix_kernel<R, false, true><<<blocks, 256, 0, s>>>(a, ring);
        else linear_flather_fix_kernel<R, false, false><<<blocks, 256, 0, s>>>(a, ring);
        hook(CAT_LINEAR_EDGE, 1);
    }
    if (c.n_forcing) launch_leapfrog_forcing<R>(a, p, c, sc, s, hook);
    if (c.fw) launch_nlfric<R>(a, p, flather ? ring : nullptr, s, hook);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// leapfrog_nonlinear (domain_mod_leapfrog_nonlinear_include.f90): the linear
// leapfrog's stage sweep, boundary and forcing, then upwind advection of the
// momenta from a lagged depth, the momentum update with nonlinear pressure
// gradient, Coriolis, spherical metric terms and semi-implicit friction, and
// the dry-cell outflow limiter.  A secondary solver: one kernel per stage of
// the reference's algorithm, reading the old momenta throughout (the
// reference's row carries and thread-boundary copies only serve that).
// Work planes (pitch P): lag0, advection UUH, UVH, VUH, VVH, fluxes
// EW-UH, NS-UH, NS-VH, EW-VH (ny + 1 rows each).
namespace nl {

template <typename R> struct NLArgs {
    LinArgs<R> a;
    const R *nsq;
    R *lag0;
    R *adv[4];      // UUH, UVH, VUH, VVH
    R *flx[4];      // EW-UH, NS-UH, NS-VH, EW-VH
    const R *fw;    // friction_work, UH then VH plane
    int64_t plane;  // elements per work plane
};

template <typename R>
__device__ __forceinline__ bool wet(const NLArgs<R> &n, int i, int r)
{
    const int64_t o = (int64_t)r * n.a.p.pitch + i;
    return n.a.p.stg_o[o] > n.a.p.elv[o] + K<R>::min_depth();
}

// depth at the time of the previous momentum update (:227-230): rows
// 0..ny-2 average the old and the new depth, the last row keeps the old.
template <typename R>
__device__ __forceinline__ R lag(const NLArgs<R> &n, int i, int r)
{
    const int64_t o = (int64_t)r * n.a.p.pitch + i;
    const R d0 = n.lag0[o];
    if (r > n.a.p.ny - 2) return d0;
    const R dn = n.a.p.stg_o[o] - n.a.p.elv[o];
    return K<R>::half() * (d0 + ((R(0) > dn) ? R(0) : dn));
}

template <typename R>
__global__ void lag0_kernel(NLArgs<R> n)
{
    const int i = blockIdx.x * 32 + threadIdx.x, r = blockIdx.y * 8 + threadIdx.y;
    if (i >= n.a.p.nx || r >= n.a.p.ny) return;
    const int64_t o = (int64_t)r * n.a.p.pitch + i;
    const R dp = n.a.p.stg[o] - n.a.p.elv[o];
    n.lag0[o] = (R(0) > dp) ? R(0) : dp;   // max(depth, 0)
}

template <typename R>
__global__ void stage_kernel(NLArgs<R> n)
{
    const LinArgs<R> &a = n.a;
    const int i = blockIdx.x * 32 + threadIdx.x, r = blockIdx.y * 8 + threadIdx.y;
    if (i >= a.p.nx || r >= a.p.ny) return;
    const int64_t o = (int64_t)r * a.p.pitch + i;
    const bool interior = (i >= 1) && (i <= a.p.nx - 2) && (r >= 1) && (r <= a.p.ny - 2);
    if (interior) a.p.stg_o[o] = swept_stage(a, i, r);
    else if (!(a.bc_stage && on_bc_ring(i, r, a.p.nx, a.p.ny, a.bext))) a.p.stg_o[o] = a.p.stg[o];
}

// The advection terms with the reference's edge extrapolations folded in
// as index remaps (:236-333).
template <typename R>
__global__ void advection_kernel(NLArgs<R> n)
{
    const int nx = n.a.p.nx, ny = n.a.p.ny;
    const int i = blockIdx.x * 32 + threadIdx.x, r = blockIdx.y * 8 + threadIdx.y;
    if (i >= nx || r >= ny) return;
    const int64_t P = n.a.p.pitch, o = (int64_t)r * P + i;
    const R half = K<R>::half(), mad = K<R>::min_depth(), quarter = R(0.25);
    const R *uh = n.a.p.uh, *vh = n.a.p.vh;
    auto inv_d = [&](R dl) -> R { return (dl > mad) ? R(1) / dl : R(0); };
    // UUH, UVH at (i+1/2, j), rows 0..ny-2; the last row copies row ny-2
    {
        const int rr = (r <= ny - 2) ? r : ny - 2;
        const int jm1 = (rr - 1 > 0) ? rr - 1 : 0;
        const int iu = (i <= nx - 2) ? i : nx - 2;
        const int64_t ou = (int64_t)rr * P + iu;
        const R dl = half * (lag(n, iu, rr) + lag(n, iu + 1, rr));
        n.adv[0][o] = (uh[ou] * uh[ou]) * inv_d(dl);
        const int iv = (i <= nx - 3) ? i : nx - 3;
        const int64_t ov = (int64_t)rr * P + iv;
        const R dv = half * (lag(n, iv, rr) + lag(n, iv + 1, rr));
        n.adv[1][o] = uh[ov] * inv_d(dv) * quarter *
                      (vh[(int64_t)jm1 * P + iv] + vh[(int64_t)jm1 * P + iv + 1] + vh[ov] + vh[ov + 1]);
    }
    // VVH at (i, j+1/2), rows 0..ny-2; VUH rows 0..ny-3 and columns 1..,
    // the rest copied from column 1 and row ny-3
    {
        const int rr = (r <= ny - 2) ? r : ny - 2;
        const int64_t ov = (int64_t)rr * P + i;
        const R dl = half * (lag(n, i, rr) + lag(n, i, rr + 1));
        n.adv[3][o] = vh[ov] * vh[ov] * inv_d(dl);
        const int ru = (r <= ny - 3) ? r : ny - 3;
        const int iu = (i >= 1) ? i : 1;
        const int64_t ou = (int64_t)ru * P + iu;
        const R du = half * (lag(n, iu, ru) + lag(n, iu, ru + 1));
        n.adv[2][o] = vh[ou] * inv_d(du) * quarter * (uh[ou - 1] + uh[ou] + uh[ou - 1 + P] + uh[ou + P]);
    }
}

// Upwind fluxes of UH and VH (:340-498).  Flux planes have ny + 1 rows.
template <typename R>
__global__ void flux_kernel(NLArgs<R> n)
{
    const int nx = n.a.p.nx, ny = n.a.p.ny;
    const int i = blockIdx.x * 32 + threadIdx.x, r = blockIdx.y * 8 + threadIdx.y;
    if (i > nx || r > ny) return;
    const int64_t P = n.a.p.pitch, o = (int64_t)r * P + i;
    const R half = K<R>::half(), zero = R(0);
    const R *uh = n.a.p.uh, *vh = n.a.p.vh;
    const Metrics<R> &m = n.a.m;
    const R *UUH = n.adv[0], *UVH = n.adv[1], *VUH = n.adv[2], *VVH = n.adv[3];
    // EW flux of UH at cell centres, rows 0..ny-2
    if (i < nx) {
        R f = zero;
        if (r <= ny - 2) {
            if (i == 0) f = UUH[o] * m.dyl[0];
            else if (i == nx - 1) f = UUH[o] * m.dyl[nx - 1];
            else {
                const R sm = uh[o] + uh[o - 1];
                f = m.dyl[i] * ((sm > zero) ? UUH[o - 1] : UUH[o]);
                if (sm == zero) f = m.dyl[i] * half * (UUH[o - 1] + UUH[o]);
            }
            if (!wet(n, i, r)) f = zero;
        }
        n.flx[0][o] = f;
    }
    // NS flux of UH on the bottom edge of row r (rows jl = max(r-1,0), ju = r)
    if (i < nx) {
        R f = zero;
        if (i <= nx - 2 && r <= ny - 1) {
            const int jl = (r - 1 > 0) ? r - 1 : 0, ju = r;
            const int64_t ol = (int64_t)jl * P + i, ou = (int64_t)ju * P + i;
            const R sm = vh[ol] + vh[ol + 1];
            f = m.dxb[r] * ((sm > zero) ? UVH[ol] : UVH[ou]);
            if (sm == zero) f = m.dxb[r] * half * (UVH[ol] + UVH[ou]);
            if (!(wet(n, i, ju) && wet(n, i + 1, ju) && wet(n, i, jl) && wet(n, i + 1, jl))) f = zero;
        }
        n.flx[1][o] = f;
    }
    // NS flux of VH on the bottom edge of row r
    if (i < nx) {
        R f = zero;
        if (i <= nx - 2 && r <= ny - 1) {
            const int jm1 = (r - 1 > 0) ? r - 1 : 0;
            const int64_t om = (int64_t)jm1 * P + i;
            const R w = half * (m.dxb[r] + m.dxb[r + 1]);
            const R sm = vh[o] + vh[om];
            f = w * ((sm > zero) ? VVH[om] : VVH[o]);
            if (sm == zero) f = w * half * (VVH[om] + VVH[o]);
            if (!wet(n, i, r)) f = zero;
        }
        n.flx[2][o] = f;
    }
    // EW flux of VH at the west face of column i, rows 0..ny-2; column 0
    // takes column 1's upwind value before its tie and wet/dry treatment
    if (i < nx) {
        R f = zero;
        if (r <= ny - 2) {
            const int ic = (i >= 1) ? i : 1;
            const int64_t oc = (int64_t)r * P + ic;
            const R sm = uh[oc - 1] + uh[oc - 1 + P];
            f = m.dyl[ic - 1] * ((sm > zero) ? VUH[oc - 1] : VUH[oc]);
            if (i >= 1) {
                if (sm == zero) f = m.dyl[i - 1] * half * (VUH[oc - 1] + VUH[oc]);
                if (!(wet(n, i - 1, r) && wet(n, i, r) && wet(n, i - 1, r + 1) && wet(n, i, r + 1))) f = zero;
            }
        }
        n.flx[3][o] = f;
    }
}

template <typename R, bool SPH, bool COR>
__global__ void momentum_kernel(NLArgs<R> n)
{
    const LinArgs<R> &a = n.a;
    const int nx = a.p.nx, ny = a.p.ny;
    const int i = blockIdx.x * 32 + threadIdx.x, r = blockIdx.y * 8 + threadIdx.y;
    if (i >= nx || r >= ny) return;
    const int64_t P = a.p.pitch, o = (int64_t)r * P + i;
    const R *uh = a.p.uh, *vh = a.p.vh, *st = a.p.stg_o, *el = a.p.elv;
    if (i > nx - 2 || r > ny - 2) {
        a.p.uh_o[o] = uh[o];
        a.p.vh_o[o] = vh[o];
        return;
    }
    const R g = K<R>::gravity(), half = K<R>::half(), one = K<R>::one(), zero = K<R>::zero();
    const R mad = K<R>::min_depth();
    const R dt = a.dt;
    const R inv_cell_area_dt = dt / a.m.area[r];
    const R inv_cell_area_dt_g = g * inv_cell_area_dt;
    const R inv_cell_area_dt_vh = dt / (half * (a.m.area[r] + a.m.area[r + 1]));
    const R inv_cell_area_dt_vh_g = g * inv_cell_area_dt_vh;
    const int64_t oe = o + 1, on = o + P;
    R h_jph = half * ((st[on] + st[o]) - (el[on] + el[o]));
    if (h_jph < mad) h_jph = zero;
    R h_iph = half * ((st[oe] + st[o]) - (el[oe] + el[o]));
    if (h_iph < mad) h_iph = zero;
    const bool jw1 = st[on] > el[on] + mad, jw0 = st[o] > el[o] + mad;
    const R h_jph_wet_strict = (jw1 && jw0) ? one : zero;
    const R h_jph_wet = ((h_jph_wet_strict > zero) || (jw1 && st[on] > el[o] + mad) || (jw0 && st[o] > el[on] + mad))
                            ? one : zero;
    const bool iw1 = st[oe] > el[oe] + mad, iw0 = jw0;
    const R h_iph_wet_strict = (iw1 && iw0) ? one : zero;
    const R h_iph_wet = ((h_iph_wet_strict > zero) || (iw1 && st[oe] > el[o] + mad) || (iw0 && st[o] > el[oe] + mad))
                            ? one : zero;
    const int rm = (r > 0) ? r - 1 : 0, im = (i > 0) ? i - 1 : 0;
    const R vh_iph_jmh = half * (vh[(int64_t)rm * P + i] + vh[(int64_t)rm * P + i + 1]);
    const R vh_iph_jph = half * (vh[o] + vh[oe]);
    const R uh_i_j = half * (uh[o] + uh[(int64_t)r * P + im]);
    const R uh_i_jp1 = half * (uh[on] + uh[(int64_t)(r + 1) * P + im]);
    const R u0 = uh[o], v0 = vh[o];
    const R tv = half * (vh_iph_jmh + vh_iph_jph);
    const R tu = half * (uh_i_j + uh_i_jp1);
    const R fm_uh = one / ((one + a.lin_fric_dt) + dt * n.fw[o] * R(sqrt(u0 * u0 + tv * tv)));
    const R fm_vh = one / ((one + a.lin_fric_dt) + dt * n.fw[n.plane + o] * R(sqrt(v0 * v0 + tu * tu)));
    R u = u0 * h_iph_wet - inv_cell_area_dt_g * h_iph * h_iph_wet * (st[oe] - st[o]) * a.m.dyl[i + 1];
    R v = v0 * h_jph_wet - inv_cell_area_dt_vh_g * h_jph * h_jph_wet * (st[on] - st[o]) * a.m.dxb[r + 1];
    const R *F0 = n.flx[0], *F1 = n.flx[1], *F2 = n.flx[2], *F3 = n.flx[3];
    u = u - inv_cell_area_dt * R(1) * h_iph_wet * ((F0[oe] - F0[o]) + (F1[on] - F1[o]));
    v = v - inv_cell_area_dt_vh * R(1) * h_jph_wet * ((F3[oe] - F3[o]) + (F2[on] - F2[o]));
    if (COR) {
        const R dthc = dt * a.m.cor[r] * half * ((h_iph_wet_strict > zero) ? one : zero);
        const R dthc_jph = dt * a.m.cor_be[r + 1] * half * ((h_jph_wet_strict > zero) ? one : zero);
        u = u + dthc * (vh_iph_jmh + vh_iph_jph);
        v = v - dthc_jph * (uh_i_j + uh_i_jp1);
    }
    if (SPH) {
        R inv_depth_local = zero;
        if (h_iph_wet_strict > zero) inv_depth_local = one / h_iph;
        const R tan_uvh = dt * a.m.tanlat[r] * u0 * half * (vh_iph_jmh + vh_iph_jph) * inv_depth_local;
        inv_depth_local = zero;
        if (h_jph_wet_strict > zero) inv_depth_local = one / h_jph;
        const R tan_uuh = dt * half * (a.m.tanlat[r] + a.m.tanlat[r + 1]) * half * (uh_i_jp1 + uh_i_j) * half *
                          (uh_i_jp1 + uh_i_j) * inv_depth_local;
        u = u + tan_uvh;
        v = v - tan_uuh;
    }
    a.p.uh_o[o] = fm_uh * u;
    a.p.vh_o[o] = fm_vh * v;
}

// No outflow from dry cells (:855-880), per face.
template <typename R>
__global__ void dry_outflow_kernel(NLArgs<R> n)
{
    const int nx = n.a.p.nx, ny = n.a.p.ny;
    const int i = blockIdx.x * 32 + threadIdx.x, r = blockIdx.y * 8 + threadIdx.y;
    if (i >= nx || r > ny - 2) return;
    const int64_t P = n.a.p.pitch, o = (int64_t)r * P + i;
    const R mad = K<R>::min_depth();
    auto dry = [&](int64_t q) { return n.a.p.stg_o[q] < n.a.p.elv[q] + mad; };
    R u = n.a.p.uh_o[o], v = n.a.p.vh_o[o];
    if ((dry(o) && u > R(0)) || (i + 1 <= nx - 1 && dry(o + 1) && u < R(0))) n.a.p.uh_o[o] = R(0);
    if ((dry(o) && v > R(0)) || (dry(o + P) && v < R(0))) n.a.p.vh_o[o] = R(0);
}

}  // namespace nl

// one_leapfrog_nonlinear_step (timestepping_alternatives_include.f90:
// 439-447) on the whole domain.  c.nl_work holds the 9 work planes of
// pitch x (ny + 1) elements; c.fw the friction work.
template <typename R>
cudaError_t launch_leapfrog_nonlinear_step(const StepPlanes<R> &p, const Metrics<R> &m, const StepConfig &c, R dt,
                                           DevScalars *sc, cudaStream_t s, const LaunchHook &hook)
{
    LinArgs<R> a = make_args<R>(p, m, c, dt);
    a.xl = 0; a.xu = p.nx - 1; a.yl = 0; a.yu = p.ny - 1;   // the reference fixes the whole domain
    nl::NLArgs<R> n;
    n.a = a;
    n.nsq = p.manning_sq;
    const int64_t wplane = p.pitch * (int64_t)(p.ny + 1);
    R *w = (R *)c.nl_work;
    n.lag0 = w;
    for (int k = 0; k < 4; k++) n.adv[k] = w + (1 + k) * wplane;
    for (int k = 0; k < 4; k++) n.flx[k] = w + (5 + k) * wplane;
    n.fw = (const R *)c.fw;
    n.plane = p.pitch * (int64_t)p.ny;
    const dim3 block(32, 8), g1((p.nx + 31) / 32, (p.ny + 7) / 8), g2((p.nx + 32) / 32, (p.ny + 8) / 8);
    auto run = [&](int cat, auto &&launch) {
        hook(cat, 0);
        launch();
        hook(cat, 1);
    };
    run(CAT_LINEAR_EDGE, [&] { nl::lag0_kernel<R><<<g1, block, 0, s>>>(n); });
    run(CAT_LINEAR_EDGE, [&] { linear_edge_kernel<R><<<1, 512, 0, s>>>(a, sc, c.exterior_cells_width, c.bf); });
    run(CAT_LINEAR_MAIN, [&] { nl::stage_kernel<R><<<g1, block, 0, s>>>(n); });
    if (c.bc_kind == 3)   // flather_boundary
        run(CAT_LINEAR_EDGE, [&] {
            launch_leapfrog_boundary<R>(p.nx, p.ny, p.pitch, p.stg_o, const_cast<R *>(p.uh), const_cast<R *>(p.vh),
                                        p.elv, m, c, dt, sc, s);
        });
    if (c.n_forcing) {
        ForcingClock clk{};
        clk.mode = FORCE_LEAPFROG;
        clk.dt = (double)dt;
        launch_forcing<R>(c, clk, p.pitch, p.stg_o, const_cast<R *>(p.uh), const_cast<R *>(p.vh), p.elv, sc, s,
                          hook, CAT_LINEAR_EDGE);
    }
    run(CAT_LINEAR_EDGE, [&] {
        if (c.chezy)
            friction_work_kernel<R, true><<<g1, block, 0, s>>>(a, p.manning_sq, (R *)c.fw, 0, 1, 0, p.nx - 1, 0,
                                                               p.ny - 1);
        else
            friction_work_kernel<R, false><<<g1, block, 0, s>>>(a, p.manning_sq, (R *)c.fw, 0, 1, 0, p.nx - 1, 0,
                                                                p.ny - 1);
    });
    run(CAT_LINEAR_MAIN, [&] { nl::advection_kernel<R><<<g1, block, 0, s>>>(n); });
    run(CAT_LINEAR_MAIN, [&] { nl::flux_kernel<R><<<g2, block, 0, s>>>(n); });
    run(CAT_LINEAR_MAIN, [&] {
        if (c.spherical && c.coriolis) nl::momentum_kernel<R, true, true><<<g1, block, 0, s>>>(n);
        else if (c.spherical) nl::momentum_kernel<R, true, false><<<g1, block, 0, s>>>(n);
        else nl::momentum_kernel<R, false, false><<<g1, block, 0, s>>>(n);
    });
    run(CAT_LINEAR_MAIN, [&] { nl::dry_outflow_kernel<R><<<g1, block, 0, s>>>(n); });
    if (p.max_stage)
        run(CAT_MAXSTAGE, [&] {
            launch_update_max_stage<R>(p.nx, p.ny, p.pitch, p.stg_o, p.max_stage, c, s);
        });
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_linear_map(const StepPlanes<R> &p, const Metrics<R> &m, const StepConfig &c, R dt,
                              const int *sites, int n_sites, double *rec, cudaStream_t s, const LaunchHook &hook)
{
    LinArgs<R> a = make_args<R>(p, m, c, dt);
    a.bc_stage = 0;
    a.bc_fn_ring = 0;
    a.sites = sites;
    a.n_sites = n_sites;
    a.rec = rec;
    hook(CAT_LINEAR_MAIN, 0);
    const bool cor = c.coriolis != 0, tl = c.truely_linear != 0;
    constexpr int CPL = 16 / (int)sizeof(R);   // the aligned wide strips of the plain step
    if (cor && tl) launch_wide<R, true, true, CPL>(a, s);
    else if (cor && !tl) launch_wide<R, true, false, CPL>(a, s);
    else if (!cor && tl) launch_wide<R, false, true, CPL>(a, s);
    else launch_wide<R, false, false, CPL>(a, s);
    hook(CAT_LINEAR_MAIN, 1);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_linear_batch(const StepPlanes<R> &p0, int64_t inst_stride, int64_t max_stride, int nbatch,
                                const Metrics<R> &m, const StepConfig &c, R dt, int tile_cfg, cudaStream_t s,
                                const LaunchHook &hook)
{
    LinArgs<R> a = make_args<R>(p0, m, c, dt);
    a.bc_stage = 0;
    a.bc_fn_ring = 0;
    a.nbatch = nbatch;
    a.inst_stride = inst_stride;
    a.max_stride = max_stride;
    hook(CAT_LINEAR_MAIN, 0);
    launch_main<R>(a, c, tile_cfg, s);
    hook(CAT_LINEAR_MAIN, 1);
    return cudaGetLastError();
}

int linear_tile_config_count() { return kNumTileCfgs; }

bool linear_step_fuses_gauges(const StepConfig &c, int nx, int ny) { return fuses_gauges(c, nx, ny); }

bool linear_bulk_launched() { return g_bulk_launched.load(std::memory_order_relaxed); }

cudaError_t linear_wait_expired(unsigned *count, bool clear, cudaStream_t s)
{
    // the count of the stream's device (the caller's current device may differ)
    int cur = 0, dev = 0;
    cudaError_t e = cudaGetDevice(&cur);
    if (e == cudaSuccess && s) e = cudaStreamGetDevice(s, &dev);
    else dev = cur;
    if (e != cudaSuccess) return e;
    if (dev != cur && (e = cudaSetDevice(dev)) != cudaSuccess) return e;
    struct Restore {
        int d, c;
        ~Restore() { if (d != c) cudaSetDevice(c); }
    } restore{dev, cur};
    void *addr = nullptr;
    e = cudaGetSymbolAddress(&addr, g_linear_wait_expired);
    if (e != cudaSuccess) return e;
    unsigned h = 0;
    e = cudaMemcpyAsync(&h, addr, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && clear && h) {
        e = cudaMemsetAsync(addr, 0, sizeof(h), s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (count) *count = h;
    return e;
}

template <typename R>
cudaError_t launch_update_max_stage(int nx, int ny, int64_t pitch, const R *stg, R *max_stage, const StepConfig &c,
                                    cudaStream_t s)
{
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8);
    max_stage_kernel<R><<<grid, block, 0, s>>>(nx, ny, pitch, stg, max_stage, c.xl, c.xu, c.yl, c.yu, nullptr, 1);
    return cudaGetLastError();
}

// Static steps (static_before_time, domain_mod.f90:1706-1716): the clock
// advances by the step's dt (when given) and the step is counted; nothing
// else changes.
__global__ void static_step_kernel(DevScalars *sc, double dt, int has_dt)
{
    const double time0 = sc->time;
    sc->time0 = time0;
    if (has_dt) sc->time = sc->time + dt;
    sc->boundary_flux_evolve_integral = 0.0;
    sc->boundary_flux_time_integral = sc->boundary_flux_time_integral + 0.0;
    sc->evolve_step_dt = sc->time - time0;
    sc->nsteps_advanced += 1;
}

cudaError_t launch_static_step(DevScalars *sc, double dt, int has_dt, cudaStream_t s)
{
    static_step_kernel<<<1, 1, 0, s>>>(sc, dt, has_dt);
    return cudaGetLastError();
}

// update_max_quantities with the optional max_U_variables
// (domain_mod.f90:2243-2404), one thread per cell of xL..xU x yL..yU, after
// a step (gated like max_stage_kernel) or before the first one (every 1).
template <typename R>
__global__ void max_u_kernel(int nx, int ny, int64_t P, const R *stg, const R *uh, const R *vh, const R *elv,
                             R *max_stage, int xl, int xu, int yl, int yu, MaxUConfig mu, R msl,
                             const DevScalars *sc, int every)
{
    if (every > 1 && (sc->nsteps_advanced - 1) % every != 0) return;
    if (every == 0 && sc->nsteps_advanced != 0) return;   // before the first step only
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (i < xl || i > xu || r < yl || r > yu || i >= nx || r >= ny) return;
    const int64_t o = (int64_t)r * P + i;
    const R mad = K<R>::min_depth(), zero = R(0), one = R(1), half = K<R>::half();
    const R s = stg[o], e = elv[o];
    const bool ok = mu.include_dry || (s > e + mad);
    R *pl = (R *)mu.planes;
    const int64_t q = (int64_t)r * nx + i;   // extra planes: nx x ny, i fastest
    if (mu.mask & 1) {
        if (s > max_stage[o] && ok) {
            max_stage[o] = s;
            pl[q] = R(sc->time);
        }
    } else if (ok) {
        const R m = max_stage[o];
        max_stage[o] = (s > m) ? s : m;
    }
    if (mu.mask & 2) {
        R v;
        if (mu.staggered) {
            // 0.5 * sum(x(i:ip1)) with ip1 = min(i+1, nx): on the last column
            // (row) the slice holds the cell alone, so the face depth is half
            // the cell's own depth.
            const bool has_e = (i + 1 < nx), has_n = (r + 1 < ny);
            const int64_t oe = (int64_t)r * P + (has_e ? i + 1 : i), on = (int64_t)(has_n ? r + 1 : r) * P + i;
            R de, dn;
            if (mu.truely_linear) {
                de = has_e ? half * ((msl - e) + (msl - elv[oe])) : half * (msl - e);
                dn = has_n ? half * ((msl - e) + (msl - elv[on])) : half * (msl - e);
            } else {
                de = has_e ? half * ((s - e) + (stg[oe] - elv[oe])) : half * (s - e);
                dn = has_n ? half * ((s - e) + (stg[on] - elv[on])) : half * (s - e);
            }
            const R dei = (de > mad) ? one / de : zero, dni = (dn > mad) ? one / dn : zero;
            const R u = uh[o], w = vh[o];
            v = R(sqrt(u * u * (dei * dei) + w * w * (dni * dni)));
        } else {
            const R ld = s - e;
            const R ldi = (ld > mad) ? one / ld : zero;
            const R u = uh[o], w = vh[o];
            v = R(sqrt((u * u + w * w) * (ldi * ldi)));
        }
        R *m = pl + mu.plane;
        m[q] = (v > m[q]) ? v : m[q];
    }
    if (mu.mask & 4) {
        const R u = uh[o], w = vh[o];
        const R v = R(sqrt(u * u + w * w));
        R *m = pl + 2 * mu.plane;
        m[q] = (v > m[q]) ? v : m[q];
    }
    if (mu.mask & 8) {
        R *m = pl + 3 * mu.plane;
        if ((s - e) > mad && s > R(mu.arrival) && m[q] < zero) m[q] = R(sc->time);
    }
    if (mu.mask & 16) {
        R *m = pl + 4 * mu.plane;
        if (ok) m[q] = (s < m[q]) ? s : m[q];
    }
}

template <typename R>
cudaError_t launch_update_max_u(int nx, int ny, int64_t pitch, const R *stg, const R *uh, const R *vh, const R *elv,
                                R *max_stage, const StepConfig &c, const MaxUConfig &mu, const DevScalars *sc,
                                int every, cudaStream_t s)
{
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8);
    max_u_kernel<R><<<grid, block, 0, s>>>(nx, ny, pitch, stg, uh, vh, elv, max_stage, c.xl, c.xu, c.yl, c.yu, mu,
                                           R(c.msl_linear), sc, every);
    return cudaGetLastError();
}
template cudaError_t launch_update_max_u<double>(int, int, int64_t, const double *, const double *, const double *,
                                                 const double *, double *, const StepConfig &, const MaxUConfig &,
                                                 const DevScalars *, int, cudaStream_t);
template cudaError_t launch_update_max_u<float>(int, int, int64_t, const float *, const float *, const float *,
                                                const float *, float *, const StepConfig &, const MaxUConfig &,
                                                const DevScalars *, int, cudaStream_t);

template <typename R>
cudaError_t launch_update_max_stage_every(int nx, int ny, int64_t pitch, const R *stg, R *max_stage,
                                          const StepConfig &c, const DevScalars *sc, int every, cudaStream_t s)
{
    dim3 block(32, 8);
    dim3 grid((nx + 31) / 32, (ny + 7) / 8);
    max_stage_kernel<R><<<grid, block, 0, s>>>(nx, ny, pitch, stg, max_stage, c.xl, c.xu, c.yl, c.yu, sc, every);
    return cudaGetLastError();
}
template cudaError_t launch_update_max_stage_every<double>(int, int, int64_t, const double *, double *,
                                                           const StepConfig &, const DevScalars *, int, cudaStream_t);
template cudaError_t launch_update_max_stage_every<float>(int, int, int64_t, const float *, float *,
                                                          const StepConfig &, const DevScalars *, int, cudaStream_t);

template <typename R>
cudaError_t launch_gauges(int64_t pitch, const R *stg, const R *uh, const R *vh, const int *site_ij, int n,
                          double *records, int capacity, DevScalars *sc, cudaStream_t s)
{
    gauge_kernel<R><<<1, 256, 0, s>>>(pitch, stg, uh, vh, site_ij, n, records, capacity, sc);
    return cudaGetLastError();
}

template cudaError_t launch_leapfrog_nonlinear_step<double>(const StepPlanes<double> &, const Metrics<double> &,
                                                             const StepConfig &, double, DevScalars *, cudaStream_t,
                                                             const LaunchHook &);
template cudaError_t launch_leapfrog_nonlinear_step<float>(const StepPlanes<float> &, const Metrics<float> &,
                                                            const StepConfig &, float, DevScalars *, cudaStream_t,
                                                            const LaunchHook &);
template cudaError_t launch_linear_step<double>(const StepPlanes<double> &, const Metrics<double> &,
                                                const StepConfig &, double, DevScalars *, cudaStream_t,
                                                const LaunchHook &, const AuxStream *);
template cudaError_t launch_linear_step<float>(const StepPlanes<float> &, const Metrics<float> &,
                                               const StepConfig &, float, DevScalars *, cudaStream_t,
                                               const LaunchHook &, const AuxStream *);
template cudaError_t launch_linear_map<double>(const StepPlanes<double> &, const Metrics<double> &,
                                               const StepConfig &, double, const int *, int, double *, cudaStream_t,
                                               const LaunchHook &);
template cudaError_t launch_linear_map<float>(const StepPlanes<float> &, const Metrics<float> &, const StepConfig &,
                                              float, const int *, int, double *, cudaStream_t, const LaunchHook &);
template cudaError_t launch_linear_batch<double>(const StepPlanes<double> &, int64_t, int64_t, int,
                                                 const Metrics<double> &, const StepConfig &, double, int,
                                                 cudaStream_t, const LaunchHook &);
template cudaError_t launch_linear_batch<float>(const StepPlanes<float> &, int64_t, int64_t, int,
                                                const Metrics<float> &, const StepConfig &, float, int, cudaStream_t,
                                                const LaunchHook &);
template cudaError_t launch_update_max_stage<double>(int, int, int64_t, const double *, double *,
                                                     const StepConfig &, cudaStream_t);
template cudaError_t launch_update_max_stage<float>(int, int, int64_t, const float *, float *,
                                                    const StepConfig &, cudaStream_t);
template cudaError_t launch_gauges<double>(int64_t, const double *, const double *, const double *, const int *,
                                           int, double *, int, DevScalars *, cudaStream_t);
template cudaError_t launch_gauges<float>(int64_t, const float *, const float *, const float *, const int *, int,
                                          double *, int, DevScalars *, cudaStream_t);

}  // namespace swals
