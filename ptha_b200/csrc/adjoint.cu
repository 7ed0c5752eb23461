// adjoint.cu -- discrete adjoint of the truly linear leapfrog step.
//
// The truly linear step of domain_mod_linear_solver_include.f90:58-571 (no
// boundary routine, fixed dt) is a linear map x' = M x on x = (STG, UH, VH):
//   stage:    S'(i,j) = S - dt/A_j [(U(i)-U(i-1)) dyl_i + V(j) dxb_{j+1} - V(j-1) dxb_j]   (interior IS)
//   momentum: U'(i,j) = m [U - gdt/A_j hU (S'(i+1)-S'(i)) dyl_{i+1} + cU (4 old V)]       (region IM)
//             V'(i,j) = m [V - gdt/A_{j+1/2} hV (S'(j+1)-S'(j)) dxb_{j+1} - cV (4 old U)]
// with the face depths hU, hV fixed by ELV, the Coriolis 2-point averages
// clamped at i=1, j=1 as in the reference, and m the implicit linear-friction
// factor.  This file applies M^T without atomics: one CTA gathers, for its
// tile, the momentum-transpose contributions, forms the total stage adjoint
// on the tile plus an east/north halo, then applies the stage transpose.
// Reads lambda' (3 planes) and ELV, writes lambda (3 planes): the same 56 B
// per cell (FP64) as a forward step.
//
// The reference has no adjoint; its correctness is checked by the
// dot-product identity <M d, l> = <d, M^T l>, by central finite differences
// of the oracle's forward model and by the oracle forward as tangent linear.
#include "domain_internal.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

constexpr int ABX = 32;
constexpr int ABY = 16;
constexpr int ATY = 8;

template <typename R>
struct AdjArgs {
    int nx, ny;
    int64_t P;
    const R *ls, *lu, *lv;   // adjoint of the step's outputs
    R *ls_o, *lu_o, *lv_o;   // adjoint of the step's inputs
    const R *elv;
    swals::Metrics<R> m;
    int xl, xu, yl, yu;
    R dt, msl, mult;         // mult: linear friction factor (1 without friction)
};

__device__ __forceinline__ bool in_im(int i, int r, int xl, int xu, int yl, int yu)
{
    return i >= xl && i <= xu - 1 && r >= yl && r <= yu - 1;
}
__device__ __forceinline__ bool in_is(int i, int r, int xl, int xu, int yl, int yu)
{
    return i >= xl + 1 && i <= xu - 1 && r >= yl + 1 && r <= yu - 1;
}

template <typename R, bool COR>
__global__ void __launch_bounds__(ABX *ATY) linear_adjoint_kernel(const AdjArgs<R> a)
{
    constexpr int W = ABX + 2;   // window columns i0-1 .. i0+ABX
    constexpr int H = ABY + 2;   // window rows    r0-1 .. r0+ABY
    constexpr int NT = ABX * ATY;
    __shared__ R s_lu[H][W], s_lv[H][W], s_ls[H][W];
    __shared__ R s_el[H + 1][W + 1];
    __shared__ R s_aU[H][W], s_aV[H][W], s_cU[H][W], s_cV[H][W];
    __shared__ R s_lst[ABY + 1][ABX + 1];

    const int nx = a.nx, ny = a.ny;
    const int64_t P = a.P;
    const int i0 = blockIdx.x * ABX, r0 = blockIdx.y * ABY;
    const int tid = threadIdx.y * ABX + threadIdx.x;
    const R g = swals::K<R>::gravity(), half = R(0.5), mad = swals::K<R>::min_depth(), zero = R(0), one = R(1);

    for (int q = tid; q < H * W; q += NT) {
        const int rr = q / W, cc = q - rr * W;
        const int r = r0 - 1 + rr, i = i0 - 1 + cc;
        R lu = zero, lv = zero, ls = zero;
        if (r >= 0 && r < ny && i >= 0 && i < nx) {
            const int64_t o = (int64_t)r * P + i;
            lu = a.lu[o]; lv = a.lv[o]; ls = a.ls[o];
        }
        s_lu[rr][cc] = lu; s_lv[rr][cc] = lv; s_ls[rr][cc] = ls;
    }
    for (int q = tid; q < (H + 1) * (W + 1); q += NT) {
        const int rr = q / (W + 1), cc = q - rr * (W + 1);
        const int r = r0 - 1 + rr, i = i0 - 1 + cc;
        s_el[rr][cc] = (r >= 0 && r < ny && i >= 0 && i < nx) ? a.elv[(int64_t)r * P + i] : zero;
    }
    __syncthreads();

    // Face coefficients of the momentum update on the window (zero outside IM).
    for (int q = tid; q < H * W; q += NT) {
        const int rr = q / W, cc = q - rr * W;
        const int r = r0 - 1 + rr, i = i0 - 1 + cc;
        R aU = zero, aV = zero, cU = zero, cV = zero;
        if (r >= 0 && r < ny && i >= 0 && i < nx && in_im(i, r, a.xl, a.xu, a.yl, a.yu)) {
            const R e0 = s_el[rr][cc], e_e = s_el[rr][cc + 1], e_n = s_el[rr + 1][cc];
            const bool wi = (e0 < -mad + a.msl) && (e_e < -mad + a.msl);
            const R hU = wi ? (a.msl - half * (e_e + e0)) : zero;
            const bool wj = (e_n < -mad + a.msl) && (e0 < -mad + a.msl);
            const R hV = wj ? (a.msl - half * (e_n + e0)) : zero;
            const R gU = g * a.dt / a.m.area[r];
            const R gV = g * a.dt / (half * (a.m.area[r] + a.m.area[r + 1]));
            aU = a.mult * (gU * hU * a.m.dyl[i + 1]);
            aV = a.mult * (gV * hV * a.m.dxb[r + 1]);
            if (COR) {
                cU = a.mult * (a.dt * a.m.cor[r] * half * ((hU > zero) ? one : zero)) * half;
                cV = a.mult * (a.dt * a.m.cor_be[r + 1] * half * ((hV > zero) ? one : zero)) * half;
            }
        }
        s_aU[rr][cc] = aU; s_aV[rr][cc] = aV; s_cU[rr][cc] = cU; s_cV[rr][cc] = cV;
    }
    __syncthreads();

    // Total adjoint of the new stage on the tile plus east/north halo.
    for (int q = tid; q < (ABY + 1) * (ABX + 1); q += NT) {
        const int rr = q / (ABX + 1), cc = q - rr * (ABX + 1);
        const int w = cc + 1, h = rr + 1;
        s_lst[rr][cc] = s_ls[h][w] + s_aU[h][w] * s_lu[h][w] + s_aV[h][w] * s_lv[h][w]
                        - s_aU[h][w - 1] * s_lu[h][w - 1] - s_aV[h - 1][w] * s_lv[h - 1][w];
    }
    __syncthreads();

#pragma unroll
    for (int k = 0; k < ABY / ATY; k++) {
        const int rr = threadIdx.y + k * ATY, cc = threadIdx.x;
        const int r = r0 + rr, i = i0 + cc;
        if (r >= ny || i >= nx) continue;
        const int w = cc + 1, h = rr + 1;
        const R idm = in_im(i, r, a.xl, a.xu, a.yl, a.yu) ? a.mult : one;
        R lU = idm * s_lu[h][w];
        R lV = idm * s_lv[h][w];
        if (COR) {
            // V'(i',r') uses U(i,r) through 1/2 (U(i') + U(max(i'-1,0))) at rows r' and r'+1.
#pragma unroll
            for (int dr = 0; dr >= -1; dr--) {
#pragma unroll
                for (int di = 0; di <= 1; di++) {
                    const int ip = i + di;
                    const R cnt = R((ip == i) ? 1 : 0) + R(((ip - 1 > 0 ? ip - 1 : 0) == i) ? 1 : 0);
                    lU = lU - s_cV[h + dr][w + di] * cnt * s_lv[h + dr][w + di];
                }
            }
            // U'(i',r') uses V(i,r) through 1/2 (V(i') + V(i'+1)) at rows max(r'-1,0) and r'.
#pragma unroll
            for (int dr = 0; dr <= 1; dr++) {
#pragma unroll
                for (int di = -1; di <= 0; di++) {
                    const int rp = r + dr;
                    const R cnt = R((rp == r) ? 1 : 0) + R(((rp - 1 > 0 ? rp - 1 : 0) == r) ? 1 : 0);
                    lV = lV + s_cU[h + dr][w + di] * cnt * s_lu[h + dr][w + di];
                }
            }
        }
        const R lst = s_lst[rr][cc];
        const R c_r = a.dt / a.m.area[r];
        if (in_is(i, r, a.xl, a.xu, a.yl, a.yu)) {
            lU = lU - c_r * a.m.dyl[i] * lst;
            lV = lV - c_r * a.m.dxb[r + 1] * lst;
        }
        if (in_is(i + 1, r, a.xl, a.xu, a.yl, a.yu)) lU = lU + c_r * a.m.dyl[i + 1] * s_lst[rr][cc + 1];
        if (in_is(i, r + 1, a.xl, a.xu, a.yl, a.yu)) lV = lV + (a.dt / a.m.area[r + 1]) * a.m.dxb[r + 1] * s_lst[rr + 1][cc];
        const int64_t o = (int64_t)r * P + i;
        a.ls_o[o] = lst;
        a.lu_o[o] = lU;
        a.lv_o[o] = lV;
    }
}

// Streaming form of the same transpose (the forward's register-row design):
// a warp owns 30 columns (lanes 1..30; lanes 0 and 31 carry the neighbour
// columns) and marches down SH rows.  Rows r+2 and r+3 are in flight while
// row r is produced: row r+1's face coefficients and total stage adjoint are
// formed from rows r+1 and r+2, then row r's outputs from rows r-1..r+1.
// Values outside the domain are zero, as in the tile kernel, and every
// expression keeps the tile kernel's order.  With `resid` set, the gauge
// adjoint of this step (lambda_STG(site) += resid[g], gauges in order) is
// added where lambda_STG is loaded, so no separate injection launch is needed.
constexpr int AOUT = 30;

template <typename R>
struct ARow { R ls, lu, lv, e, ee; };  // ee: ELV one column east

template <typename R>
struct ACoef { R aU, aV, cU, cV; };

template <typename R, bool COR>
__global__ void __launch_bounds__(128) linear_adjoint_stream_kernel(const AdjArgs<R> a, int SH, int nstrips, int total,
                                                                    const int *sites, int ng, const double *resid)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int nx = a.nx, ny = a.ny;
    const int64_t P = a.P;
    const R g = swals::K<R>::gravity(), half = R(0.5), mad = swals::K<R>::min_depth(), zero = R(0), one = R(1);

    for (int w = blockIdx.x * 4 + (threadIdx.x >> 5); w < total; w += gridDim.x * 4) {
        const int sx = w % nstrips, sy = w / nstrips;
        const int ra = sy * SH, rb = min(ra + SH, ny);
        const int i = sx * AOUT - 1 + lane;
        const bool in_x = (i >= 0 && i < nx);
        const bool out = (lane >= 1 && lane <= AOUT && i < nx);
        // Gauges whose adjoint is injected into the rows this warp loads.
        const unsigned long long gmask =
            resid ? swals::gauges_in(sites, ng, sx * AOUT - 1, sx * AOUT + AOUT, ra - 1, rb + 2) : 0ull;

        auto load = [&](int r) -> ARow<R> {
            ARow<R> v;
            v.ls = v.lu = v.lv = v.e = v.ee = zero;
            if (in_x && r >= 0 && r < ny) {
                const int64_t o = (int64_t)r * P + i;
                v.ls = a.ls[o]; v.lu = a.lu[o]; v.lv = a.lv[o]; v.e = a.elv[o];
                if (i + 1 < nx) v.ee = a.elv[o + 1];
                if (gmask) {
                    if (ng > 64) {
                        for (int q = 0; q < ng; q++)
                            if (sites[2 * q] == i && sites[2 * q + 1] == r) v.ls = v.ls + R(resid[q]);
                    } else {
                        for (unsigned long long m = gmask; m; m &= m - 1) {
                            const int q = __ffsll((long long)m) - 1;
                            if (sites[2 * q] == i && sites[2 * q + 1] == r) v.ls = v.ls + R(resid[q]);
                        }
                    }
                }
            }
            return v;
        };
        // Row constants g dt/area(r), g dt/mean area(r, r+1) and dt/area(r),
        // the same in every lane: lane L evaluates them for row base + L of
        // a 32-row chunk, and the rows take them by shuffle (the same
        // divisions, once per row instead of once per cell).
        int base = ra - 1;
        R f_gu = zero, f_gv = zero, f_c = zero;
        auto chunk = [&](int b) {
            base = b;
            const int rr = min(max(b + lane, 0), ny - 1);
            const int rn = min(rr + 1, ny - 1);
            f_gu = g * a.dt / a.m.area[rr];
            f_gv = g * a.dt / (half * (a.m.area[rr] + a.m.area[rn]));
            f_c = a.dt / a.m.area[rr];
        };
        chunk(ra - 1);
        // Face coefficients of row r from its ELV and the ELV of row r+1 (zero outside IM).
        auto coef = [&](int r, R e0, R e_e, R e_n) -> ACoef<R> {
            ACoef<R> c;
            c.aU = c.aV = c.cU = c.cV = zero;
            const R gU = __shfl_sync(FULL, f_gu, r - base);
            const R gV = __shfl_sync(FULL, f_gv, r - base);
            if (in_x && r >= 0 && r < ny && in_im(i, r, a.xl, a.xu, a.yl, a.yu)) {
                const bool wi = (e0 < -mad + a.msl) && (e_e < -mad + a.msl);
                const R hU = wi ? (a.msl - half * (e_e + e0)) : zero;
                const bool wj = (e_n < -mad + a.msl) && (e0 < -mad + a.msl);
                const R hV = wj ? (a.msl - half * (e_n + e0)) : zero;
                c.aU = a.mult * (gU * hU * a.m.dyl[i + 1]);
                c.aV = a.mult * (gV * hV * a.m.dxb[r + 1]);
                if (COR) {
                    c.cU = a.mult * (a.dt * a.m.cor[r] * half * ((hU > zero) ? one : zero)) * half;
                    c.cV = a.mult * (a.dt * a.m.cor_be[r + 1] * half * ((hV > zero) ? one : zero)) * half;
                }
            }
            return c;
        };
        // Total stage adjoint of row r from rows r (value, coefficients) and r-1.
        auto lst_of = [&](const ARow<R> &v, const ACoef<R> &c, R aV_s, R lv_s) -> R {
            const R pw = __shfl_up_sync(FULL, c.aU * v.lu, 1);
            return v.ls + c.aU * v.lu + c.aV * v.lv - pw - aV_s * lv_s;
        };

        // Prologue: rows ra-1 .. ra+2 loaded, coefficients of rows ra-1 and ra,
        // total stage adjoint of row ra.
        ARow<R> vm = load(ra - 1), v0 = load(ra), v1 = load(ra + 1), v2 = load(ra + 2);
        ACoef<R> cm = coef(ra - 1, vm.e, vm.ee, v0.e);
        ACoef<R> c0 = coef(ra, v0.e, v0.ee, v1.e);
        R lst0 = lst_of(v0, c0, cm.aV, vm.lv);

        for (int r = ra; r < rb; r++) {
            if (r + 1 - base > 31) chunk(r);   // warp-uniform
            const ARow<R> v3 = load(r + 3);
            const ACoef<R> c1 = coef(r + 1, v1.e, v1.ee, v2.e);
            const R lst1 = lst_of(v1, c1, c0.aV, v0.lv);

            const R lst_e = __shfl_down_sync(FULL, lst0, 1);
            const R cvlv_e0 = __shfl_down_sync(FULL, c0.cV * v0.lv, 1);   // (cV*1)*lV at (i+1, r)
            const R cvlv_em = __shfl_down_sync(FULL, cm.cV * vm.lv, 1);   // at (i+1, r-1)
            const R culu_w0 = __shfl_up_sync(FULL, c0.cU * v0.lu, 1);     // at (i-1, r)
            const R culu_w1 = __shfl_up_sync(FULL, c1.cU * v1.lu, 1);     // at (i-1, r+1)
            const R c_r = __shfl_sync(FULL, f_c, r - base);              // dt / area(r)
            const R c_r1 = __shfl_sync(FULL, f_c, r + 1 - base);         // dt / area(r+1)
            if (out) {
                const R idm = in_im(i, r, a.xl, a.xu, a.yl, a.yu) ? a.mult : one;
                R lU = idm * v0.lu;
                R lV = idm * v0.lv;
                if (COR) {
                    // U'(i',r') and V'(i',r') terms in the tile kernel's order;
                    // (c * cnt) * l with cnt in {1, 2} equals cnt * (c * l).
                    const R cnt_i = R(1) + R((i == 0) ? 1 : 0);
                    lU = lU - c0.cV * cnt_i * v0.lv;
                    lU = lU - cvlv_e0;
                    lU = lU - cm.cV * cnt_i * vm.lv;
                    lU = lU - cvlv_em;
                    const R cnt_r = R(1) + R((r == 0) ? 1 : 0);
                    lV = lV + cnt_r * culu_w0;
                    lV = lV + c0.cU * cnt_r * v0.lu;
                    lV = lV + culu_w1;
                    lV = lV + c1.cU * R(1) * v1.lu;
                }
                if (in_is(i, r, a.xl, a.xu, a.yl, a.yu)) {
                    lU = lU - c_r * a.m.dyl[i] * lst0;
                    lV = lV - c_r * a.m.dxb[r + 1] * lst0;
                }
                if (in_is(i + 1, r, a.xl, a.xu, a.yl, a.yu)) lU = lU + c_r * a.m.dyl[i + 1] * lst_e;
                if (in_is(i, r + 1, a.xl, a.xu, a.yl, a.yu)) lV = lV + c_r1 * a.m.dxb[r + 1] * lst1;
                const int64_t o = (int64_t)r * P + i;
                a.ls_o[o] = lst0;
                a.lu_o[o] = lU;
                a.lv_o[o] = lV;
            }
            vm = v0; v0 = v1; v1 = v2; v2 = v3;
            cm = c0; c0 = c1;
            lst0 = lst1;
        }
    }
}

// lambda_STG(site) += weight * gauge adjoint, one thread (sites may repeat).
template <typename R>
__global__ void inject_kernel(R *ls, int64_t P, const int *site_ij, int n, const double *gadj)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int g = 0; g < n; g++) {
        const int64_t o = (int64_t)site_ij[2 * g + 1] * P + site_ij[2 * g];
        ls[o] = ls[o] + R(gadj[g]);
    }
}

// Kernel choice: streaming unless SWALS_ADJOINT_KERNEL=tile.
bool adjoint_tile()
{
    static int t = -1;
    if (t < 0) {
        const char *e = getenv("SWALS_ADJOINT_KERNEL");
        t = (e && strcmp(e, "tile") == 0) ? 1 : 0;
    }
    return t == 1;
}

// One adjoint step lambda_out = M^T (lambda_in + C^T resid): with `resid`
// (n gauges at `sites`) the injection is fused into the streaming kernel.
template <typename R>
cudaError_t adjoint_step(swals_domain *d, R *const in[3], R *const out[3], double dt, const int *sites = nullptr,
                         int ng = 0, const double *resid = nullptr)
{
    AdjArgs<R> a;
    a.nx = d->nx; a.ny = d->ny; a.P = d->pitch;
    a.ls = in[0]; a.lu = in[1]; a.lv = in[2];
    a.ls_o = out[0]; a.lu_o = out[1]; a.lv_o = out[2];
    a.elv = (const R *)d->elv;
    a.m = swals::metrics_of<R>(d);
    a.xl = d->cfg.xl; a.xu = d->cfg.xu; a.yl = d->cfg.yl; a.yu = d->cfg.yu;
    a.dt = R(dt);
    a.msl = R(d->cfg.msl_linear);
    const R lfc = R(d->cfg.linear_friction_coeff);
    a.mult = (lfc != R(0)) ? (R(1) / (R(1) + a.dt * lfc)) : R(1);
    swals::LaunchHook hook = swals::hook_of(d);
    if (adjoint_tile()) {
        if (resid && ng > 0) {
            inject_kernel<R><<<1, 32, 0, d->stream>>>(const_cast<R *>(in[0]), d->pitch, sites, ng, resid);
            d->launches++;
        }
        dim3 block(ABX, ATY), grid((d->nx + ABX - 1) / ABX, (d->ny + ABY - 1) / ABY);
        hook(swals::CAT_LINEAR_MAIN, 0);
        if (d->cfg.coriolis) linear_adjoint_kernel<R, true><<<grid, block, 0, d->stream>>>(a);
        else linear_adjoint_kernel<R, false><<<grid, block, 0, d->stream>>>(a);
        hook(swals::CAT_LINEAR_MAIN, 1);
        return cudaGetLastError();
    }
    // Rows per segment: up to 128, while every SM still gets about 24 warps.
    const int nstrips = (d->nx + AOUT - 1) / AOUT;
    int sh = 128;
    while (sh > 8 && (int64_t)nstrips * ((d->ny + sh - 1) / sh) < 148 * 24) sh /= 2;
    const int total = nstrips * ((d->ny + sh - 1) / sh);
    const int gx = std::min((total + 3) / 4, 1 << 20);
    hook(swals::CAT_LINEAR_MAIN, 0);
    if (d->cfg.coriolis)
        linear_adjoint_stream_kernel<R, true><<<gx, 128, 0, d->stream>>>(a, sh, nstrips, total, sites, ng, resid);
    else
        linear_adjoint_stream_kernel<R, false><<<gx, 128, 0, d->stream>>>(a, sh, nstrips, total, sites, ng, resid);
    hook(swals::CAT_LINEAR_MAIN, 1);
    return cudaGetLastError();
}

// The domain's adjoint scratch, grown to at least `need` bytes.
cudaError_t workspace(swals_domain *d, size_t need, void **out)
{
    if (d->ws_bytes < need) {
        cudaStreamSynchronize(d->stream);
        if (d->ws) cudaFree(d->ws);
        d->ws = nullptr;
        d->ws_bytes = 0;
        cudaError_t e = cudaMalloc(&d->ws, need);
        if (e != cudaSuccess) return e;
        d->ws_bytes = need;
    }
    *out = d->ws;
    return cudaSuccess;
}

int check_adjoint_domain(swals_domain *d)
{
    if (strncmp(d->desc.timestepping_method, "linear", 6) != 0 || d->desc.timestepping_method[6] > ' ')
        return swals::api_fail(SWALS_ERR_UNSUPPORTED, "the adjoint is implemented for timestepping_method='linear'");
    if (!d->cfg.truely_linear)
        return swals::api_fail(SWALS_ERR_UNSUPPORTED, "the adjoint needs linear_solver_is_truely_linear=.true.");
    if (d->cfg.n_forcing)
        return swals::api_fail(SWALS_ERR_UNSUPPORTED, "forcing patches are not supported here");
    if (d->cfg.bc_kind != SWALS_BC_NONE)
        return swals::api_fail(SWALS_ERR_UNSUPPORTED, "the adjoint supports walls via elevation only");
    return SWALS_OK;
}

int copy_plane3(swals_domain *d, void *dev3[3], void *host, bool to_dev)
{
    const size_t es = d->fp64 ? 8 : 4;
    for (int v = 0; v < 3; v++) {
        char *h = (char *)host + (size_t)v * d->nx * d->ny * es;
        cudaError_t e;
        if (to_dev)
            e = cudaMemcpy2DAsync(dev3[v], d->pitch * es, h, d->nx * es, d->nx * es, d->ny, cudaMemcpyHostToDevice,
                                  d->stream);
        else
            e = cudaMemcpy2DAsync(h, d->nx * es, dev3[v], d->pitch * es, d->nx * es, d->ny, cudaMemcpyDeviceToHost,
                                  d->stream);
        if (e != cudaSuccess) return swals::api_cuda_fail(e, "adjoint copy");
    }
    cudaError_t e = cudaStreamSynchronize(d->stream);
    if (e != cudaSuccess) return swals::api_cuda_fail(e, "adjoint copy sync");
    return SWALS_OK;
}

// Pure adjoint sweep: lambda_N+1 = 0; for n = N..1: lambda += C^T g_n;
// lambda = M^T lambda.  Returns lambda_0 = dL/dx_0.
template <typename R>
int adjoint_sweep(swals_domain *d, int nsteps, double dt, const double *gadj_host, void *grad_host,
                  const void *lambda_seed_host)
{
    const int64_t plane = d->pitch * (int64_t)d->ny;
    const size_t es = sizeof(R);
    const int ng = d->n_gauges > 0 ? d->n_gauges : (int)(d->h_sites.size() / 2);
    void *buf = nullptr;
    const size_t need = 6 * plane * es + sizeof(double) * (size_t)nsteps * (ng > 0 ? ng : 1) + 2 * sizeof(int) * (ng + 1);
    cudaError_t e = workspace(d, need, &buf);
    if (e != cudaSuccess) return swals::api_cuda_fail(e, "adjoint workspace");
    R *lam[2][3];
    for (int b = 0; b < 2; b++)
        for (int v = 0; v < 3; v++) lam[b][v] = (R *)buf + (b * 3 + v) * plane;
    double *d_g = (double *)((char *)buf + 6 * plane * es);
    int *d_sites = (int *)(d_g + (size_t)nsteps * (ng > 0 ? ng : 1));
    int rc = SWALS_OK;
    e = cudaMemsetAsync(buf, 0, 6 * plane * es, d->stream);
    if (e == cudaSuccess && ng > 0) {
        e = cudaMemcpyAsync(d_g, gadj_host, sizeof(double) * (size_t)nsteps * ng, cudaMemcpyHostToDevice, d->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_sites, d->h_sites.data(), sizeof(int) * 2 * ng, cudaMemcpyHostToDevice, d->stream);
    }
    if (e != cudaSuccess) rc = swals::api_cuda_fail(e, "adjoint setup");
    int cur = 0;
    if (rc == SWALS_OK && lambda_seed_host) {
        void *dst[3] = {lam[0][0], lam[0][1], lam[0][2]};
        rc = copy_plane3(d, dst, (void *)lambda_seed_host, true);
    }
    for (int n = nsteps; n >= 1 && rc == SWALS_OK; n--) {
        const bool inj = ng > 0 && gadj_host;
        e = adjoint_step<R>(d, lam[cur], lam[1 - cur], dt, inj ? d_sites : nullptr, inj ? ng : 0,
                            inj ? d_g + (size_t)(n - 1) * ng : nullptr);
        if (e != cudaSuccess) rc = swals::api_cuda_fail(e, "adjoint step");
        cur = 1 - cur;
    }
    if (rc == SWALS_OK) {
        void *src[3] = {lam[cur][0], lam[cur][1], lam[cur][2]};
        rc = copy_plane3(d, src, grad_host, false);
    }
    cudaStreamSynchronize(d->stream);
    return rc;
}

// One interior update x' = M x of the forward (no boundary routine, bookkeeping
// or max_stage, which the misfit does not involve), optionally recording the
// new stage at the gauges into rec.
template <typename R>
cudaError_t map_step(swals_domain *d, R *const in[3], R *const out[3], double dt, const int *sites, int ng,
                     double *rec, cudaStream_t stream = nullptr)
{
    swals::StepPlanes<R> p;
    p.nx = d->nx; p.ny = d->ny; p.pitch = d->pitch;
    p.stg = in[0]; p.uh = in[1]; p.vh = in[2];
    p.stg_o = out[0]; p.uh_o = out[1]; p.vh_o = out[2];
    p.elv = (R *)d->elv;
    p.max_stage = nullptr;
    p.manning_sq = nullptr;
    return swals::launch_linear_map<R>(p, swals::metrics_of<R>(d), d->cfg, R(dt), sites, ng, rec,
                                       stream ? stream : d->stream, swals::hook_of(d));
}

// Residuals of `count` recorded steps against the target, and each step's
// half squared misfit (the loss is summed over steps in forward order at
// the end, so it does not depend on the checkpoint spacing).
__global__ void segment_residual_kernel(const double *rec, const double *target, int count, int ng, double *resid,
                                        double *step_half)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int q = 0; q < ng; q++) {
            const double rsd = rec[(size_t)t * ng + q] - target[(size_t)t * ng + q];
            resid[(size_t)t * ng + q] = rsd;
            acc += rsd * rsd;
        }
        step_half[t] = 0.5 * acc;
    }
}

__global__ void loss_sum_kernel(const double *step_half, int n, double *loss)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double l = 0.0;
    for (int k = 0; k < n; k++) l += step_half[k];
    *loss = l;
}

// Misfit gradient with checkpointing: a forward sweep from the domain's
// current state keeps a copy of the state every K steps (and nothing else);
// then, for each segment from the last, the segment's forward steps are
// recomputed from its checkpoint, recording the gauge stage, the segment's
// residuals are formed, and the adjoint runs back through the segment with
// the residuals injected as it goes.  Per timestep that is one forward map,
// one recomputed forward map and one adjoint launch.  The recomputation of
// segment s-1 does not depend on the adjoint through segment s, so it runs
// on the domain's side stream, into a second buffer set, while the adjoint
// runs on the main stream: the two grids are smaller than one wave of the
// GPU each and fill it together.
template <typename R>
int misfit_gradient(swals_domain *d, int nsteps, double dt, const double *target_host, int K, double *loss_out,
                    void *grad_host)
{
    const int ng = (int)(d->h_sites.size() / 2);
    if (ng <= 0) return swals::api_fail(SWALS_ERR_INVALID_ARGUMENT, "gauges must be set up first");
    const int64_t plane = d->pitch * (int64_t)d->ny;
    const size_t es = sizeof(R);
    const int nseg = (nsteps + K - 1) / K;
    size_t need = (size_t)(6 + 12 + 3 * nseg) * plane * es;          // lambda x2, state x2 x2 sets, checkpoints
    need += sizeof(double) * ((size_t)nsteps * ng + 4 * (size_t)K * ng + (size_t)nsteps + 8);
    need += sizeof(int) * 2 * (size_t)ng + 1024;
    void *buf = nullptr;
    cudaError_t e = workspace(d, need, &buf);
    if (e != cudaSuccess) return swals::api_cuda_fail(e, "misfit-gradient workspace");
    char *p = (char *)buf;
    R *lam[2][3], *xs[2][2][3];   // xs[set][ping-pong][variable]
    for (int b = 0; b < 2; b++)
        for (int v = 0; v < 3; v++) { lam[b][v] = (R *)p; p += plane * es; }
    for (int q = 0; q < 2; q++)
        for (int b = 0; b < 2; b++)
            for (int v = 0; v < 3; v++) { xs[q][b][v] = (R *)p; p += plane * es; }
    R *ckpt = (R *)p; p += (size_t)3 * nseg * plane * es;
    double *d_target = (double *)p; p += sizeof(double) * (size_t)nsteps * ng;
    double *d_rec[2], *d_resid[2];
    for (int q = 0; q < 2; q++) { d_rec[q] = (double *)p; p += sizeof(double) * (size_t)K * ng; }
    for (int q = 0; q < 2; q++) { d_resid[q] = (double *)p; p += sizeof(double) * (size_t)K * ng; }
    double *d_half = (double *)p; p += sizeof(double) * (size_t)nsteps;
    double *d_loss = (double *)p; p += sizeof(double) * 8;
    int *d_sites = (int *)p;

    int rc = SWALS_OK;
    auto ck = [&](cudaError_t err, const char *w) { if (err != cudaSuccess && rc == SWALS_OK) rc = swals::api_cuda_fail(err, w); };
    // The side stream of the domain (created here on first use).
    const bool overlap = !d->timers_on;
    if (overlap && !d->aux.stream) {
        ck(cudaStreamCreateWithFlags(&d->aux.stream, cudaStreamNonBlocking), "side stream");
        ck(cudaEventCreateWithFlags(&d->aux.fork, cudaEventDisableTiming), "event");
        ck(cudaEventCreateWithFlags(&d->aux.join, cudaEventDisableTiming), "event");
    }
    ck(cudaMemsetAsync(lam[0][0], 0, 3 * plane * es, d->stream), "memset");
    ck(cudaMemcpyAsync(d_target, target_host, sizeof(double) * (size_t)nsteps * ng, cudaMemcpyHostToDevice, d->stream),
       "target upload");
    ck(cudaMemcpyAsync(d_sites, d->h_sites.data(), sizeof(int) * 2 * ng, cudaMemcpyHostToDevice, d->stream), "sites");
    for (int v = 0; v < 3; v++)
        ck(cudaMemcpyAsync(xs[0][0][v], d->planes[d->cur][v], plane * es, cudaMemcpyDeviceToDevice, d->stream), "x0");

    // The per-segment step sequences.  For an even K a full segment leaves
    // the buffer parity unchanged, so each sequence is captured once as a
    // CUDA graph and replayed for every full segment.
    auto fwd_seq = [&](int count) {   // xs[0][0] -> xs[0][0] after an even count
        int c = 0;
        for (int n = 0; n < count; n++) {
            ck(map_step<R>(d, xs[0][c], xs[0][1 - c], dt, nullptr, 0, nullptr), "forward");
            c = 1 - c;
        }
        return c;
    };
    auto rec_seq = [&](int count, int set, cudaStream_t st) {   // recompute, recording the gauge stage
        int c = 0;
        for (int n = 0; n < count; n++) {
            ck(map_step<R>(d, xs[set][c], xs[set][1 - c], dt, d_sites, ng, d_rec[set] + (size_t)n * ng, st),
               "recompute");
            c = 1 - c;
        }
        return c;
    };
    auto adj_seq = [&](int count, int lc, int set) {   // adjoint back through `count` steps
        for (int t = count; t > 0; t--) {
            ck(adjoint_step<R>(d, lam[lc], lam[1 - lc], dt, d_sites, ng, d_resid[set] + (size_t)(t - 1) * ng),
               "adjoint");
            lc = 1 - lc;
        }
        return lc;
    };
    const bool graphs = (K % 2 == 0) && K <= nsteps && !d->timers_on;
    if (graphs && (d->adj_K != K || d->adj_ng != ng || d->adj_dt != dt || d->adj_ws != d->ws || !d->adj_graph[0])) {
        for (auto &g : d->adj_graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        d->adj_K = 0;
        const int64_t l0 = d->launches;
        for (int q = 0; q < 7 && rc == SWALS_OK; q++) {
            ck(cudaStreamBeginCapture(d->stream, cudaStreamCaptureModeThreadLocal), "capture");
            if (q == 0) fwd_seq(K);
            else if ((q - 1) % 3 == 0) rec_seq(K, (q - 1) / 3, d->stream);
            else adj_seq(K, (q - 2) % 3, (q - 2) / 3);
            cudaGraph_t gr = nullptr;
            ck(cudaStreamEndCapture(d->stream, &gr), "end capture");
            if (gr) {
                ck(cudaGraphInstantiate(&d->adj_graph[q], gr, 0), "instantiate");
                cudaGraphDestroy(gr);
            }
        }
        d->launches = l0;
        if (rc == SWALS_OK) { d->adj_K = K; d->adj_ng = ng; d->adj_dt = dt; d->adj_ws = d->ws; }
    }

    // Forward sweep with checkpoints (every segment starts in xs[0][0]).
    int cur = 0;
    for (int sgm = 0; sgm < nseg && rc == SWALS_OK; sgm++) {
        const int n0 = sgm * K, cnt = (n0 + K < nsteps) ? K : nsteps - n0;
        for (int v = 0; v < 3; v++)
            ck(cudaMemcpyAsync(ckpt + ((size_t)sgm * 3 + v) * plane, xs[0][cur][v], plane * es,
                               cudaMemcpyDeviceToDevice, d->stream), "checkpoint");
        if (graphs && cnt == K && cur == 0) {
            ck(cudaGraphLaunch(d->adj_graph[0], d->stream), "forward graph");
            d->launches += K;
        } else {
            // A last, shorter segment (no state is needed after it).
            int c = cur;
            for (int n = 0; n < cnt; n++) {
                ck(map_step<R>(d, xs[0][c], xs[0][1 - c], dt, nullptr, 0, nullptr), "forward");
                c = 1 - c;
            }
            cur = c;
        }
    }
    // Recompute segment sgm into buffer set `set` on stream st, then its residuals.
    auto recompute = [&](int sgm, int set, cudaStream_t st) {
        const int n0 = sgm * K, n1 = (n0 + K < nsteps) ? n0 + K : nsteps;
        const int cnt = n1 - n0;
        for (int v = 0; v < 3; v++)
            ck(cudaMemcpyAsync(xs[set][0][v], ckpt + ((size_t)sgm * 3 + v) * plane, plane * es,
                               cudaMemcpyDeviceToDevice, st), "restore");
        if (graphs && cnt == K) {
            ck(cudaGraphLaunch(d->adj_graph[1 + 3 * set], st), "recompute graph");
            d->launches += K;
        } else {
            rec_seq(cnt, set, st);
        }
        segment_residual_kernel<<<1, 128, 0, st>>>(d_rec[set], d_target + (size_t)n0 * ng, cnt, ng, d_resid[set],
                                                   d_half + n0);
        ck(cudaGetLastError(), "residuals");
    };
    // Backward, segment by segment from the last; segment sgm's buffers are
    // set sgm & 1, and the recomputation of sgm-1 overlaps the adjoint of sgm.
    recompute(nseg - 1, (nseg - 1) & 1, d->stream);
    int lc = 0;
    for (int sgm = nseg - 1; sgm >= 0 && rc == SWALS_OK; sgm--) {
        const int set = sgm & 1;
        const int n0 = sgm * K, n1 = (n0 + K < nsteps) ? n0 + K : nsteps;
        const int cnt = n1 - n0;
        if (sgm > 0) {
            // the side stream may reuse set 1-set once the adjoint of sgm+1
            // (issued before this point on the main stream) is done with it
            cudaStream_t st = overlap ? d->aux.stream : d->stream;
            if (overlap) {
                ck(cudaEventRecord(d->aux.fork, d->stream), "fork");
                ck(cudaStreamWaitEvent(st, d->aux.fork, 0), "fork wait");
            }
            recompute(sgm - 1, 1 - set, st);
            if (overlap) ck(cudaEventRecord(d->aux.join, st), "join");
        }
        if (graphs && cnt == K) {
            ck(cudaGraphLaunch(d->adj_graph[2 + 3 * set + lc], d->stream), "adjoint graph");
            d->launches += K;
        } else {
            lc = adj_seq(cnt, lc, set);
        }
        if (sgm > 0 && overlap) ck(cudaStreamWaitEvent(d->stream, d->aux.join, 0), "join wait");
    }
    loss_sum_kernel<<<1, 32, 0, d->stream>>>(d_half, nsteps, d_loss);
    double loss = 0.0;
    ck(cudaMemcpyAsync(&loss, d_loss, sizeof(double), cudaMemcpyDeviceToHost, d->stream), "loss");
    if (rc == SWALS_OK) {
        void *src[3] = {lam[lc][0], lam[lc][1], lam[lc][2]};
        rc = copy_plane3(d, src, grad_host, false);
    }
    cudaStreamSynchronize(d->stream);
    if (loss_out) *loss_out = loss;
    return rc;
}

}  // namespace

extern "C" {

int swals_gpu_adjoint_linear(swals_domain *d, int32_t nsteps, double timestep, const double *gauge_adjoint,
                             const void *lambda_seed, void *grad_U0)
{
    if (!d || nsteps < 0 || !grad_U0) return swals::api_fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    int rc = check_adjoint_domain(d);
    if (rc) return rc;
    return d->fp64 ? adjoint_sweep<double>(d, nsteps, timestep, gauge_adjoint, grad_U0, lambda_seed)
                   : adjoint_sweep<float>(d, nsteps, timestep, gauge_adjoint, grad_U0, lambda_seed);
}

int swals_gpu_misfit_gradient_linear(swals_domain *d, int32_t nsteps, double timestep, const double *target,
                                     int32_t checkpoint_every, double *loss, void *grad_U0)
{
    if (!d || nsteps < 1 || !target || !grad_U0 || checkpoint_every < 1)
        return swals::api_fail(SWALS_ERR_INVALID_ARGUMENT, "bad argument");
    int rc = check_adjoint_domain(d);
    if (rc) return rc;
    return d->fp64 ? misfit_gradient<double>(d, nsteps, timestep, target, checkpoint_every, loss, grad_U0)
                   : misfit_gradient<float>(d, nsteps, timestep, target, checkpoint_every, loss, grad_U0);
}

}  // extern "C"
