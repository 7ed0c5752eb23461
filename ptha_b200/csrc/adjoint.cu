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

// Residual of the recorded gauge stage against a target: out[g] = y[g] - d[g].
__global__ void residual_kernel(const double *records3, const double *target, int n, double *out, double *loss)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double acc = 0.0;
    for (int g = 0; g < n; g++) {
        const double rsd = records3[3 * g] - target[g];
        out[g] = rsd;
        acc += rsd * rsd;
    }
    *loss += 0.5 * acc;
}

template <typename R>
struct Work {
    swals_domain *d;
    int64_t plane;
    R *lam[2][3];
    R *x[2][3];
    swals::DevScalars *sc;
    int *sites;
    double *records, *gadj, *loss;
};

template <typename R>
cudaError_t adjoint_step(swals_domain *d, R *const in[3], R *const out[3], double dt)
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
    dim3 block(ABX, ATY), grid((d->nx + ABX - 1) / ABX, (d->ny + ABY - 1) / ABY);
    swals::LaunchHook hook = swals::hook_of(d);
    hook(swals::CAT_LINEAR_MAIN, 0);
    if (d->cfg.coriolis) linear_adjoint_kernel<R, true><<<grid, block, 0, d->stream>>>(a);
    else linear_adjoint_kernel<R, false><<<grid, block, 0, d->stream>>>(a);
    hook(swals::CAT_LINEAR_MAIN, 1);
    return cudaGetLastError();
}

template <typename R>
cudaError_t forward_step(swals_domain *d, R *const in[3], R *const out[3], double dt, swals::DevScalars *sc)
{
    swals::StepPlanes<R> p;
    p.nx = d->nx; p.ny = d->ny; p.pitch = d->pitch;
    p.stg = in[0]; p.uh = in[1]; p.vh = in[2];
    p.stg_o = out[0]; p.uh_o = out[1]; p.vh_o = out[2];
    p.elv = (R *)d->elv;
    p.max_stage = nullptr;
    p.manning_sq = nullptr;
    return swals::launch_linear_step<R>(p, swals::metrics_of<R>(d), d->cfg, R(dt), sc, d->stream,
                                        swals::hook_of(d));
}

int check_adjoint_domain(swals_domain *d)
{
    if (strncmp(d->desc.timestepping_method, "linear", 6) != 0 || d->desc.timestepping_method[6] > ' ')
        return swals::api_fail(SWALS_ERR_UNSUPPORTED, "the adjoint is implemented for timestepping_method='linear'");
    if (!d->cfg.truely_linear)
        return swals::api_fail(SWALS_ERR_UNSUPPORTED, "the adjoint needs linear_solver_is_truely_linear=.true.");
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
    cudaError_t e = cudaMalloc(&buf, need);
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
        if (ng > 0 && gadj_host) {
            inject_kernel<R><<<1, 32, 0, d->stream>>>(lam[cur][0], d->pitch, d_sites, ng, d_g + (size_t)(n - 1) * ng);
            d->launches++;
        }
        e = adjoint_step<R>(d, lam[cur], lam[1 - cur], dt);
        if (e != cudaSuccess) rc = swals::api_cuda_fail(e, "adjoint step");
        cur = 1 - cur;
    }
    if (rc == SWALS_OK) {
        void *src[3] = {lam[cur][0], lam[cur][1], lam[cur][2]};
        rc = copy_plane3(d, src, grad_host, false);
    }
    cudaStreamSynchronize(d->stream);
    cudaFree(buf);
    return rc;
}

// Misfit gradient with checkpointing: forward from the domain's current
// state keeping a copy every K steps (and nothing else), then for each
// segment from the last: recompute its forward steps from the checkpoint to
// get the gauge residuals, and run the adjoint back through it.
template <typename R>
int misfit_gradient(swals_domain *d, int nsteps, double dt, const double *target_host, int K, double *loss_out,
                    void *grad_host)
{
    const int ng = (int)(d->h_sites.size() / 2);
    if (ng <= 0) return swals::api_fail(SWALS_ERR_INVALID_ARGUMENT, "gauges must be set up first");
    const int64_t plane = d->pitch * (int64_t)d->ny;
    const size_t es = sizeof(R);
    const int nseg = (nsteps + K - 1) / K;
    size_t need = (size_t)(6 + 6 + 3 * nseg) * plane * es;          // lambda x2, state x2, checkpoints
    need += sizeof(double) * ((size_t)nsteps * ng + (size_t)K * ng * 3 + (size_t)ng + 8);
    need += sizeof(int) * 2 * (size_t)ng + sizeof(swals::DevScalars) + 1024;
    void *buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, need);
    if (e != cudaSuccess) return swals::api_cuda_fail(e, "misfit-gradient workspace");
    char *p = (char *)buf;
    R *lam[2][3], *x[2][3];
    for (int b = 0; b < 2; b++)
        for (int v = 0; v < 3; v++) { lam[b][v] = (R *)p; p += plane * es; }
    for (int b = 0; b < 2; b++)
        for (int v = 0; v < 3; v++) { x[b][v] = (R *)p; p += plane * es; }
    R *ckpt = (R *)p; p += (size_t)3 * nseg * plane * es;
    double *d_target = (double *)p; p += sizeof(double) * (size_t)nsteps * ng;
    double *d_rec = (double *)p; p += sizeof(double) * (size_t)K * ng * 3;
    double *d_resid = (double *)p; p += sizeof(double) * (size_t)ng;
    double *d_loss = (double *)p; p += sizeof(double) * 8;
    int *d_sites = (int *)p; p += sizeof(int) * 2 * (size_t)ng;
    p = (char *)(((uintptr_t)p + 255) & ~(uintptr_t)255);
    swals::DevScalars *sc = (swals::DevScalars *)p;

    int rc = SWALS_OK;
    auto ck = [&](cudaError_t err, const char *w) { if (err != cudaSuccess && rc == SWALS_OK) rc = swals::api_cuda_fail(err, w); };
    ck(cudaMemsetAsync(buf, 0, need, d->stream), "memset");
    ck(cudaMemcpyAsync(d_target, target_host, sizeof(double) * (size_t)nsteps * ng, cudaMemcpyHostToDevice, d->stream),
       "target upload");
    ck(cudaMemcpyAsync(d_sites, d->h_sites.data(), sizeof(int) * 2 * ng, cudaMemcpyHostToDevice, d->stream), "sites");
    // x_0 = the domain's current state
    for (int v = 0; v < 3; v++)
        ck(cudaMemcpyAsync(x[0][v], d->planes[d->cur][v], plane * es, cudaMemcpyDeviceToDevice, d->stream), "x0");

    // Forward with checkpoints (loss accumulated on the device).
    int cur = 0;
    for (int n = 0; n < nsteps && rc == SWALS_OK; n++) {
        if (n % K == 0)
            for (int v = 0; v < 3; v++)
                ck(cudaMemcpyAsync(ckpt + ((size_t)(n / K) * 3 + v) * plane, x[cur][v], plane * es,
                                   cudaMemcpyDeviceToDevice, d->stream), "checkpoint");
        ck(forward_step<R>(d, x[cur], x[1 - cur], dt, sc), "forward");
        cur = 1 - cur;
        ck(cudaMemsetAsync(&sc->gauge_records, 0, sizeof(int), d->stream), "rec reset");
        ck(swals::launch_gauges<R>(d->pitch, x[cur][0], x[cur][1], x[cur][2], d_sites, ng, d_rec, 1, sc, d->stream),
           "gauges");
        residual_kernel<<<1, 32, 0, d->stream>>>(d_rec, d_target + (size_t)n * ng, ng, d_resid, d_loss);
    }
    // Backward, segment by segment from the last.
    int lc = 0;
    for (int s = nseg - 1; s >= 0 && rc == SWALS_OK; s--) {
        const int n0 = s * K, n1 = (n0 + K < nsteps) ? n0 + K : nsteps;
        for (int v = 0; v < 3; v++)
            ck(cudaMemcpyAsync(x[0][v], ckpt + ((size_t)s * 3 + v) * plane, plane * es, cudaMemcpyDeviceToDevice,
                               d->stream), "restore");
        ck(cudaMemsetAsync(&sc->gauge_records, 0, sizeof(int), d->stream), "rec reset");
        int xc = 0;
        for (int n = n0; n < n1; n++) {   // recompute the segment, recording gauges
            ck(forward_step<R>(d, x[xc], x[1 - xc], dt, sc), "recompute");
            xc = 1 - xc;
            ck(swals::launch_gauges<R>(d->pitch, x[xc][0], x[xc][1], x[xc][2], d_sites, ng, d_rec, K, sc,
                                       d->stream), "gauges");
        }
        for (int n = n1; n > n0; n--) {   // adjoint back through the segment
            residual_kernel<<<1, 32, 0, d->stream>>>(d_rec + (size_t)(n - 1 - n0) * ng * 3, d_target + (size_t)(n - 1) * ng,
                                                     ng, d_resid, d_loss + 1);
            inject_kernel<R><<<1, 32, 0, d->stream>>>(lam[lc][0], d->pitch, d_sites, ng, d_resid);
            ck(adjoint_step<R>(d, lam[lc], lam[1 - lc], dt), "adjoint");
            lc = 1 - lc;
        }
    }
    double loss = 0.0;
    ck(cudaMemcpyAsync(&loss, d_loss, sizeof(double), cudaMemcpyDeviceToHost, d->stream), "loss");
    if (rc == SWALS_OK) {
        void *src[3] = {lam[lc][0], lam[lc][1], lam[lc][2]};
        rc = copy_plane3(d, src, grad_host, false);
    }
    cudaStreamSynchronize(d->stream);
    cudaFree(buf);
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
