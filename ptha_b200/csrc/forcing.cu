// forcing.cu -- forcing patches (forcing_mod.f90) on sm_100a.
//
// A forcing patch adds forcing_work to U(i0:i1, j0:j1, k0:k1) at a constant
// rate between start_time and end_time (add_forcing_work_to_U_over_time,
// forcing_mod.f90:80-156, with the default identity forcing_time_function):
// for an update of U over (time - dt, time) the patch adds
//     (min(time, end) - max(time - dt, start)) / (end - start)
// of its work (all of it when start == end), nothing when the update does
// not overlap [start, end].  Patches are applied in the order they were
// added (apply_forcing_patch_array, :241-262).
//
// The time and dt come from the device scalars, in the same expressions as
// the boundary kernels use, so a step that is captured in a CUDA graph
// applies each patch exactly when the reference would.
#include "swals_kernels.h"

namespace swals {
namespace {

template <typename R>
__device__ __forceinline__ void forcing_time(const ForcingClock &clk, const DevScalars *sc, double &t, R &dt)
{
    if (clk.mode == FORCE_EXPLICIT) {   // domain%apply_forcing(dt) at domain%time
        t = sc->time;
        dt = R(clk.dt);
    } else if (clk.mode == FORCE_LEAPFROG) {
        // after the stage sweep: domain%time = time0 + dt/2 (linear_solver_include.f90:117-123)
        dt = R(clk.dt);
        t = sc->time0 + (double)(dt * K<R>::half());
    } else {
        double dtd;
        if (clk.dt_from_cfl) {
            const double bits_max = __longlong_as_double((long long)sc->max_dt_inv_bits);
            const R inv = R(fmax(clk.max_dt_inv_init, bits_max));
            dtd = (double)(R(1) / inv);
        } else {
            dtd = (double)R(clk.dt_fixed);
        }
        t = sc->time;
        for (int k = 0; k < clk.n_dt; k++) t = t + dtd;
        dt = R(dtd);
        if (clk.dt_extra != 0.0) {
            dt = R(dtd) * R(clk.dt_extra);
            t = t + (double)dt;
        }
    }
}

template <typename R>
__global__ void __launch_bounds__(256) forcing_kernel(ForcingPatch p, ForcingClock clk, int64_t P, R *stg, R *uh,
                                                      R *vh, R *elv, const DevScalars *sc)
{
    double td;
    R dt;
    forcing_time<R>(clk, sc, td, dt);
    const R time = R(td), start = R(p.start_time), end = R(p.end_time);
    if (!(((time - dt) <= end) && (time >= start))) return;
    const R uf = (start == end) ? R(1) : (rmin(time, end) - rmax(time - dt, start)) / (end - start);
    const int ni = p.i1 - p.i0 + 1, nj = p.j1 - p.j0 + 1;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ni * nj) return;
    const int i = p.i0 + q % ni, r = p.j0 + q / ni;
    const int64_t o = (int64_t)r * P + i;
    const R *w = (const R *)p.work;
    for (int k = p.k0; k <= p.k1; k++) {
        R *pl = (k == 0) ? stg : (k == 1) ? uh : (k == 2) ? vh : elv;
        pl[o] = pl[o] + uf * w[(int64_t)(k - p.k0) * ni * nj + q];
    }
}

template <typename R>
__global__ void forcing_box_copy_kernel(ForcingPatch p, int64_t P, const R *src, R *dst)
{
    const int ni = p.i1 - p.i0 + 1, nj = p.j1 - p.j0 + 1;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ni * nj) return;
    dst[q] = src[(int64_t)(p.j0 + q / ni) * P + p.i0 + q % ni];
}

// max_stage over the box after the leapfrog step: the step kernel folded in
// the stage before the forcing; update_max_quantities sees the stage after.
template <typename R>
__global__ void forcing_max_kernel(ForcingPatch p, int64_t P, const R *stg, R *max_stage, int xl, int xu, int yl,
                                   int yu)
{
    const int ni = p.i1 - p.i0 + 1, nj = p.j1 - p.j0 + 1;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ni * nj) return;
    const int i = p.i0 + q % ni, r = p.j0 + q / ni;
    if (i < xl || i > xu || r < yl || r > yu) return;
    const int64_t o = (int64_t)r * P + i;
    const R mx = ((const R *)p.saved_max)[q];
    const R sv = stg[o];
    max_stage[o] = (sv > mx) ? sv : mx;
}

int cells(const ForcingPatch &p) { return (p.i1 - p.i0 + 1) * (p.j1 - p.j0 + 1); }

}  // namespace

template <typename R>
cudaError_t launch_forcing(const StepConfig &c, const ForcingClock &clk, int64_t pitch, R *stg, R *uh, R *vh,
                           R *elv, const DevScalars *sc, cudaStream_t s, const LaunchHook &hook, int cat)
{
    for (int k = 0; k < c.n_forcing; k++) {
        const ForcingPatch &p = c.forcing[k];
        hook(cat, 0);
        forcing_kernel<R><<<(cells(p) + 255) / 256, 256, 0, s>>>(p, clk, pitch, stg, uh, vh, elv, sc);
        hook(cat, 1);
    }
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_forcing_save_max(const StepConfig &c, int64_t pitch, const R *max_stage, cudaStream_t s,
                                    const LaunchHook &hook, int cat)
{
    for (int k = 0; k < c.n_forcing; k++) {
        const ForcingPatch &p = c.forcing[k];
        if (p.k0 != 0 || !p.saved_max) continue;
        hook(cat, 0);
        forcing_box_copy_kernel<R><<<(cells(p) + 255) / 256, 256, 0, s>>>(p, pitch, max_stage, (R *)p.saved_max);
        hook(cat, 1);
    }
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_forcing_restore_max(const StepConfig &c, int64_t pitch, const R *stg, R *max_stage,
                                       cudaStream_t s, const LaunchHook &hook, int cat)
{
    for (int k = 0; k < c.n_forcing; k++) {
        const ForcingPatch &p = c.forcing[k];
        if (p.k0 != 0 || !p.saved_max) continue;
        hook(cat, 0);
        forcing_max_kernel<R><<<(cells(p) + 255) / 256, 256, 0, s>>>(p, pitch, stg, max_stage, c.xl, c.xu, c.yl,
                                                                     c.yu);
        hook(cat, 1);
    }
    return cudaGetLastError();
}

#define SWALS_INST_FORCING(R)                                                                                  \
    template cudaError_t launch_forcing<R>(const StepConfig &, const ForcingClock &, int64_t, R *, R *, R *,   \
                                           R *, const DevScalars *, cudaStream_t, const LaunchHook &, int);    \
    template cudaError_t launch_forcing_save_max<R>(const StepConfig &, int64_t, const R *, cudaStream_t,      \
                                                    const LaunchHook &, int);                                   \
    template cudaError_t launch_forcing_restore_max<R>(const StepConfig &, int64_t, const R *, R *,           \
                                                       cudaStream_t, const LaunchHook &, int);
SWALS_INST_FORCING(double)
SWALS_INST_FORCING(float)

}  // namespace swals
