// swals_common.cuh -- shared definitions for the sm_100a SWALS kernels.
//
// Device layout (one domain):
//   STG, UH, VH, ELV planes, each ny rows of `pitch` elements, row j holding
//   cells i = 0..nx-1 (the reference's U(i+1, j+1, k)); pitch is a multiple
//   of 32 elements so every row starts on a 256-byte boundary (FP64) and
//   every warp-wide row access is whole 128-byte sectors.
//   State planes (STG, UH, VH) exist in 3 copies so a step reads one copy
//   and writes another (no in-place races between CTAs); ELV, max_stage and
//   manning_squared exist once.
//   1-D metric arrays (dxb, dyl, area, coriolis, ...) hold the reference's
//   Fortran arrays shifted to 0-based: dxb0[j] = distance_bottom_edge(j+1).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace swals {

// global_mod.f90:37-55, domain_mod.f90:111-117, spherical_mod.f90:9-17.
template <typename R> struct K {
    static __host__ __device__ __forceinline__ R gravity() { return R(9.8); }
    static __host__ __device__ __forceinline__ R half() { return R(0.5); }
    static __host__ __device__ __forceinline__ R one() { return R(1.0); }
    static __host__ __device__ __forceinline__ R zero() { return R(0.0); }
    static __host__ __device__ __forceinline__ R min_depth() { return R(1.0e-05); }
    static __host__ __device__ __forceinline__ R wall_elevation() { return R(1.0e+6); }
    // HUGE(1.0_dp) of the state precision.
    static __host__ __device__ __forceinline__ R huge() { return sizeof(R) == 8 ? R(1.7976931348623157e308) : R(3.4028234663852886e38f); }
    static __host__ __device__ __forceinline__ R limiter_coef1() { return R(0.1); }
    static __host__ __device__ __forceinline__ R limiter_coef2() { return R(0.3); }
    static __host__ __device__ __forceinline__ R limiter_coef3() { return R(100.0); }
};

template <typename R> __device__ __forceinline__ R rmin(R a, R b) { return (b < a) ? b : a; }
template <typename R> __device__ __forceinline__ R rmax(R a, R b) { return (b > a) ? b : a; }

// Friction power law pow(x, p), p = fl(-7/3) (Manning) or -2 (Chezy), for
// x >= minimum_allowed_depth (update_U_DE1_inner_include.f90:72-75).  The
// oracle evaluates the same operation sequence, so both give the same bits
// whatever libm is present; every step is an IEEE operation (no FMA
// contraction in this library), plus integer work on the float bits.
//   Chezy: the correctly rounded 1/x^2 (x^2 as a double-double, compensated
//   reciprocal).
//   Manning: the inverse cube root y = x^(-1/3) by Newton's iteration
//   y <- y + y (1 - x y^3)/3, seeded from the float bits of x
//   (bits(y) = K - bits(x)/3, the linear-in-the-exponent estimate of
//   x^(-1/3), K fitted for the least relative error, 3.4%), two iterations
//   in FP32 and two in FP64; then x^(-7/3) = y / (x x), and the exponent's
//   own rounding, x^p = x^(-7/3) x^eps with eps = fl(-7/3) + 7/3, as the
//   factor 1 + eps ln(x) with ln(x) from the float bits (log2 x ~ exponent
//   + mantissa fraction; the term is below 2e-15, so its 9% error is far
//   below an ulp).  Within 3 ulp of the exact power over 1e-5 <= x <=
//   1e5 (checked against 300-bit arithmetic), about 40 instructions against
//   the ~400 of a correctly rounded evaluation.
struct DD { double hi, lo; };
__device__ __forceinline__ DD dd_two_prod(double a, double b) { DD r; r.hi = a * b; r.lo = fma(a, b, -r.hi); return r; }
__device__ __forceinline__ DD dd_fast_two_sum(double a, double b) { DD r; r.hi = a + b; r.lo = b - (r.hi - a); return r; }
__device__ __forceinline__ DD dd_recip(DD p)
{
    const double y0 = 1.0 / p.hi;
    DD t = dd_two_prod(p.hi, y0);
    t.lo += p.lo * y0;
    const double e = (1.0 - t.hi) - t.lo;
    return dd_fast_two_sum(y0, y0 * e);
}
constexpr unsigned kRcbrtSeed = 0x54a237fbu;
constexpr double kEpsLn2 = -1.0260639457488826e-16;   // (fl(-7/3) + 7/3) ln 2
template <bool CHEZY>
__device__ __forceinline__ double pow_friction(double x)
{
    if (CHEZY) return dd_recip(dd_two_prod(x, x)).hi;
    const float xf = __double2float_rn(x);
    const unsigned ix = __float_as_uint(xf);
    float y = __uint_as_float(kRcbrtSeed - ix / 3u);
    const float third_f = 1.0f / 3.0f;
    y = y + y * ((1.0f - xf * (y * y * y)) * third_f);
    y = y + y * ((1.0f - xf * (y * y * y)) * third_f);
    double yd = (double)y;
    yd = yd + yd * ((1.0 - x * (yd * yd * yd)) * (1.0 / 3.0));
    yd = yd + yd * ((1.0 - x * (yd * yd * yd)) * (1.0 / 3.0));
    const double v = yd / (x * x);
    const double t = kEpsLn2 * ((double)ix * (1.0 / 8388608.0) - 127.0);
    return v + v * t;
}

// Correctly rounded depth**p, p = fl(1 - 1/6), of the Shiono-Knight eddy
// viscosity (compute_fluxes_DE1_inner_include.f90:1000-1002), depth >= 0.
// Double-double arithmetic: the Newton-corrected cube root, its
// Newton-corrected square root (x**(1/6)), the compensated quotient
// x / x**(1/6), and the factor x**eps = 1 + eps*ln(x), eps = p - 5/6.  The
// oracle evaluates the same definition (checked there against 300-bit
// arithmetic).
__device__ __forceinline__ double pow_eddy_cr(double x)
{
    if (x == 0.0) return 0.0;
    const double c0 = cbrt(x);
    const DD s = dd_two_prod(c0, c0);
    DD t = dd_two_prod(s.hi, c0);
    t.lo += s.lo * c0;
    const double r = (x - t.hi) - t.lo;
    const DD c = dd_fast_two_sum(c0, r / (3.0 * c0 * c0));
    const double q0 = sqrt(c.hi);
    const DD q2 = dd_two_prod(q0, q0);
    const double rq = ((c.hi - q2.hi) - q2.lo) + c.lo;
    const DD q = dd_fast_two_sum(q0, rq / (2.0 * q0));
    const double y0 = x / q.hi;
    DD pq = dd_two_prod(y0, q.hi);
    pq.lo += y0 * q.lo;
    const DD y = dd_fast_two_sum(y0, ((x - pq.hi) - pq.lo) / q.hi);
    const double p = 1.0 - 1.0 / 6.0;
    const double eps = fma(p, 6.0, -5.0) / 6.0;
    const double tl = eps * log(x);
    return dd_fast_two_sum(y.hi, y.lo + y.hi * tl).hi;
}

// Correctly rounded cosh for the device boundary functions, in double-double
// arithmetic: a = k ln2 + r with a double-double ln2 and |r| <= ln2/2,
// exp(r) by the Horner form of its Taylor series to r^22/22!, exp(-|a|) by a
// compensated reciprocal.  Only IEEE operations, fma, rint and ldexp are used,
// so host and device evaluate it to the same bits.
__host__ __device__ __forceinline__ DD dd_two_sum_hd(double a, double b)
{
    DD r; r.hi = a + b; const double bb = r.hi - a; r.lo = (a - (r.hi - bb)) + (b - bb); return r;
}
__host__ __device__ __forceinline__ DD dd_fts_hd(double a, double b) { DD r; r.hi = a + b; r.lo = b - (r.hi - a); return r; }
__host__ __device__ __forceinline__ DD dd_tp_hd(double a, double b) { DD r; r.hi = a * b; r.lo = fma(a, b, -r.hi); return r; }
__host__ __device__ __forceinline__ DD dd_mul_hd(DD a, DD b)
{
    DD p = dd_tp_hd(a.hi, b.hi);
    p.lo += a.hi * b.lo + a.lo * b.hi;
    return dd_fts_hd(p.hi, p.lo);
}
__host__ __device__ __forceinline__ DD dd_div_d_hd(DD x, double n)
{
    const double q1 = x.hi / n;
    const DD p = dd_tp_hd(q1, n);
    const double e = (((x.hi - p.hi) - p.lo) + x.lo) / n;
    return dd_fts_hd(q1, e);
}
__host__ __device__ __forceinline__ double cosh_cr(double a)
{
    const double x = fabs(a);
    if (x > 700.0) return x * 1.0e308;  // overflow to +inf, as cosh does
    const double ln2_hi = 6.93147180559945286227e-01, ln2_lo = 2.31904681384629955842e-17;
    const double k = rint(x * 1.44269504088896338700e+00);
    const DD p = dd_tp_hd(k, ln2_hi);
    DD t = dd_two_sum_hd(x, -p.hi);
    t.lo = (t.lo - p.lo) - k * ln2_lo;
    const DD r = dd_fts_hd(t.hi, t.lo);
    DD s; s.hi = 1.0; s.lo = 0.0;
    for (int n = 22; n >= 1; n--) {
        DD q = dd_div_d_hd(dd_mul_hd(r, s), (double)n);
        DD u = dd_two_sum_hd(1.0, q.hi);
        u.lo += q.lo;
        s = dd_fts_hd(u.hi, u.lo);
    }
    const int ki = (int)k;
    DD E; E.hi = ldexp(s.hi, ki); E.lo = ldexp(s.lo, ki);
    // 1/E
    const double y0 = 1.0 / E.hi;
    DD w = dd_tp_hd(E.hi, y0);
    w.lo += E.lo * y0;
    const double e = (1.0 - w.hi) - w.lo;
    const DD inv = dd_fts_hd(y0, y0 * e);
    DD sum = dd_two_sum_hd(E.hi, inv.hi);
    sum.lo += E.lo + inv.lo;
    sum = dd_fts_hd(sum.hi, sum.lo);
    return 0.5 * sum.hi + 0.5 * sum.lo;
}

// Metric arrays, 0-based copies of the Fortran arrays.
template <typename R> struct Metrics {
    const R *dxb;     // ny+1: distance_bottom_edge
    const R *dyl;     // nx+1: distance_left_edge
    const R *area;    // ny:   area_cell_y
    const R *cor;     // ny:   coriolis
    const R *cor_be;  // ny+1: coriolis_bottom_edge
    const R *tanlat;  // ny:   tanlat_on_radius_earth
    const R *x;       // nx
    const R *y;       // ny
};

// Device-side scalar state of a domain (time, timestep, reductions).
struct DevScalars {
    double time;
    double dt;                 // timestep used by the current step
    double max_dt;             // domain%max_dt
    unsigned long long max_dt_inv_bits;  // running max of 1/dt (positive doubles order as integers)
    unsigned long long nonfinite;        // nonzero when a stability check found NaN/Inf
    long long negative_depth_fix_counter;
    long long nsteps_advanced;
    double time0;              // time at the start of the current step
    double boundary_flux_store[4];
    double boundary_flux_evolve_integral;
    double boundary_flux_time_integral;
    double dt_last_update;
    double evolve_step_dt;
    int    gauge_records;      // number of gauge records written
    int    blocks_done;        // CTAs of the running step kernel past their gauge records (reset by the last)
    double bf_col0[2][2];      // the boundary function's (stage, elevation) at column 0 for times
                               // time + dt and time + 2 dt of an adaptive rk2 step (its stage-1
                               // update kernel writes them; the stage-boundary kernels read them)
};

// Boundary-function parameters (SWALS_BF_*), evaluated on the device.
struct BoundaryFn {
    int kind;
    int pad;
    double p[8];
};

__host__ __device__ inline int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

// Analytic boundary_function values [stage, uh, vh, elev] at cell (i,j)
// (0-based), time t.  i0/j0 tests use the 0-based cell index.
template <typename R>
__device__ __forceinline__ void boundary_function(const BoundaryFn &bf, const R *x, double t, int i, int j,
                                                  R &stg, R &elv)
{
    (void)j;
    if (bf.kind == 1) {  // SWALS_BF_SOLITARY_WEST_WALLS
        R H = R(bf.p[0]), dep = R(bf.p[1]), x0 = R(bf.p[2]);
        if (i == 0) {
            R k = R(sqrt(R(3.0) * H / (R(4.0) * dep * dep * dep)));
            R c = R(sqrt(K<R>::gravity() * (dep + H)));
            R arg = k * (x[0] - x0 - c * R(t));
            R ch = R(cosh_cr((double)arg));
            stg = H / (ch * ch);
            elv = -dep;
        } else {
            stg = K<R>::wall_elevation();
            elv = K<R>::wall_elevation();
        }
    } else {
        stg = R(0);
        elv = R(0);
    }
}

// flather_boundary (boundary_mod.f90:502-730) for one ring cell (i, j),
// 0-based.  The inner neighbour holds stage s_in, elevation e_in, normal
// momentum qn_in (UH on the west/east edges, VH on the south/north edges) and
// transverse momentum qt_in; e is the ring cell's elevation.  lo: the west or
// south edge (inflow has positive normal velocity).  The 'outside' state is
// the boundary function's (whose momenta are zero for the device kinds), or
// at rest at stage max(msl_linear, e) without one.  Returns the ring cell's
// stage, normal and transverse momentum; its elevation is unchanged.
template <typename R>
__device__ __forceinline__ void flather_cell(const BoundaryFn &bf, const R *x, double t, int i, int j, R msl, bool lo,
                                             R s_in, R qn_in, R qt_in, R e_in, R e, R &s_out, R &qn_out, R &qt_out)
{
    const R mad = K<R>::min_depth();
    const R depth_inside = s_in - e_in;
    R stage_outside, depth_outside;
    const R u_outside = R(0);
    if (bf.kind == 0) {
        stage_outside = (msl > e) ? msl : e;
        depth_outside = stage_outside - e;
    } else {
        R bs, be;
        boundary_function<R>(bf, x, t, i, j, bs, be);
        stage_outside = bs;
        depth_outside = bs - be;
    }
    if (depth_inside > mad && depth_outside > mad) {
        const R depth_inside_inv = R(1) / depth_inside;
        const R sqrt_g_on_di = sqrt(K<R>::gravity() * depth_inside_inv);
        R w1, w2, w3;
        if (lo) {
            w1 = u_outside + sqrt_g_on_di * stage_outside;
            w2 = (qn_in < R(0)) ? qt_in * depth_inside_inv : R(0);
            w3 = qn_in * depth_inside_inv - sqrt_g_on_di * s_in;
            s_out = (-w3 + w1) / (R(2) * sqrt_g_on_di);
        } else {
            w1 = u_outside - sqrt_g_on_di * stage_outside;
            w2 = (qn_in > R(0)) ? qt_in * depth_inside_inv : R(0);
            w3 = qn_in * depth_inside_inv + sqrt_g_on_di * s_in;
            s_out = (w3 - w1) / (R(2) * sqrt_g_on_di);
        }
        qn_out = (w3 + w1) * K<R>::half() * depth_inside;
        qt_out = w2 * depth_inside;
    } else {
        s_out = stage_outside;
        qn_out = R(0);
        qt_out = R(0);
    }
}

}  // namespace swals
