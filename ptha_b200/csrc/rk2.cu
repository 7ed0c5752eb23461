// rk2.cu -- nonlinear finite-volume steps ('rk2', 'euler') on sm_100a.
//
// Restates, per Euler stage, in ONE fused kernel:
//   compute_depth_and_velocity            domain_mod.f90:1360-1419
//   compute_fluxes_DE1_low_fr_diffusion   compute_fluxes_alternatives_include.f90:25-36
//     -> DE1_inner_include.f90:78-727 (NS/EW edge loops),
//        :735-862 (theta wet/dry limiter + MC gradients),
//        extrapolation_limiting_mod.f90:44-79 (MC limiter)
//   update_U_manning / _chezy             update_U_DE1_inner_include.f90:14-99
//   the CFL max-reduction                 DE1_inner_include.f90:426-430,712-727
// and the rk2 driver (timestepping_alternatives_include.f90:64-146): stage 2
// averages with the backed-up state in the same pass.
//
// Each CTA owns a 32x8 tile of cells.  It stages the tile plus a 2-cell cross
// halo (the 5-point stencil of the limiter) in shared memory after the
// depth/velocity fix-ups, computes the limited gradients, then every NS and
// EW edge touching the tile (edges on tile borders are recomputed by both
// neighbours, ~8% extra), then updates its cells.  Fluxes, depth, velocity
// and explicit sources never reach HBM.  Edge loop bounds follow the
// reference exactly: edges exist only for i=2..nx, j=2..ny (1-based); the
// outer NS/EW gradients are zero; explicit_source of row 1 stays zero.
// Arithmetic order mirrors the reference statement by statement and the
// library is compiled without FMA contraction, so FP64 results equal the
// IEEE-strict oracle except where a libm function (pow) differs.
#include "rk2_common.cuh"

#include <cstdlib>
#include <cstring>

namespace swals {
namespace {
using namespace fv;

constexpr int TX = 32;
constexpr int TY = 8;
constexpr int NT = TX * TY;
constexpr int CW = TX + 4;   // cell window columns (i0-2 .. i0+TX+1)
constexpr int CH = TY + 4;   // cell window rows    (r0-2 .. r0+TY+1)

// Structure-of-arrays shared-memory tiles (one array per field, so a warp's
// accesses to one field are consecutive words).
template <typename R, int H, int W>
struct CellTile {
    R stg[H][W], dep[H][W], u[H][W], v[H][W], elv[H][W];
    __device__ __forceinline__ Cell<R> get(int r, int c) const
    {
        Cell<R> x;
        x.stg = stg[r][c]; x.dep = dep[r][c]; x.u = u[r][c]; x.v = v[r][c]; x.elv = elv[r][c];
        return x;
    }
    __device__ __forceinline__ void set(int r, int c, const Cell<R> &x)
    {
        stg[r][c] = x.stg; dep[r][c] = x.dep; u[r][c] = x.u; v[r][c] = x.v; elv[r][c] = x.elv;
    }
};
template <typename R, int H, int W>
struct GradTile {
    R ds[H][W], dd[H][W], du[H][W], dv[H][W];
    __device__ __forceinline__ Grad<R> get(int r, int c) const
    {
        Grad<R> g;
        g.ds = ds[r][c]; g.dd = dd[r][c]; g.du = du[r][c]; g.dv = dv[r][c];
        return g;
    }
    __device__ __forceinline__ void set(int r, int c, const Grad<R> &g)
    {
        ds[r][c] = g.ds; dd[r][c] = g.dd; du[r][c] = g.du; dv[r][c] = g.dv;
    }
};
template <typename R, int H, int W>
struct EdgeTile {
    R f0[H][W], f1[H][W], f2[H][W];
    double es_pos[H][W], es_neg[H][W];
    __device__ __forceinline__ EdgeRes<R> get(int r, int c) const
    {
        EdgeRes<R> e;
        e.f[0] = f0[r][c]; e.f[1] = f1[r][c]; e.f[2] = f2[r][c]; e.es_pos = es_pos[r][c]; e.es_neg = es_neg[r][c];
        return e;
    }
    __device__ __forceinline__ void set(int r, int c, const EdgeRes<R> &e)
    {
        f0[r][c] = e.f[0]; f1[r][c] = e.f[1]; f2[r][c] = e.f[2]; es_pos[r][c] = e.es_pos; es_neg[r][c] = e.es_neg;
    }
};

template <typename R>
struct Smem {
    CellTile<R, CH, CW> cell;
    GradTile<R, TY + 2, TX> gns;     // NS gradients, rows r0-1 .. r0+TY, cols i0 .. i0+TX-1
    GradTile<R, TY, TX + 2> gew;     // EW gradients, rows r0 .. r0+TY-1, cols i0-1 .. i0+TX
    EdgeTile<R, TY + 1, TX> ens;     // NS edges r0 .. r0+TY
    EdgeTile<R, TY, TX + 1> eew;     // EW edges i0 .. i0+TX
    double red[NT / 32];
    long long negfix[NT / 32];
};

template <typename R, int MODE, bool SPH, bool COR, int FRIC, bool EDDY>
__global__ void __launch_bounds__(NT, 3) rk2_stage_kernel(const Rk2Args<R> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem<R> &S = *reinterpret_cast<Smem<R> *>(smem_raw);

    const int nx = a.nx, ny = a.ny;
    const int64_t P = a.P;
    const int i0 = blockIdx.x * TX, r0 = blockIdx.y * TY;
    const int tid = threadIdx.x;
    const R mad = K<R>::min_depth();

    // ---- Phase A: cells with the depth/velocity fix-ups (domain_mod.f90:1387-1412)
    long long negfix = 0;
    for (int q = tid; q < CH * CW; q += NT) {
        const int rr = q / CW, cc = q - rr * CW;
        const int r = r0 - 2 + rr, i = i0 - 2 + cc;
        Cell<R> c;
        c.stg = R(0); c.dep = R(0); c.u = R(0); c.v = R(0); c.elv = R(0);
        if (r >= 0 && r < ny && i >= 0 && i < nx) {
            const int64_t o = (int64_t)r * P + i;
            R s = a.stg[o], e = a.elv[o];
            R dep = s - e;
            if (dep > mad) {
                R depth_inv = R(1) / dep;
                c.u = a.uh[o] * depth_inv;
                c.v = a.vh[o] * depth_inv;
            } else {
                if (dep < R(0)) {
                    dep = R(0);
                    s = e;
                    if (rr >= 2 && rr < 2 + TY && cc >= 2 && cc < 2 + TX) negfix += 1;
                }
            }
            c.stg = s; c.dep = dep; c.elv = e;
        }
        S.cell.set(rr, cc, c);
    }
    __syncthreads();

    // ---- Phase B: limited gradients (DE1_inner_include.f90:735-862)
    for (int q = tid; q < (TY + 2) * TX; q += NT) {
        const int rr = q / TX, cc = q - rr * TX;        // cell (i0+cc, r0-1+rr)
        const int r = r0 - 1 + rr, i = i0 + cc;
        Grad<R> g; g.ds = R(0); g.dd = R(0); g.du = R(0); g.dv = R(0);
        if (r > 0 && r < ny - 1 && i < nx) {
            const Cell<R> lo = S.cell.get(rr, cc + 2), c = S.cell.get(rr + 1, cc + 2), up = S.cell.get(rr + 2, cc + 2);
            const R th = theta_wd<R>(lo.dep, c.dep, up.dep, a.theta);
            g.ds = mc_half_gradient<R>(c.stg, lo.stg, up.stg, th);
            g.dd = mc_half_gradient<R>(c.dep, lo.dep, up.dep, th);
            g.du = mc_half_gradient<R>(c.u, lo.u, up.u, th);
            g.dv = mc_half_gradient<R>(c.v, lo.v, up.v, th);
        }
        S.gns.set(rr, cc, g);
    }
    for (int q = tid; q < TY * (TX + 2); q += NT) {
        const int rr = q / (TX + 2), cc = q - rr * (TX + 2);  // cell (i0-1+cc, r0+rr)
        const int r = r0 + rr, i = i0 - 1 + cc;
        Grad<R> g; g.ds = R(0); g.dd = R(0); g.du = R(0); g.dv = R(0);
        if (i > 0 && i < nx - 1 && r < ny) {
            const Cell<R> lo = S.cell.get(rr + 2, cc), c = S.cell.get(rr + 2, cc + 1), up = S.cell.get(rr + 2, cc + 2);
            const R th = theta_wd<R>(lo.dep, c.dep, up.dep, a.theta);
            g.ds = mc_half_gradient<R>(c.stg, lo.stg, up.stg, th);
            g.dd = mc_half_gradient<R>(c.dep, lo.dep, up.dep, th);
            g.du = mc_half_gradient<R>(c.u, lo.u, up.u, th);
            g.dv = mc_half_gradient<R>(c.v, lo.v, up.v, th);
        }
        S.gew.set(rr, cc, g);
    }
    __syncthreads();

    // ---- Phase C: edges touching the tile
    double cfl = 0.0;
    const R inv2 = R(1) / (a.m.dyl[0] * a.half_cfl);  // dx_cfl_half_inv(2): NS edges
    for (int q = tid; q < (TY + 1) * TX; q += NT) {
        const int rr = q / TX, cc = q - rr * TX;        // edge between (i, r-1) and (i, r)
        const int r = r0 + rr, i = i0 + cc;
        EdgeRes<R> e;
        e.f[0] = R(0); e.f[1] = R(0); e.f[2] = R(0); e.es_pos = 0.0; e.es_neg = 0.0;
        if (r >= 1 && r <= ny - 1 && i >= 1 && i <= nx - 1) {
            double cand;
            edge_flux<R, true, EDDY>(S.cell.get(rr + 1, cc + 2), S.gns.get(rr, cc), S.cell.get(rr + 2, cc + 2),
                                     S.gns.get(rr + 1, cc), a.m.dxb[r], inv2, e, cand, a.flux_variant,
                                     EDDY ? a.ev[(int64_t)(r - 1) * a.P + i] : R(0),
                                     EDDY ? a.ev[(int64_t)r * a.P + i] : R(0), EDDY ? a.m.dyl[i] : R(1));
            cfl = fmax(cfl, cand);
            if (MODE != MODE_CFL && a.lines) {
                if (r == ny - a.n_ext && i >= a.n_ext && i <= nx - a.n_ext - 1) a.lines[i] = (double)e.f[0];
                if (r == a.n_ext && i >= a.n_ext && i <= nx - a.n_ext - 1) a.lines[nx + ny + i] = (double)e.f[0];
            }
        }
        if (MODE != MODE_CFL) S.ens.set(rr, cc, e);
    }
    for (int q = tid; q < TY * (TX + 1); q += NT) {
        const int rr = q / (TX + 1), cc = q - rr * (TX + 1);  // edge between (i-1, r) and (i, r)
        const int r = r0 + rr, i = i0 + cc;
        EdgeRes<R> e;
        e.f[0] = R(0); e.f[1] = R(0); e.f[2] = R(0); e.es_pos = 0.0; e.es_neg = 0.0;
        if (r >= 1 && r <= ny - 1 && i >= 1 && i <= nx - 1) {
            const R inv1 = R(1) / (a.m.dxb[r] * a.half_cfl);  // dx_cfl_half_inv(1)
            double cand;
            const int64_t oe = (int64_t)r * a.P + i;
            edge_flux<R, false, EDDY>(S.cell.get(rr + 2, cc + 1), S.gew.get(rr, cc), S.cell.get(rr + 2, cc + 2),
                                      S.gew.get(rr, cc + 1), a.m.dyl[i], inv1, e, cand, a.flux_variant,
                                      EDDY ? a.ev[oe - 1] : R(0), EDDY ? a.ev[oe] : R(0),
                                      EDDY ? R(0.5) * (a.m.dxb[r] + a.m.dxb[r + 1]) : R(1));
            cfl = fmax(cfl, cand);
            if (MODE != MODE_CFL && a.lines) {
                if (i == nx - a.n_ext && r >= a.n_ext && r <= ny - a.n_ext - 1) a.lines[nx + r] = (double)e.f[0];
                if (i == a.n_ext && r >= a.n_ext && r <= ny - a.n_ext - 1) a.lines[2 * nx + ny + r] = (double)e.f[0];
            }
        }
        if (MODE != MODE_CFL) S.eew.set(rr, cc, e);
    }

    // Block max of the CFL candidates and the negative-depth count.
    const int lane = tid & 31, warp = tid >> 5;
    if (a.write_cfl || MODE == MODE_CFL) {
        for (int o = 16; o > 0; o >>= 1) cfl = fmax(cfl, __shfl_down_sync(0xffffffffu, cfl, o));
        if (lane == 0) S.red[warp] = cfl;
    }
    if (MODE != MODE_CFL) {
        for (int o = 16; o > 0; o >>= 1) negfix += __shfl_down_sync(0xffffffffu, negfix, o);
        if (lane == 0) S.negfix[warp] = negfix;
    }
    __syncthreads();
    if (tid == 0) {
        if (a.write_cfl || MODE == MODE_CFL) {
            double mx = S.red[0];
            for (int w = 1; w < NT / 32; w++) mx = fmax(mx, S.red[w]);
            if (mx > 0.0) atomic_max_pos_double(&a.sc->max_dt_inv_bits, mx);
        }
        if (MODE != MODE_CFL) {
            long long n = 0;
            for (int w = 0; w < NT / 32; w++) n += S.negfix[w];
            if (n) atomicAdd((unsigned long long *)&a.sc->negative_depth_fix_counter, (unsigned long long)n);
        }
    }
    if (MODE == MODE_CFL) return;

    // ---- Phase D: update_U (update_U_DE1_inner_include.f90:38-96)
    const int cc = tid & (TX - 1), rr = tid / TX;
    const int i = i0 + cc, r = r0 + rr;
    if (i >= nx || r >= ny) return;

    const R dt = stage_dt<R>(a);
    fv_update<R, MODE, SPH, COR, FRIC>(a, i, r, S.cell.get(rr + 2, cc + 2), S.ens.get(rr, cc), S.ens.get(rr + 1, cc),
                                       S.eew.get(rr, cc), S.eew.get(rr, cc + 1), dt, dt / a.m.area[r]);
}


// ---------------------------------------------------------------------------
// Boundary routines on the non-staggered grid (boundary_mod.f90:21-75 and
// :78-163).  The reference applies them in two OpenMP loops: a west/east pass
// over j, then a south/north pass over i, so a corner cell ends with its
// south/north value, and that value reads the west/east result of the cell
// next to it in the column.  Here one thread owns one ring cell; the corner
// threads recompute that west/east value themselves instead of reading it,
// so no thread reads a cell another thread writes and the kernel needs no
// grid-wide ordering.
//   STAGE_MODE 1: in place on the stage output (stage 1 of rk2, euler).
//   STAGE_MODE 2: rk2 stage 2.  The stage kernel already wrote the averaged
//                 state; the ring's inputs are the pre-average values the
//                 stage kernel saved in the side buffer, and the boundary
//                 values are averaged with the backed-up U0 ring here.
template <typename R>
struct BcArgs {
    int nx, ny;
    int64_t P;
    int kind;               // SWALS_BC_*
    int bext[4];            // N,E,S,W
    BoundaryFn bf;
    R msl;                  // msl_linear (flather's default outside stage)
    const R *x;
    R *stg, *uh, *vh;       // stage output planes
    const R *stg0, *uh0, *vh0;  // backup U0 (mode 2)
    R *elv;
    const R *side;          // mode 2: saved pre-average outer two rings
    R *max_stage;
    int pre_bf;             // column 0's boundary-function values from sc->bf_col0[n_dt - 1]
    int stage_mode;
    int dt_from_cfl;
    double dt_fixed;
    double max_dt_inv_init;
    int n_dt;               // boundary time = time0 + n_dt * dt (n_dt additions) ...
    R dt_extra;             // ... + dt * dt_extra when nonzero (midpoint half step, rk2n last step)
    DevScalars *sc;
    int leapfrog_half;      // a leapfrog step's boundary: time = time0 + dt/2 (dt = dt_fixed)
};

template <typename R> struct RingVal { R s, uh, vh, e; };

// Stage-output value of a cell in the outer two rings or the interior
// (mode 2 reads the saved pre-average copy; every cell of the outer two
// rings has both a column and a row copy).
template <typename R>
__device__ __forceinline__ R bc_get(const BcArgs<R> &a, int i, int r, int v)
{
    if (a.stage_mode == 2) {
        const int nx = a.nx, ny = a.ny;
        int k = -1;
        if (i == 0) k = 0; else if (i == 1) k = 1; else if (i == nx - 2) k = 2; else if (i == nx - 1) k = 3;
        if (k >= 0) return a.side[((int64_t)k * ny + r) * 3 + v];
        k = (r == 0) ? 0 : (r == 1) ? 1 : (r == ny - 1) ? 3 : 2;
        return a.side[(int64_t)4 * ny * 3 + ((int64_t)k * nx + i) * 3 + v];
    }
    const R *pl = (v == 0) ? a.stg : (v == 1) ? a.uh : a.vh;
    return pl[(int64_t)r * a.P + i];
}

// West/east pass value of ring cell (i, r), i in {0, nx-1}.  fs, fe: the
// boundary function's stage and elevation at column i (KIND 2; the device
// boundary functions do not depend on the row, so a corner thread evaluates
// the function once for its own cell and its column neighbour).
template <typename R, int KIND>
__device__ __forceinline__ RingVal<R> we_value(const BcArgs<R> &a, int i, int r, double t, R fs, R fe)
{
    const int in = (i == 0) ? 1 : a.nx - 2;
    RingVal<R> v;
    if (KIND == 1) {  // transmissive: all four variables from the inner neighbour
        v.e = a.elv[(int64_t)r * a.P + in];
        v.s = bc_get(a, in, r, 0); v.uh = bc_get(a, in, r, 1); v.vh = bc_get(a, in, r, 2);
    } else if (KIND == 3) {  // flather: normal momentum UH
        v.e = a.elv[(int64_t)r * a.P + i];
        flather_cell<R>(a.bf, a.x, t, i, r, a.msl, i == 0, bc_get(a, in, r, 0), bc_get(a, in, r, 1),
                        bc_get(a, in, r, 2), a.elv[(int64_t)r * a.P + in], v.e, v.s, v.uh, v.vh);
    } else {
        v.s = fs;
        v.e = fe;
        v.uh = bc_get(a, in, r, 1);
        v.vh = R(0);
    }
    return v;
}

// KIND (= a.kind) is a template parameter so that each boundary routine's
// kernel carries only its own code.
template <typename R, int KIND>
__global__ void __launch_bounds__(256) rk2_boundary_kernel(const BcArgs<R> a)
{
    const int nx = a.nx, ny = a.ny;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    // Ring cells, each once: rows 0 and ny-1 in full, then columns 0 and
    // nx-1 for rows 1..ny-2.
    int i, r;
    if (q < 2 * nx) { i = q % nx; r = (q < nx) ? 0 : ny - 1; }
    else if (q < 2 * nx + 2 * (ny - 2)) { const int p = q - 2 * nx; r = 1 + p % (ny - 2); i = (p < ny - 2) ? 0 : nx - 1; }
    else return;
    const bool sn = (r == 0 && a.bext[2]) || (r == ny - 1 && a.bext[0]);
    const bool we = (i == 0 && a.bext[3]) || (i == nx - 1 && a.bext[1]);
    if (!sn && !we) return;

    double dtd;
    if (a.dt_from_cfl) {
        double bits_max = __longlong_as_double((long long)a.sc->max_dt_inv_bits);
        R inv = R(fmax(a.max_dt_inv_init, bits_max));
        dtd = (double)(R(1) / inv);
    } else {
        dtd = (double)R(a.dt_fixed);
    }
    double t;
    if (a.leapfrog_half) {
        t = a.sc->time0 + (double)(R(dtd) * K<R>::half());
    } else {
        t = a.sc->time;
        for (int k = 0; k < a.n_dt; k++) t = t + dtd;
        if (a.dt_extra != R(0)) t = t + (double)(R(dtd) * a.dt_extra);
    }

    R fs = R(0), fe = R(0);
    if (KIND != 1 && KIND != 3) {
        if (a.pre_bf && i == 0) {
            fs = R(a.sc->bf_col0[a.n_dt - 1][0]);
            fe = R(a.sc->bf_col0[a.n_dt - 1][1]);
        } else {
            boundary_function<R>(a.bf, a.x, t, i, r, fs, fe);
        }
    }
    RingVal<R> v;
    if (sn) {
        const int rn = (r == 0) ? 1 : ny - 2;
        // The column neighbour after the west/east pass.
        RingVal<R> nb;
        const bool nb_we = (i == 0 && a.bext[3]) || (i == nx - 1 && a.bext[1]);
        if (nb_we) {
            nb = we_value<R, KIND>(a, i, rn, t, fs, fe);
        } else {
            nb.e = a.elv[(int64_t)rn * a.P + i];
            nb.s = bc_get(a, i, rn, 0); nb.uh = bc_get(a, i, rn, 1); nb.vh = bc_get(a, i, rn, 2);
        }
        if (KIND == 1) {
            v = nb;
        } else if (KIND == 3) {  // flather: normal momentum VH
            v.e = a.elv[(int64_t)r * a.P + i];
            flather_cell<R>(a.bf, a.x, t, i, r, a.msl, r == 0, nb.s, nb.vh, nb.uh, nb.e, v.e, v.s, v.vh, v.uh);
        } else {
            v.s = fs;
            v.e = fe;
            v.uh = R(0);
            v.vh = nb.vh;
        }
    } else {
        v = we_value<R, KIND>(a, i, r, t, fs, fe);
    }

    const int64_t o = (int64_t)r * a.P + i;
    a.elv[o] = v.e;
    if (a.stage_mode != 2) {
        a.stg[o] = v.s; a.uh[o] = v.uh; a.vh[o] = v.vh;
        return;
    }
    // rk2 average of the ring cell and its max_stage.
    const R s = R(0.5) * (v.s + a.stg0[o]);
    a.stg[o] = s;
    a.uh[o] = R(0.5) * (v.uh + a.uh0[o]);
    a.vh[o] = R(0.5) * (v.vh + a.vh0[o]);
    if (a.max_stage) {
        R mx = a.max_stage[o];
        a.max_stage[o] = (s > mx) ? s : mx;
    }
}

template <typename R>
cudaError_t launch_boundary(const BcArgs<R> &b, cudaStream_t s)
{
    const int n = 2 * b.nx + 2 * (b.ny - 2);
    const int blocks = (n + 255) / 256;
    if (b.kind == 1) rk2_boundary_kernel<R, 1><<<blocks, 256, 0, s>>>(b);
    else if (b.kind == 3) rk2_boundary_kernel<R, 3><<<blocks, 256, 0, s>>>(b);
    else rk2_boundary_kernel<R, 2><<<blocks, 256, 0, s>>>(b);
    return cudaGetLastError();
}

// End of a step: domain%max_dt, time, boundary-flux integrals, counters
// (timestepping_alternatives_include.f90:36-50,121-144; domain_mod.f90:1800-1810).
// kind: FIN_RK2 (two Euler stages averaged), FIN_EULER, FIN_MIDPOINT (the
// store of the midpoint's fluxes), FIN_RK2N (n = 5 Euler steps, the last
// one shortened, timestepping_alternatives_include.f90:149-270).  `lines` holds one set of
// 2 nx + 2 ny boundary-flux line values per flux evaluation.
enum { FIN_RK2 = 0, FIN_EULER = 1, FIN_MIDPOINT = 2, FIN_RK2N = 3 };
constexpr int RK2N_N = 5;   // rk2n_n_value (domain_mod.f90:90)

// The step's point gauges, recorded by the finalize kernel from the step's
// final planes (n = 0: none): records[rec][g][STG, UH, VH], as the
// separate gauge kernel stores them.
template <typename R>
struct FinGauges {
    const R *stg, *uh, *vh;
    int64_t P;
    const int *sites;
    int n;
    double *records;
    int capacity;
};

template <typename R>
FinGauges<R> fin_gauges(const StepConfig &c, R *const pl[3], int64_t pitch)
{
    FinGauges<R> g{};
    if (c.g_n > 0) {
        g.stg = pl[0]; g.uh = pl[1]; g.vh = pl[2];
        g.P = pitch;
        g.sites = c.g_sites;
        g.n = c.g_n;
        g.records = c.g_records;
        g.capacity = c.g_capacity;
    }
    return g;
}

template <typename R, int KIND>
__global__ void __launch_bounds__(1024) rk2_finalize_kernel(int nx, int ny, int n_ext, const double *lines,
                                                            int dt_from_cfl, double dt_fixed, double max_dt_inv_init,
                                                            DevScalars *sc, FinGauges<R> g)
{
    constexpr int NSETS = (KIND == FIN_EULER) ? 1 : (KIND == FIN_RK2N) ? RK2N_N : 2;
    __shared__ double red[4 * NSETS][32];
    // gauges first: every read of the record count precedes thread 0's update
    // below (the __syncthreads of the reduction lies between)
    const int rec = g.n ? sc->gauge_records : 0;
    if (rec < g.capacity)
        for (int q = threadIdx.x; q < g.n; q += blockDim.x) {
            const int64_t o = (int64_t)g.sites[2 * q + 1] * g.P + g.sites[2 * q];
            double *dst = g.records + ((int64_t)rec * g.n + q) * 3;
            dst[0] = (double)g.stg[o];
            dst[1] = (double)g.uh[o];
            dst[2] = (double)g.vh[o];
        }
    double acc[4 * NSETS];
#pragma unroll
    for (int k = 0; k < 4 * NSETS; k++) acc[k] = 0.0;
    const int L = 2 * nx + 2 * ny;
#pragma unroll 4
    for (int q = threadIdx.x; q < L; q += blockDim.x) {
        int line, idx;
        if (q < nx) { line = 0; idx = q; }
        else if (q < nx + ny) { line = 1; idx = q - nx; }
        else if (q < 2 * nx + ny) { line = 2; idx = q - nx - ny; }
        else { line = 3; idx = q - 2 * nx - ny; }
        const int lim = (line == 0 || line == 2) ? nx : ny;
        if (idx < n_ext || idx > lim - n_ext - 1) continue;
#pragma unroll
        for (int k = 0; k < NSETS; k++) {
            const double v = lines[(int64_t)k * L + q];
#pragma unroll
            for (int l = 0; l < 4; l++)
                if (line == l) acc[4 * k + l] += v;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4 * NSETS; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    // the warps' partial sums, combined by warp 0 (lane w holds warp w's)
    if (warp != 0) return;
    const int nw = blockDim.x >> 5;
    double s[4 * NSETS];
#pragma unroll
    for (int k = 0; k < 4 * NSETS; k++) {
        double v = (lane < nw) ? red[k][lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        s[k] = v;
    }
    if (lane != 0) return;
    double bits_max = __longlong_as_double((long long)sc->max_dt_inv_bits);
    R max_dt_inv = R(fmax(max_dt_inv_init, bits_max));
    const double max_dt = (double)(R(1) / max_dt_inv);
    const double dt = dt_from_cfl ? max_dt : (double)R(dt_fixed);
    const double time0 = sc->time;
    double store[NSETS][4], tot[NSETS];
    for (int q = 0; q < NSETS; q++) {
        store[q][0] = s[4 * q]; store[q][1] = s[4 * q + 1]; store[q][2] = -s[4 * q + 2]; store[q][3] = -s[4 * q + 3];
        tot[q] = 0.0;
        for (int k = 0; k < 4; k++) tot[q] += store[q][k];
    }
    double integral;
    double dt_last = dt;
    double t_end = time0 + dt;
    int last = 0;
    if (KIND == FIN_RK2) {
        integral = 0.0 + dt * tot[0];
        integral = integral + dt * tot[1];
        integral = 0.5 * integral;
        last = 1;
    } else if (KIND == FIN_EULER) {
        integral = 0.0 + dt * tot[0];
    } else if (KIND == FIN_MIDPOINT) {
        integral = tot[1] * dt;
        last = 1;
    } else {
        const R n_inverse = R(1) / (R(1) * R(RK2N_N));
        integral = 0.0;
        for (int q = 0; q < NSETS - 1; q++) integral = integral + dt * tot[q];
        integral = integral * (double)(R(RK2N_N) - R(1)) * (double)n_inverse;
        const R reduced_dt = (R(1) * R(RK2N_N) - R(1)) * n_inverse * R(dt);
        integral = integral + (double)reduced_dt * tot[NSETS - 1];
        dt_last = (double)reduced_dt;
        t_end = time0 + (double)(R(dt) * R(RK2N_N - 1));
        last = NSETS - 1;
    }
    for (int k = 0; k < 4; k++) sc->boundary_flux_store[k] = store[last][k];
    sc->boundary_flux_evolve_integral = integral;
    sc->boundary_flux_time_integral += integral;
    sc->max_dt = max_dt;
    sc->dt = dt;
    sc->dt_last_update = dt_last;
    sc->time0 = time0;
    sc->time = t_end;
    sc->evolve_step_dt = sc->time - time0;
    sc->nsteps_advanced += 1;
    sc->max_dt_inv_bits = 0ull;
    if (g.n) sc->gauge_records = rec + 1;
}

template <typename R, int MODE, bool SPH, bool COR, int FRIC, bool EDDY>
cudaError_t launch_stage_tile(const Rk2Args<R> &a, cudaStream_t s)
{
    static bool configured = false;
    const size_t smem = sizeof(Smem<R>);
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(rk2_stage_kernel<R, MODE, SPH, COR, FRIC, EDDY>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        // Prefer shared memory over L1 so three CTAs fit per SM.
        e = cudaFuncSetAttribute(rk2_stage_kernel<R, MODE, SPH, COR, FRIC, EDDY>,
                                 cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    dim3 grid((a.nx + TX - 1) / TX, (a.ny + TY - 1) / TY);
    rk2_stage_kernel<R, MODE, SPH, COR, FRIC, EDDY><<<grid, NT, smem, s>>>(a);
    return cudaGetLastError();
}

// The eddy-viscosity fluxes are a separate instantiation (the CFL pass never
// needs them), so the default kernels carry none of their code.
template <typename R, int MODE, bool SPH, bool COR, int FRIC>
cudaError_t launch_stage(const Rk2Args<R> &a, cudaStream_t s)
{
    if constexpr (MODE != MODE_CFL) {
        if (a.flux_variant & FLUX_EDDY) return launch_stage_tile<R, MODE, SPH, COR, FRIC, true>(a, s);
    }
    return launch_stage_tile<R, MODE, SPH, COR, FRIC, false>(a, s);
}

}  // namespace

template <typename R, int MODE, bool SPH, bool COR, int FRIC>
cudaError_t launch_stage_stream(const fv::Rk2Args<R> &a, cudaStream_t s);

namespace {

// Stage kernel variant: register streaming (default) or shared-memory tiles,
// chosen by SWALS_FV_KERNEL=stream|tile.
bool use_stream_kernel()
{
    // read at every launch, so that a process can switch forms between steps
    const char *e = getenv("SWALS_FV_KERNEL");
    return !(e && strcmp(e, "tile") == 0);
}

template <typename R, int MODE, bool SPH, bool COR, int FRIC>
cudaError_t launch_stage_any(const Rk2Args<R> &a, cudaStream_t s)
{
    if (use_stream_kernel()) return launch_stage_stream<R, MODE, SPH, COR, FRIC>(a, s);
    return launch_stage<R, MODE, SPH, COR, FRIC>(a, s);
}

// The update of one cell from its loaded inputs.
template <typename R, int FRIC>
__device__ __forceinline__ void update_cell(const Rk2Args<R> &a, int i, int r, R sv, R ev, R uh_in, R vh_in,
                                            const CellFlux<R> &f, R dt, R area, long long &negfix)
{
    // compute_depth_and_velocity (domain_mod.f90:1387-1412)
    Cell<R> c;
    R dep = sv - ev;
    c.u = R(0); c.v = R(0);
    if (dep > K<R>::min_depth()) {
        const R depth_inv = R(1) / dep;
        c.u = uh_in * depth_inv;
        c.v = vh_in * depth_inv;
    } else if (dep < R(0)) {
        dep = R(0);
        sv = ev;
        negfix += 1;
    }
    c.stg = sv; c.dep = dep; c.elv = ev;
    // U(i,j,UH/VH) after the fix-ups (fixed_momenta)
    const bool wet = c.dep > K<R>::min_depth();
    const R Um_uh = wet ? uh_in : R(0), Um_vh = wet ? vh_in : R(0);
    fv_apply<R, MODE_STAGE1, FRIC>(a, i, r, c, Um_uh, Um_vh, f, dt, dt / area);
}

// Cells per thread and CTAs per SM of the stage-1 update.  Measured on the
// 2048^2 FP64 step: one cell, 4 CTAs 0.081 ms (0.097 with the stored terms
// loaded after the depth test); two cells, 3 CTAs 0.077 ms (0.88 of the
// measured HBM bandwidth for its 104 B a cell); two cells, 2 CTAs 0.093.
#ifndef SWALS_UPDATE_CELLS
#define SWALS_UPDATE_CELLS 2
#endif
#ifndef SWALS_UPDATE_MINB
#define SWALS_UPDATE_MINB 3
#endif

// Stage-1 update of an adaptive step from the per-cell flux and source sums
// the flux pass stored (cell_flux): the same fix-ups and fv_apply as the
// stage kernels, SWALS_UPDATE_CELLS adjacent cells per thread.  Every load
// of a cell is issued before its first branch, so that the cell costs one
// memory round trip: the state, the stored update terms, the stage dt (one
// line for all threads), the row's area and (into L1, for the friction
// branch) n^2.  A memory-latency-bound kernel.
template <typename R, bool SPH, bool COR, int FRIC>
__global__ void __launch_bounds__(256, SWALS_UPDATE_MINB) rk2_update_kernel(const Rk2Args<R> a)
{
    constexpr int NC = SWALS_UPDATE_CELLS;
    const int i0 = (blockIdx.x * 32 + threadIdx.x) * NC;
    const int r = blockIdx.y * 8 + threadIdx.y;
    const int nx = a.nx, ny = a.ny;
    if (a.pre_bf && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y < 2) {
        // Column 0's boundary-function values at the step's two stage
        // boundaries (time + dt, time + dt + dt, as the boundary kernel forms
        // them), one per warp, off the boundary kernels' critical path.
        const double bits_max = __longlong_as_double((long long)a.sc->max_dt_inv_bits);
        const R inv = R(fmax(a.max_dt_inv_init, bits_max));
        const double dtd = (double)(R(1) / inv);
        double t = a.sc->time + dtd;
        if (threadIdx.y == 1) t = t + dtd;
        R fs, fe;
        boundary_function<R>(a.bf, a.bf_x, t, 0, 0, fs, fe);
        a.sc->bf_col0[threadIdx.y][0] = (double)fs;
        a.sc->bf_col0[threadIdx.y][1] = (double)fe;
    }
    long long negfix = 0;
    if (i0 < nx && r < ny) {
        const int64_t o0 = (int64_t)r * a.P + i0;
        R sv[NC], ev[NC], uh_in[NC], vh_in[NC];
        CellFlux<R> f[NC];
#pragma unroll
        for (int q = 0; q < NC; q++) {
            if (i0 + q < nx) {
                const int64_t o = o0 + q;
                if (FRIC != FRIC_NONE) asm volatile("prefetch.global.L1 [%0];" ::"l"(a.nsq + o));
                sv[q] = a.stg[o]; ev[q] = a.elv[o]; uh_in[q] = a.uh[o]; vh_in[q] = a.vh[o];
                f[q].d[0] = a.cs.d[0][o]; f[q].d[1] = a.cs.d[1][o]; f[q].d[2] = a.cs.d[2][o];
                f[q].eu = a.cs.eu[o]; f[q].ev = a.cs.ev[o];
            }
        }
        const R dt = stage_dt<R>(a);
        const R area = a.m.area[r];
#pragma unroll
        for (int q = 0; q < NC; q++)
            if (i0 + q < nx) update_cell<R, FRIC>(a, i0 + q, r, sv[q], ev[q], uh_in[q], vh_in[q], f[q], dt, area, negfix);
    }
    for (int off = 16; off > 0; off >>= 1) negfix += __shfl_down_sync(0xffffffffu, negfix, off);
    if ((threadIdx.x & 31) == 0 && negfix)
        atomicAdd((unsigned long long *)&a.sc->negative_depth_fix_counter, (unsigned long long)negfix);
}

template <typename R, bool SPH, bool COR, int FRIC>
cudaError_t launch_flux_pass(const Rk2Args<R> &a, cudaStream_t s)
{
    return launch_stage_stream<R, MODE_FLUX, SPH, COR, FRIC>(a, s);
}

template <typename R, bool SPH, bool COR, int FRIC>
cudaError_t launch_update(const Rk2Args<R> &a, cudaStream_t s)
{
    constexpr int NC = SWALS_UPDATE_CELLS;
    dim3 block(32, 8), grid((a.nx + 32 * NC - 1) / (32 * NC), (a.ny + 7) / 8);
    rk2_update_kernel<R, SPH, COR, FRIC><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

// Run F<R, SPH, COR, FRIC>(a, s) for the step configuration.
#define SWALS_DISPATCH_FV(FN)                                                                          \
    const int fric = c.nofriction ? FRIC_NONE : (c.chezy ? FRIC_CHEZY : FRIC_MANNING);                 \
    if (c.spherical) {                                                                                 \
        if (c.coriolis) {                                                                              \
            if (fric == FRIC_MANNING) return FN<R, true, true, FRIC_MANNING>(a, s);                    \
            if (fric == FRIC_CHEZY) return FN<R, true, true, FRIC_CHEZY>(a, s);                        \
            return FN<R, true, true, FRIC_NONE>(a, s);                                                 \
        }                                                                                              \
        if (fric == FRIC_MANNING) return FN<R, true, false, FRIC_MANNING>(a, s);                       \
        if (fric == FRIC_CHEZY) return FN<R, true, false, FRIC_CHEZY>(a, s);                           \
        return FN<R, true, false, FRIC_NONE>(a, s);                                                    \
    }                                                                                                  \
    if (fric == FRIC_MANNING) return FN<R, false, false, FRIC_MANNING>(a, s);                          \
    if (fric == FRIC_CHEZY) return FN<R, false, false, FRIC_CHEZY>(a, s);                              \
    return FN<R, false, false, FRIC_NONE>(a, s);

// get_eddy_viscosity (DE1_inner_include.f90:864-1017) for every cell of the
// stage input, before the fluxes that use it: constant when
// eddy_visc_constants(2) is 0, else constant + Shiono-Knight
// (c2 depth**(5/6) sqrt(n^2 g speed^2)), clipped to
// 0.25 min(2dx, 2dy)^2 / (2 dt_last_update + 1e-10); columns 1 and nx take
// the clipped values of columns 2 and nx-1 (nx >= 3).
template <typename R>
__global__ void __launch_bounds__(256) eddy_visc_kernel(const Rk2Args<R> a)
{
    const int i = blockIdx.x * 32 + threadIdx.x, r = blockIdx.y * 8 + threadIdx.y;
    const int nx = a.nx, ny = a.ny;
    if (i >= nx || r >= ny) return;
    const int is = (i < 1) ? 1 : ((i > nx - 2) ? nx - 2 : i);
    const int64_t o = (int64_t)r * a.P + is;
    R dep = a.stg[o] - a.elv[o], u = R(0), v = R(0);
    if (dep > K<R>::min_depth()) {
        const R depth_inv = R(1) / dep;
        u = a.uh[o] * depth_inv;
        v = a.vh[o] * depth_inv;
    } else if (dep < R(0)) {
        dep = R(0);
    }
    R ev;
    if (a.ev_c2 == R(0))
        ev = a.ev_c1;
    else
        ev = a.ev_c1 + a.ev_c2 * R(pow_eddy_cr((double)dep)) * R(sqrt(a.nsq[o] * K<R>::gravity() * (u * u + v * v)));
    const R two_dx = a.m.dxb[r] + a.m.dxb[r + 1];
    const R two_dy = a.m.dyl[is] + a.m.dyl[is + 1];
    const R lim = R(0.25) * rmin(two_dx * two_dx, two_dy * two_dy) /
                  (R(2.0) * R(a.sc->dt_last_update) + R(1.0e-10));
    a.ev[(int64_t)r * a.P + i] = rmin(ev, lim);
}

// domain%dt_last_update = dt of the update just made (update_U_DE1_inner_include.f90:17).
template <typename R>
__global__ void dt_last_update_kernel(const Rk2Args<R> a)
{
    a.sc->dt_last_update = (double)stage_dt<R>(a);
}

template <typename R>
cudaError_t launch_eddy_visc(const Rk2Args<R> &a, cudaStream_t s)
{
    dim3 block(32, 8), grid((a.nx + 31) / 32, (a.ny + 7) / 8);
    eddy_visc_kernel<R><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_dt_last_update(const Rk2Args<R> &a, cudaStream_t s)
{
    dt_last_update_kernel<R><<<1, 1, 0, s>>>(a);
    return cudaGetLastError();
}

template <typename R>
cudaError_t dispatch_flux(const Rk2Args<R> &a, const StepConfig &c, cudaStream_t s)
{
    if (a.flux_variant & FLUX_EDDY) {
        const cudaError_t e = launch_eddy_visc<R>(a, s);
        if (e != cudaSuccess) return e;
    }
    SWALS_DISPATCH_FV(launch_flux_pass)
}

template <typename R>
cudaError_t dispatch_update_fv(const Rk2Args<R> &a, const StepConfig &c, cudaStream_t s) { SWALS_DISPATCH_FV(launch_update) }

template <typename R>
cudaError_t dispatch_update(const Rk2Args<R> &a, const StepConfig &c, cudaStream_t s)
{
    const cudaError_t e = dispatch_update_fv<R>(a, c, s);
    if (e != cudaSuccess || !(a.flux_variant & FLUX_EDDY)) return e;
    return launch_dt_last_update<R>(a, s);
}

template <typename R, int MODE>
cudaError_t dispatch_stage_fv(const Rk2Args<R> &a, const StepConfig &c, cudaStream_t s);

// A stage kernel launch; with eddy viscosity, the viscosity of the stage
// input first and, after an update, dt_last_update.  The CFL pass does not
// depend on the viscosity and runs without it.
template <typename R, int MODE>
cudaError_t dispatch_stage(const Rk2Args<R> &a, const StepConfig &c, cudaStream_t s)
{
    if (!(a.flux_variant & FLUX_EDDY)) return dispatch_stage_fv<R, MODE>(a, c, s);
    if (MODE == MODE_CFL) {
        Rk2Args<R> b = a;
        b.flux_variant &= ~FLUX_EDDY;
        return dispatch_stage_fv<R, MODE>(b, c, s);
    }
    cudaError_t e = launch_eddy_visc<R>(a, s);
    if (e == cudaSuccess) e = dispatch_stage_fv<R, MODE>(a, c, s);
    if (e == cudaSuccess) e = launch_dt_last_update<R>(a, s);
    return e;
}

template <typename R, int MODE>
cudaError_t dispatch_stage_fv(const Rk2Args<R> &a, const StepConfig &c, cudaStream_t s)
{
    const int fric = c.nofriction ? FRIC_NONE : (c.chezy ? FRIC_CHEZY : FRIC_MANNING);
    if (c.spherical) {
        if (c.coriolis) {
            if (fric == FRIC_MANNING) return launch_stage_any<R, MODE, true, true, FRIC_MANNING>(a, s);
            if (fric == FRIC_CHEZY) return launch_stage_any<R, MODE, true, true, FRIC_CHEZY>(a, s);
            return launch_stage_any<R, MODE, true, true, FRIC_NONE>(a, s);
        }
        if (fric == FRIC_MANNING) return launch_stage_any<R, MODE, true, false, FRIC_MANNING>(a, s);
        if (fric == FRIC_CHEZY) return launch_stage_any<R, MODE, true, false, FRIC_CHEZY>(a, s);
        return launch_stage_any<R, MODE, true, false, FRIC_NONE>(a, s);
    }
    if (fric == FRIC_MANNING) return launch_stage_any<R, MODE, false, false, FRIC_MANNING>(a, s);
    if (fric == FRIC_CHEZY) return launch_stage_any<R, MODE, false, false, FRIC_CHEZY>(a, s);
    return launch_stage_any<R, MODE, false, false, FRIC_NONE>(a, s);
}

}  // namespace

namespace {

// Stage arguments common to every stage of a finite-volume step.
template <typename R>
Rk2Args<R> fv_args(int nx, int ny, int64_t pitch, R *elv, R *manning_sq, const Metrics<R> &m, const StepConfig &c,
                   double dt, const Rk2Buffers &buf, DevScalars *sc)
{
    Rk2Args<R> a;
    a.nx = nx; a.ny = ny; a.P = pitch;
    a.elv = elv; a.nsq = manning_sq; a.max_stage = nullptr; a.m = m;
    a.theta = R(c.theta); a.half_cfl = R(0.5) * R(c.cfl);
    a.lin_fric = R(c.linear_friction_coeff);
    a.dt_fixed = dt;
    a.max_dt_inv_init = (double)(R(1) / R(c.maximum_timestep));
    a.n_ext = c.exterior_cells_width;
    a.bc_ring = 0;
    for (int k = 0; k < 4; k++) a.bext[k] = c.bext[k];
    a.side = reinterpret_cast<R *>(buf.side);
    a.sc = sc;
    a.stg0 = nullptr; a.uh0 = nullptr; a.vh0 = nullptr;
    a.cs = CellSums<R>{};
    a.flux_variant = c.flux_variant;
    a.dt_scale = R(1);
    a.base0 = 0;
    a.lines = nullptr;
    a.write_cfl = 0;
    a.dt_from_cfl = 0;
    a.ev = reinterpret_cast<R *>(c.eddy_visc);
    a.ev_c1 = R(c.eddy_visc_constants[0]);
    a.ev_c2 = R(c.eddy_visc_constants[1]);
    if (!a.ev) a.flux_variant &= ~FLUX_EDDY;
    a.pre_bf = 0;
    a.bf = c.bf;
    a.bf_x = m.x;
    return a;
}

// Boundary-kernel arguments of a step.
template <typename R>
BcArgs<R> bc_args(const Rk2Args<R> &a, const StepConfig &c, double dt)
{
    BcArgs<R> b;
    b.nx = a.nx; b.ny = a.ny; b.P = a.P; b.kind = c.bc_kind;
    for (int k = 0; k < 4; k++) b.bext[k] = c.bext[k];
    b.bf = c.bf; b.msl = R(c.msl_linear); b.x = a.m.x; b.elv = const_cast<R *>(a.elv); b.side = a.side;
    b.max_stage = nullptr;
    b.dt_extra = R(0);
    b.dt_from_cfl = a.dt_from_cfl; b.dt_fixed = dt; b.max_dt_inv_init = a.max_dt_inv_init; b.sc = a.sc;
    b.stg0 = nullptr; b.uh0 = nullptr; b.vh0 = nullptr;
    b.n_dt = 1;
    b.stage_mode = 1;
    b.leapfrog_half = 0;
    b.pre_bf = a.pre_bf;
    return b;
}

// The first flux evaluation of a step, from planes[A] into planes[B]
// (one_euler_step's compute_fluxes + update_U): with stored edges and an
// adaptive dt, a flux pass (edges, CFL maximum, boundary-flux lines) and an
// update once dt is known; otherwise a CFL pass (adaptive only) and the fused
// stage kernel.  `a` carries dt_scale and max_stage; returns with a's planes
// and dt flags set as the stage used them.
template <typename R>
cudaError_t first_stage(Rk2Args<R> &a, R *const planes[3][3], int A, int B, bool has_dt, const Rk2Buffers &buf,
                        double *lines, const StepConfig &c, cudaStream_t s, const LaunchHook &hook)
{
    cudaError_t e;
    const bool stored = !has_dt && buf.edges && use_stream_kernel();
    if (stored) {
        char *q = reinterpret_cast<char *>(buf.edges);
        const int64_t plane = a.P * (int64_t)a.ny;
        auto take_r = [&]() { R *p = reinterpret_cast<R *>(q); q += plane * sizeof(R); return p; };
        auto take_d = [&]() { double *p = reinterpret_cast<double *>(q); q += plane * sizeof(double); return p; };
        // doubles first (8-byte alignment whatever R is)
        a.cs.eu = take_d(); a.cs.ev = take_d();
        for (int k = 0; k < 3; k++) a.cs.d[k] = take_r();
        Rk2Args<R> p = a;
        p.stg = planes[A][0]; p.uh = planes[A][1]; p.vh = planes[A][2];
        p.stg_o = nullptr; p.uh_o = nullptr; p.vh_o = nullptr;
        p.dt_from_cfl = 0; p.write_cfl = 1; p.lines = lines;
        hook(CAT_CFL, 0);
        e = dispatch_flux<R>(p, c, s);
        hook(CAT_CFL, 1);
        if (e != cudaSuccess) return e;
    } else if (!has_dt) {
        // Adaptive: the CFL of U0 must be known before the first update.
        Rk2Args<R> p = a;
        p.stg = planes[A][0]; p.uh = planes[A][1]; p.vh = planes[A][2];
        p.stg_o = nullptr; p.uh_o = nullptr; p.vh_o = nullptr;
        p.dt_from_cfl = 0; p.write_cfl = 1; p.lines = nullptr;
        hook(CAT_CFL, 0);
        e = dispatch_stage<R, MODE_CFL>(p, c, s);
        hook(CAT_CFL, 1);
        if (e != cudaSuccess) return e;
    }
    a.stg = planes[A][0]; a.uh = planes[A][1]; a.vh = planes[A][2];
    a.stg_o = planes[B][0]; a.uh_o = planes[B][1]; a.vh_o = planes[B][2];
    a.dt_from_cfl = has_dt ? 0 : 1;
    a.write_cfl = has_dt ? 1 : 0;
    a.lines = lines;
    if (!stored) a.pre_bf = 0;   // only the update kernel stores the boundary-function values
    hook(CAT_STAGE1, 0);
    e = stored ? dispatch_update<R>(a, c, s) : dispatch_stage<R, MODE_STAGE1>(a, c, s);
    hook(CAT_STAGE1, 1);
    return e;
}

// A later Euler stage with the first stage's dt (rk2 / rk2n sub-steps,
// midpoint full step): planes[in] -> planes[out], no CFL accumulation.
template <typename R>
cudaError_t later_stage(Rk2Args<R> a, R *const planes[3][3], int in, int out, bool has_dt, double *lines,
                        const StepConfig &c, cudaStream_t s, const LaunchHook &hook, int cat)
{
    a.stg = planes[in][0]; a.uh = planes[in][1]; a.vh = planes[in][2];
    a.stg_o = planes[out][0]; a.uh_o = planes[out][1]; a.vh_o = planes[out][2];
    a.dt_from_cfl = has_dt ? 0 : 1;
    a.write_cfl = 0;
    a.lines = lines;
    hook(cat, 0);
    cudaError_t e = dispatch_stage<R, MODE_STAGE1>(a, c, s);
    hook(cat, 1);
    return e;
}

bool has_bc(const StepConfig &c) { return c.bc_kind == 1 || c.bc_kind == 2 || c.bc_kind == 3; }

// The end of update_U into planes[P_] (domain_mod.f90:1564-1582):
// update_boundary, then apply_forcing, at the update's time time0 + n_dt dt
// (+ dt * extra, which is then the update's dt).
template <typename R>
cudaError_t end_of_update(BcArgs<R> &b, const StepConfig &c, R *const planes[3][3], int P_, int n_dt, R extra,
                          cudaStream_t s, const LaunchHook &hook, int cat)
{
    b.stg = planes[P_][0]; b.uh = planes[P_][1]; b.vh = planes[P_][2];
    b.stage_mode = 1; b.n_dt = n_dt; b.dt_extra = extra;
    cudaError_t e = cudaSuccess;
    if (has_bc(c)) {
        hook(cat, 0);
        e = launch_boundary<R>(b, s);
        hook(cat, 1);
        if (e != cudaSuccess) return e;
    }
    if (c.n_forcing) {
        ForcingClock clk{};
        clk.mode = FORCE_FV_STAGE;
        clk.n_dt = n_dt;
        clk.dt_extra = (double)extra;
        clk.dt_from_cfl = b.dt_from_cfl;
        clk.dt_fixed = b.dt_fixed;
        clk.max_dt_inv_init = b.max_dt_inv_init;
        e = launch_forcing<R>(c, clk, b.P, b.stg, b.uh, b.vh, b.elv, b.sc, s, hook, cat);
    }
    return e;
}

// rk2's average U = (U + U0) / 2 (timestepping_alternatives_include.f90:
// 124-135), for the unfused stage 2 (forcing patches present).
template <typename R>
__global__ void rk2_average_kernel(int nx, int ny, int64_t P, R *u0, R *u1, R *u2, const R *b0, const R *b1,
                                   const R *b2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
    if (i >= nx) return;
    const int64_t o = (int64_t)r * P + i;
    u0[o] = R(0.5) * (u0[o] + b0[o]);
    u1[o] = R(0.5) * (u1[o] + b1[o]);
    u2[o] = R(0.5) * (u2[o] + b2[o]);
}

}  // namespace

template <typename R>
cudaError_t launch_rk2_step(R *const planes[3][3], int &cur, R *elv, R *max_stage, R *manning_sq, int nx, int ny,
                            int64_t pitch, const Metrics<R> &m, const StepConfig &c, bool has_dt, double dt,
                            bool euler_only, const Rk2Buffers &buf, DevScalars *sc, cudaStream_t s,
                            const LaunchHook &hook)
{
    const int A = cur, B = (cur + 1) % 3, C = (cur + 2) % 3;
    const bool bc = has_bc(c);
    double *lines1 = reinterpret_cast<double *>(buf.partials);
    double *lines2 = lines1 + (2 * nx + 2 * ny);
    const double max_dt_inv_init = (double)(R(1) / R(c.maximum_timestep));
    cudaError_t e;

    // Stage 1: U0 -> B.  With the stage-from-function boundary (bc_kind 2)
    // the stage-1 update kernel (adaptive steps) evaluates column 0's
    // boundary function for the two stage boundaries (n_dt 1 and 2 below).
    Rk2Args<R> a = fv_args<R>(nx, ny, pitch, elv, manning_sq, m, c, dt, buf, sc);
    a.pre_bf = (c.bc_kind == 2) ? 1 : 0;
    e = first_stage<R>(a, planes, A, B, has_dt, buf, lines1, c, s, hook);
    if (e != cudaSuccess) return e;

    BcArgs<R> b = bc_args<R>(a, c, dt);
    if ((e = end_of_update<R>(b, c, planes, B, 1, R(0), s, hook, CAT_BC1)) != cudaSuccess) return e;
    if (euler_only) {
        if (max_stage) {
            hook(CAT_MAXSTAGE, 0);
            e = launch_update_max_stage<R>(nx, ny, pitch, planes[B][0], max_stage, c, s);
            hook(CAT_MAXSTAGE, 1);
            if (e != cudaSuccess) return e;
        }
        hook(CAT_FINALIZE, 0);
        rk2_finalize_kernel<R, FIN_EULER><<<1, 1024, 0, s>>>(nx, ny, c.exterior_cells_width, lines1,
                                                             a.dt_from_cfl, dt, max_dt_inv_init, sc,
                                                             fin_gauges<R>(c, planes[B], pitch));
        hook(CAT_FINALIZE, 1);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        cur = B;
        return cudaSuccess;
    }
    if (c.n_forcing) {
        // Stage 2 as an Euler step, its boundary and forcing, then the average.
        e = later_stage<R>(a, planes, B, C, has_dt, lines2, c, s, hook, CAT_STAGE2);
        if (e != cudaSuccess) return e;
        if ((e = end_of_update<R>(b, c, planes, C, 2, R(0), s, hook, CAT_BC2)) != cudaSuccess) return e;
        hook(CAT_STAGE2, 0);
        rk2_average_kernel<R><<<dim3((nx + 255) / 256, ny), 256, 0, s>>>(
            nx, ny, pitch, planes[C][0], planes[C][1], planes[C][2], planes[A][0], planes[A][1], planes[A][2]);
        hook(CAT_STAGE2, 1);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (max_stage) {
            hook(CAT_MAXSTAGE, 0);
            e = launch_update_max_stage<R>(nx, ny, pitch, planes[C][0], max_stage, c, s);
            hook(CAT_MAXSTAGE, 1);
            if (e != cudaSuccess) return e;
        }
        hook(CAT_FINALIZE, 0);
        rk2_finalize_kernel<R, FIN_RK2><<<1, 1024, 0, s>>>(nx, ny, c.exterior_cells_width, lines1, a.dt_from_cfl,
                                                           dt, max_dt_inv_init, sc,
                                                           fin_gauges<R>(c, planes[C], pitch));
        hook(CAT_FINALIZE, 1);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        cur = C;
        return cudaSuccess;
    }
    // Stage 2: B -> C, averaged with U0 (A)
    Rk2Args<R> a2 = a;
    a2.stg = planes[B][0]; a2.uh = planes[B][1]; a2.vh = planes[B][2];
    a2.stg0 = planes[A][0]; a2.uh0 = planes[A][1]; a2.vh0 = planes[A][2];
    a2.stg_o = planes[C][0]; a2.uh_o = planes[C][1]; a2.vh_o = planes[C][2];
    a2.dt_from_cfl = has_dt ? 0 : 1;
    a2.write_cfl = 0;
    a2.lines = lines2;
    a2.bc_ring = bc ? 1 : 0;
    a2.max_stage = max_stage;
    hook(CAT_STAGE2, 0);
    e = dispatch_stage<R, MODE_STAGE2>(a2, c, s);
    hook(CAT_STAGE2, 1);
    if (e != cudaSuccess) return e;
    if (bc) {
        b.stg = planes[C][0]; b.uh = planes[C][1]; b.vh = planes[C][2];
        b.stg0 = planes[A][0]; b.uh0 = planes[A][1]; b.vh0 = planes[A][2];
        b.stage_mode = 2; b.n_dt = 2; b.max_stage = max_stage;
        hook(CAT_BC2, 0);
        e = launch_boundary<R>(b, s);
        hook(CAT_BC2, 1);
        if (e != cudaSuccess) return e;
    }
    hook(CAT_FINALIZE, 0);
    rk2_finalize_kernel<R, FIN_RK2><<<1, 1024, 0, s>>>(nx, ny, c.exterior_cells_width, lines1, a.dt_from_cfl,
                                              dt, max_dt_inv_init, sc, fin_gauges<R>(c, planes[C], pitch));
    hook(CAT_FINALIZE, 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cur = C;
    return cudaSuccess;
}

namespace {

// rk2n: backup_U = (backup_U - U) / n (timestepping_alternatives_include.f90:211-220).
template <typename R>
__global__ void rk2n_backup_kernel(int nx, int ny, int64_t P, R *b0, R *b1, R *b2, const R *u0, const R *u1,
                                   const R *u2, R n_inverse)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
    if (i >= nx) return;
    const int64_t o = (int64_t)r * P + i;
    b0[o] = (b0[o] - u0[o]) * n_inverse;
    b1[o] = (b1[o] - u1[o]) * n_inverse;
    b2[o] = (b2[o] - u2[o]) * n_inverse;
}

// rk2n: U = U + backup_U (:237-247), then update_max_quantities (max_stage
// over the active region, dry cells included).
template <typename R>
__global__ void rk2n_final_kernel(int nx, int ny, int64_t P, R *u0, R *u1, R *u2, const R *b0, const R *b1,
                                  const R *b2, R *max_stage, int xl, int xu, int yl, int yu)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
    if (i >= nx) return;
    const int64_t o = (int64_t)r * P + i;
    const R st = u0[o] + b0[o];
    u0[o] = st;
    u1[o] = u1[o] + b1[o];
    u2[o] = u2[o] + b2[o];
    if (max_stage && i >= xl && i <= xu && r >= yl && r <= yu) {
        const R mx = max_stage[o];
        max_stage[o] = (st > mx) ? st : mx;
    }
}

}  // namespace

// one_midpoint_step (timestepping_alternatives_include.f90:273-337):
// U0 (A) -> the midpoint state (B) with dt/2, then the full step of U0 with
// the midpoint's fluxes, depth and velocity (C).
template <typename R>
cudaError_t launch_midpoint_step(R *const planes[3][3], int &cur, R *elv, R *max_stage, R *manning_sq, int nx, int ny,
                                 int64_t pitch, const Metrics<R> &m, const StepConfig &c, bool has_dt, double dt,
                                 const Rk2Buffers &buf, DevScalars *sc, cudaStream_t s, const LaunchHook &hook)
{
    const int A = cur, B = (cur + 1) % 3, C = (cur + 2) % 3;
    const bool bc = has_bc(c);
    double *lines1 = reinterpret_cast<double *>(buf.partials);
    double *lines2 = lines1 + (2 * nx + 2 * ny);
    cudaError_t e;

    Rk2Args<R> a = fv_args<R>(nx, ny, pitch, elv, manning_sq, m, c, dt, buf, sc);
    a.dt_scale = K<R>::half();
    e = first_stage<R>(a, planes, A, B, has_dt, buf, lines1, c, s, hook);
    if (e != cudaSuccess) return e;
    BcArgs<R> b = bc_args<R>(a, c, dt);
    // update_U(dt/2) ends with update_boundary and apply_forcing at time + dt/2
    if ((e = end_of_update<R>(b, c, planes, B, 0, K<R>::half(), s, hook, CAT_BC1)) != cudaSuccess) return e;
    Rk2Args<R> a2 = a;
    a2.dt_scale = R(1);
    a2.base0 = 1;
    a2.stg0 = planes[A][0]; a2.uh0 = planes[A][1]; a2.vh0 = planes[A][2];
    e = later_stage<R>(a2, planes, B, C, has_dt, lines2, c, s, hook, CAT_STAGE2);
    if (e != cudaSuccess) return e;
    if ((e = end_of_update<R>(b, c, planes, C, 1, R(0), s, hook, CAT_BC2)) != cudaSuccess) return e;
    if (max_stage) {
        hook(CAT_MAXSTAGE, 0);
        e = launch_update_max_stage<R>(nx, ny, pitch, planes[C][0], max_stage, c, s);
        hook(CAT_MAXSTAGE, 1);
        if (e != cudaSuccess) return e;
    }
    hook(CAT_FINALIZE, 0);
    rk2_finalize_kernel<R, FIN_MIDPOINT><<<1, 1024, 0, s>>>(nx, ny, c.exterior_cells_width, lines1,
                                                            has_dt ? 0 : 1, dt, a.max_dt_inv_init, sc,
                                                            fin_gauges<R>(c, planes[C], pitch));
    hook(CAT_FINALIZE, 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cur = C;
    return cudaSuccess;
}

// one_rk2n_step (timestepping_alternatives_include.f90:149-270) with n = 5:
// A holds the backup; n-1 Euler steps A -> B -> C -> B -> C, backup =
// (backup - U)/n, a last step C -> B with (n-1)/n of dt, and U = B + backup.
// `dt` is the caller's timestep (n-1 sub-steps of dt/(n-1)).
template <typename R>
cudaError_t launch_rk2n_step(R *const planes[3][3], int &cur, R *elv, R *max_stage, R *manning_sq, int nx, int ny,
                             int64_t pitch, const Metrics<R> &m, const StepConfig &c, bool has_dt, double dt,
                             const Rk2Buffers &buf, DevScalars *sc, cudaStream_t s, const LaunchHook &hook)
{
    const int A = cur, B = (cur + 1) % 3, C = (cur + 2) % 3;
    const bool bc = has_bc(c);
    const int L = 2 * nx + 2 * ny;
    double *lines = reinterpret_cast<double *>(buf.partials);
    const R n_inverse = R(1) / (R(1) * R(RK2N_N));
    // dt_first_step = timestep / (n - 1)
    const double dt_sub = has_dt ? (double)(R(dt) / (R(RK2N_N) - R(1))) : 0.0;
    cudaError_t e;

    Rk2Args<R> a = fv_args<R>(nx, ny, pitch, elv, manning_sq, m, c, dt_sub, buf, sc);
    e = first_stage<R>(a, planes, A, B, has_dt, buf, lines, c, s, hook);
    if (e != cudaSuccess) return e;
    BcArgs<R> b = bc_args<R>(a, c, dt_sub);
    auto boundary = [&](int P_, int n_dt, R extra) -> cudaError_t {
        return end_of_update<R>(b, c, planes, P_, n_dt, extra, s, hook, CAT_BC1);
    };
    if ((e = boundary(B, 1, R(0))) != cudaSuccess) return e;
    // sub-steps 2 .. n-1
    const int seq[RK2N_N] = {B, C, B, C, B};
    for (int k = 1; k < RK2N_N - 1; k++) {
        e = later_stage<R>(a, planes, seq[k - 1], seq[k], has_dt, lines + (int64_t)k * L, c, s, hook, CAT_STAGE2);
        if (e != cudaSuccess) return e;
        if ((e = boundary(seq[k], k + 1, R(0))) != cudaSuccess) return e;
    }
    const int U4 = seq[RK2N_N - 2], U5 = seq[RK2N_N - 1];
    const dim3 eg((nx + 255) / 256, ny);
    hook(CAT_FINALIZE, 0);
    rk2n_backup_kernel<R><<<eg, 256, 0, s>>>(nx, ny, pitch, planes[A][0], planes[A][1], planes[A][2], planes[U4][0],
                                            planes[U4][1], planes[U4][2], n_inverse);
    hook(CAT_FINALIZE, 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // the last sub-step, (n-1)/n of dt
    Rk2Args<R> a5 = a;
    a5.dt_scale = (R(1) * R(RK2N_N) - R(1)) * n_inverse;
    e = later_stage<R>(a5, planes, U4, U5, has_dt, lines + (int64_t)(RK2N_N - 1) * L, c, s, hook, CAT_STAGE2);
    if (e != cudaSuccess) return e;
    if ((e = boundary(U5, RK2N_N - 1, a5.dt_scale)) != cudaSuccess) return e;
    hook(CAT_MAXSTAGE, 0);
    rk2n_final_kernel<R><<<eg, 256, 0, s>>>(nx, ny, pitch, planes[U5][0], planes[U5][1], planes[U5][2],
                                           planes[A][0], planes[A][1], planes[A][2], max_stage, c.xl, c.xu, c.yl,
                                           c.yu);
    hook(CAT_MAXSTAGE, 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    hook(CAT_FINALIZE, 0);
    rk2_finalize_kernel<R, FIN_RK2N><<<1, 1024, 0, s>>>(nx, ny, c.exterior_cells_width, lines, has_dt ? 0 : 1,
                                              dt_sub, a.max_dt_inv_init, sc, fin_gauges<R>(c, planes[U5], pitch));
    hook(CAT_FINALIZE, 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cur = U5;
    return cudaSuccess;
}

#define SWALS_INST_FV_STEPS(R)                                                                                      \
    template cudaError_t launch_midpoint_step<R>(R *const[3][3], int &, R *, R *, R *, int, int, int64_t,           \
                                                 const Metrics<R> &, const StepConfig &, bool, double,              \
                                                 const Rk2Buffers &, DevScalars *, cudaStream_t, const LaunchHook &); \
    template cudaError_t launch_rk2n_step<R>(R *const[3][3], int &, R *, R *, R *, int, int, int64_t,               \
                                             const Metrics<R> &, const StepConfig &, bool, double,                  \
                                             const Rk2Buffers &, DevScalars *, cudaStream_t, const LaunchHook &);
SWALS_INST_FV_STEPS(double)
SWALS_INST_FV_STEPS(float)

template cudaError_t launch_rk2_step<double>(double *const[3][3], int &, double *, double *, double *, int, int,
                                             int64_t, const Metrics<double> &, const StepConfig &, bool, double,
                                             bool, const Rk2Buffers &, DevScalars *, cudaStream_t,
                                             const LaunchHook &);
template cudaError_t launch_rk2_step<float>(float *const[3][3], int &, float *, float *, float *, int, int,
                                            int64_t, const Metrics<float> &, const StepConfig &, bool, double,
                                            bool, const Rk2Buffers &, DevScalars *, cudaStream_t,
                                            const LaunchHook &);

// update_boundary after the stage sweep of 'leapfrog_nonlinear'
// (domain_mod_leapfrog_nonlinear_include.f90:122-140) for flather_boundary:
// the ring of the new stage and of the (not yet updated) momenta, in place,
// at time0 + dt/2, by the finite-volume boundary kernel (west/east pass,
// then south/north with the corners from the first).
template <typename R>
cudaError_t launch_leapfrog_boundary(int nx, int ny, int64_t pitch, R *stg, R *uh, R *vh, R *elv, const Metrics<R> &m,
                                     const StepConfig &c, R dt, DevScalars *sc, cudaStream_t s)
{
    BcArgs<R> b;
    b.nx = nx; b.ny = ny; b.P = pitch; b.kind = c.bc_kind;
    for (int k = 0; k < 4; k++) b.bext[k] = c.bext[k];
    b.bf = c.bf; b.msl = R(c.msl_linear); b.x = m.x;
    b.stg = stg; b.uh = uh; b.vh = vh; b.elv = elv;
    b.stg0 = nullptr; b.uh0 = nullptr; b.vh0 = nullptr; b.side = nullptr; b.max_stage = nullptr;
    b.stage_mode = 1;
    b.dt_from_cfl = 0; b.dt_fixed = (double)dt; b.max_dt_inv_init = 0.0;
    b.n_dt = 0; b.dt_extra = R(0); b.sc = sc;
    b.leapfrog_half = 1;
    b.pre_bf = 0;
    return launch_boundary<R>(b, s);
}
template cudaError_t launch_leapfrog_boundary<double>(int, int, int64_t, double *, double *, double *, double *,
                                                      const Metrics<double> &, const StepConfig &, double,
                                                      DevScalars *, cudaStream_t);
template cudaError_t launch_leapfrog_boundary<float>(int, int, int64_t, float *, float *, float *, float *,
                                                     const Metrics<float> &, const StepConfig &, float, DevScalars *,
                                                     cudaStream_t);

}  // namespace swals
