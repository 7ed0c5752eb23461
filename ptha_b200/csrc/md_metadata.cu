// md_metadata.cu -- the multidomain nesting metadata builder, native host
// code: setup_multidomain + setup_multidomain_domains for one image
// (multidomain_mod.f90:2663-3553).
//
// From the domains' interior extents it computes
//  * each domain's nesting-layer width (compute_multidomain_nesting_layer_
//    width, :620-716; get_domain_nesting_layer_thickness, :1803-1852) and
//    widens the domain by that many cells on its nesting boundaries
//    (:2860-2895);
//  * the priority domain of every cell (find_priority_domain_containing_xy,
//    :1538-1677: the finest domain whose interior bounding box holds the
//    cell centre, by the point_in_poly crossing test);
//  * the receive boxes (convert_priority_domain_info_to_boxes, :718-958:
//    row-wise runs of the priority domain within nest_layer_width of the
//    domain's own priority cells, merged over rows while the runs match);
//  * the send boxes (:3090-3140) and the pairing of every receive box that
//    needs communication with its send box (:3170-3330).
// Coordinates use the reference's expressions in IEEE double, so the
// integer boxes equal the reference's.  The result feeds swals_gpu_md_create.
#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "domain_internal.h"

struct swals_md_metadata {
    std::vector<swals_md_exchange> exchanges;
    std::vector<std::vector<int32_t>> pind, pimg;   // per domain, i fastest (nx x ny)
    std::vector<std::vector<std::array<int64_t, 6>>> recv_metadata;
};

namespace {

using swals::api_fail;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return api_fail(code, buf);
}

// timestepping_metadata_mod.f90:60-160: halo cells one evolve_one_step consumes.
int nesting_thickness_of(const char *m)
{
    static const struct { const char *name; int w; } tab[] = {
        {"rk2", 4}, {"rk2n", 10}, {"midpoint", 4}, {"euler", 2}, {"linear", 2},
        {"leapfrog_linear_plus_nonlinear_friction", 2}, {"cliffs", 2}, {"leapfrog_nonlinear", 3}};
    for (const auto &t : tab)
        if (strcmp(m, t.name) == 0) return t.w;
    return -1;
}

long nint(double v) { return (long)std::floor(std::fabs(v) + 0.5) * (v >= 0 ? 1 : -1); }

struct Dom {
    swals_nest_domain_desc *d;
    double dx[2];
    double bbox[4][2];   // ll, lr, ur, ul
};

// check_periodic for one coordinate (multidomain_mod.f90:280-346).
double periodic_shift(double v, double lo, double hi, bool adjust, bool *flag)
{
    const bool below = v < lo, above = v > hi;
    if (flag) *flag = below || above;
    if (!adjust) return v;
    if (below) return (hi - lo) + v;
    if (above) return (-(hi - lo)) + v;
    return v;
}

// point_in_poly (util/points_in_poly_mod.f90:31-58) on the 4-vertex box.
bool inside_rectangle(const double b[4][2], double px, double py)
{
    bool inside = false;
    for (int i = 0; i < 4; i++) {
        const int j = (i == 0) ? 3 : i - 1;
        const bool crosses = (b[i][1] > py) != (b[j][1] > py);
        if (crosses) {
            const double g0 = (b[j][0] - b[i][0]) * (py - b[i][1]) / (b[j][1] - b[i][1]) + b[i][0];
            if (px < g0) inside = !inside;
        }
    }
    return inside;
}

// find_priority_domain_containing_xy for one point: (1-based index or -1,
// image, dx of the chosen domain).  Returns nonzero on an overlap of two
// domains with the same cell size.
int priority_of(const std::vector<Dom> &doms, double x, double y, const double pxs[2], const double pys[2],
                int *ind, int *img, double ddx[2])
{
    *ind = -1;
    *img = -1;
    const double big = -std::sqrt(DBL_MAX - 1.0e6);
    ddx[0] = big;
    ddx[1] = big;
    const double px = periodic_shift(x, pxs[0], pxs[1], true, nullptr);
    const double py = periodic_shift(y, pys[0], pys[1], true, nullptr);
    for (size_t di = 0; di < doms.size(); di++) {
        const Dom &d = doms[di];
        bool zero = true;
        for (int k = 0; k < 4; k++) zero = zero && d.bbox[k][0] == 0.0 && d.bbox[k][1] == 0.0;
        if (zero) continue;
        if (!inside_rectangle(d.bbox, px, py)) continue;
        const double area1 = d.dx[0] * d.dx[1];
        const double area2 = ddx[0] * ddx[1];
        if (area1 < area2) {
            *ind = (int)di + 1;
            *img = 1;
            ddx[0] = d.dx[0];
            ddx[1] = d.dx[1];
        } else if (std::fabs(area1 - area2) < 1.0e-2 * std::min(area1, area2)) {
            return fail(SWALS_ERR_INVALID_ARGUMENT, "domains with the same cell size overlap around (%.17g, %.17g)", x,
                        y);
        }
    }
    return 0;
}

// get_domain_xs_ys (multidomain_mod.f90:1854-1880).
double xs_of(const swals_nest_domain_desc *d, int i) { return d->lower_left[0] + ((i - 0.5) * d->lw[0]) / d->nx[0]; }
double ys_of(const swals_nest_domain_desc *d, int j) { return d->lower_left[1] + ((j - 0.5) * d->lw[1]) / d->nx[1]; }
// domain%x, domain%y (domain_mod.f90:941).
double x_of(const swals_nest_domain_desc *d, int i) { return d->lower_left[0] + ((i - 0.5) / (d->nx[0] * 1.0)) * d->lw[0]; }
double y_of(const swals_nest_domain_desc *d, int j) { return d->lower_left[1] + ((j - 0.5) / (d->nx[1] * 1.0)) * d->lw[1]; }

// find_priority_nesting_domains_along_a_boundary (multidomain_mod.f90:
// 1679-1800): cell centres one cell outside boundary b (1..4 = N, E, S, W),
// extended by one cell past each end.
void boundary_points(const Dom &D, int b, std::vector<double> &xs, std::vector<double> &ys)
{
    const swals_nest_domain_desc *d = D.d;
    const int width = 1;
    const double dx = D.dx[0], dy = D.dx[1];
    if (b == 1 || b == 3) {
        const int n1 = d->nx[0], n2 = n1 + 2 * width;
        xs.assign(n2, 0.0);
        for (int i = 0; i < n1; i++) xs[width + i] = xs_of(d, i + 1);
        for (int i = 1; i <= width; i++) {
            xs[i - 1] = xs_of(d, 1) - (width - (i - 1)) * dx;
            xs[n2 - (width - i) - 1] = xs_of(d, n1) + i * dx;
        }
        const double yv = (b == 1) ? ys_of(d, d->nx[1]) + dy * width : ys_of(d, 1) - dy * width;
        ys.assign(n2, yv);
    } else {
        const int n1 = d->nx[1], n2 = n1 + 2 * width;
        ys.assign(n2, 0.0);
        for (int j = 0; j < n1; j++) ys[width + j] = ys_of(d, j + 1);
        for (int i = 1; i <= width; i++) {
            ys[i - 1] = ys_of(d, 1) - (width - (i - 1)) * dy;
            ys[n2 - (width - i) - 1] = ys_of(d, n1) + i * dy;
        }
        const double xv = (b == 2) ? xs_of(d, d->nx[0]) + dx * width : xs_of(d, 1) - dx * width;
        xs.assign(n2, xv);
    }
}

// get_domain_nesting_layer_thickness (multidomain_mod.f90:1803-1852).
int layer_thickness(const swals_nest_domain_desc *d, double mpdr, int extra_halo_buffer, int extra_cells_in_halo)
{
    int required = nesting_thickness_of(d->timestepping_method);
    if (d->use_eddy_viscosity) required = (required * 3) / 2;
    long thickness = (long)required * d->timestepping_refinement_factor + extra_cells_in_halo;
    if (thickness < d->minimum_nesting_layer_thickness) thickness = d->minimum_nesting_layer_thickness;
    const long r = nint(mpdr);
    if (r > 1)
        thickness = ((long)std::ceil(thickness * 1.0 / mpdr) + extra_halo_buffer) * r;
    else
        thickness = (long)std::ceil(thickness * 1.0 / mpdr) * r;
    return (int)thickness;
}

// convert_priority_domain_info_to_boxes (multidomain_mod.f90:718-958): rows
// (ind, img, iL, iU, jL, jU), 1-based, in the reference's order (a box is
// appended on the first row where its run no longer appears; boxes open at
// the last row follow in creation order).
int priority_boxes(const std::vector<int32_t> &pind, const std::vector<int32_t> &pimg, int nx, int ny, int halo,
                   int myindex, const std::vector<bool> &in_px, const std::vector<bool> &in_py,
                   std::vector<std::array<int64_t, 6>> &out)
{
    // is_in_active_region (:2021-2045): within `halo` cells (Chebyshev) of
    // one of the domain's own priority cells; a 2-D prefix sum of the mask.
    std::vector<int64_t> c((size_t)(nx + 1) * (ny + 1), 0);
    auto C = [&](int i, int j) -> int64_t & { return c[(size_t)j * (nx + 1) + i]; };
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const size_t q = (size_t)j * nx + i;
            const int64_t m = (pind[q] == myindex && pimg[q] == 1) ? 1 : 0;
            C(i + 1, j + 1) = m + C(i, j + 1) + C(i + 1, j) - C(i, j);
        }
    auto active = [&](int i, int j) {
        const int i0 = std::max(i - halo, 0), i1 = std::min(i + halo, nx - 1) + 1;
        const int j0 = std::max(j - halo, 0), j1 = std::min(j + halo, ny - 1) + 1;
        return C(i1, j1) - C(i0, j1) - C(i1, j0) + C(i0, j0) > 0;
    };
    struct Run { int64_t ind, img, s, e; };
    std::vector<std::array<int64_t, 6>> cand;
    std::vector<Run> runs;
    for (int j = 0; j < ny; j++) {
        runs.clear();
        int64_t pi = -2, pm = -2;
        bool pp = false;
        for (int i = 0; i < nx; i++) {
            const size_t q = (size_t)j * nx + i;
            const bool a = active(i, j);
            const int64_t ni = a ? pind[q] : 0, nm = a ? pimg[q] : 0;
            if (i == 0 || ni != pi || nm != pm || in_px[i] != pp) runs.push_back({ni, nm, i + 1, i + 1});
            else runs.back().e = i + 1;
            pi = ni; pm = nm; pp = in_px[i];
        }
        if (j == 0) {
            for (const Run &r : runs) cand.push_back({r.ind, r.img, r.s, r.e, 1, -1});
            continue;
        }
        auto same = [](const std::array<int64_t, 6> &c0, const Run &r) {
            return c0[0] == r.ind && c0[1] == r.img && c0[2] == r.s && c0[3] == r.e;
        };
        const bool py_now = in_py[j], py_prev = in_py[j - 1];
        std::vector<std::array<int64_t, 6>> keep;
        for (auto &c0 : cand) {
            bool found = false;
            for (const Run &r : runs) found = found || (same(c0, r) && py_prev == py_now);
            if (found) keep.push_back(c0);
            else { c0[5] = j; out.push_back(c0); }
        }
        for (const Run &r : runs) {
            bool found = false;
            for (const auto &c0 : cand) found = found || (same(c0, r) && py_prev == py_now);
            if (!found) keep.push_back({r.ind, r.img, r.s, r.e, (int64_t)j + 1, -1});
        }
        cand.swap(keep);
        if (j == ny - 1) {
            for (auto &c0 : cand) { c0[5] = ny; out.push_back(c0); }
            cand.clear();
        }
    }
    if (ny == 1) {
        for (auto &c0 : cand) { c0[5] = 1; out.push_back(c0); }
    }
    for (const auto &b : out) {
        if (b[0] == 0) continue;
        for (int64_t j = b[4] - 1; j < b[5]; j++)
            for (int64_t i = b[2] - 1; i < b[3]; i++) {
                const size_t q = (size_t)j * nx + i;
                if (pind[q] != b[0] || pimg[q] != b[1] || in_px[i] != in_px[b[2] - 1] || in_py[j] != in_py[b[4] - 1])
                    return fail(SWALS_ERR_INVALID_ARGUMENT, "inconsistent box in priority-domain metadata");
            }
    }
    return 0;
}

}  // namespace

extern "C" {

int swals_md_build_metadata(swals_nest_domain_desc *domains, int32_t n, int32_t extra_halo_buffer,
                            int32_t extra_cells_in_halo, const double periodic_xs[2], const double periodic_ys[2],
                            swals_md_metadata **out)
{
    if (!domains || n < 1 || !out) return fail(SWALS_ERR_INVALID_ARGUMENT, "swals_md_build_metadata: bad arguments");
    *out = nullptr;
    const double pxs[2] = {periodic_xs ? periodic_xs[0] : -DBL_MAX, periodic_xs ? periodic_xs[1] : DBL_MAX};
    const double pys[2] = {periodic_ys ? periodic_ys[0] : -DBL_MAX, periodic_ys ? periodic_ys[1] : DBL_MAX};
    std::vector<Dom> doms((size_t)n);
    for (int k = 0; k < n; k++) {
        swals_nest_domain_desc *d = &domains[k];
        if (d->nx[0] < 1 || d->nx[1] < 1 || nesting_thickness_of(d->timestepping_method) < 0 ||
            d->timestepping_refinement_factor < 1)
            return fail(SWALS_ERR_INVALID_ARGUMENT, "domain %d: bad extent, method or refinement factor", k + 1);
        Dom &D = doms[k];
        D.d = d;
        D.dx[0] = d->lw[0] / (1.0 * d->nx[0]);
        D.dx[1] = d->lw[1] / (1.0 * d->nx[1]);
        bool zero = true;
        for (int q = 0; q < 8; q++) zero = zero && d->interior_bounding_box[q] == 0.0;
        if (zero) {   // create_all_bbox_and_dx (multidomain_mod.f90:960-1060)
            const double *ll = d->lower_left, *lw = d->lw;
            const double b[4][2] = {{ll[0], ll[1]}, {ll[0] + lw[0] * 1.0, ll[1] + lw[1] * 0.0},
                                    {ll[0] + lw[0], ll[1] + lw[1]}, {ll[0] + lw[0] * 0.0, ll[1] + lw[1] * 1.0}};
            for (int q = 0; q < 4; q++) {
                d->interior_bounding_box[2 * q] = b[q][0];
                d->interior_bounding_box[2 * q + 1] = b[q][1];
            }
        }
        for (int q = 0; q < 4; q++) {
            D.bbox[q][0] = d->interior_bounding_box[2 * q];
            D.bbox[q][1] = d->interior_bounding_box[2 * q + 1];
        }
    }

    // Nesting-layer width (multidomain_mod.f90:636-716).
    std::vector<double> xs, ys;
    for (int k = 0; k < n; k++) {
        swals_nest_domain_desc *d = doms[k].d;
        double mpdr = 1.0;
        for (int b = 1; b <= 4; b++) {
            boundary_points(doms[k], b, xs, ys);
            double dmax[2] = {-DBL_MAX, -DBL_MAX};
            bool any_img = false;
            for (size_t q = 0; q < xs.size(); q++) {
                int ind, img;
                double ddx[2];
                if (priority_of(doms, xs[q], ys[q], pxs, pys, &ind, &img, ddx)) return SWALS_ERR_INVALID_ARGUMENT;
                dmax[0] = std::max(dmax[0], ddx[0]);
                dmax[1] = std::max(dmax[1], ddx[1]);
                any_img = any_img || img > 0;
            }
            if (dmax[0] > 0 && dmax[1] > 0) {
                const double r0 = (double)nint(dmax[0] / doms[k].dx[0]), r1 = (double)nint(dmax[1] / doms[k].dx[1]);
                mpdr = std::max(mpdr, std::max(r0, r1));
            }
            d->is_nesting_boundary[b - 1] = any_img ? 1 : 0;
        }
        d->max_parent_dx_ratio = mpdr;
        d->nest_layer_width = layer_thickness(d, mpdr, extra_halo_buffer, extra_cells_in_halo);
    }

    // Widen the nesting boundaries (multidomain_mod.f90:2860-2895).
    for (int k = 0; k < n; k++) {
        swals_nest_domain_desc *d = doms[k].d;
        const int w = d->nest_layer_width;
        const double *dx = doms[k].dx;
        for (int b = 1; b <= 4; b++) {
            if (!d->is_nesting_boundary[b - 1]) continue;
            if (b == 2 || b == 4) { d->lw[0] = d->lw[0] + w * dx[0]; d->nx[0] = d->nx[0] + w; }
            if (b == 1 || b == 3) { d->lw[1] = d->lw[1] + w * dx[1]; d->nx[1] = d->nx[1] + w; }
            if (b == 3) d->lower_left[1] = d->lower_left[1] - w * dx[1];
            if (b == 4) d->lower_left[0] = d->lower_left[0] - w * dx[0];
        }
    }

    swals_md_metadata *M = new swals_md_metadata();
    M->pind.resize(n);
    M->pimg.resize(n);
    M->recv_metadata.resize(n);
    auto bail = [&](int code) { delete M; return code; };

    // Priority domains and receive boxes (:2897-3030).
    for (int k = 0; k < n; k++) {
        swals_nest_domain_desc *d = doms[k].d;
        const int nx = d->nx[0], ny = d->nx[1];
        std::vector<int32_t> &pind = M->pind[k], &pimg = M->pimg[k];
        pind.assign((size_t)nx * ny, 0);
        pimg.assign((size_t)nx * ny, 0);
        std::vector<bool> in_px(nx), in_py(ny);
        for (int i = 0; i < nx; i++) { bool f; periodic_shift(xs_of(d, i + 1), pxs[0], pxs[1], false, &f); in_px[i] = f; }
        for (int j = 0; j < ny; j++) { bool f; periodic_shift(ys_of(d, j + 1), pys[0], pys[1], false, &f); in_py[j] = f; }
        for (int j = 0; j < ny; j++) {
            const double y = ys_of(d, j + 1);
            for (int i = 0; i < nx; i++) {
                int ind, img;
                double ddx[2];
                if (priority_of(doms, xs_of(d, i + 1), y, pxs, pys, &ind, &img, ddx)) return bail(SWALS_ERR_INVALID_ARGUMENT);
                if (ind < 0)
                    return bail(fail(SWALS_ERR_INVALID_ARGUMENT, "domain %d: cells outside every domain (row %d)", k + 1,
                                     j + 1));
                for (int q = 0; q < 2; q++)
                    if (ddx[q] > 1.0001 * d->max_parent_dx_ratio * doms[k].dx[q])
                        return bail(fail(SWALS_ERR_INVALID_ARGUMENT,
                                         "domain %d: nesting boundary overlaps a domain coarser than its parent", k + 1));
                pind[(size_t)j * nx + i] = ind;
                pimg[(size_t)j * nx + i] = img;
            }
        }
        if (priority_boxes(pind, pimg, nx, ny, d->nest_layer_width, k + 1, in_px, in_py, M->recv_metadata[k]))
            return bail(SWALS_ERR_INVALID_ARGUMENT);
    }

    // Receive rows as coordinates; rows that need communication (:3050-3080).
    struct RecvRow { int64_t ind, img; double xlo, xhi, ylo, yhi; int cnt; };
    std::vector<std::vector<RecvRow>> recv_rows(n);
    for (int k = 0; k < n; k++) {
        const swals_nest_domain_desc *d = doms[k].d;
        int counter = 0;
        for (const auto &b : M->recv_metadata[k]) {
            const double tx0 = x_of(d, (int)b[2]), tx1 = x_of(d, (int)b[3]);
            const double ty0 = y_of(d, (int)b[4]), ty1 = y_of(d, (int)b[5]);
            bool fc, fd;
            periodic_shift(tx1, pxs[0], pxs[1], false, &fc);
            periodic_shift(ty1, pys[0], pys[1], false, &fd);
            const bool in_per = fc || fd;   // check_periodic's flag of the second corner
            RecvRow r;
            r.ind = b[0]; r.img = b[1];
            r.xlo = tx0 - 0.5 * doms[k].dx[0]; r.xhi = tx1 + 0.5 * doms[k].dx[0];
            r.ylo = ty0 - 0.5 * doms[k].dx[1]; r.yhi = ty1 + 0.5 * doms[k].dx[1];
            const bool real = !(((!in_per) && b[0] == k + 1 && b[1] == 1) || b[0] < 1);
            r.cnt = real ? ++counter : -1;
            recv_rows[k].push_back(r);
        }
    }

    // Send metadata (:3090-3140): per sender, rows (ind, img, iL, iU, jL, jU, recv_row, in_periodic).
    std::vector<std::vector<std::array<int64_t, 8>>> send_meta(n);
    for (int k = 0; k < n; k++) {
        const swals_nest_domain_desc *d = doms[k].d;
        const int nx = d->nx[0], ny = d->nx[1];
        for (int jj = 0; jj < n; jj++) {
            for (size_t i = 0; i < recv_rows[jj].size(); i++) {
                const RecvRow &r = recv_rows[jj][i];
                if (r.ind != k + 1 || r.img != 1) continue;
                const double *tdx = doms[jj].dx;
                bool f1x, f1y, f2x, f2y;
                const double p1x = periodic_shift(r.xlo + 0.5 * tdx[0], pxs[0], pxs[1], true, &f1x);
                const double p1y = periodic_shift(r.ylo + 0.5 * tdx[1], pys[0], pys[1], true, &f1y);
                const double p2x = periodic_shift(r.xhi - 0.5 * tdx[0], pxs[0], pxs[1], true, &f2x);
                const double p2y = periodic_shift(r.yhi - 0.5 * tdx[1], pys[0], pys[1], true, &f2y);
                const bool in_per = f2x || f2y;
                const double tx0 = p1x - 0.5 * 1.0 * tdx[0], tx1 = p2x - 0.5 * -1.0 * tdx[0];
                const double ty0 = p1y - 0.5 * 1.0 * tdx[1], ty1 = p2y - 0.5 * -1.0 * tdx[1];
                int64_t c0 = 0, c1 = 0, c2 = 0, c3 = 0;
                for (int q = 1; q <= nx; q++) { const double x = x_of(d, q); c0 += x < tx0; c1 += x < tx1; }
                for (int q = 1; q <= ny; q++) { const double y = y_of(d, q); c2 += y < ty0; c3 += y < ty1; }
                send_meta[k].push_back({(int64_t)jj + 1, 1, c0 + 1, c1, c2 + 1, c3, (int64_t)i, in_per ? 1 : 0});
            }
        }
    }

    // Pair the real receive rows with their send rows (:3170-3330).
    for (int jd = 0; jd < n; jd++) {
        for (size_t i = 0; i < recv_rows[jd].size(); i++) {
            if (recv_rows[jd][i].cnt < 1) continue;
            int sender = -1, srow = -1;
            for (int k = 0; k < n && sender < 0; k++)
                for (size_t q = 0; q < send_meta[k].size(); q++) {
                    const auto &s = send_meta[k][q];
                    if ((!s[7] && s[0] - 1 == k) || s[0] < 1) continue;
                    if (s[0] - 1 == jd && s[6] == (int64_t)i) { sender = k; srow = (int)q; }
                }
            if (sender < 0) return bail(fail(SWALS_ERR_INVALID_ARGUMENT, "domain %d: receive box %d has no sender", jd + 1, (int)i + 1));
            const auto &s = send_meta[sender][srow];
            const auto &b = M->recv_metadata[jd][i];
            swals_md_exchange e;
            e.sender = sender;
            e.receiver = jd;
            for (int q = 0; q < 4; q++) { e.send_box[q] = (int32_t)s[2 + q]; e.recv_box[q] = (int32_t)b[2 + q]; }
            e.recv_row = (int32_t)i;
            e.send_row = srow;
            M->exchanges.push_back(e);
        }
    }
    *out = M;
    return SWALS_OK;
}

int swals_md_metadata_exchanges(const swals_md_metadata *m, swals_md_exchange *out, int32_t capacity, int32_t *count)
{
    if (!m || !count) return fail(SWALS_ERR_INVALID_ARGUMENT, "swals_md_metadata_exchanges: NULL argument");
    *count = (int32_t)m->exchanges.size();
    if (out) {
        if (capacity < *count) return fail(SWALS_ERR_INVALID_ARGUMENT, "exchange capacity %d < %d", capacity, *count);
        std::copy(m->exchanges.begin(), m->exchanges.end(), out);
    }
    return SWALS_OK;
}

int swals_md_metadata_priority(const swals_md_metadata *m, int32_t domain, int32_t *index_out, int32_t *image_out)
{
    if (!m || domain < 0 || domain >= (int32_t)m->pind.size())
        return fail(SWALS_ERR_INVALID_ARGUMENT, "swals_md_metadata_priority: bad domain");
    if (index_out) std::copy(m->pind[domain].begin(), m->pind[domain].end(), index_out);
    if (image_out) std::copy(m->pimg[domain].begin(), m->pimg[domain].end(), image_out);
    return SWALS_OK;
}

int swals_md_metadata_recv_boxes(const swals_md_metadata *m, int32_t domain, int64_t *rows_out, int32_t capacity,
                                 int32_t *count)
{
    if (!m || !count || domain < 0 || domain >= (int32_t)m->recv_metadata.size())
        return fail(SWALS_ERR_INVALID_ARGUMENT, "swals_md_metadata_recv_boxes: bad arguments");
    const auto &rm = m->recv_metadata[domain];
    *count = (int32_t)rm.size();
    if (rows_out) {
        if (capacity < *count) return fail(SWALS_ERR_INVALID_ARGUMENT, "recv box capacity %d < %d", capacity, *count);
        for (size_t q = 0; q < rm.size(); q++)
            for (int k = 0; k < 6; k++) rows_out[q * 6 + k] = rm[q][k];
    }
    return SWALS_OK;
}

void swals_md_metadata_free(swals_md_metadata *m) { delete m; }

}  // extern "C"
