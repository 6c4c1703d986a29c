// oracle_psf.cpp -- TEST INFRASTRUCTURE ONLY (the oracle): PSF arithmetic.
// See oracle_psf.hpp for the scope and the parity status.
#include "oracle_psf.hpp"

#include <algorithm>
#include <cstring>
#include <set>

namespace orc {

namespace {
inline int64_t clampi(int64_t v, int64_t lo, int64_t hi) { return v < lo ? lo : (v > hi ? hi : v); }
}  // namespace

std::string load_psf(const cpb_psf_desc* d, Psf& out) {
    if (!d) return "psf descriptor is NULL";
    out = Psf();
    out.kind = d->kind;
    if (d->kind == CPB_PSF_CIRCULAR_GAUSSIAN) {
        out.fwhm = d->fwhm;
        return "";
    }
    if (d->kind != CPB_PSF_GRIDDED_IMAGE && d->kind != CPB_PSF_IMAGE) return "unsupported PSF kind";
    int nn = d->n_nodes;
    if (nn < 1) return "`psfs` must be non-empty";
    if (d->kind == CPB_PSF_IMAGE && nn != 1) return "ImagePSF takes exactly one node";
    if (d->eltype != CPB_F32 && d->eltype != CPB_F64) return "unsupported PSF eltype";
    for (int k = 0; k < nn; ++k) {
        Node nd;
        nd.ny = d->node_ny[k];
        nd.nx = d->node_nx[k];
        if (nd.ny < 4 || nd.nx < 4) return "each axis of `data` must have at least 4 samples";
        nd.data.resize(nd.ny * nd.nx);
        for (int64_t q = 0; q < nd.ny * nd.nx; ++q) {
            double v = d->eltype == CPB_F64 ? ((const double*)d->node_data[k])[q]
                                            : (double)((const float*)d->node_data[k])[q];
            if (!std::isfinite(v)) return "all elements of `data` must be finite";
            nd.data[q] = v;
        }
        nd.sx = (double)d->node_os[2 * k];
        nd.sy = (double)d->node_os[2 * k + 1];
        if (!(nd.sx > 0 && nd.sy > 0)) return "`oversampling` values must be positive";
        nd.oy = d->node_origin[2 * k];
        nd.ox = d->node_origin[2 * k + 1];
        if (!std::isfinite(nd.oy) || !std::isfinite(nd.ox)) return "`origin` must be finite";
        nd.fill = d->node_fill_value ? d->node_fill_value[k] : 0.0;
        out.nodes.push_back(std::move(nd));
    }
    if (d->kind == CPB_PSF_IMAGE || nn == 1) {
        out.ygrid = {d->grid_y ? d->grid_y[0] : 0.0};
        out.xgrid = {d->grid_x ? d->grid_x[0] : 0.0};
        out.index_grid = {0};
        return "";
    }
    // GriddedPSFModel constructor: complete rectangular grid (gridded_psf.jl:106-134).
    for (int k = 0; k < nn; ++k)
        if (!std::isfinite(d->grid_y[k]) || !std::isfinite(d->grid_x[k]))
            return "`grid_y` and `grid_x` must be finite";
    std::set<double> ys(d->grid_y, d->grid_y + nn), xs(d->grid_x, d->grid_x + nn);
    out.ygrid.assign(ys.begin(), ys.end());
    out.xgrid.assign(xs.begin(), xs.end());
    size_t gny = out.ygrid.size(), gnx = out.xgrid.size();
    if (gnx < 2 || gny < 2)
        return "`grid_y` and `grid_x` must each contain at least 2 unique values unless a single PSF is supplied";
    if ((size_t)nn != gny * gnx) return "`grid_y`/`grid_x` positions do not form a complete rectangular grid";
    out.index_grid.assign(gny * gnx, -1);
    for (int k = 0; k < nn; ++k) {
        size_t iy = std::lower_bound(out.ygrid.begin(), out.ygrid.end(), d->grid_y[k]) - out.ygrid.begin();
        size_t ix = std::lower_bound(out.xgrid.begin(), out.xgrid.end(), d->grid_x[k]) - out.xgrid.begin();
        int& slot = out.index_grid[iy + ix * gny];
        if (slot != -1) return "duplicate node position";
        slot = k;
    }
    return "";
}

void bicubic(const double* data, int64_t ny, int64_t nx, double y, double x, double fill,
             double& v, double& dfdy, double& dfdx) {
    bool inb = std::isfinite(x) && std::isfinite(y) && x >= 1.0 && x <= (double)nx && y >= 1.0 && y <= (double)ny;
    double xxc = inb ? x : 1.0, yyc = inb ? y : 1.0;
    int64_t lx = clampi((int64_t)std::floor(xxc), 1, nx - 1);
    int64_t ly = clampi((int64_t)std::floor(yyc), 1, ny - 1);
    double dx = xxc - (double)lx, dy = yyc - (double)ly;
    int64_t ix[4] = {clampi(lx - 1, 1, nx), lx, lx + 1, clampi(lx + 2, 1, nx)};
    int64_t iy[4] = {clampi(ly - 1, 1, ny), ly, ly + 1, clampi(ly + 2, 1, ny)};
    double row[4], drow[4];
    for (int r = 0; r < 4; ++r) {
        const double* col = data + (iy[r] - 1);
        cubic4(col[(ix[0] - 1) * ny], col[(ix[1] - 1) * ny], col[(ix[2] - 1) * ny], col[(ix[3] - 1) * ny], dx,
               row[r], drow[r]);
    }
    double value, dy_, dx_, unused;
    cubic4(row[0], row[1], row[2], row[3], dy, value, dy_);
    cubic4(drow[0], drow[1], drow[2], drow[3], dy, dx_, unused);
    v = inb ? value : fill;
    dfdy = inb ? dy_ : 0.0;
    dfdx = inb ? dx_ : 0.0;
}

void corner_point(const Node& nd, double Y, double X, double py, double px, double& pv, double& pdv, double& pdu) {
    double u = nd.sx * (px - X) + nd.ox;
    double v = nd.sy * (py - Y) + nd.oy;
    int64_t nyd = nd.ny, nxd = nd.nx;
    bool inb = std::isfinite(u) && std::isfinite(v) && u >= 1.0 && u <= (double)nxd && v >= 1.0 && v <= (double)nyd;
    double uc = inb ? u : 1.0, vc = inb ? v : 1.0;
    int64_t lx = clampi((int64_t)std::floor(uc), 1, nxd - 1);
    int64_t ly = clampi((int64_t)std::floor(vc), 1, nyd - 1);
    double du = uc - (double)lx, dv = vc - (double)ly;
    int64_t ix[4] = {clampi(lx - 1, 1, nxd), lx, lx + 1, clampi(lx + 2, 1, nxd)};
    int64_t iy[4] = {clampi(ly - 1, 1, nyd), ly, ly + 1, clampi(ly + 2, 1, nyd)};
    double row[4], drow[4];
    for (int r = 0; r < 4; ++r) {
        double a = nd.at(iy[r], ix[0]), b = nd.at(iy[r], ix[1]), c = nd.at(iy[r], ix[2]), e = nd.at(iy[r], ix[3]);
        double c1 = (c - a) / 2;
        double c4 = c - b - c1;
        double c2 = 3 * c4 - (e - b) / 2 + c1;
        double c3 = c4 - c2;
        row[r] = du * (du * (du * c3 + c2) + c1) + b;
        drow[r] = du * (3 * du * c3 + 2 * c2) + c1;
    }
    double cv1 = (row[2] - row[0]) / 2;
    double cv4 = row[2] - row[1] - cv1;
    double cv2 = 3 * cv4 - (row[3] - row[1]) / 2 + cv1;
    double cv3 = cv4 - cv2;
    double val = dv * (dv * (dv * cv3 + cv2) + cv1) + row[1];
    double dpdv = dv * (3 * dv * cv3 + 2 * cv2) + cv1;
    double cu1 = (drow[2] - drow[0]) / 2;
    double cu4 = drow[2] - drow[1] - cu1;
    double cu2 = 3 * cu4 - (drow[3] - drow[1]) / 2 + cu1;
    double cu3 = cu4 - cu2;
    double dpdu = dv * (dv * (dv * cu3 + cu2) + cu1) + drow[1];
    pv = inb ? val : nd.fill;
    pdv = inb ? dpdv : 0.0;
    pdu = inb ? dpdu : 0.0;
}

void grid_corners_dw(const Psf& psf, double Y, double X, Corner c[4]) {
    if (psf.nodes.size() == 1) {
        c[0] = {0, 1.0, 0.0, 0.0};
        for (int k = 1; k < 4; ++k) c[k] = {-1, 0.0, 0.0, 0.0};
        return;
    }
    const auto& yg = psf.ygrid;
    const auto& xg = psf.xgrid;
    int64_t gny = (int64_t)yg.size(), gnx = (int64_t)xg.size();
    // searchsortedlast: index of the last element <= value (1-based), 0 if none.
    int64_t iy = std::upper_bound(yg.begin(), yg.end(), Y) - yg.begin();
    int64_t ix = std::upper_bound(xg.begin(), xg.end(), X) - xg.begin();
    iy = clampi(iy, 1, gny - 1);
    ix = clampi(ix, 1, gnx - 1);
    double y0 = yg[iy - 1], y1 = yg[iy], x0 = xg[ix - 1], x1 = xg[ix];
    double Yc = std::min(std::max(Y, y0), y1);
    double Xc = std::min(std::max(X, x0), x1);
    double cy = (Y > y0 && Y < y1) ? 1.0 : 0.0;
    double cx = (X > x0 && X < x1) ? 1.0 : 0.0;
    double invnorm = 1.0 / ((x1 - x0) * (y1 - y0));
    double dy1 = y1 - Yc, dy0 = Yc - y0, dx1 = x1 - Xc, dx0 = Xc - x0;
    auto ig = [&](int64_t a, int64_t b) { return psf.index_grid[(a - 1) + (b - 1) * gny]; };
    c[0] = {ig(iy, ix), dx1 * dy1 * invnorm, -dx1 * cy * invnorm, -dy1 * cx * invnorm};
    c[1] = {ig(iy, ix + 1), dx0 * dy1 * invnorm, -dx0 * cy * invnorm, dy1 * cx * invnorm};
    c[2] = {ig(iy + 1, ix), dx1 * dy0 * invnorm, dx1 * cy * invnorm, -dy0 * cx * invnorm};
    c[3] = {ig(iy + 1, ix + 1), dx0 * dy0 * invnorm, dx0 * cy * invnorm, dy0 * cx * invnorm};
}

namespace {
// Gridded value + chain-rule derivatives at one pixel, summing only the
// corners that carry weight or weight derivative (the reference's remaining
// corners contribute exact zeros).
void gridded_point(const Psf& psf, double Y, double X, double py, double px, double& s, double& dsdY, double& dsdX) {
    Corner c[4];
    grid_corners_dw(psf, Y, X, c);
    s = 0;
    dsdY = 0;
    dsdX = 0;
    for (int k = 0; k < 4; ++k) {
        if (c[k].idx < 0) continue;
        if (c[k].w == 0.0 && c[k].dwdy == 0.0 && c[k].dwdx == 0.0) continue;
        const Node& nd = psf.nodes[c[k].idx];
        double pv, pdv, pdu;
        corner_point(nd, Y, X, py, px, pv, pdv, pdu);
        s += c[k].w * pv;
        dsdY += c[k].dwdy * pv - c[k].w * nd.sy * pdv;
        dsdX += c[k].dwdx * pv - c[k].w * nd.sx * pdu;
    }
}
}  // namespace

double evaluate(const Psf& psf, const StarP& s, double py, double px) {
    if (psf.kind == CPB_PSF_CIRCULAR_GAUSSIAN) {
        double dx = px - s.x, dy = py - s.y;
        double sq = (dx * dx + dy * dy) / (s.fwhm * s.fwhm);
        double norm = -(M_PI * (s.fwhm * s.fwhm) / gauss_pre());
        double amp = s.flux / norm;
        return amp * std::exp(gauss_pre() * sq) + s.bkg;
    }
    if (psf.kind == CPB_PSF_IMAGE) {
        const Node& nd = psf.nodes[0];
        double u = nd.sx * (px - s.x) + nd.ox;
        double v = nd.sy * (py - s.y) + nd.oy;
        double p, a, b;
        bicubic(nd.data.data(), nd.ny, nd.nx, v, u, nd.fill, p, a, b);
        return s.flux * p + s.bkg;
    }
    double sv, dY, dX;
    gridded_point(psf, s.y, s.x, py, px, sv, dY, dX);
    return s.flux * sv + s.bkg;
}

double evaluate_fg(const Psf& psf, const StarP& s, double py, double px, double g[3]) {
    if (psf.kind == CPB_PSF_CIRCULAR_GAUSSIAN) {
        double gp = gauss_pre();
        double dx = px - s.x, dy = py - s.y;
        double f2 = s.fwhm * s.fwhm;
        double sq = (dx * dx + dy * dy) / f2;
        double norm = -(M_PI * f2 / gp);
        double amp = s.flux / norm;
        double gg = std::exp(gp * sq);
        double Ag = amp * gg;
        double gf2 = gp / f2;
        g[0] = -2 * Ag * gf2 * dy;
        g[1] = -2 * Ag * gf2 * dx;
        g[2] = gg / norm;
        return amp * gg + s.bkg;
    }
    if (psf.kind == CPB_PSF_IMAGE) {
        const Node& nd = psf.nodes[0];
        double u = nd.sx * (px - s.x) + nd.ox;
        double v = nd.sy * (py - s.y) + nd.oy;
        double p, dpdv, dpdu;
        bicubic(nd.data.data(), nd.ny, nd.nx, v, u, nd.fill, p, dpdv, dpdu);
        g[0] = -s.flux * nd.sy * dpdv;
        g[1] = -s.flux * nd.sx * dpdu;
        g[2] = p;
        return s.flux * p + s.bkg;
    }
    double sv, dY, dX;
    gridded_point(psf, s.y, s.x, py, px, sv, dY, dX);
    g[0] = s.flux * dY;
    g[1] = s.flux * dX;
    g[2] = sv;
    return s.flux * sv + s.bkg;
}

}  // namespace orc
