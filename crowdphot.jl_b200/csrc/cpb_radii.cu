// cpb_radii.cu -- model_rad = :auto: per-star model-render radii (host side).
//
// Restates, for the library's device path,
//   _model_radii (:auto branch)       src/photometry/psf_photometry_simultaneous.jl:209-243
//   curve_of_growth                    src/curve_of_growth.jl:143-212
//   CircularAperture ExactOverlap      src/apertures.jl:52-66, 93-103, 160-166, 196-290
// The unit PSF's annular surface brightness depends only on the PSF, R_cap and
// (for the Gaussian) its FWHM, so it is computed once per PSF handle and kept.
// Arithmetic is FP64 throughout.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "cpb_internal.cuh"

namespace cpb {
namespace {

const double kPi = 3.141592653589793;

// Exact area of a unit pixel / circle overlap (apertures.jl:196-290).
double area_triangle(double x0, double y0, double x1, double y1, double x2, double y2) {
    return std::fabs(x0 * (y1 - y2) + x1 * (y2 - y0) + x2 * (y0 - y1)) / 2;
}

double area_arc(double x0, double y0, double x1, double y1, double r) {
    const double a = std::sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0));
    const double th = 2 * std::asin(a / (2 * r));
    return r * r * (th - std::sin(th)) / 2;
}

// Rectangle [xmin, xmax] x [ymin, ymax] in the first quadrant (0 <= xmin, 0 <= ymin).
double overlap_core(double xmin, double ymin, double xmax, double ymax, double r) {
    if (xmin * xmin + ymin * ymin > r * r) return 0.0;
    if (xmax * xmax + ymax * ymax < r * r) return (xmax - xmin) * (ymax - ymin);
    const double d1 = std::sqrt(xmax * xmax + ymin * ymin);
    const double d2 = std::sqrt(xmin * xmin + ymax * ymax);
    if (d1 < r && d2 < r) {
        const double x1 = std::sqrt(r * r - ymax * ymax), y1 = ymax;
        const double x2 = xmax, y2 = std::sqrt(r * r - xmax * xmax);
        return (xmax - xmin) * (ymax - ymin) - area_triangle(x1, y1, x2, y2, xmax, ymax) +
               area_arc(x1, y1, x2, y2, r);
    }
    if (d1 < r) {
        const double x1 = xmin, y1 = std::sqrt(r * r - xmin * xmin);
        const double x2 = xmax, y2 = std::sqrt(r * r - xmax * xmax);
        return area_arc(x1, y1, x2, y2, r) + area_triangle(x1, y1, x1, ymin, xmax, ymin) +
               area_triangle(x1, y1, x2, ymin, x2, y2);
    }
    if (d2 < r) {
        const double x1 = std::sqrt(r * r - ymin * ymin), y1 = ymin;
        const double x2 = std::sqrt(r * r - ymax * ymax), y2 = ymax;
        return area_arc(x1, y1, x2, y2, r) + area_triangle(x1, y1, xmin, y1, xmin, ymax) +
               area_triangle(x1, y1, xmin, y2, x2, y2);
    }
    const double x1 = std::sqrt(r * r - ymin * ymin), y1 = ymin;
    const double x2 = xmin, y2 = std::sqrt(r * r - xmin * xmin);
    return area_arc(x1, y1, x2, y2, r) + area_triangle(x1, y1, x2, y2, xmin, ymin);
}

// Any rectangle, split at the axes into first-quadrant pieces.
double overlap_single(double xmin, double ymin, double xmax, double ymax, double r) {
    if (r <= 0) return 0.0;
    if (0 <= xmin) {
        if (0 <= ymin) return overlap_core(xmin, ymin, xmax, ymax, r);
        if (0 >= ymax) return overlap_core(-ymax, xmin, -ymin, xmax, r);
        return overlap_single(xmin, ymin, xmax, 0, r) + overlap_single(xmin, 0, xmax, ymax, r);
    }
    if (0 >= xmax) {
        if (0 <= ymin) return overlap_core(-xmax, ymin, -xmin, ymax, r);
        if (0 >= ymax) return overlap_core(-xmax, -ymax, -xmin, -ymin, r);
        return overlap_single(xmin, ymin, xmax, 0, r) + overlap_single(xmin, 0, xmax, ymax, r);
    }
    if (0 <= ymin) return overlap_single(xmin, ymin, 0, ymax, r) + overlap_single(0, ymin, xmax, ymax, r);
    if (0 >= ymax) return overlap_single(xmin, ymin, 0, ymax, r) + overlap_single(0, ymin, xmax, ymax, r);
    return overlap_single(xmin, ymin, 0, 0, r) + overlap_single(0, ymin, xmax, 0, r) +
           overlap_single(xmin, 0, 0, ymax, r) + overlap_single(0, 0, xmax, ymax, r);
}

// aperture_weight(::CircularAperture at the origin, i, j, ExactOverlap()).
double aperture_weight(int i, int j, double r) {
    const double dy = (double)i, dx = (double)j;
    const double d2 = dx * dx + dy * dy;
    const double dr = std::sqrt(2.0) / 2;
    if (d2 > (r + dr) * (r + dr)) return 0.0;
    if (r > dr && d2 < (r - dr) * (r - dr)) return 1.0;
    if (r <= 0) return 0.0;
    return overlap_single(dx - 0.5, dy - 0.5, dx + 0.5, dy + 0.5, r);
}

// bicubic_interpolate value of one node at detector offset (dy, dx) = pixel
// minus star centre (empirical_models.jl:185-292).
double node_value(const cpb_psf* ps, const DevNode& nd, double dy, double dx) {
    const double* data = ps->h_data64.data() + nd.off;
    const double u = nd.sx * dx + nd.ox;
    const double v = nd.sy * dy + nd.oy;
    const int nyd = nd.ny, nxd = nd.nx;
    if (!(std::isfinite(u) && std::isfinite(v) && u >= 1 && u <= nxd && v >= 1 && v <= nyd)) return nd.fill;
    const int lx = std::min(std::max((int)std::floor(u), 1), nxd - 1);
    const int ly = std::min(std::max((int)std::floor(v), 1), nyd - 1);
    const double du = u - lx, dv = v - ly;
    auto cl = [](int t, int n) { return std::min(std::max(t, 1), n) - 1; };
    const int ix[4] = {cl(lx - 1, nxd), lx - 1, lx, cl(lx + 2, nxd)};
    const int iy[4] = {cl(ly - 1, nyd), ly - 1, ly, cl(ly + 2, nyd)};
    double row[4];
    for (int r = 0; r < 4; ++r) {
        const double a = data[iy[r] + (int64_t)ix[0] * nyd], b = data[iy[r] + (int64_t)ix[1] * nyd];
        const double c = data[iy[r] + (int64_t)ix[2] * nyd], e = data[iy[r] + (int64_t)ix[3] * nyd];
        const double k1 = (c - a) / 2, k4 = c - b - k1, k2 = 3 * k4 - (e - b) / 2 + k1, k3 = k4 - k2;
        row[r] = du * (du * (du * k3 + k2) + k1) + b;
    }
    const double v1 = (row[2] - row[0]) / 2, v4 = row[2] - row[1] - v1, v2 = 3 * v4 - (row[3] - row[1]) / 2 + v1,
                 v3 = v4 - v2;
    return dv * (dv * (dv * v3 + v2) + v1) + row[1];
}

// Node weights of GriddedPSFModel at (Y, X) (_grid_corners_dw, gridded_psf.jl:176-208,
// weights only); single-node and ImagePSF models: node 0 with weight 1.
int host_corners(const cpb_psf* ps, double Y, double X, int idx[4], double wts[4]) {
    const DevPsf& P = ps->dev;
    if (P.n_nodes == 1 || P.kind != CPB_PSF_GRIDDED_IMAGE) {
        idx[0] = 0;
        wts[0] = 1.0;
        return 1;
    }
    const auto& yg = ps->h_ygrid;
    const auto& xg = ps->h_xgrid;
    const int gny = (int)yg.size(), gnx = (int)xg.size();
    int iy = 0, ix = 0;
    for (int k = 0; k < gny; ++k) iy += yg[k] <= Y ? 1 : 0;
    for (int k = 0; k < gnx; ++k) ix += xg[k] <= X ? 1 : 0;
    iy = std::min(std::max(iy, 1), gny - 1);
    ix = std::min(std::max(ix, 1), gnx - 1);
    const double y0 = yg[iy - 1], y1 = yg[iy], x0 = xg[ix - 1], x1 = xg[ix];
    const double Yc = std::min(std::max(Y, y0), y1), Xc = std::min(std::max(X, x0), x1);
    const double inv = 1.0 / ((x1 - x0) * (y1 - y0));
    const double w4[4] = {(x1 - Xc) * (y1 - Yc) * inv, (Xc - x0) * (y1 - Yc) * inv, (x1 - Xc) * (Yc - y0) * inv,
                          (Xc - x0) * (Yc - y0) * inv};
    const int i4[4] = {ps->h_index_grid[(iy - 1) + (ix - 1) * gny], ps->h_index_grid[(iy - 1) + ix * gny],
                       ps->h_index_grid[iy + (ix - 1) * gny], ps->h_index_grid[iy + ix * gny]};
    int k = 0;
    for (int q = 0; q < 4; ++q)
        if (w4[q] != 0.0) {
            idx[k] = i4[q];
            wts[k] = w4[q];
            ++k;
        }
    return k;
}

}  // namespace

// The unit model (flux = 1, bkg = 0) centred at (Y, X), at pixel (i, j).
double host_unit_value(const cpb_psf* ps, double fwhm, double Y, double X, int i, int j) {
    if (ps->dev.kind == CPB_PSF_CIRCULAR_GAUSSIAN) {
        const double g = -4.0 * std::log(2.0);
        const double r2 = ((double)i - Y) * ((double)i - Y) + ((double)j - X) * ((double)j - X);
        const double norm = -(kPi * fwhm * fwhm / g);
        return (1.0 / norm) * std::exp(g * r2 / (fwhm * fwhm));
    }
    int idx[4];
    double wts[4];
    const int nc = host_corners(ps, Y, X, idx, wts);
    double s = 0;
    for (int k = 0; k < nc; ++k) s += wts[k] * node_value(ps, ps->h_nodes[idx[k]], (double)i - Y, (double)j - X);
    return s;
}

// PSF.extent of the model centred at (Y, X) (PSF.jl:285-296, empirical_models.jl:167-176,
// gridded_psf.jl:281-300): (ymin, ymax, xmin, xmax).
void host_extent(const cpb_psf* ps, double fwhm, double Y, double X, double e[4]) {
    if (ps->dev.kind == CPB_PSF_CIRCULAR_GAUSSIAN) {
        const double a = 5.0 * fwhm / 2;  // fwhm_factor 5, no rotation
        e[0] = Y - a;
        e[1] = Y + a;
        e[2] = X - a;
        e[3] = X + a;
        return;
    }
    int idx[4];
    double wts[4];
    const int nc = host_corners(ps, Y, X, idx, wts);
    for (int k = 0; k < nc; ++k) {
        const DevNode& nd = ps->h_nodes[idx[k]];
        const double lo_y = Y - (nd.oy - 1.0) / nd.sy, hi_y = Y + ((double)nd.ny - nd.oy) / nd.sy;
        const double lo_x = X - (nd.ox - 1.0) / nd.sx, hi_x = X + ((double)nd.nx - nd.ox) / nd.sx;
        if (k == 0) {
            e[0] = lo_y;
            e[1] = hi_y;
            e[2] = lo_x;
            e[3] = hi_x;
        } else {
            e[0] = std::min(e[0], lo_y);
            e[1] = std::max(e[1], hi_y);
            e[2] = std::min(e[2], lo_x);
            e[3] = std::max(e[3], hi_x);
        }
    }
}

namespace {

// The unit model (y = x = 0, flux = 1, bkg = 0) at pixel (i, j).
double unit_value(const cpb_psf* ps, int i, int j) { return host_unit_value(ps, 0.0, 0.0, 0.0, i, j); }

// Annular mean surface brightness of the unit PSF for radii 1..R_cap
// (_model_radii, :226-236), from its curve of growth.
std::vector<double> unit_sb(const cpb_psf* ps, double fwhm, int R_cap) {
    std::vector<double> cog(R_cap);
    if (ps->dev.kind == CPB_PSF_CIRCULAR_GAUSSIAN) {
        // analytic overload (curve_of_growth.jl:180-195); integral(model) = flux = 1
        const double g = -4.0 * std::log(2.0);
        for (int r = 1; r <= R_cap; ++r) cog[r - 1] = 1.0 * (1.0 - std::exp(g * ((double)r * r) / (fwhm * fwhm)));
    } else {
        // generic curve_of_growth: exact-overlap apertures over the unit model's pixels
        const int W = 2 * R_cap + 1;
        std::vector<double> val((size_t)W * W);
        for (int j = -R_cap; j <= R_cap; ++j)
            for (int i = -R_cap; i <= R_cap; ++i) val[(i + R_cap) + (size_t)(j + R_cap) * W] = unit_value(ps, i, j);
        for (int r = 1; r <= R_cap; ++r) {
            double flux = 0;
            for (int j = -r; j <= r; ++j)
                for (int i = -r; i <= r; ++i) {
                    const double w = aperture_weight(i, j, (double)r);
                    if (!(w > 0)) continue;
                    flux += w * val[(i + R_cap) + (size_t)(j + R_cap) * W];
                }
            cog[r - 1] = flux;
        }
    }
    std::vector<double> sb(R_cap);
    double prev = 0;
    for (int r = 1; r <= R_cap; ++r) {
        const double ee = cog[r - 1] / cog[R_cap - 1];
        sb[r - 1] = std::max((ee - prev) / (kPi * (double)(r * r - (r - 1) * (r - 1))), 0.0);
        prev = ee;
    }
    return sb;
}

}  // namespace

void model_radii_auto(const cpb_psf* psf, double fwhm, double nsigma, int R_fit, int R_cap,
                      std::vector<double>& w_sample, const std::vector<double>& flux, std::vector<int32_t>& out) {
    // sigma_bg from the 0.84 quantile (type 7) of the positive finite weights
    std::vector<double> ws;
    ws.reserve(w_sample.size());
    for (double v : w_sample)
        if (v > 0 && std::isfinite(v)) ws.push_back(v);
    if (ws.empty()) throw ArgError{"model_rad=:auto found no positive finite weights to estimate the noise"};
    std::sort(ws.begin(), ws.end());
    const double h = (double)(ws.size() - 1) * 0.84;
    const size_t lo = (size_t)std::floor(h);
    const size_t hi = std::min(lo + 1, ws.size() - 1);
    const double wval = ws[lo] + (h - (double)lo) * (ws[hi] - ws[lo]);
    const double sigma_bg = wval > 0 ? std::sqrt(1.0 / wval) : 1.0;
    cpb_psf* ps = const_cast<cpb_psf*>(psf);
    std::vector<double> sb;
    {
        std::lock_guard<std::mutex> lk(ps->cog_mu);
        const auto key = std::make_pair(R_cap, psf->dev.kind == CPB_PSF_CIRCULAR_GAUSSIAN ? fwhm : 0.0);
        auto it = ps->cog_sb.find(key);
        if (it == ps->cog_sb.end()) it = ps->cog_sb.emplace(key, unit_sb(psf, fwhm, R_cap)).first;
        sb = it->second;
    }
    const double thr = nsigma * sigma_bg;
    out.resize(flux.size());
    for (size_t j = 0; j < flux.size(); ++j) {
        const double F = std::max(flux[j], 0.0);
        int r = R_fit;
        while (r < R_cap && F * sb[r - 1] > thr) ++r;
        out[j] = r;
    }
}

}  // namespace cpb
