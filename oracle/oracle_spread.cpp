// oracle_spread.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// CPU restatement of the spread_model pieces of the per-star diagnostics:
//   _exp_disk_kernel_bandlimited  src/photometry/psf_photometry_diagnostics.jl:82-108
//   _spread_fwhm                  src/photometry/psf_photometry_diagnostics.jl:121-133
//   correlate!(g, ms, K, :zero)   src/correlation.jl:122-141 (zero border)
// The band-limited 1-D profile of each Gaussian component,
//   I(m; v) = integral over k in [-1/2, 1/2] of exp(-a k^2) cos(2 pi k m),
// is integrated here by Gauss-Legendre quadrature on a few panels (written
// apart from the product's own quadrature; the reference evaluates the closed
// form through the complex error function); tests/test_oracle_spread.py pins
// it against that closed form evaluated with scipy's complex erf.
#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

#include "oracle_psf.hpp"

namespace orc {

namespace {
const double kPi = 3.141592653589793;
// The Tractor's 6-Gaussian circular exponential profile (amplitudes, variances
// in units of the half-light radius squared), as the reference tabulates it.
const double kAmp[6] = {1.99485977e-4, 2.61612679e-3, 1.89726655e-2, 1.00186544e-1, 3.68534484e-1, 5.09490694e-1};
const double kVar[6] = {1.20078965e-3, 8.84526493e-3, 3.91463084e-2, 1.39976817e-1, 4.60962500e-1, 1.50159566e0};

// Gauss-Legendre nodes and weights on [-1, 1] (Newton iteration on P_n).
void gl_nodes(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < (n + 1) / 2; ++i) {
        double z = std::cos(kPi * (i + 0.75) / (n + 0.5)), pd = 0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            pd = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / pd;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; ++k) {
            const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        pd = n * (z * p1 - p0) / (z * z - 1.0);
        x[i] = -z;
        x[n - 1 - i] = z;
        w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * pd * pd);
    }
}

// I(m; a) by 40-point Gauss-Legendre on 1 + |m| / 3 equal panels of
// [-1/2, 1/2] (at most about 1.5 cosine periods a panel, where 40 nodes are
// exact to rounding).
double band_profile(double a, int m) {
    if (kPi * kPi * (double)m * m / a > 690) return 0.0;  // the reference's overflow cutoff
    static const struct Nodes {
        std::vector<double> x, w;
        Nodes() { gl_nodes(40, x, w); }
    } G;
    const int panels = 1 + std::abs(m) / 3;
    const double hw = 0.5 / panels;
    double I = 0;
    for (int p = 0; p < panels; ++p) {
        const double mid = -0.5 + (2 * p + 1) * hw;
        for (size_t q = 0; q < G.x.size(); ++q) {
            const double k = mid + hw * G.x[q];
            I += hw * G.w[q] * std::exp(-a * k * k) * std::cos(2 * kPi * k * m);
        }
    }
    return I;
}
}  // namespace

void exp_disk_kernel(double fwhm, int half, std::vector<double>& K) {
    const int n = 2 * half + 1;
    const double re = fwhm / 16 * 1.67834699;
    K.assign((size_t)n * n, 0.0);
    std::vector<double> Iv(n);
    for (int c = 0; c < 6; ++c) {
        const double a = 2 * kPi * kPi * re * re * kVar[c];
        for (int m = -half; m <= half; ++m) Iv[m + half] = band_profile(a, m);
        for (int jj = 0; jj < n; ++jj)
            for (int ii = 0; ii < n; ++ii) K[ii + (size_t)jj * n] += kAmp[c] * Iv[ii] * Iv[jj];
    }
    double tot = 0;
    for (double v : K) tot += v;
    for (double& v : K) v /= tot;
}

// PSF.extent of the unit model at (Y, X): +-2.5 fwhm for the Gaussian
// (PSF.jl:285-291, fwhm_factor 5, no rotation); the node's data extent for an
// ImagePSF (empirical_models.jl:167-176); the union over the weighted corner
// nodes for a gridded model (gridded_psf.jl:281-297).
static void unit_extent(const Psf& psf, double Y, double X, double e[4]) {
    if (psf.kind == CPB_PSF_CIRCULAR_GAUSSIAN) {
        const double a = 5 * psf.fwhm / 2;
        e[0] = Y - a, e[1] = Y + a, e[2] = X - a, e[3] = X + a;
        return;
    }
    Corner c[4];
    grid_corners_dw(psf, Y, X, c);
    bool first = true;
    for (int k = 0; k < 4; ++k) {
        if (c[k].idx < 0 || c[k].w == 0.0) continue;
        const Node& nd = psf.nodes[c[k].idx];
        const double ylo = Y - (nd.oy - 1) / nd.sy, yhi = Y + ((double)nd.ny - nd.oy) / nd.sy;
        const double xlo = X - (nd.ox - 1) / nd.sx, xhi = X + ((double)nd.nx - nd.ox) / nd.sx;
        if (first) {
            e[0] = ylo, e[1] = yhi, e[2] = xlo, e[3] = xhi;
            first = false;
        } else {
            e[0] = std::min(e[0], ylo), e[1] = std::max(e[1], yhi);
            e[2] = std::min(e[2], xlo), e[3] = std::max(e[3], xhi);
        }
    }
    if (first) e[0] = e[1] = Y, e[2] = e[3] = X;
}

double spread_fwhm(const Psf& psf, double Y, double X) {
    // the reference's PSF.extent(Int, m) raises an InexactError on a non-finite
    // position; here spread_model is then off
    if (!(std::isfinite(Y) && std::isfinite(X))) return std::numeric_limits<double>::quiet_NaN();
    double e[4];
    unit_extent(psf, Y, X, e);
    const StarP s{Y, X, 1.0, 0.0, psf.fwhm};
    double s1 = 0, s2 = 0;
    for (int64_t j = (int64_t)std::floor(e[2]); j <= (int64_t)std::ceil(e[3]); ++j)
        for (int64_t i = (int64_t)std::floor(e[0]); i <= (int64_t)std::ceil(e[1]); ++i) {
            const double g = evaluate(psf, s, (double)i, (double)j);
            s1 += g;
            s2 += g * g;
        }
    return std::sqrt(s1 * s1 / s2 * 2 * std::log(2.0) / kPi);
}

bool spread_kernel(const Psf& psf, double param, double y1, double x1, double fit_rad, std::vector<double>& K,
                   int& half) {
    const double f = std::isnan(param) ? spread_fwhm(psf, y1, x1) : param;
    if (!(std::isfinite(f) && f > 0)) return false;
    half = (int)std::ceil(fit_rad);
    exp_disk_kernel(f, half, K);
    return true;
}

void correlate_zero(const double* ms, int h, int w, const std::vector<double>& K, int half, double* g) {
    const int n = 2 * half + 1;
    for (int c = 0; c < w; ++c)
        for (int r = 0; r < h; ++r) {
            double acc = 0;
            for (int q = -half; q <= half; ++q)
                for (int p = -half; p <= half; ++p) {
                    const int rr = r + p, cc = c + q;
                    if (rr >= 0 && rr < h && cc >= 0 && cc < w) acc += K[(p + half) + (size_t)(q + half) * n] * ms[rr + cc * h];
                }
            g[r + c * h] = acc;
        }
}

}  // namespace orc

extern "C" int orc_exp_disk_kernel(double fwhm, int half, double* K) {
    if (!K || half < 0 || !(std::isfinite(fwhm) && fwhm > 0)) return -1;
    std::vector<double> k;
    orc::exp_disk_kernel(fwhm, half, k);
    std::copy(k.begin(), k.end(), K);
    return 0;
}

extern "C" double orc_spread_fwhm(const cpb_psf_desc* desc, double y, double x) {
    orc::Psf psf;
    if (!orc::load_psf(desc, psf).empty()) return std::nan("");
    return orc::spread_fwhm(psf, y, x);
}
