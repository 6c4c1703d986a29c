// cpb_spread.cu -- the spread_model reference disk, host side (fit_all_stars and
// cpb_exp_disk_kernel; the simultaneous fits build theirs on the device with
// spread_disk_block, whose quadrature rule spread_rule supplies).
//
// Restates, for the diagnostics of the device fits,
//   _spread_fwhm                      src/photometry/psf_photometry_diagnostics.jl:121-133
//   _exp_disk_kernel_bandlimited      :82-108
// The band-limited profile of each mixture component,
//   I(m; v) = integral over k in [-1/2, 1/2] of exp(-a k^2) cos(2 pi k m),
//   a = 2 pi^2 re^2 v,  re = 1.67834699 fwhm / 16,
// is integrated here by composite Gauss-Legendre quadrature (32 nodes on each
// of max(4, 2 half) panels: the integrand is entire and makes at most half/2
// cycles per panel, so each panel is exact to rounding), instead of the
// reference's closed form through the complex error function -- the same
// number to rounding.  The reference's cutoff (I = 0 where pi^2 m^2 / a > 690,
// where its closed form would overflow) is kept as it is.
#include <algorithm>
#include <cmath>
#include <vector>

#include "cpb_internal.cuh"

namespace cpb {

double host_unit_value(const cpb_psf* ps, double fwhm, double Y, double X, int i, int j);
void host_extent(const cpb_psf* ps, double fwhm, double Y, double X, double e[4]);

namespace {

const double kPi = 3.141592653589793;
// Mixture-of-Gaussians circular exponential profile (Hogg & Lang, The Tractor):
// amplitudes and variances in units of the half-light radius squared.
const double kExpAmp[6] = {1.99485977e-4, 2.61612679e-3, 1.89726655e-2, 1.00186544e-1, 3.68534484e-1, 5.09490694e-1};
const double kExpVar[6] = {1.20078965e-3, 8.84526493e-3, 3.91463084e-2, 1.39976817e-1, 4.60962500e-1, 1.50159566e0};

// Gauss-Legendre nodes and weights on [-1, 1] (Newton iteration on P_n).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < (n + 1) / 2; ++i) {
        double z = std::cos(kPi * (i + 0.75) / (n + 0.5)), dp = 0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; ++k) {
            const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        dp = n * (z * p1 - p0) / (z * z - 1.0);
        x[i] = -z;
        x[n - 1 - i] = z;
        w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

}  // namespace

// _spread_fwhm: the Gaussian-equivalent FWHM of the unit render at (Y, X),
// sqrt(ea 2 ln2 / pi) with ea = (sum g)^2 / sum g^2 over the PSF's integer extent.
double spread_fwhm(const cpb_psf* psf, double fwhm, double Y, double X) {
    // the reference's PSF.extent(Int, m) raises an InexactError on a non-finite
    // position; here spread_model is then off
    if (!(std::isfinite(Y) && std::isfinite(X))) return std::nan("");
    double e[4];
    host_extent(psf, fwhm, Y, X, e);
    const int ylo = (int)std::floor(e[0]), yhi = (int)std::ceil(e[1]);
    const int xlo = (int)std::floor(e[2]), xhi = (int)std::ceil(e[3]);
    double s1 = 0, s2 = 0;
    for (int j = xlo; j <= xhi; ++j)
        for (int i = ylo; i <= yhi; ++i) {
            const double g = host_unit_value(psf, fwhm, Y, X, i, j);
            s1 += g;
            s2 += g * g;
        }
    const double ea = s1 * s1 / s2;
    return std::sqrt(ea * 2 * std::log(2.0) / kPi);
}

// The six band-limited component profiles I_c(m), m = -half..half, of
// _exp_disk_kernel_bandlimited(fwhm; half), their support half-widths and the
// weights alpha_c = a_c / total that make sum_c alpha_c I_c I_c' the kernel
// normalised to sum 1.
void exp_disk_components(double fwhm, int half, SpreadHost& S) {
    const int n = 2 * half + 1;
    const double re = fwhm / 16 * 1.67834699;
    std::vector<double> gx, gw;
    gauss_legendre(32, gx, gw);
    const int panels = std::max(4, 2 * half);
    const double hw = 0.5 / panels;  // half-width of one panel on [-1/2, 1/2]
    S.kh = half;
    S.I.assign((size_t)6 * n, 0.0);
    double total = 0;
    for (int c = 0; c < 6; ++c) {
        const double a = 2 * kPi * kPi * re * re * kExpVar[c];
        double* Iv = S.I.data() + (size_t)c * n;
        S.L[c] = 0;
        double sum = 0;
        for (int m = -half; m <= half; ++m) {
            double I = 0;
            if (!(kPi * kPi * (double)m * m / a > 690)) {
                for (int pnl = 0; pnl < panels; ++pnl) {
                    const double mid = -0.5 + (2 * pnl + 1) * hw;
                    for (size_t q = 0; q < gx.size(); ++q) {
                        const double k = mid + hw * gx[q];
                        I += hw * gw[q] * std::exp(-a * k * k) * std::cos(2 * kPi * k * m);
                    }
                }
            }
            Iv[m + half] = I;
            if (I != 0.0) S.L[c] = std::max(S.L[c], std::abs(m));
            sum += I;
        }
        total += kExpAmp[c] * sum * sum;
    }
    for (int c = 0; c < 6; ++c) S.alpha[c] = kExpAmp[c] / total;
}

// The quadrature rule and mixture constants of the device disk builder
// (spread_disk_block): 32 Gauss-Legendre nodes and weights on [-1, 1], the six
// amplitudes and the six variances.
void spread_rule(double* out) {
    std::vector<double> gx, gw;
    gauss_legendre(kSpreadGL, gx, gw);
    for (int q = 0; q < kSpreadGL; ++q) {
        out[q] = gx[q];
        out[kSpreadGL + q] = gw[q];
    }
    for (int c = 0; c < 6; ++c) {
        out[2 * kSpreadGL + c] = kExpAmp[c];
        out[2 * kSpreadGL + 6 + c] = kExpVar[c];
    }
}

// _exp_disk_kernel_bandlimited(fwhm; half): (2 half + 1)^2, column-major, sum 1.
void exp_disk_kernel(double fwhm, int half, std::vector<double>& K) {
    SpreadHost S;
    exp_disk_components(fwhm, half, S);
    const int n = 2 * half + 1;
    K.assign((size_t)n * n, 0.0);
    for (int c = 0; c < 6; ++c) {
        const double* Iv = S.I.data() + (size_t)c * n;
        for (int jj = 0; jj < n; ++jj)
            for (int ii = 0; ii < n; ++ii) K[ii + (size_t)jj * n] += S.alpha[c] * Iv[ii] * Iv[jj];
    }
}

// The spread_model kernel of one fit: the disk FWHM is `param` when given
// (NaN: derived from the PSF at the catalogue's first star, as the reference
// does), the support half = ceil(fit_rad).  Returns false when spread_model
// is off (a non-finite or non-positive disk FWHM).
bool spread_kernel(const cpb_psf* psf, double psf_fwhm, double param, double y1, double x1, double fit_rad,
                   SpreadHost& out) {
    const double f = std::isnan(param) ? spread_fwhm(psf, psf_fwhm, y1, x1) : param;
    if (!(std::isfinite(f) && f > 0)) return false;
    exp_disk_components(f, (int)std::ceil(fit_rad), out);
    return true;
}

}  // namespace cpb

// ---- C ABI -------------------------------------------------------------------
extern "C" CPB_API int cpb_exp_disk_kernel(double fwhm, int32_t half, double* K) {
    if (!K || half < 0 || half > 4096 || !(std::isfinite(fwhm) && fwhm > 0)) return CPB_ERR_ARGUMENT;
    std::vector<double> k;
    cpb::exp_disk_kernel(fwhm, half, k);
    std::copy(k.begin(), k.end(), K);
    return 0;
}
