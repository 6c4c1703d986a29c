// oracle_sim.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// Single-threaded FP64 restatement of CrowdPhot.fit_all_stars_simultaneous
// (src/photometry/psf_photometry_simultaneous.jl:953-1431) used as the
// correctness checker and as the timed CPU baseline.  The product library
// never links this file.  Each step cites the reference lines it follows.
// Deviations (documented, not silent):
//   * catalogue stars with non-finite y/x are excluded (valid = false) instead
//     of raising Julia's InexactError from round(Int, NaN);
//   * a negative Morton anchor raises CPB_ERR_ARGUMENT (Julia raises
//     InexactError from UInt64(negative)) -- same outcome: the call fails;
//   * solver = :lsmr runs the LSMR restatement (oracle_lsqr.hpp) in place of
//     LSQR, as krylov_solve! does; model_rad = :auto follows _model_radii with the unit
//     PSF's curve of growth (analytic for the Gaussian, exact-overlap apertures
//     otherwise), in FP64 whatever the image eltype;
//   * spread_model / spread_model_err are not computed (NaN).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <vector>

#include "oracle_lsqr.hpp"
#include "oracle_psf.hpp"

using namespace orc;

namespace {

const double kEps = std::numeric_limits<double>::epsilon();
const double kNaN = std::numeric_limits<double>::quiet_NaN();

inline double load(const void* p, int et, int64_t i) {
    return et == CPB_F64 ? ((const double*)p)[i] : (double)((const float*)p)[i];
}

void set_err(char* buf, int len, const std::string& s) {
    if (buf && len > 0) {
        std::snprintf(buf, (size_t)len, "%s", s.c_str());
    }
}

// _morton2d (:163-174).
uint64_t spread_bits(uint64_t v) {
    v &= 0x00000000ffffffffULL;
    v = (v | (v << 16)) & 0x0000ffff0000ffffULL;
    v = (v | (v << 8)) & 0x00ff00ff00ff00ffULL;
    v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0fULL;
    v = (v | (v << 2)) & 0x3333333333333333ULL;
    v = (v | (v << 1)) & 0x5555555555555555ULL;
    return v;
}
uint64_t morton2d(int64_t y, int64_t x) { return spread_bits((uint64_t)y) | (spread_bits((uint64_t)x) << 1); }

// _ring_offsets (:181-190).
void ring_offsets(int R, std::vector<int>& dy, std::vector<int>& dx) {
    dy.clear();
    dx.clear();
    for (int r = 0; r <= R; ++r)
        for (int a = -r; a <= r; ++a)
            for (int b = -r; b <= r; ++b) {
                if (std::max(std::abs(a), std::abs(b)) != r) continue;
                dy.push_back(a);
                dx.push_back(b);
            }
}

// Julia round(Int, v): half to even (default rounding mode of nearbyint).
inline int64_t jround(double v) { return (int64_t)std::nearbyint(v); }

struct Stamp {
    int p = 0, S2 = 0, R = 0;
    int64_t n = 0;
    std::vector<double> values;   // p x S2 x n (k fastest)
    std::vector<int32_t> pixels;  // S2 x n, 1-based, 0 = unusable
    std::vector<double> colnorm;  // p x n
};

struct Fit {
    const Psf* psf;
    int p;
    int grad_col[3];           // 1 = dy, 2 = dx, 3 = dflux for free param k
    int k_y = -1, k_x = -1;    // position of y / x in the free list
    double fixed_y, fixed_x, fixed_flux, fixed_bkg, fwhm;
    int64_t ny, nx;
    std::vector<int> dy_off, dx_off;      // column-major fit box
    std::vector<int> mdy_off, mdx_off;    // ring-ordered model box
    std::vector<int64_t> ay, ax;          // anchors (active order)
    std::vector<int> model_R;
    std::vector<int64_t> model_S2;

    // model_from_vector (psf_fitting.jl:23-26): free params from theta, the rest fixed.
    StarP star(const double* th) const {
        StarP s{fixed_y, fixed_x, fixed_flux, fixed_bkg, fwhm};
        for (int k = 0; k < p; ++k) {
            if (grad_col[k] == 1) s.y = th[k];
            else if (grad_col[k] == 2) s.x = th[k];
            else s.flux = th[k];
        }
        return s;
    }
};

// _fill_stamps! (:342-399 generic, :437-543 gridded): live columns only.
void fill_stamps(const Fit& F, Stamp& st, const double* theta, const std::vector<double>& w,
                 const std::vector<uint8_t>& live) {
    const int p = st.p, S2 = st.S2;
    for (int64_t a = 0; a < st.n; ++a) {
        if (!live[a]) continue;
        for (int k = 0; k < p; ++k) st.colnorm[k + p * a] = 0.0;
        StarP s = F.star(theta + a * p);
        for (int m = 0; m < S2; ++m) {
            int32_t fi = st.pixels[m + (int64_t)S2 * a];
            if (fi == 0) continue;
            double gy = (double)(F.ay[a] + F.dy_off[m]);
            double gx = (double)(F.ax[a] + F.dx_off[m]);
            double g[3];
            evaluate_fg(*F.psf, s, gy, gx, g);
            double sw = std::sqrt(w[fi - 1]);
            for (int k = 0; k < p; ++k) {
                double raw = sw * g[F.grad_col[k] - 1];
                st.values[k + p * (m + (int64_t)S2 * a)] = raw;
                st.colnorm[k + p * a] += raw * raw;
            }
        }
    }
    for (int64_t a = 0; a < st.n; ++a) {
        if (!live[a]) continue;
        for (int k = 0; k < p; ++k) {
            double cn = std::sqrt(st.colnorm[k + p * a]);
            cn = cn < kEps ? kEps : cn;
            st.colnorm[k + p * a] = cn;
            double inv = 1.0 / cn;
            for (int m = 0; m < S2; ++m) st.values[k + p * (m + (int64_t)S2 * a)] *= inv;
        }
    }
}

// _render_model! (:545-577 generic ring order; :605-673 gridded column-major box).
void render_model(const Fit& F, std::vector<double>& model, const double* theta, const std::vector<uint8_t>& live,
                  bool all) {
    std::fill(model.begin(), model.end(), 0.0);
    const int64_t n = (int64_t)F.ay.size();
    for (int64_t a = 0; a < n; ++a) {
        if (!all && !live[a]) continue;
        StarP s = F.star(theta + a * F.p);
        int64_t ay = F.ay[a], ax = F.ax[a];
        if (F.psf->kind == CPB_PSF_GRIDDED_IMAGE) {
            int R = F.model_R[a];
            for (int jj = 0; jj < 2 * R + 1; ++jj)
                for (int ii = 0; ii < 2 * R + 1; ++ii) {
                    int64_t gy = ay - R + ii, gx = ax - R + jj;
                    double val = evaluate(*F.psf, s, (double)gy, (double)gx);
                    if (gy < 1 || gy > F.ny || gx < 1 || gx > F.nx) continue;
                    model[(gy - 1) + (gx - 1) * F.ny] += val;
                }
        } else {
            for (int64_t mi = 0; mi < F.model_S2[a]; ++mi) {
                int64_t gy = ay + F.mdy_off[mi], gx = ax + F.mdx_off[mi];
                if (gy < 1 || gy > F.ny || gx < 1 || gx > F.nx) continue;
                model[(gy - 1) + (gx - 1) * F.ny] += evaluate(*F.psf, s, (double)gy, (double)gx);
            }
        }
    }
}

// _freeze_star! (:739-754).
void freeze_star(const Fit& F, std::vector<double>& data_work, const double* theta, int64_t j) {
    StarP s = F.star(theta + j * F.p);
    for (int64_t mi = 0; mi < F.model_S2[j]; ++mi) {
        int64_t gy = F.ay[j] + F.mdy_off[mi], gx = F.ax[j] + F.mdx_off[mi];
        if (gy < 1 || gy > F.ny || gx < 1 || gx > F.nx) continue;
        data_work[(gy - 1) + (gx - 1) * F.ny] -= evaluate(*F.psf, s, (double)gy, (double)gx);
    }
}

// apply_JT! (:55-85).
void apply_JT(const Stamp& st, const double* u, const std::vector<uint8_t>& live, double* z) {
    const int p = st.p, S2 = st.S2;
    std::fill(z, z + p * st.n, 0.0);
    for (int64_t a = 0; a < st.n; ++a) {
        if (!live[a]) continue;
        for (int k = 0; k < p; ++k) {
            double acc = 0;
            for (int m = 0; m < S2; ++m) {
                int32_t fi = st.pixels[m + (int64_t)S2 * a];
                acc += st.values[k + p * (m + (int64_t)S2 * a)] * u[fi == 0 ? 0 : fi - 1];
            }
            z[a * p + k] = acc;
        }
    }
}

// apply_J! (:95-137).
void apply_J(const Stamp& st, const double* v, const std::vector<uint8_t>& live, double* y, int64_t npix) {
    const int p = st.p, S2 = st.S2;
    std::fill(y, y + npix, 0.0);
    for (int64_t a = 0; a < st.n; ++a) {
        if (!live[a]) continue;
        for (int m = 0; m < S2; ++m) {
            double acc = 0;
            for (int k = 0; k < p; ++k) acc += st.values[k + p * (m + (int64_t)S2 * a)] * v[a * p + k];
            int32_t fi = st.pixels[m + (int64_t)S2 * a];
            if (fi != 0) y[fi - 1] += acc;
        }
    }
}

// Cholesky inverse with the pinv fallback (levenberg_marquardt.jl:366-388).
bool chol_inverse(const std::vector<double>& A, int n, std::vector<double>& inv);
void pinv_sym(const std::vector<double>& A, int n, std::vector<double>& inv);

}  // namespace

namespace orc {
bool chol_inverse_ext(const std::vector<double>& A, int n, std::vector<double>& inv) { return chol_inverse(A, n, inv); }
void pinv_sym_ext(const std::vector<double>& A, int n, std::vector<double>& inv) { pinv_sym(A, n, inv); }
}  // namespace orc

namespace {

// cholesky!(Symmetric(A)) (upper) then F \ I.  Returns false on a non-positive pivot.
bool chol_inverse(const std::vector<double>& A, int n, std::vector<double>& inv) {
    std::vector<double> U(n * n, 0.0);  // column-major upper factor, A = U'U
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i <= j; ++i) {
            double s = A[i + j * n];
            for (int k = 0; k < i; ++k) s -= U[k + i * n] * U[k + j * n];
            if (i == j) {
                if (!(s > 0)) return false;
                U[j + j * n] = std::sqrt(s);
            } else {
                U[i + j * n] = s / U[i + i * n];
            }
        }
    }
    inv.assign(n * n, 0.0);
    for (int c = 0; c < n; ++c) {
        std::vector<double> y(n, 0.0), x(n, 0.0);
        for (int i = 0; i < n; ++i) {  // U' y = e_c
            double s = (i == c) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) s -= U[k + i * n] * y[k];
            y[i] = s / U[i + i * n];
        }
        for (int i = n - 1; i >= 0; --i) {  // U x = y
            double s = y[i];
            for (int k = i + 1; k < n; ++k) s -= U[i + k * n] * x[k];
            x[i] = s / U[i + i * n];
        }
        for (int i = 0; i < n; ++i) inv[i + c * n] = x[i];
    }
    return true;
}

// pinv via a cyclic Jacobi eigendecomposition of the (symmetric) matrix; the
// singular values are |eigenvalues|, cut at eps*n*max (Julia's default rtol).
void pinv_sym(const std::vector<double>& A0, int n, std::vector<double>& inv) {
    std::vector<double> A(A0), V(n * n, 0.0);
    for (int i = 0; i < n; ++i) V[i + i * n] = 1.0;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
            double s = 0.5 * (A[i + j * n] + A[j + i * n]);
            A[i + j * n] = A[j + i * n] = s;
        }
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) off += A[i + j * n] * A[i + j * n];
        if (off < 1e-300) break;
        for (int pp = 0; pp < n; ++pp)
            for (int q = pp + 1; q < n; ++q) {
                double apq = A[pp + q * n];
                if (apq == 0) continue;
                double app = A[pp + pp * n], aqq = A[q + q * n];
                double tau = (aqq - app) / (2 * apq);
                double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1 + tau * tau));
                double c = 1 / std::sqrt(1 + t * t), s = t * c;
                for (int k = 0; k < n; ++k) {
                    double akp = A[k + pp * n], akq = A[k + q * n];
                    A[k + pp * n] = c * akp - s * akq;
                    A[k + q * n] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    double apk = A[pp + k * n], aqk = A[q + k * n];
                    A[pp + k * n] = c * apk - s * aqk;
                    A[q + k * n] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = V[k + pp * n], vkq = V[k + q * n];
                    V[k + pp * n] = c * vkp - s * vkq;
                    V[k + q * n] = s * vkp + c * vkq;
                }
            }
    }
    double smax = 0;
    for (int i = 0; i < n; ++i) smax = std::max(smax, std::fabs(A[i + i * n]));
    double tol = kEps * n * smax;
    inv.assign(n * n, 0.0);
    for (int e = 0; e < n; ++e) {
        double lam = A[e + e * n];
        if (!(std::fabs(lam) > tol)) continue;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) inv[i + j * n] += V[i + e * n] * V[j + e * n] / lam;
    }
}

}  // namespace

namespace orc {
// covariance! (levenberg_marquardt.jl:366-388); reweighted scales by cost/dof.
void covariance(const std::vector<double>& A, int n, bool reweighted, double cost, double dof,
                std::vector<double>& cov) {
    if (!chol_inverse(A, n, cov)) pinv_sym(A, n, cov);
    if (reweighted)
        for (auto& e : cov) e *= cost / dof;
}
}  // namespace orc

extern "C" {

// _ring_offsets for tests: writes (2R+1)^2 pairs.
int orc_ring_offsets(int R, int32_t* dy, int32_t* dx) {
    std::vector<int> a, b;
    ring_offsets(R, a, b);
    for (size_t i = 0; i < a.size(); ++i) {
        dy[i] = a[i];
        dx[i] = b[i];
    }
    return (int)a.size();
}

uint64_t orc_morton2d(int64_t y, int64_t x) { return morton2d(y, x); }

// apply_J! / apply_JT! on a caller-provided stamp (tests of the operator).
void orc_apply_J(int p, int S2, int64_t n, int64_t npix, const double* values, const int32_t* pixels,
                 const uint8_t* live, const double* v, double* y) {
    Stamp st;
    st.p = p;
    st.S2 = S2;
    st.n = n;
    st.values.assign(values, values + (int64_t)p * S2 * n);
    st.pixels.assign(pixels, pixels + (int64_t)S2 * n);
    std::vector<uint8_t> lv(live, live + n);
    apply_J(st, v, lv, y, npix);
}

void orc_apply_JT(int p, int S2, int64_t n, const double* values, const int32_t* pixels, const uint8_t* live,
                  const double* u, double* z) {
    Stamp st;
    st.p = p;
    st.S2 = S2;
    st.n = n;
    st.values.assign(values, values + (int64_t)p * S2 * n);
    st.pixels.assign(pixels, pixels + (int64_t)S2 * n);
    std::vector<uint8_t> lv(live, live + n);
    apply_JT(st, u, lv, z);
}

// The damped LSQR step on a caller-provided stamp operator.
int orc_lsqr_stamp(int p, int S2, int64_t n, int64_t npix, const double* values, const int32_t* pixels,
                   const uint8_t* live, const double* rhs, double lambda, int itmax, double atol, double btol,
                   double* x) {
    Stamp st;
    st.p = p;
    st.S2 = S2;
    st.n = n;
    st.values.assign(values, values + (int64_t)p * S2 * n);
    st.pixels.assign(pixels, pixels + (int64_t)S2 * n);
    std::vector<uint8_t> lv(live, live + n);
    auto Av = [&](const double* v, double* y) { apply_J(st, v, lv, y, npix); };
    auto Atu = [&](const double* u, double* z) { apply_JT(st, u, lv, z); };
    LsqrStats s = lsqr(npix, p * n, Av, Atu, rhs, lambda, itmax, atol, btol, x);
    return s.iters;
}

// Dense LSQR (tests against scipy): A is m x n column-major.
int orc_lsqr_dense(int64_t m, int64_t n, const double* A, const double* b, double lambda, int itmax, double atol,
                   double btol, double* x) {
    auto Av = [&](const double* v, double* y) {
        for (int64_t i = 0; i < m; ++i) {
            double s = 0;
            for (int64_t j = 0; j < n; ++j) s += A[i + j * m] * v[j];
            y[i] = s;
        }
    };
    auto Atu = [&](const double* u, double* z) {
        for (int64_t j = 0; j < n; ++j) {
            double s = 0;
            for (int64_t i = 0; i < m; ++i) s += A[i + j * m] * u[i];
            z[j] = s;
        }
    };
    LsqrStats s = lsqr(m, n, Av, Atu, b, lambda, itmax, atol, btol, x);
    return s.iters;
}

// Dense LSMR (tests against scipy): A is m x n column-major.
int orc_lsmr_dense(int64_t m, int64_t n, const double* A, const double* b, double lambda, int itmax, double atol,
                   double btol, double* x) {
    auto Av = [&](const double* v, double* y) {
        for (int64_t i = 0; i < m; ++i) {
            double s = 0;
            for (int64_t j = 0; j < n; ++j) s += A[i + j * m] * v[j];
            y[i] = s;
        }
    };
    auto Atu = [&](const double* u, double* z) {
        for (int64_t j = 0; j < n; ++j) {
            double s = 0;
            for (int64_t i = 0; i < m; ++i) s += A[i + j * m] * u[i];
            z[j] = s;
        }
    };
    LsqrStats s = lsmr(m, n, Av, Atu, b, lambda, itmax, atol, btol, x);
    return s.iters;
}

// _fill_stamps! on a caller-provided stamp (frozen-column preservation test).
int orc_fill_stamps(const cpb_psf_desc* desc, int free_mask, double fixed_y, double fixed_x, double fixed_flux,
                    double fixed_bkg, double fwhm, int R, int64_t n, int64_t ny, int64_t nx, const int32_t* pixels,
                    const int64_t* anchor_y, const int64_t* anchor_x, const double* theta, const double* w,
                    const uint8_t* live, double* values, double* colnorm) {
    Psf psf;
    if (!load_psf(desc, psf).empty()) return CPB_ERR_ARGUMENT;
    Fit F;
    F.psf = &psf;
    F.p = 0;
    if (free_mask & CPB_FREE_Y) F.grad_col[F.p++] = 1;
    if (free_mask & CPB_FREE_X) F.grad_col[F.p++] = 2;
    if (free_mask & CPB_FREE_FLUX) F.grad_col[F.p++] = 3;
    F.fixed_y = fixed_y;
    F.fixed_x = fixed_x;
    F.fixed_flux = fixed_flux;
    F.fixed_bkg = fixed_bkg;
    F.fwhm = fwhm;
    F.ny = ny;
    F.nx = nx;
    for (int dx = -R; dx <= R; ++dx)
        for (int dy = -R; dy <= R; ++dy) {
            F.dy_off.push_back(dy);
            F.dx_off.push_back(dx);
        }
    F.ay.assign(anchor_y, anchor_y + n);
    F.ax.assign(anchor_x, anchor_x + n);
    Stamp st;
    st.p = F.p;
    st.S2 = (2 * R + 1) * (2 * R + 1);
    st.n = n;
    st.values.assign(values, values + (int64_t)st.p * st.S2 * n);
    st.colnorm.assign(colnorm, colnorm + (int64_t)st.p * n);
    st.pixels.assign(pixels, pixels + (int64_t)st.S2 * n);
    std::vector<double> wv(w, w + ny * nx);
    std::vector<uint8_t> lv(live, live + n);
    fill_stamps(F, st, theta, wv, lv);
    std::memcpy(values, st.values.data(), st.values.size() * sizeof(double));
    std::memcpy(colnorm, st.colnorm.data(), st.colnorm.size() * sizeof(double));
    return 0;
}

// evaluate / evaluate_fg for tests: f[n], g[3n] (dy, dx, dflux).
int orc_psf_eval(const cpb_psf_desc* desc, double y, double x, double flux, double bkg, double fwhm, int64_t n,
                 const double* py, const double* px, double* f, double* g) {
    Psf psf;
    if (!load_psf(desc, psf).empty()) return CPB_ERR_ARGUMENT;
    StarP s{y, x, flux, bkg, fwhm};
    for (int64_t i = 0; i < n; ++i) {
        if (g) f[i] = evaluate_fg(psf, s, py[i], px[i], g + 3 * i);
        else f[i] = evaluate(psf, s, py[i], px[i]);
    }
    return 0;
}

// bicubic_interpolate for tests.
void orc_bicubic(const double* data, int64_t ny, int64_t nx, int64_t n, const double* y, const double* x,
                 double fill, double* out) {
    for (int64_t i = 0; i < n; ++i) bicubic(data, ny, nx, y[i], x[i], fill, out[3 * i], out[3 * i + 1], out[3 * i + 2]);
}

// Exact pixel / circle overlap (apertures.jl:196-290, the photutils algorithm):
// area of the rectangle [x0, x1] x [y0, y1] inside the circle of radius r at
// the origin, by splitting the rectangle at the axes into first-quadrant pieces.
static double tri_area(double ax, double ay, double bx, double by, double cx, double cy) {
    return std::fabs(ax * (by - cy) + bx * (cy - ay) + cx * (ay - by)) / 2;
}
static double seg_area(double ax, double ay, double bx, double by, double r) {
    double chord = std::sqrt((bx - ax) * (bx - ax) + (by - ay) * (by - ay));
    double th = 2 * std::asin(chord / (2 * r));
    return r * r * (th - std::sin(th)) / 2;
}
static double quad_overlap(double x0, double y0, double x1, double y1, double r) {  // 0 <= x0, 0 <= y0
    double r2 = r * r;
    if (x0 * x0 + y0 * y0 > r2) return 0.0;
    if (x1 * x1 + y1 * y1 < r2) return (x1 - x0) * (y1 - y0);
    bool c1 = std::sqrt(x1 * x1 + y0 * y0) < r, c2 = std::sqrt(x0 * x0 + y1 * y1) < r;
    if (c1 && c2) {
        double px = std::sqrt(r2 - y1 * y1), qy = std::sqrt(r2 - x1 * x1);
        return (x1 - x0) * (y1 - y0) - tri_area(px, y1, x1, qy, x1, y1) + seg_area(px, y1, x1, qy, r);
    }
    if (c1) {
        double py = std::sqrt(r2 - x0 * x0), qy = std::sqrt(r2 - x1 * x1);
        return seg_area(x0, py, x1, qy, r) + tri_area(x0, py, x0, y0, x1, y0) + tri_area(x0, py, x1, y0, x1, qy);
    }
    if (c2) {
        double px = std::sqrt(r2 - y0 * y0), qx = std::sqrt(r2 - y1 * y1);
        return seg_area(px, y0, qx, y1, r) + tri_area(px, y0, x0, y0, x0, y1) + tri_area(px, y0, x0, y1, qx, y1);
    }
    double px = std::sqrt(r2 - y0 * y0), qy = std::sqrt(r2 - x0 * x0);
    return seg_area(px, y0, x0, qy, r) + tri_area(px, y0, x0, qy, x0, y0);
}
static double rect_overlap(double x0, double y0, double x1, double y1, double r) {
    if (r <= 0) return 0.0;
    if (x0 >= 0) {
        if (y0 >= 0) return quad_overlap(x0, y0, x1, y1, r);
        if (y1 <= 0) return quad_overlap(-y1, x0, -y0, x1, r);
        return rect_overlap(x0, y0, x1, 0, r) + rect_overlap(x0, 0, x1, y1, r);
    }
    if (x1 <= 0) {
        if (y0 >= 0) return quad_overlap(-x1, y0, -x0, y1, r);
        if (y1 <= 0) return quad_overlap(-x1, -y1, -x0, -y0, r);
        return rect_overlap(x0, y0, x1, 0, r) + rect_overlap(x0, 0, x1, y1, r);
    }
    if (y0 >= 0 || y1 <= 0) return rect_overlap(x0, y0, 0, y1, r) + rect_overlap(0, y0, x1, y1, r);
    return rect_overlap(x0, y0, 0, 0, r) + rect_overlap(0, y0, x1, 0, r) + rect_overlap(x0, 0, 0, y1, r) +
           rect_overlap(0, 0, x1, y1, r);
}
// aperture_weight(CircularAperture(yc, xc, r), i, j, ExactOverlap()) (apertures.jl:93-103, 160-166).
static double exact_weight(double yc, double xc, double r, int64_t i, int64_t j) {
    double dy = (double)i - yc, dx = (double)j - xc, d2 = dx * dx + dy * dy, h = std::sqrt(2.0) / 2;
    if (d2 > (r + h) * (r + h)) return 0.0;
    if (r > h && d2 < (r - h) * (r - h)) return 1.0;
    return rect_overlap(dx - 0.5, dy - 0.5, dx + 0.5, dy + 0.5, r);
}

extern "C" {
double orc_exact_overlap(double dx, double dy, double r) { return rect_overlap(dx - 0.5, dy - 0.5, dx + 0.5, dy + 0.5, r); }
double orc_aperture_weight(double yc, double xc, double r, int64_t i, int64_t j) { return exact_weight(yc, xc, r, i, j); }
}

// curve_of_growth (curve_of_growth.jl:143-173) of the unit model
// (y = x = 0, flux = 1, bkg = 0) at radii 1..R_cap; the Gaussian uses its
// analytic overload (:180-195).
static void unit_curve_of_growth(const Psf& psf, int R_cap, std::vector<double>& cog) {
    cog.assign(R_cap, 0.0);
    if (psf.kind == CPB_PSF_CIRCULAR_GAUSSIAN) {
        for (int r = 1; r <= R_cap; ++r)
            cog[r - 1] = 1.0 * (1.0 - std::exp(gauss_pre() * ((double)r * (double)r) / (psf.fwhm * psf.fwhm)));
        return;
    }
    StarP unit{0.0, 0.0, 1.0, 0.0, psf.fwhm};
    for (int r = 1; r <= R_cap; ++r) {
        // bounding_axes (apertures.jl:52-66) of a circle of integer radius at the origin: -r..r
        double tot = 0;
        for (int64_t j = -r; j <= r; ++j)
            for (int64_t i = -r; i <= r; ++i) {
                double w = exact_weight(0.0, 0.0, (double)r, i, j);
                if (!(w > 0)) continue;
                tot += w * evaluate(psf, unit, (double)i, (double)j);
            }
        cog[r - 1] = tot;
    }
}

// _model_radii, :auto branch (:209-243), any supported PSF.
static int model_radii_auto(const Psf& psf, double nsigma, int R_fit, int R_cap, int64_t nw, const double* w,
                            int64_t n, const double* flux, int32_t* out) {
    int64_t step = std::max<int64_t>(1, nw / 65536);
    std::vector<double> ws;
    for (int64_t i = 0; i < nw; i += step)
        if (w[i] > 0 && std::isfinite(w[i])) ws.push_back(w[i]);
    if (ws.empty()) return CPB_ERR_ARGUMENT;
    std::sort(ws.begin(), ws.end());
    double h = (double)(ws.size() - 1) * 0.84;  // quantile, type 7
    size_t lo = (size_t)std::floor(h);
    size_t hi = std::min(lo + 1, ws.size() - 1);
    double wval = ws[lo] + (h - (double)lo) * (ws[hi] - ws[lo]);
    double sigma_bg = wval > 0 ? std::sqrt(1.0 / wval) : 1.0;
    std::vector<double> cog, sb(R_cap);
    unit_curve_of_growth(psf, R_cap, cog);
    double prev = 0;
    for (int r = 1; r <= R_cap; ++r) {
        double ee = cog[r - 1] / cog[R_cap - 1];
        sb[r - 1] = std::max((ee - prev) / (M_PI * (double)(r * r - (r - 1) * (r - 1))), 0.0);
        prev = ee;
    }
    double thr = nsigma * sigma_bg;
    for (int64_t j = 0; j < n; ++j) {
        double Fj = std::max(flux[j], 0.0);
        int r = R_fit;
        while (r < R_cap && Fj * sb[r - 1] > thr) ++r;
        out[j] = r;
    }
    return 0;
}

extern "C" {
// The unit model's curve of growth at radii 1..R_cap (tests).
int orc_unit_curve_of_growth(const cpb_psf_desc* desc, double fwhm, int R_cap, double* out) {
    Psf psf;
    if (!load_psf(desc, psf).empty()) return CPB_ERR_ARGUMENT;
    psf.fwhm = fwhm;
    std::vector<double> cog;
    unit_curve_of_growth(psf, R_cap, cog);
    std::copy(cog.begin(), cog.end(), out);
    return 0;
}
int orc_model_radii_auto(const cpb_psf_desc* desc, double fwhm, double nsigma, int R_fit, int R_cap, int64_t nw,
                         const double* w, int64_t n, const double* flux, int32_t* out) {
    Psf psf;
    if (!load_psf(desc, psf).empty()) return CPB_ERR_ARGUMENT;
    psf.fwhm = fwhm;
    return model_radii_auto(psf, nsigma, R_fit, R_cap, nw, w, n, flux, out);
}
}

// _model_radii, :auto branch (:209-243) for CircularGaussianPSF, whose curve
// of growth is analytic (curve_of_growth.jl:180-195).  w: inverse-weight vector.
int orc_model_radii_auto_gaussian(double fwhm, double nsigma, int R_fit, int R_cap, int64_t nw, const double* w,
                                  int64_t n, const double* flux, int32_t* out) {
    int64_t step = std::max<int64_t>(1, nw / 65536);
    std::vector<double> ws;
    for (int64_t i = 0; i < nw; i += step)
        if (w[i] > 0 && std::isfinite(w[i])) ws.push_back(w[i]);
    if (ws.empty()) return CPB_ERR_ARGUMENT;
    std::sort(ws.begin(), ws.end());
    // quantile type 7
    double h = (double)(ws.size() - 1) * 0.84;
    size_t lo = (size_t)std::floor(h);
    size_t hi = std::min(lo + 1, ws.size() - 1);
    double wval = ws[lo] + (h - (double)lo) * (ws[hi] - ws[lo]);
    double sigma_bg = wval > 0 ? std::sqrt(1.0 / wval) : 1.0;
    std::vector<double> cog(R_cap), sb(R_cap);
    for (int r = 1; r <= R_cap; ++r)
        cog[r - 1] = 1.0 * (1.0 - std::exp(gauss_pre() * ((double)r * (double)r) / (fwhm * fwhm)));
    double prev = 0;
    for (int r = 1; r <= R_cap; ++r) {
        double ee = cog[r - 1] / cog[R_cap - 1];
        sb[r - 1] = std::max((ee - prev) / (M_PI * (double)(r * r - (r - 1) * (r - 1))), 0.0);
        prev = ee;
    }
    double thr = nsigma * sigma_bg;
    for (int64_t j = 0; j < n; ++j) {
        double Fj = std::max(flux[j], 0.0);
        int r = R_fit;
        while (r < R_cap && Fj * sb[r - 1] > thr) ++r;
        out[j] = r;
    }
    return 0;
}

// fit_all_stars_simultaneous (:953-1431).
int orc_fit_simultaneous(const cpb_psf_desc* desc, const cpb_sim_params* P, const void* image, int32_t eltype,
                         int64_t ny, int64_t nx, const void* inv_var, const void* background, int64_t n_stars,
                         const double* y0, const double* x0, const double* flux0, cpb_sim_result* out, char* errbuf,
                         int errlen) {
    auto fail = [&](const std::string& m) {
        set_err(errbuf, errlen, m);
        return CPB_ERR_ARGUMENT;
    };
    // argument checks in the reference's order (:984-997)
    if (!(P->max_iter > 0)) return fail("max_iter must be positive");
    if (!(P->inner_iterations > 0)) return fail("inner_iterations must be positive");
    if (!(P->linear_tol > 0)) return fail("linear_tol must be positive");
    if (!(P->max_trials > 0)) return fail("max_trials must be positive");
    if (!P->model_rad_auto && !(P->model_rad > 0))
        return fail("model_rad must be :auto or a positive real");
    const double model_rad_max = P->model_rad_max < 0 ? 10 * P->fit_rad : P->model_rad_max;
    if (!(model_rad_max >= P->fit_rad)) return fail("model_rad_max must be >= fit_rad");
    if (!(P->model_rad_nsigma > 0)) return fail("model_rad_nsigma must be positive");
    if (P->solver != CPB_SOLVER_LSQR && P->solver != CPB_SOLVER_LSMR)
        return fail("solver must be :lsqr or :lsmr");
    if (P->damping == CPB_DAMP_LEVENBERG)
        return fail(
            "LevenbergDamping is not supported by fit_all_stars_simultaneous: it conflicts with the "
            "column-equilibrated x_tol scaling. Use MarquardtDamping.");
    if (!(P->fit_rad > 0)) return fail("fit_rad must be positive");
    if (eltype != CPB_F32 && eltype != CPB_F64) return fail("unsupported image eltype");

    Psf psf;
    {
        std::string e = load_psf(desc, psf);
        if (!e.empty()) return fail(e);
    }
    const bool reweighted =
        P->covariance == CPB_COV_REWEIGHTED || (P->covariance == CPB_COV_AUTO && inv_var == nullptr);
    out->n_active = 0;
    out->n_union = 0;
    out->n_trials = 0;
    out->n_lsqr_iters = 0;
    out->model_px_evals = 0;
    out->lsqr_px_macs = 0;
    out->device_seconds = 0;
    const int64_t npix = ny * nx;
    auto put_nan_diag = [&](int64_t i) {
        if (out->qfit) out->qfit[i] = kNaN;
        if (out->qfit_expected) out->qfit_expected[i] = kNaN;
        if (out->qfit_z) out->qfit_z[i] = kNaN;
        if (out->crowding) out->crowding[i] = kNaN;
        if (out->spread_model) out->spread_model[i] = kNaN;
        if (out->spread_model_err) out->spread_model_err[i] = kNaN;
    };
    if (n_stars == 0) {
        out->n_passes = 0;
        out->n_failed = 0;
        if (out->residual) std::fill(out->residual, out->residual + npix, 0.0);
        return 0;
    }
    // free set (:1015-1051)
    Fit F;
    F.psf = &psf;
    F.p = 0;
    if (P->free_mask & CPB_FREE_Y) F.grad_col[F.p++] = 1;
    if (P->free_mask & CPB_FREE_X) F.grad_col[F.p++] = 2;
    if (P->free_mask & CPB_FREE_FLUX) F.grad_col[F.p++] = 3;
    if (P->free_mask & ~(CPB_FREE_Y | CPB_FREE_X | CPB_FREE_FLUX))
        return fail(
            "fit_all_stars_simultaneous fits only (y, x, flux) per star. Fix `bkg` (subtract the background "
            "first and pass `fixed = (; bkg = zero(eltype(image)))`), and fix all shape parameters.");
    if (F.p == 0) return fail("all model parameters are fixed; nothing to fit");
    const int p = F.p;
    for (int k = 0; k < p; ++k) {
        if (F.grad_col[k] == 1) F.k_y = k;
        if (F.grad_col[k] == 2) F.k_x = k;
    }
    F.fixed_y = P->fixed_y;
    F.fixed_x = P->fixed_x;
    F.fixed_flux = P->fixed_flux;
    F.fixed_bkg = P->fixed_bkg;
    F.fwhm = psf.kind == CPB_PSF_CIRCULAR_GAUSSIAN ? P->fixed_fwhm : 0.0;
    F.ny = ny;
    F.nx = nx;

    // data and weights (:1056-1084)
    std::vector<double> data(npix), w(npix);
    for (int64_t q = 0; q < npix; ++q) {
        data[q] = load(image, eltype, q) - (background ? load(background, eltype, q) : 0.0);
    }
    if (!inv_var) {
        for (int64_t q = 0; q < npix; ++q)
            if (!std::isfinite(data[q]))
                return fail(
                    "the image contains non-finite values but `inv_var` was not provided; pass `inv_var` to "
                    "mask them or clean the image first");
        std::fill(w.begin(), w.end(), 1.0);
    } else {
        for (int64_t q = 0; q < npix; ++q) {
            double wv = load(inv_var, eltype, q);
            w[q] = (std::isfinite(wv) && wv > 0) ? wv : 0.0;
        }
    }
    for (int64_t q = 0; q < npix; ++q)
        if (!std::isfinite(data[q])) {
            data[q] = 0.0;
            w[q] = 0.0;
        }

    // _build_stamps! (:245-323)
    const int R = (int)std::ceil(P->fit_rad);
    const int S = 2 * R + 1, S2 = S * S;
    for (int dx = -R; dx <= R; ++dx)
        for (int dy = -R; dy <= R; ++dy) {
            F.dy_off.push_back(dy);
            F.dx_off.push_back(dx);
        }
    std::vector<int64_t> anc_y(n_stars), anc_x(n_stars);
    std::vector<uint8_t> valid(n_stars, 1);
    std::vector<int64_t> active;
    std::vector<int32_t> pix_all((size_t)S2 * n_stars, 0);
    for (int64_t i = 0; i < n_stars; ++i) {
        bool fin = std::isfinite(y0[i]) && std::isfinite(x0[i]);
        anc_y[i] = fin ? jround(y0[i]) : 0;
        anc_x[i] = fin ? jround(x0[i]) : 0;
        bool any = false;
        if (fin)
            for (int m = 0; m < S2; ++m) {
                int64_t gy = anc_y[i] + F.dy_off[m], gx = anc_x[i] + F.dx_off[m];
                if (gy >= 1 && gy <= ny && gx >= 1 && gx <= nx) {
                    int64_t fi = gy + (gx - 1) * ny;
                    if (w[fi - 1] > 0) {
                        pix_all[m + (size_t)S2 * i] = (int32_t)fi;
                        any = true;
                    }
                }
            }
        bool ok = any && fin && std::isfinite(flux0[i]);
        if (ok) active.push_back(i);
        else valid[i] = 0;
    }
    for (int64_t i : active)
        if (anc_y[i] < 0 || anc_x[i] < 0)
            return fail("InexactError: a star's integer anchor is negative (Morton key of a negative coordinate)");
    std::stable_sort(active.begin(), active.end(), [&](int64_t a, int64_t b) {
        return morton2d(anc_y[a], anc_x[a]) < morton2d(anc_y[b], anc_x[b]);
    });
    const int64_t n_act = (int64_t)active.size();
    const int n_failed = (int)(n_stars - n_act);
    out->n_active = n_act;
    if (out->dbg_active)
        for (int64_t j = 0; j < n_act; ++j) out->dbg_active[j] = (int32_t)active[j];

    // outputs that do not depend on the solve
    auto write_fixed_outputs = [&](std::vector<double>& oy, std::vector<double>& ox, std::vector<double>& of) {
        for (int64_t i = 0; i < n_stars; ++i) {
            if (!(P->free_mask & CPB_FREE_Y)) oy[i] = P->fixed_y;
            if (!(P->free_mask & CPB_FREE_X)) ox[i] = P->fixed_x;
            if (!(P->free_mask & CPB_FREE_FLUX)) of[i] = P->fixed_flux;
        }
    };
    if (n_act == 0) {  // _empty_simultaneous_result (:1433-1445)
        for (int64_t i = 0; i < n_stars; ++i) {
            out->y[i] = y0[i];
            out->x[i] = x0[i];
            out->flux[i] = flux0[i];
            out->bkg[i] = 0.0;
            out->y_err[i] = (P->free_mask & CPB_FREE_Y) ? kNaN : 0.0;
            out->x_err[i] = (P->free_mask & CPB_FREE_X) ? kNaN : 0.0;
            out->flux_err[i] = (P->free_mask & CPB_FREE_FLUX) ? kNaN : 0.0;
            out->bkg_err[i] = 0.0;
            out->converged[i] = 0;
            out->valid[i] = valid[i];
            if (out->chisq) out->chisq[i] = 0.0;
            put_nan_diag(i);
            out->n_iter[i] = 0;
        }
        out->n_passes = 0;
        out->n_failed = (int32_t)n_stars;
        if (out->residual) std::fill(out->residual, out->residual + npix, 0.0);
        return 0;
    }
    Stamp st;
    st.p = p;
    st.S2 = S2;
    st.R = R;
    st.n = n_act;
    st.pixels.resize((size_t)S2 * n_act);
    F.ay.resize(n_act);
    F.ax.resize(n_act);
    for (int64_t j = 0; j < n_act; ++j) {
        std::memcpy(&st.pixels[(size_t)S2 * j], &pix_all[(size_t)S2 * active[j]], sizeof(int32_t) * S2);
        F.ay[j] = anc_y[active[j]];
        F.ax[j] = anc_x[active[j]];
    }
    if (out->dbg_pixels) std::memcpy(out->dbg_pixels, st.pixels.data(), sizeof(int32_t) * st.pixels.size());

    // _touched_pixels (:329-335)
    std::vector<uint8_t> mask(npix, 0);
    for (int32_t fi : st.pixels)
        if (fi != 0) mask[fi - 1] = 1;
    std::vector<int64_t> U;
    for (int64_t q = 0; q < npix; ++q)
        if (mask[q]) U.push_back(q);
    out->n_union = (int64_t)U.size();

    // model radii (:1111-1124)
    if (P->model_rad_auto && !inv_var)
        return fail(
            "model_rad=:auto requires inv_var (it needs a noise scale); pass inv_var or an explicit scalar "
            "model_rad");
    const int R_fit = R;
    if (P->model_rad_auto) {
        const int R_cap = (int)std::ceil(model_rad_max);
        std::vector<double> fl(n_act);
        for (int64_t j = 0; j < n_act; ++j) fl[j] = flux0[active[j]];
        std::vector<int32_t> mr(n_act);
        if (model_radii_auto(psf, P->model_rad_nsigma, R_fit, R_cap, npix, w.data(), n_act, fl.data(), mr.data()) != 0)
            return fail("model_rad=:auto found no positive finite weights to estimate the noise");
        F.model_R.assign(mr.begin(), mr.end());
    } else {
        const int R_cap = (int)std::ceil(std::max(P->model_rad, P->fit_rad));
        int r = (int)std::ceil(P->model_rad);
        r = std::min(std::max(r, R_fit), R_cap);
        F.model_R.assign(n_act, r);
    }
    int R_max = *std::max_element(F.model_R.begin(), F.model_R.end());
    ring_offsets(R_max, F.mdy_off, F.mdx_off);
    F.model_S2.resize(n_act);
    for (int64_t j = 0; j < n_act; ++j)
        F.model_S2[j] = (int64_t)(2 * F.model_R[j] + 1) * (2 * F.model_R[j] + 1);
    if (out->dbg_model_R)
        for (int64_t j = 0; j < n_act; ++j) out->dbg_model_R[j] = F.model_R[j];

    // working buffers (:1129-1166)
    const int64_t n = (int64_t)p * n_act;
    std::vector<double> theta(n), b_scaled(n), d_scaled(n), delta(n), D(n), theta_c(n);
    for (int64_t j = 0; j < n_act; ++j)
        for (int k = 0; k < p; ++k) {
            int gc = F.grad_col[k];
            double v = gc == 1 ? y0[active[j]] : (gc == 2 ? x0[active[j]] : flux0[active[j]]);
            theta[j * p + k] = v;
        }
    st.values.assign((size_t)p * S2 * n_act, 0.0);
    st.colnorm.assign((size_t)p * n_act, 0.0);
    std::vector<double> model_img(npix, 0.0), model_cand(npix, 0.0), wt_resid(npix, 0.0), mrhs(npix, 0.0);
    std::vector<uint8_t> live(n_act, 1), star_conv(n_act, 0);
    std::vector<int32_t> frozen_at(n_act, 0);
    std::vector<double> data_work(data);

    auto residual_cost = [&]() {  // _residual_cost! (:675-684)
        double cost = 0;
        for (int64_t q : U) {
            double r = model_img[q] - data_work[q];
            double wr = std::sqrt(w[q]) * r;
            wt_resid[q] = wr;
            cost += wr * wr;
        }
        return cost;
    };
    auto cand_cost = [&]() {  // _cost! (:686-693)
        double cost = 0;
        for (int64_t q : U) {
            double r = model_cand[q] - data_work[q];
            cost += w[q] * r * r;
        }
        return cost;
    };
    auto count_live = [&]() {
        int64_t c = 0;
        for (auto l : live) c += l;
        return c;
    };
    auto model_evals = [&](bool fill) {
        double e = 0;
        for (int64_t j = 0; j < n_act; ++j)
            if (live[j]) e += fill ? (double)S2 : (double)F.model_S2[j];
        return e;
    };

    // initial fill and cost (:1171-1176)
    fill_stamps(F, st, theta.data(), w, live);
    render_model(F, model_img, theta.data(), live, false);
    double cost = residual_cost();
    D.assign(st.colnorm.begin(), st.colnorm.end());
    const double dof = (double)std::max<int64_t>((int64_t)U.size() - n, 1);
    double lam = P->lambda_init;
    int n_run = 0;
    auto Av = [&](const double* v, double* y) { apply_J(st, v, live, y, npix); };
    auto Atu = [&](const double* u, double* z) { apply_JT(st, u, live, z); };

    // outer loop (:1186-1284)
    for (int iter = 1; iter <= P->max_iter; ++iter) {
        int64_t nl = count_live();
        out->model_px_evals += model_evals(true) + model_evals(false);
        fill_stamps(F, st, theta.data(), w, live);
        render_model(F, model_img, theta.data(), live, false);
        cost = residual_cost();
        for (int64_t q = 0; q < npix; ++q) mrhs[q] = -wt_resid[q];
        apply_JT(st, wt_resid.data(), live, b_scaled.data());
        out->lsqr_px_macs += (double)nl * S2;
        const double C_r = cost / dof;
        double gnorm = 0;
        for (int64_t i = 0; i < n; ++i) {
            double bt = st.colnorm[i] * b_scaled[i];
            double Aii = st.colnorm[i] * st.colnorm[i];
            gnorm = std::max(gnorm, std::fabs(bt) / (std::sqrt(Aii * C_r) + kEps));
        }
        if (gnorm <= P->g_tol) {
            for (int64_t j = 0; j < n_act; ++j)
                if (live[j]) {
                    live[j] = 0;
                    frozen_at[j] = iter - 1;
                    star_conv[j] = 1;
                }
            n_run = iter - 1;
            break;
        }
        bool accepted = false, f_conv = false;
        for (int trial = 1; trial <= P->max_trials; ++trial) {
            out->n_trials += 1;
            double lam_solve = std::sqrt(lam);
            // krylov_solve!(ws, J_op, mrhs; λ, itmax, atol, btol) with the workspace of `solver` (:1222-1224)
            LsqrStats ls = (P->solver == CPB_SOLVER_LSMR ? lsmr : lsqr)(
                npix, n, Av, Atu, mrhs.data(), lam_solve, P->inner_iterations, P->linear_tol, P->linear_tol,
                d_scaled.data());
            out->n_lsqr_iters += ls.iters;
            out->lsqr_px_macs += 2.0 * ls.iters * nl * S2 + (double)nl * S2;
            for (int64_t i = 0; i < n; ++i) delta[i] = d_scaled[i] / st.colnorm[i];
            // _cap_position_step! (:700-716)
            if (F.k_y >= 0 || F.k_x >= 0) {
                for (int64_t a = 0; a < n_act; ++a) {
                    int64_t base = a * p;
                    double dy = F.k_y < 0 ? 0.0 : delta[base + F.k_y];
                    double dx = F.k_x < 0 ? 0.0 : delta[base + F.k_x];
                    double len = std::sqrt(dy * dy + dx * dx);
                    if (!(len > P->max_step)) continue;
                    double sc = P->max_step / len;
                    if (F.k_y >= 0) delta[base + F.k_y] *= sc;
                    if (F.k_x >= 0) delta[base + F.k_x] *= sc;
                }
            }
            for (int64_t i = 0; i < n; ++i) d_scaled[i] = st.colnorm[i] * delta[i];
            for (int64_t i = 0; i < n; ++i) theta_c[i] = theta[i] + delta[i];
            render_model(F, model_cand, theta_c.data(), live, false);
            out->model_px_evals += model_evals(false);
            double cost_cand = cand_cost();
            double dcost = cost - cost_cand;
            f_conv = (cost_cand < cost) && (dcost / cost <= P->f_tol);
            if (cost_cand < cost) {
                accepted = true;
                for (int64_t i = 0; i < n; ++i) theta[i] += delta[i];
                cost = cost_cand;
                lam = std::max(lam / P->lambda_down, P->lambda_min);
                for (int64_t i = 0; i < n; ++i) D[i] = std::max(D[i], st.colnorm[i]);
                break;
            } else {
                lam = std::min(lam * P->lambda_up, P->lambda_max);
            }
        }
        n_run = iter;
        if (f_conv) {
            for (int64_t j = 0; j < n_act; ++j)
                if (live[j]) {
                    live[j] = 0;
                    frozen_at[j] = iter;
                    star_conv[j] = 1;
                }
            break;
        }
        if (accepted) {
            for (int64_t j = 0; j < n_act; ++j) {
                if (!live[j]) continue;
                // _x_tol_local (:810-823)
                double num = 0, xn = 0;
                for (int k = 0; k < p; ++k) {
                    int64_t i = j * p + k;
                    double v = (D[i] / st.colnorm[i]) * d_scaled[i];
                    num += v * v;
                    double xv = D[i] * theta[i];
                    xn += xv * xv;
                }
                bool xt = std::sqrt(num) <= P->x_tol * (std::sqrt(xn) + P->x_tol);
                // _g_tol_local (:789-801)
                double gn = 0;
                for (int k = 0; k < p; ++k) {
                    int64_t i = j * p + k;
                    double bt = st.colnorm[i] * b_scaled[i];
                    double Aii = st.colnorm[i] * st.colnorm[i];
                    gn = std::max(gn, std::fabs(bt) / (std::sqrt(Aii * C_r) + kEps));
                }
                bool gt = gn <= P->g_tol;
                if (xt || gt) {
                    freeze_star(F, data_work, theta.data(), j);
                    live[j] = 0;
                    frozen_at[j] = iter;
                    star_conv[j] = 1;
                }
            }
            if (count_live() == 0) break;
        }
    }

    // final bookkeeping (:1289-1300)
    std::vector<double> oy(y0, y0 + n_stars), ox(x0, x0 + n_stars), of(flux0, flux0 + n_stars);
    for (int64_t j = 0; j < n_act; ++j)
        for (int k = 0; k < p; ++k) {
            int gc = F.grad_col[k];
            double v = theta[j * p + k];
            if (gc == 1) oy[active[j]] = v;
            else if (gc == 2) ox[active[j]] = v;
            else of[active[j]] = v;
        }
    write_fixed_outputs(oy, ox, of);
    std::vector<double> ey(n_stars, kNaN), ex(n_stars, kNaN), ef(n_stars, kNaN);
    for (int64_t i = 0; i < n_stars; ++i) {
        if (!(P->free_mask & CPB_FREE_Y)) ey[i] = 0.0;
        if (!(P->free_mask & CPB_FREE_X)) ex[i] = 0.0;
        if (!(P->free_mask & CPB_FREE_FLUX)) ef[i] = 0.0;
    }
    // errors (:1302-1329)
    std::vector<uint8_t> all_live(n_act, 1);
    fill_stamps(F, st, theta.data(), w, all_live);
    for (int64_t j = 0; j < n_act; ++j) {
        std::vector<double> blk(p * p, 0.0);
        for (int m = 0; m < S2; ++m) {
            if (st.pixels[m + (size_t)S2 * j] == 0) continue;
            for (int k = 0; k < p; ++k)
                for (int l = 0; l < p; ++l)
                    blk[k + l * p] += st.values[k + p * (m + (size_t)S2 * j)] * st.values[l + p * (m + (size_t)S2 * j)];
        }
        for (int k = 0; k < p; ++k)
            for (int l = 0; l < p; ++l) blk[k + l * p] *= st.colnorm[k + p * j] * st.colnorm[l + p * j];
        double tr = 0;
        for (int k = 0; k < p; ++k) tr += blk[k + k * p];
        for (int k = 0; k < p; ++k) blk[k + k * p] += 1.0e-12 * tr;
        std::vector<double> cov;
        covariance(blk, p, reweighted, cost, dof, cov);
        for (int k = 0; k < p; ++k) {
            double e = std::sqrt(std::max(0.0, cov[k + k * p]));
            int gc = F.grad_col[k];
            if (gc == 1) ey[active[j]] = e;
            else if (gc == 2) ex[active[j]] = e;
            else ef[active[j]] = e;
        }
    }
    // validity gate (:1332-1337)
    for (int64_t i = 0; i < n_stars; ++i)
        if (valid[i] && !(std::isfinite(oy[i]) && std::isfinite(ox[i]) && std::isfinite(of[i]) && of[i] > 0))
            valid[i] = 0;
    // final render against the original data (:1344-1356)
    render_model(F, model_img, theta.data(), all_live, true);
    std::vector<double> resid(npix);
    for (int64_t q = 0; q < npix; ++q) resid[q] = data[q] - model_img[q];
    if (out->residual) std::memcpy(out->residual, resid.data(), sizeof(double) * npix);

    for (int64_t i = 0; i < n_stars; ++i) {
        out->y[i] = oy[i];
        out->x[i] = ox[i];
        out->flux[i] = of[i];
        out->bkg[i] = P->fixed_bkg;
        out->y_err[i] = ey[i];
        out->x_err[i] = ex[i];
        out->flux_err[i] = ef[i];
        out->bkg_err[i] = 0.0;
        out->valid[i] = valid[i];
        out->converged[i] = 0;
        out->n_iter[i] = 0;
        if (out->chisq) out->chisq[i] = 0.0;
        put_nan_diag(i);
    }
    // spread_model reference disk: one field-constant kernel sized from the
    // catalogue's first star's parameters after the bookkeeping above
    // (params[row_y, 1], params[row_x, 1], :1289-1299, :1361-1365): its fitted
    // position when active, its catalogue position otherwise, fixed values
    std::vector<double> spread_K;
    int spread_half = 0;
    const bool have_spread =
        n_stars > 0 && spread_kernel(psf, P->spread_model_fwhm, out->y[0], out->x[0], P->fit_rad, spread_K, spread_half);
    // per-star diagnostics (:1382-1397 chisq; psf_photometry_diagnostics.jl:154-231)
    for (int64_t j = 0; j < n_act; ++j) {
        int64_t i = active[j];
        out->converged[i] = star_conv[j];
        out->n_iter[i] = live[j] ? n_run : frozen_at[j];
        if (!valid[i]) continue;
        StarP s = F.star(theta.data() + j * p);
        int64_t ylo = (int64_t)std::floor(s.y - P->fit_rad), yhi = (int64_t)std::ceil(s.y + P->fit_rad);
        int64_t xlo = (int64_t)std::floor(s.x - P->fit_rad), xhi = (int64_t)std::ceil(s.x + P->fit_rad);
        ylo = std::max<int64_t>(ylo, 1);
        yhi = std::min<int64_t>(yhi, ny);
        xlo = std::max<int64_t>(xlo, 1);
        xhi = std::min<int64_t>(xhi, nx);
        if (ylo > yhi || xlo > xhi) continue;
        // _star_diagnostics! (qfit, qfit_expected, qfit_z, crowding, spread_model)
        double flux = s.flux, bkg = s.bkg;
        if (flux > 0) {
            const int h = (int)(yhi - ylo + 1), w = (int)(xhi - xlo + 1);
            std::vector<double> ms((size_t)h * w), gs;
            for (int c = 0; c < w; ++c)
                for (int r = 0; r < h; ++r) ms[r + (size_t)c * h] = evaluate(psf, s, (double)(ylo + r), (double)(xlo + c));
            const bool do_spread = have_spread;
            if (do_spread) {
                gs.resize(ms.size());
                correlate_zero(ms.data(), h, w, spread_K, spread_half, gs.data());
            }
            double inv_flux = 1.0 / flux, qv = 0, num_clean = 0, num_dirty = 0, den = 0;
            double Sp = 0, Sq = 0, Sp0 = 0, Sq0 = 0, SqG = 0;
            double sig_sum = 0, sig2_sum = 0;
            int64_t ngood = 0;
            for (int64_t gx = xlo; gx <= xhi; ++gx)
                for (int64_t gy = ylo; gy <= yhi; ++gy) {
                    int64_t q = (gy - 1) + (gx - 1) * ny;
                    const size_t e = (size_t)(gy - ylo) + (size_t)(gx - xlo) * h;
                    double mv = ms[e];
                    double wp = inv_var ? load(inv_var, eltype, q) : 1.0;
                    if (std::isfinite(wp) && wp > 0) {
                        qv += std::fabs(resid[q]);
                        double Pp = (mv - bkg) * inv_flux;
                        double wP = wp * Pp;
                        double p_i = resid[q] + mv - bkg;
                        num_clean += wP * p_i;
                        double img = load(image, eltype, q) - (background ? load(background, eltype, q) : 0.0);
                        num_dirty += wP * (img - bkg);
                        den += wP * Pp;
                        if (do_spread) {
                            double g_i = (gs[e] - bkg) * inv_flux;
                            Sp += wP * p_i;
                            Sq += wp * g_i * p_i;
                            Sp0 += wP * Pp;
                            Sq0 += wp * Pp * g_i;
                            SqG += wp * g_i * g_i;
                        }
                    }
                    if (inv_var) {
                        double iv = load(inv_var, eltype, q);
                        if (std::isfinite(iv) && iv > 0) {
                            double si = 1.0 / std::sqrt(iv);
                            sig_sum += si;
                            sig2_sum += si * si;
                            ngood += 1;
                        }
                    }
                }
            if (out->qfit) out->qfit[i] = qv * inv_flux;
            if (out->crowding && den > 0 && num_clean > 0 && num_dirty > 0)
                out->crowding[i] = 2.5 * std::log10(num_dirty / num_clean);
            if (do_spread && Sp > 0) {
                if (out->spread_model) out->spread_model[i] = Sq / Sp - Sq0 / Sp0;
                if (inv_var && out->spread_model_err) {
                    double v = Sp * Sp * SqG + Sq * Sq * Sp0 - 2 * Sq * Sp * Sq0;
                    out->spread_model_err[i] = std::sqrt(std::max(0.0, v)) / (Sp * Sp);
                }
            }
            if (inv_var) {
                if (out->qfit_expected) out->qfit_expected[i] = std::sqrt(2.0 / M_PI) * sig_sum * inv_flux;
                if (out->qfit_z && sig2_sum > 0 && ngood > p) {
                    double dof_factor = std::sqrt(1.0 - (double)p / (double)ngood);
                    double numz = qv - std::sqrt(2.0 / M_PI) * dof_factor * sig_sum;
                    double denz = std::sqrt((1.0 - 2.0 / M_PI) * sig2_sum) * dof_factor;
                    out->qfit_z[i] = numz / denz;
                }
            }
        }
        // chisq (:1382-1397)
        double num = 0;
        int64_t ng = 0;
        for (int64_t gx = xlo; gx <= xhi; ++gx)
            for (int64_t gy = ylo; gy <= yhi; ++gy) {
                int64_t q = (gy - 1) + (gx - 1) * ny;
                double iv = inv_var ? load(inv_var, eltype, q) : 1.0;
                if (std::isfinite(iv) && iv > 0) {
                    num += iv * (resid[q] * resid[q]);
                    ng += 1;
                }
            }
        int64_t den = ng - p;
        if (out->chisq && den > 0) out->chisq[i] = num / (double)den;
    }
    out->n_passes = n_run;
    out->n_failed = n_failed;
    return 0;
}

}  // extern "C"
