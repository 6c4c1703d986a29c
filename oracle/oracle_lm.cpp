// oracle_lm.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// FP64 restatement of CrowdPhot.PSF.fit_star for the three supported PSF kinds
// and of the LM driver lm_irls without IRLS:
//   _prepare_fit_star_inputs   src/psf/psf_fitting.jl:36-101
//   fit_star(CircularGaussianPSF) + _accum_circular_gaussian!  :314-451
//   fit_star(ImagePSF) + _accum_image_psf!                    :1086-1173
//   fit_star(GriddedPSFModel{ImagePSF}) + _accum_gridded_imagepsf!  :1177-1517
//   lm_irls, damp!, covariance!  src/levenberg_marquardt.jl:64-99, 361-680
// Only tests/, smoke() and bench.py's CPU legs load it.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <atomic>
#include <thread>
#include <vector>

#include "oracle_psf.hpp"

using namespace orc;

namespace orc {
void covariance(const std::vector<double>& A, int n, bool reweighted, double cost, double dof,
                std::vector<double>& cov);
}

namespace {

const double kEps = std::numeric_limits<double>::epsilon();

struct Cutout {
    const double* pix;  // column-major ny x nx
    const double* iv;   // nullable
    int ny, nx, y1, x1;
};

// Accumulates cost, b (np) and A (np x np, column-major) over the cutout at
// the full parameter vector `full` (Gaussian: y,x,fwhm,flux,bkg; else y,x,flux,bkg),
// then projects onto the free set (psf_fitting.jl:423-450, 1165-1172, 1500-1516).
double accum(const Psf& psf, const Cutout& c, const std::vector<double>& wts, const double* full, const int* fidx,
             int nf, double* A, double* b) {
    const bool gauss = psf.kind == CPB_PSF_CIRCULAR_GAUSSIAN;
    const int np = gauss ? 5 : 4;
    double Af[25] = {0}, bf[5] = {0}, cost = 0;
    double Y = full[0], X = full[1];
    if (gauss) {
        const double gp = gauss_pre();
        double fwhm = full[2], flux = full[3], bkg = full[4];
        double f2 = fwhm * fwhm;
        double norm = -(M_PI * f2 / gp);
        double amp = flux / norm, gf2 = gp / f2;
        for (int j = 0; j < c.nx; ++j)
            for (int i = 0; i < c.ny; ++i) {
                double dx = (double)(c.x1 + j) - X, dy = (double)(c.y1 + i) - Y;
                double sq = (dx * dx + dy * dy) / f2;
                double g = std::exp(gp * sq);
                double Ag = amp * g;
                double r = (amp * g + bkg) - c.pix[i + j * c.ny];
                double w = wts[i + j * c.ny];
                double wr = w * r;
                cost = wr * r + cost;
                double gv[5] = {-2 * Ag * gf2 * dy, -2 * Ag * gf2 * dx, -2 * Ag * (1 + gp * sq) / fwhm, g / norm, 1.0};
                for (int q = 0; q < 5; ++q) {
                    bf[q] = wr * gv[q] + bf[q];
                    for (int pq = 0; pq <= q; ++pq) Af[pq + q * 5] = (w * gv[pq]) * gv[q] + Af[pq + q * 5];
                }
            }
    } else {
        double flux = full[2], bkg = full[3];
        Corner cr[4];
        grid_corners_dw(psf, Y, X, cr);
        for (int j = 0; j < c.nx; ++j)
            for (int i = 0; i < c.ny; ++i) {
                double py = (double)(c.y1 + i), px = (double)(c.x1 + j);
                double s = 0, dsdY = 0, dsdX = 0;
                if (psf.kind == CPB_PSF_IMAGE) {
                    const Node& nd = psf.nodes[0];
                    double u = nd.sx * (px - X) + nd.ox;
                    double v = nd.sy * (py - Y) + nd.oy;
                    double p, dpdv, dpdu;
                    bicubic(nd.data.data(), nd.ny, nd.nx, v, u, nd.fill, p, dpdv, dpdu);
                    s = p;
                    dsdY = -nd.sy * dpdv;
                    dsdX = -nd.sx * dpdu;
                } else {
                    for (int k = 0; k < 4; ++k) {
                        if (cr[k].idx < 0) continue;
                        if (cr[k].w == 0.0 && cr[k].dwdy == 0.0 && cr[k].dwdx == 0.0) continue;
                        const Node& nd = psf.nodes[cr[k].idx];
                        double pv, pdv, pdu;
                        corner_point(nd, Y, X, py, px, pv, pdv, pdu);
                        s += cr[k].w * pv;
                        dsdY += cr[k].dwdy * pv - cr[k].w * nd.sy * pdv;
                        dsdX += cr[k].dwdx * pv - cr[k].w * nd.sx * pdu;
                    }
                }
                double r = (flux * s + bkg) - c.pix[i + j * c.ny];
                double w = wts[i + j * c.ny];
                double wr = w * r;
                cost = wr * r + cost;
                double gv[4] = {flux * dsdY, flux * dsdX, s, 1.0};
                for (int q = 0; q < 4; ++q) {
                    bf[q] = wr * gv[q] + bf[q];
                    for (int pq = 0; pq <= q; ++pq) Af[pq + q * 4] = (w * gv[pq]) * gv[q] + Af[pq + q * 4];
                }
            }
    }
    for (int jq = 0; jq < nf; ++jq) {
        b[jq] = bf[fidx[jq]];
        for (int iq = 0; iq < nf; ++iq) {
            int a = fidx[iq], bb = fidx[jq];
            int lo = std::min(a, bb), hi = std::max(a, bb);
            A[iq + jq * nf] = Af[lo + hi * np];
        }
    }
    return cost;
}

// cholesky!(Symmetric(A)) \ b.  Returns false on a non-positive pivot.
bool chol_solve(const double* A, int n, const double* b, double* x) {
    double U[25] = {0};
    for (int j = 0; j < n; ++j)
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
    double y[5];
    for (int i = 0; i < n; ++i) {
        double s = b[i];
        for (int k = 0; k < i; ++k) s -= U[k + i * n] * y[k];
        y[i] = s / U[i + i * n];
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = y[i];
        for (int k = i + 1; k < n; ++k) s -= U[i + k * n] * x[k];
        x[i] = s / U[i + i * n];
    }
    return true;
}

int fit_one(const Psf& psf, const cpb_lm_params* P, const double* pix, const double* inv_var, int32_t ny, int32_t nx,
            int32_t y1, int32_t x1, const double* init, double* out_params, double* cov_out, double* cost_out,
            double* cost_init_out, double* chisq_out, double* lambda_out, uint8_t* flags_out, int32_t* iters_out,
            char* errbuf, int errlen);

}  // namespace

extern "C" {

// One fit_star call.  init/out_params: np model parameters.  cov: nf*nf (nullable).
// Returns 0, or CPB_ERR_ARGUMENT with errbuf set.
int orc_fit_star(const cpb_psf_desc* desc, const cpb_lm_params* P, const double* pix, const double* inv_var,
                 int32_t ny, int32_t nx, int32_t y1, int32_t x1, const double* init, double* out_params,
                 double* cov_out, double* cost_out, double* cost_init_out, double* chisq_out, double* lambda_out,
                 uint8_t* flags_out /* converged, x, f, g */, int32_t* iters_out, char* errbuf, int errlen) {
    Psf psf;
    {
        std::string e = load_psf(desc, psf);
        if (!e.empty()) {
            if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", e.c_str());
            return CPB_ERR_ARGUMENT;
        }
    }
    return fit_one(psf, P, pix, inv_var, ny, nx, y1, x1, init, out_params, cov_out, cost_out, cost_init_out,
                   chisq_out, lambda_out, flags_out, iters_out, errbuf, errlen);
}

// n_cut fit_star calls on one loaded PSF, cutout c at pix[offsets[c]..] (column-major
// ny[c] x nx[c]); the cutouts are independent, so they are spread over `threads`
// host threads (<= 0: all hardware threads).  Per-cutout outputs as orc_fit_star's, packed:
// params n*np, cov n*nf*nf (nullable), scal n*4 (cost, cost_init, chisq, lambda),
// flags n*4, iters n, status n (0 or CPB_ERR_ARGUMENT).  Returns the threads used.
int orc_fit_star_batch(const cpb_psf_desc* desc, const cpb_lm_params* P, int64_t n_cut, const int64_t* offsets,
                       const int32_t* ny, const int32_t* nx, const int32_t* y1, const int32_t* x1, const double* pix,
                       const double* inv_var, const double* init, int np, int nf, double* params, double* cov,
                       double* scal, uint8_t* flags, int32_t* iters, int32_t* status, int threads) {
    Psf psf;
    if (!load_psf(desc, psf).empty()) return -1;
    const int used = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<int64_t> next{0};
    auto work = [&]() {
        for (;;) {
            const int64_t c0 = next.fetch_add(16);
            if (c0 >= n_cut) return;
            for (int64_t c = c0; c < std::min(n_cut, c0 + 16); ++c)
                status[c] = fit_one(psf, P, pix + offsets[c], inv_var ? inv_var + offsets[c] : nullptr, ny[c], nx[c],
                                    y1[c], x1[c], init + c * np, params + c * np, cov ? cov + c * nf * nf : nullptr,
                                    &scal[c * 4], &scal[c * 4 + 1], &scal[c * 4 + 2], &scal[c * 4 + 3], flags + c * 4,
                                    iters + c, nullptr, 0);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < used; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    return used;
}

}  // extern "C"

namespace {

int fit_one(const Psf& psf, const cpb_lm_params* P, const double* pix, const double* inv_var, int32_t ny, int32_t nx,
            int32_t y1, int32_t x1, const double* init, double* out_params, double* cov_out, double* cost_out,
            double* cost_init_out, double* chisq_out, double* lambda_out, uint8_t* flags_out, int32_t* iters_out,
            char* errbuf, int errlen) {
    auto fail = [&](const std::string& m) {
        if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", m.c_str());
        return CPB_ERR_ARGUMENT;
    };
    const bool gauss = psf.kind == CPB_PSF_CIRCULAR_GAUSSIAN;
    const int np = gauss ? 5 : 4;
    // free set in getproperties order
    const int bits_g[5] = {CPB_FREE_Y, CPB_FREE_X, CPB_FREE_FWHM, CPB_FREE_FLUX, CPB_FREE_BKG};
    const int bits_i[4] = {CPB_FREE_Y, CPB_FREE_X, CPB_FREE_FLUX, CPB_FREE_BKG};
    int fidx[5], nf = 0;
    for (int q = 0; q < np; ++q)
        if (P->free_mask & (gauss ? bits_g[q] : bits_i[q])) fidx[nf++] = q;
    if (nf == 0) return fail("all model parameters are fixed; nothing to fit");
    double full[5];
    for (int q = 0; q < np; ++q) full[q] = init[q];
    // fixed values override (model_from_vector merges `fixed`)
    double fixv_g[5] = {P->fixed_y, P->fixed_x, P->fixed_fwhm, P->fixed_flux, P->fixed_bkg};
    double fixv_i[4] = {P->fixed_y, P->fixed_x, P->fixed_flux, P->fixed_bkg};
    for (int q = 0; q < np; ++q)
        if (!(P->free_mask & (gauss ? bits_g[q] : bits_i[q]))) full[q] = gauss ? fixv_g[q] : fixv_i[q];
    const int64_t nobs = (int64_t)ny * nx;
    std::vector<double> wts(nobs, 1.0);
    if (inv_var) {
        int64_t nvalid = 0;
        for (int64_t q = 0; q < nobs; ++q) {
            double w = inv_var[q];
            if (std::isfinite(w) && w > 0) {
                wts[q] = w;
                ++nvalid;
            } else {
                wts[q] = 0.0;
            }
        }
        if (!(nvalid > nf))
            return fail("too few valid inv_var pixels (" + std::to_string(nvalid) + ") for " + std::to_string(nf) +
                        " free parameters");
    }
    const int64_t dof = nobs - nf;
    if (!(dof > 0))
        return fail("degrees of freedom must be positive; too many free parameters (" + std::to_string(nf) +
                    ") for the number of observations (" + std::to_string(nobs) + ")");
    Cutout c{pix, inv_var, ny, nx, y1, x1};
    double x[5], xc[5], A[25], b[5], Ac[25], bc[5], Ad[25], d[5], D[5];
    for (int q = 0; q < nf; ++q) x[q] = full[fidx[q]];
    auto set_full = [&](const double* xv, double* fv) {
        for (int q = 0; q < np; ++q) fv[q] = full[q];
        for (int q = 0; q < nf; ++q) fv[fidx[q]] = xv[q];
    };
    double fv[5];
    set_full(x, fv);
    double cost = accum(psf, c, wts, fv, fidx, nf, A, b);
    const double cost_init = cost;
    const double d_floor = 1.0e-6;
    for (int q = 0; q < nf; ++q) D[q] = std::sqrt(std::max(A[q + q * nf], d_floor));
    double lam = P->lambda_init;
    bool xconv = false, fconv = false, gconv = false, conv = false;
    int iter = 0;
    while (iter < P->max_iter) {
        ++iter;
        double gcos = 0;
        for (int q = 0; q < nf; ++q) gcos = std::max(gcos, std::fabs(b[q]) / (std::sqrt(A[q + q * nf] * cost) + kEps));
        if (gcos <= P->g_tol) {
            gconv = true;
            conv = true;
            break;
        }
        std::memcpy(Ad, A, sizeof(double) * nf * nf);
        if (P->damping == CPB_DAMP_MARQUARDT) {
            for (int q = 0; q < nf; ++q) Ad[q + q * nf] += lam * std::max(Ad[q + q * nf], P->min_diagonal);
        } else if (P->damping == CPB_DAMP_LEVENBERG) {
            for (int q = 0; q < nf; ++q) Ad[q + q * nf] += lam;
        }
        if (!chol_solve(Ad, nf, b, d)) {
            lam = std::min(lam * P->lambda_up, P->lambda_max);
            continue;
        }
        for (int q = 0; q < nf; ++q) d[q] *= -1;
        double db = 0, dAd = 0;
        for (int q = 0; q < nf; ++q) db += d[q] * b[q];
        for (int q = 0; q < nf; ++q)
            for (int r = 0; r < nf; ++r) dAd += d[q] * A[q + r * nf] * d[r];
        double prered = -2 * db - dAd;
        for (int q = 0; q < nf; ++q) xc[q] = x[q] + d[q];
        set_full(xc, fv);
        double cost_c = accum(psf, c, wts, fv, fidx, nf, Ac, bc);
        bool accepted = cost_c < cost;
        double dcost = cost - cost_c;
        double ratio = prered > 0 ? dcost / prered : 0.0;
        fconv = std::fabs(dcost) <= P->f_tol * (std::fabs(cost) + P->f_tol) &&
                prered <= P->f_tol * (std::fabs(cost) + P->f_tol) && 0.5 * ratio <= 1;
        double nd = 0, nx_ = 0;
        for (int q = 0; q < nf; ++q) {
            nd += (D[q] * d[q]) * (D[q] * d[q]);
            nx_ += (D[q] * x[q]) * (D[q] * x[q]);
        }
        xconv = std::sqrt(nd) <= P->x_tol * (std::sqrt(nx_) + P->x_tol) && (accepted || fconv);
        if (accepted) {
            cost = cost_c;
            lam = std::max(lam / P->lambda_down, P->lambda_min);
            std::memcpy(x, xc, sizeof(double) * nf);
            std::memcpy(A, Ac, sizeof(double) * nf * nf);
            std::memcpy(b, bc, sizeof(double) * nf);
            for (int q = 0; q < nf; ++q) D[q] = std::max(D[q], std::sqrt(A[q + q * nf]));
            if (xconv || fconv) {
                conv = true;
                break;
            }
        } else {
            if (xconv || fconv) {
                conv = true;
                break;
            }
            lam = std::min(lam * P->lambda_up, P->lambda_max);
        }
    }
    const bool reweighted = P->covariance == CPB_COV_REWEIGHTED || (P->covariance == CPB_COV_AUTO && !inv_var);
    std::vector<double> Av(A, A + nf * nf), cov;
    covariance(Av, nf, reweighted, cost, (double)dof, cov);
    set_full(x, fv);
    for (int q = 0; q < np; ++q) out_params[q] = fv[q];
    if (cov_out) std::memcpy(cov_out, cov.data(), sizeof(double) * nf * nf);
    *cost_out = cost;
    *cost_init_out = cost_init;
    *chisq_out = cost / (double)dof;
    *lambda_out = lam;
    flags_out[0] = conv;
    flags_out[1] = xconv;
    flags_out[2] = fconv;
    flags_out[3] = gconv;
    *iters_out = iter;
    return 0;
}

}  // namespace

namespace orc {
// fit_one for the other oracle files (fit_all_stars calls fit_star per star).
int fit_star_one(const Psf& psf, const cpb_lm_params* P, const double* pix, const double* inv_var, int32_t ny,
                 int32_t nx, int32_t y1, int32_t x1, const double* init, double* out_params, double* cov_out,
                 double* cost_out, double* cost_init_out, double* chisq_out, double* lambda_out, uint8_t* flags_out,
                 int32_t* iters_out) {
    return fit_one(psf, P, pix, inv_var, ny, nx, y1, x1, init, out_params, cov_out, cost_out, cost_init_out,
                   chisq_out, lambda_out, flags_out, iters_out, nullptr, 0);
}
}  // namespace orc
