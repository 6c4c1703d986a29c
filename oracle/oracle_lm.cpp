// oracle_lm.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// FP64 restatement of CrowdPhot.PSF.fit_star for the three supported PSF kinds
// and of the LM driver lm_irls, IRLS reweighting included:
//   _prepare_fit_star_inputs   src/psf/psf_fitting.jl:36-101
//   fit_star(CircularGaussianPSF) + _accum_circular_gaussian!  :314-451
//   fit_star(ImagePSF) + _accum_image_psf!                    :1086-1173
//   fit_star(GriddedPSFModel{ImagePSF}) + _accum_gridded_imagepsf!  :1177-1517
//   lm_irls, damp!, covariance!  src/levenberg_marquardt.jl:64-99, 361-680
//   MADScale / FixedScale / MScale, TukeyLoss, weight  :105-355 (HuberLoss and
//   L2DistLoss as LossFunctions.jl defines their derivatives)
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
             int nf, double* A, double* b, double* res) {
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
                res[i + j * c.ny] = r;
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
                res[i + j * c.ny] = r;
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
            char* errbuf, int errlen, double* sigma_out = nullptr);

const double kNaN = std::numeric_limits<double>::quiet_NaN();

// Statistics.median (NaN if any value is NaN; middle(a, b) = a/2 + b/2).
double median_of(std::vector<double> v) {
    for (double x : v)
        if (std::isnan(x)) return kNaN;
    std::sort(v.begin(), v.end());
    const size_t n = v.size();
    if (n == 0) return kNaN;
    return (n & 1) ? v[(n - 1) / 2] : v[n / 2 - 1] / 2 + v[n / 2] / 2;
}

// estimate_scale (:137-140 MADScale, :159 FixedScale, :201-224 MScale)
double estimate_scale(int kind, const cpb_lm_params* P, double fixed_sigma, const std::vector<double>& r) {
    if (kind == CPB_SCALE_FIXED) return fixed_sigma;
    const double med = median_of(r);
    std::vector<double> dev(r.size());
    for (size_t k = 0; k < r.size(); ++k) dev[k] = std::fabs(r[k] - med);
    const double mad = 1.4826 * median_of(dev);
    if (kind != CPB_SCALE_MSCALE) return mad;
    double sg = std::isnan(mad) ? mad : std::max(mad, kEps);
    const double n = (double)r.size();
    for (int it = 0; it < P->mscale_max_iter; ++it) {
        const double cap = 9 * (sg * sg);
        double chi = 0;
        for (double ri : r) {
            const double r2 = ri * ri;
            chi += r2 < cap ? r2 : cap;
        }
        const double sn = std::sqrt(chi / (n * P->mscale_delta));
        if (std::fabs(sn - sg) <= P->mscale_tol * std::max(sg, P->mscale_tol)) {
            sg = sn;
            break;
        }
        sg = sn;
    }
    return sg;
}

// weight(loss, r) = psi(r) / (r psi'(0)) (:337-345) for L2DistLoss (psi = 2r),
// HuberLoss(d) (psi = r inside d, d sign(r) beyond), TukeyLoss(c) (:289-313) and
// LossFunctions.jl's LogitDistLoss (loss -log(4 e^r / (1 + e^r)^2): psi = tanh(r/2),
// psi'(0) = 1/2; a third-party loss the reference's generic weight accepts).
double irls_weight(int loss, double c, double r) {
    if (std::fabs(r) < kEps * 10) return 1.0;
    if (loss == CPB_LOSS_L2DIST) return (2 * r) / (r * 2.0);
    if (loss == CPB_LOSS_HUBER) {
        const double psi = std::fabs(r) <= c ? r : c * (r > 0 ? 1.0 : -1.0);
        const double psi0 = 0.0 <= c ? 1.0 : 0.0;
        return psi / (r * psi0);
    }
    if (loss == CPB_LOSS_LOGITDIST) return std::tanh(r / 2) / (r * 0.5);
    double psi = 0.0;
    if (std::fabs(r) <= c) {
        const double rc2 = (r / c) * (r / c);
        psi = r * ((1 - rc2) * (1 - rc2));
    }
    return psi / (r * 1.0);
}

struct LMRun {
    double x[5], A[25];
    double cost = 0, cost_init = 0, lam = 0, sigma_final = kNaN, chisq = 0;
    bool conv = false, xconv = false, fconv = false, gconv = false;
    int iter = 0;
    bool reweighted = false;
};

// lm_irls (:431-680) on a generic problem: accum(x, w, A, b, res) fills the
// normal equations, the residuals and returns the cost, w being the current
// per-observation weights (nullptr: unit weights).  base: the fixed input
// weights (nullptr: none).
template <class Acc>
LMRun lm_irls_run(Acc&& accum, int n, int64_t nobs, const double* x0, const std::vector<double>* base,
                  const cpb_lm_params* P) {
    LMRun R;
    const bool do_irls = P->reweight != CPB_LOSS_NONE;
    const int64_t dof = nobs - n;
    double fixed_sigma = P->scale_value;
    int scale_kind = P->scale_estimator;
    if (scale_kind == CPB_SCALE_AUTO) {
        if (base) {
            double sm = 0;
            for (double w : *base) sm += w;
            fixed_sigma = std::sqrt(1.0 / (sm / (double)nobs));
            scale_kind = CPB_SCALE_FIXED;
        } else {
            scale_kind = CPB_SCALE_MAD;
        }
    }
    // per-thread buffers (the batch entry fits many cutouts on each host thread)
    thread_local std::vector<double> weights, res;
    const std::vector<double>* wp = base;
    if (do_irls) {
        if (base)
            weights = *base;
        else
            weights.assign(nobs, 1.0);
        wp = &weights;
    }
    res.resize(nobs);
    double x[5], xc[5], A[25], b[5], Ac[25], bc[5], Ad[25], d[5], D[5];
    std::copy(x0, x0 + n, x);
    double cost = accum(x, wp, A, b, res.data());
    R.cost_init = cost;
    const double d_floor = 1.0e-6;
    for (int q = 0; q < n; ++q) D[q] = std::sqrt(std::max(A[q + q * n], d_floor));
    double lam = P->lambda_init;
    while (R.iter < P->max_iter) {
        ++R.iter;
        double gcos = 0;
        for (int q = 0; q < n; ++q) gcos = std::max(gcos, std::fabs(b[q]) / (std::sqrt(A[q + q * n] * cost) + kEps));
        if (gcos <= P->g_tol) {
            R.gconv = R.conv = true;
            break;
        }
        std::copy(A, A + n * n, Ad);
        if (P->damping == CPB_DAMP_MARQUARDT) {
            for (int q = 0; q < n; ++q) Ad[q + q * n] += lam * std::max(Ad[q + q * n], P->min_diagonal);
        } else if (P->damping == CPB_DAMP_LEVENBERG) {
            for (int q = 0; q < n; ++q) Ad[q + q * n] += lam;
        }
        if (!chol_solve(Ad, n, b, d)) {
            lam = std::min(lam * P->lambda_up, P->lambda_max);
            continue;
        }
        for (int q = 0; q < n; ++q) d[q] *= -1;
        double db = 0, dAd = 0;
        for (int q = 0; q < n; ++q) db += d[q] * b[q];
        for (int q = 0; q < n; ++q)
            for (int r = 0; r < n; ++r) dAd += d[q] * A[q + r * n] * d[r];
        const double prered = -2 * db - dAd;
        for (int q = 0; q < n; ++q) xc[q] = x[q] + d[q];
        const double cost_c = accum(xc, wp, Ac, bc, res.data());
        const bool accepted = cost_c < cost;
        const double dcost = cost - cost_c;
        const double ratio = prered > 0 ? dcost / prered : 0.0;
        R.fconv = std::fabs(dcost) <= P->f_tol * (std::fabs(cost) + P->f_tol) &&
                  prered <= P->f_tol * (std::fabs(cost) + P->f_tol) && 0.5 * ratio <= 1;
        double nd = 0, nxv = 0;
        for (int q = 0; q < n; ++q) {
            nd += (D[q] * d[q]) * (D[q] * d[q]);
            nxv += (D[q] * x[q]) * (D[q] * x[q]);
        }
        R.xconv = std::sqrt(nd) <= P->x_tol * (std::sqrt(nxv) + P->x_tol) && (accepted || R.fconv);
        if (accepted) {
            cost = cost_c;
            lam = std::max(lam / P->lambda_down, P->lambda_min);
            std::copy(xc, xc + n, x);
            std::copy(Ac, Ac + n * n, A);
            std::copy(bc, bc + n, b);
            for (int q = 0; q < n; ++q) D[q] = std::max(D[q], std::sqrt(A[q + q * n]));
            if (R.xconv || R.fconv) {
                R.conv = true;
                break;
            }
            if (do_irls) {  // :611-645
                R.sigma_final = estimate_scale(scale_kind, P, fixed_sigma, res);
                if (R.sigma_final > kEps) {
                    double dw2 = 0, wo2 = 0, wn2 = 0;
                    for (int64_t k = 0; k < nobs; ++k) {
                        const double old_w = weights[k];
                        const double base_w = base ? (*base)[k] : 1.0;
                        const double new_w = base_w * irls_weight(P->reweight, P->loss_param, res[k] / R.sigma_final);
                        const double dw = new_w - old_w;
                        dw2 = std::fma(dw, dw, dw2);
                        wo2 = std::fma(old_w, old_w, wo2);
                        wn2 = std::fma(new_w, new_w, wn2);
                        weights[k] = new_w;
                    }
                    cost = accum(x, wp, A, b, res.data());
                    const double wchange = std::sqrt(dw2) / std::max({std::sqrt(wo2), std::sqrt(wn2), kEps});
                    if (wchange >= P->weight_reset_tol) {
                        lam = P->lambda_init;
                        for (int q = 0; q < n; ++q) D[q] = std::sqrt(std::max(A[q + q * n], d_floor));
                    }
                }
            }
        } else {
            if (R.xconv || R.fconv) {
                R.conv = true;
                break;
            }
            lam = std::min(lam * P->lambda_up, P->lambda_max);
        }
    }
    R.reweighted = P->covariance == CPB_COV_REWEIGHTED || (P->covariance == CPB_COV_AUTO && (!base || do_irls));
    const double s2 = cost / (double)dof;
    R.chisq = (!base && do_irls && !std::isnan(R.sigma_final) && R.sigma_final > kEps)
                  ? s2 / (R.sigma_final * R.sigma_final)
                  : s2;
    std::copy(x, x + n, R.x);
    std::copy(A, A + n * n, R.A);
    R.cost = cost;
    R.lam = lam;
    return R;
}

}  // namespace

extern "C" {

// One fit_star call.  init/out_params: np model parameters.  cov: nf*nf (nullable).
// Returns 0, or CPB_ERR_ARGUMENT with errbuf set.
int orc_fit_star(const cpb_psf_desc* desc, const cpb_lm_params* P, const double* pix, const double* inv_var,
                 int32_t ny, int32_t nx, int32_t y1, int32_t x1, const double* init, double* out_params,
                 double* cov_out, double* cost_out, double* cost_init_out, double* chisq_out, double* lambda_out,
                 uint8_t* flags_out /* converged, x, f, g */, int32_t* iters_out, char* errbuf, int errlen,
                 double* sigma_out /* nullable: LMResult.sigma_final */) {
    Psf psf;
    {
        std::string e = load_psf(desc, psf);
        if (!e.empty()) {
            if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", e.c_str());
            return CPB_ERR_ARGUMENT;
        }
    }
    return fit_one(psf, P, pix, inv_var, ny, nx, y1, x1, init, out_params, cov_out, cost_out, cost_init_out,
                   chisq_out, lambda_out, flags_out, iters_out, errbuf, errlen, sigma_out);
}

// n_cut fit_star calls on one loaded PSF, cutout c at pix[offsets[c]..] (column-major
// ny[c] x nx[c]); the cutouts are independent, so they are spread over `threads`
// host threads (<= 0: all hardware threads).  Per-cutout outputs as orc_fit_star's, packed:
// params n*np, cov n*nf*nf (nullable), scal n*4 (cost, cost_init, chisq, lambda),
// flags n*4, iters n, status n (0 or CPB_ERR_ARGUMENT).  Returns the threads used.
int orc_fit_star_batch(const cpb_psf_desc* desc, const cpb_lm_params* P, int64_t n_cut, const int64_t* offsets,
                       const int32_t* ny, const int32_t* nx, const int32_t* y1, const int32_t* x1, const double* pix,
                       const double* inv_var, const double* init, int np, int nf, double* params, double* cov,
                       double* scal, uint8_t* flags, int32_t* iters, int32_t* status, int threads,
                       double* sigma /* nullable, n */) {
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
                                    iters + c, nullptr, 0, sigma ? sigma + c : nullptr);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < used; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    return used;
}

// lm_irls on the straight-line problem of the reference's weight-reset test
// (test/psf/psf_fitting_tests.jl:176-233): y = x[0] * xs + x[1], unit base
// weights absent.  Returns 0 and writes the minimiser, lambda_final,
// sigma_final and the iteration count.
int orc_lm_irls_line(const double* xs, const double* ys, int n, const cpb_lm_params* P, const double* x0,
                     double* x_out, double* lambda_out, double* sigma_out, int32_t* iters_out) {
    auto acc = [&](const double* x, const std::vector<double>* w, double* A, double* b, double* res) {
        for (int k = 0; k < 4; ++k) A[k] = 0;
        b[0] = b[1] = 0;
        double cost = 0;
        for (int k = 0; k < n; ++k) {
            const double wk = w ? (*w)[k] : 1.0;
            const double r = x[0] * xs[k] + x[1] - ys[k];
            res[k] = r;
            const double wr = wk * r;
            cost = std::fma(wr, r, cost);
            A[0] = std::fma(wk * xs[k], xs[k], A[0]);
            A[1] = std::fma(wk, xs[k], A[1]);
            A[2] = std::fma(wk * xs[k], 1.0, A[2]);
            A[3] += wk;
            b[0] = std::fma(wr, xs[k], b[0]);
            b[1] += wr;
        }
        return cost;
    };
    if (n - 2 <= 0) return CPB_ERR_ARGUMENT;
    LMRun R = lm_irls_run(acc, 2, n, x0, nullptr, P);
    x_out[0] = R.x[0];
    x_out[1] = R.x[1];
    *lambda_out = R.lam;
    *sigma_out = R.sigma_final;
    *iters_out = R.iter;
    return 0;
}

// estimate_scale(kind, r) for MADScale / FixedScale(sigma) / MScale(P's delta, tol, max_iter).
double orc_estimate_scale(int kind, const cpb_lm_params* P, double sigma, const double* r, int64_t n) {
    return estimate_scale(kind, P, sigma, std::vector<double>(r, r + n));
}

// weight(loss, r) for CPB_LOSS_L2DIST / _HUBER (d = c) / _TUKEY (c).
double orc_irls_weight(int loss, double c, double r) { return irls_weight(loss, c, r); }

}  // extern "C"

namespace {

int fit_one(const Psf& psf, const cpb_lm_params* P, const double* pix, const double* inv_var, int32_t ny, int32_t nx,
            int32_t y1, int32_t x1, const double* init, double* out_params, double* cov_out, double* cost_out,
            double* cost_init_out, double* chisq_out, double* lambda_out, uint8_t* flags_out, int32_t* iters_out,
            char* errbuf, int errlen, double* sigma_out) {
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
    if (P->reweight != CPB_LOSS_NONE && !(P->weight_reset_tol >= 0))
        return fail("`weight_reset_tol` must be non-negative");
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
    double x0[5];
    for (int q = 0; q < nf; ++q) x0[q] = full[fidx[q]];
    auto set_full = [&](const double* xv, double* fv) {
        for (int q = 0; q < np; ++q) fv[q] = full[q];
        for (int q = 0; q < nf; ++q) fv[fidx[q]] = xv[q];
    };
    auto acc = [&](const double* xv, const std::vector<double>* w, double* A, double* b, double* res) {
        double fv[5];
        set_full(xv, fv);
        return accum(psf, c, w ? *w : wts, fv, fidx, nf, A, b, res);  // wts: all 1 without inv_var
    };
    LMRun R = lm_irls_run(acc, nf, nobs, x0, inv_var ? &wts : nullptr, P);
    std::vector<double> cov, Av(R.A, R.A + nf * nf);
    covariance(Av, nf, R.reweighted, R.cost, (double)dof, cov);
    double fv[5];
    set_full(R.x, fv);
    for (int q = 0; q < np; ++q) out_params[q] = fv[q];
    if (cov_out) std::memcpy(cov_out, cov.data(), sizeof(double) * nf * nf);
    *cost_out = R.cost;
    *cost_init_out = R.cost_init;
    *chisq_out = R.chisq;
    *lambda_out = R.lam;
    flags_out[0] = R.conv;
    flags_out[1] = R.xconv;
    flags_out[2] = R.fconv;
    flags_out[3] = R.gconv;
    *iters_out = R.iter;
    if (sigma_out) *sigma_out = R.sigma_final;
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
