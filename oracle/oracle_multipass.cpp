// oracle_multipass.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// Single-threaded FP64 restatement of CrowdPhot.fit_all_stars
// (src/photometry/psf_photometry_single.jl:267-469): brightness-ordered passes,
// one star at a time, each star added back (passes 2+), fitted with fit_star
// on its +-fit_rad box of the running residual and subtracted again; per-star
// diagnostics on the final pass (psf_photometry_diagnostics.jl:154-231), with
// spread_model from the band-limited exponential-disk reference kernel
// (oracle_spread.cpp; :322-326 of the reference).  Stars with non-finite positions are
// marked invalid (Julia would raise InexactError from floor(Int, NaN)).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <vector>

#include "oracle_psf.hpp"

namespace orc {
int fit_star_one(const Psf& psf, const cpb_lm_params* P, const double* pix, const double* inv_var, int32_t ny,
                 int32_t nx, int32_t y1, int32_t x1, const double* init, double* out_params, double* cov_out,
                 double* cost_out, double* cost_init_out, double* chisq_out, double* lambda_out, uint8_t* flags_out,
                 int32_t* iters_out);
}

using namespace orc;

namespace {

double ld(const void* p, int et, int64_t i) {
    return et == CPB_F64 ? ((const double*)p)[i] : (double)((const float*)p)[i];
}

StarP star_of(const double* pr, bool gauss) {
    if (gauss) return StarP{pr[0], pr[1], pr[3], pr[4], pr[2]};
    return StarP{pr[0], pr[1], pr[2], pr[3], 0.0};
}

}  // namespace

extern "C" int orc_fit_all_stars(const cpb_psf_desc* desc, const cpb_lm_params* P, double fit_rad, int n_passes,
                                 double spread_model_fwhm, const void* image, int32_t eltype, int64_t ny, int64_t nx, const void* inv_var,
                                 int64_t n, const double* init, cpb_multipass_result* out, char* errbuf, int errlen) {
    auto fail = [&](const std::string& m) {
        if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", m.c_str());
        return CPB_ERR_ARGUMENT;
    };
    if (!(n_passes > 0)) return fail("n_passes must be positive, got " + std::to_string(n_passes));
    Psf psf;
    {
        std::string e = load_psf(desc, psf);
        if (!e.empty()) return fail(e);
    }
    const bool gauss = psf.kind == CPB_PSF_CIRCULAR_GAUSSIAN;
    const int np = gauss ? 5 : 4;
    const int rf = gauss ? 3 : 2;
    const int bits_g[5] = {CPB_FREE_Y, CPB_FREE_X, CPB_FREE_FWHM, CPB_FREE_FLUX, CPB_FREE_BKG};
    const int bits_i[4] = {CPB_FREE_Y, CPB_FREE_X, CPB_FREE_FLUX, CPB_FREE_BKG};
    std::vector<int> free_idx;
    for (int q = 0; q < np; ++q)
        if (P->free_mask & (gauss ? bits_g[q] : bits_i[q])) free_idx.push_back(q);
    if (free_idx.empty()) return fail("all model parameters are fixed; nothing to fit");
    const int nf = (int)free_idx.size();
    const double NaN = std::numeric_limits<double>::quiet_NaN();
    const int64_t npix = ny * nx;

    std::vector<double> prm(init, init + n * np), err(n * np, NaN);
    for (int64_t s = 0; s < n; ++s)
        for (int q = 0; q < np; ++q)
            if (std::find(free_idx.begin(), free_idx.end(), q) == free_idx.end()) err[s * np + q] = 0.0;
    std::vector<uint8_t> valid(n, 1), conv(n, 0);
    std::vector<double> chisq(n, 0.0), diag(n * 6, NaN);
    // spread_model reference disk from the first catalogue star (:322-326)
    std::vector<double> spread_K;
    int spread_half = 0;
    const bool have_spread =
        n > 0 && spread_kernel(psf, spread_model_fwhm, init[0], init[1], fit_rad, spread_K, spread_half);
    std::vector<int32_t> niter(n, 0);
    std::vector<double> resid(npix), ivd(inv_var ? npix : 0);
    for (int64_t q = 0; q < npix; ++q) resid[q] = ld(image, eltype, q);
    for (int64_t q = 0; q < (int64_t)ivd.size(); ++q) ivd[q] = ld(inv_var, eltype, q);
    int n_failed = 0;
    auto addsub = [&](const double* pr, int ylo, int yhi, int xlo, int xhi, double sign) {
        StarP sp = star_of(pr, gauss);
        for (int j = xlo; j <= xhi; ++j)
            for (int i = ylo; i <= yhi; ++i) {
                int64_t q = (i - 1) + (int64_t)(j - 1) * ny;
                resid[q] = resid[q] + sign * evaluate(psf, sp, (double)i, (double)j);
            }
    };

    for (int pass = 1; pass <= n_passes; ++pass) {
        std::vector<int64_t> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(),
                         [&](int64_t a, int64_t b) { return prm[a * np + rf] > prm[b * np + rf]; });
        for (int64_t s : order) {
            if (!valid[s]) continue;
            const double y = prm[s * np], x = prm[s * np + 1];
            if (!(std::isfinite(y) && std::isfinite(x))) {
                valid[s] = 0;
                continue;
            }
            // +-fit_rad box clamped to the image (:343-348, utilities.jl:259-264)
            const int ylo = (int)std::max(std::floor(y - fit_rad), 1.0), yhi = (int)std::min(std::ceil(y + fit_rad), (double)ny);
            const int xlo = (int)std::max(std::floor(x - fit_rad), 1.0), xhi = (int)std::min(std::ceil(x + fit_rad), (double)nx);
            const int by = std::max(yhi - ylo + 1, 0), bx = std::max(xhi - xlo + 1, 0);
            if ((int64_t)by * bx < 3) {
                valid[s] = 0;
                continue;
            }
            std::vector<double> m(prm.begin() + s * np, prm.begin() + (s + 1) * np);
            if (pass > 1) addsub(m.data(), ylo, yhi, xlo, xhi, 1.0);
            std::vector<double> cut((size_t)by * bx), cutiv(inv_var ? (size_t)by * bx : 0);
            for (int j = 0; j < bx; ++j)
                for (int i = 0; i < by; ++i) {
                    int64_t q = (ylo - 1 + i) + (int64_t)(xlo - 1 + j) * ny;
                    cut[i + (size_t)j * by] = resid[q];
                    if (inv_var) cutiv[i + (size_t)j * by] = ivd[q];
                }
            std::vector<double> best(np), cov(nf * nf);
            double cost, cost0, chi, lam;
            uint8_t flags[4];
            int32_t iters = 0;
            int rc = fit_star_one(psf, P, cut.data(), inv_var ? cutiv.data() : nullptr, by, bx, ylo, xlo, m.data(),
                                  best.data(), cov.data(), &cost, &cost0, &chi, &lam, flags, &iters);
            if (rc != 0) {  // fit_star threw (:391-401): undo the add-back
                if (pass > 1) addsub(m.data(), ylo, yhi, xlo, xhi, -1.0);
                valid[s] = 0;
                n_failed += 1;
                continue;
            }
            std::copy(best.begin(), best.end(), prm.begin() + s * np);
            for (int a = 0; a < nf; ++a) err[s * np + free_idx[a]] = std::sqrt(std::max(0.0, cov[a + a * nf]));
            conv[s] = flags[0];
            chisq[s] = chi;
            niter[s] += iters;
            addsub(best.data(), ylo, yhi, xlo, xhi, -1.0);
            if (pass == n_passes) {  // _star_diagnostics!
                StarP sp = star_of(best.data(), gauss);
                double* d = &diag[s * 6];
                if (sp.flux > 0) {
                    std::vector<double> ms((size_t)by * bx), gs;
                    for (int j = 0; j < bx; ++j)
                        for (int i = 0; i < by; ++i)
                            ms[i + (size_t)j * by] = evaluate(psf, sp, (double)(ylo + i), (double)(xlo + j));
                    if (have_spread) {
                        gs.resize(ms.size());
                        correlate_zero(ms.data(), by, bx, spread_K, spread_half, gs.data());
                    }
                    double inv_flux = 1.0 / sp.flux, qv = 0, ncl = 0, ndi = 0, den = 0, ss = 0, ss2 = 0;
                    double Sp = 0, Sq = 0, Sp0 = 0, Sq0 = 0, SqG = 0;
                    int64_t ng = 0;
                    for (int j = xlo; j <= xhi; ++j)
                        for (int i = ylo; i <= yhi; ++i) {
                            int64_t q = (i - 1) + (int64_t)(j - 1) * ny;
                            const size_t e = (size_t)(i - ylo) + (size_t)(j - xlo) * by;
                            double mv = ms[e];
                            double wp = inv_var ? ivd[q] : 1.0;
                            if (std::isfinite(wp) && wp > 0) {
                                qv += std::fabs(resid[q]);
                                double Pp = (mv - sp.bkg) * inv_flux, wP = wp * Pp;
                                double p_i = resid[q] + mv - sp.bkg;
                                ncl += wP * p_i;
                                ndi += wP * (ld(image, eltype, q) - sp.bkg);
                                den += wP * Pp;
                                if (have_spread) {
                                    double g_i = (gs[e] - sp.bkg) * inv_flux;
                                    Sp += wP * p_i;
                                    Sq += wp * g_i * p_i;
                                    Sp0 += wP * Pp;
                                    Sq0 += wp * Pp * g_i;
                                    SqG += wp * g_i * g_i;
                                }
                            }
                            if (inv_var && std::isfinite(ivd[q]) && ivd[q] > 0) {
                                double si = 1.0 / std::sqrt(ivd[q]);
                                ss += si;
                                ss2 += si * si;
                                ng += 1;
                            }
                        }
                    d[0] = qv * inv_flux;
                    if (den > 0 && ncl > 0 && ndi > 0) d[3] = 2.5 * std::log10(ndi / ncl);
                    if (have_spread && Sp > 0) {
                        d[4] = Sq / Sp - Sq0 / Sp0;
                        if (inv_var)
                            d[5] = std::sqrt(std::max(0.0, Sp * Sp * SqG + Sq * Sq * Sp0 - 2 * Sq * Sp * Sq0)) / (Sp * Sp);
                    }
                    if (inv_var) {
                        d[1] = std::sqrt(2.0 / M_PI) * ss * inv_flux;
                        if (ss2 > 0 && ng > nf) {
                            double dof_factor = std::sqrt(1.0 - (double)nf / (double)ng);
                            d[2] = (qv - std::sqrt(2.0 / M_PI) * dof_factor * ss) /
                                   (std::sqrt((1.0 - 2.0 / M_PI) * ss2) * dof_factor);
                        }
                    }
                }
            }
        }
        for (int64_t s = 0; s < n; ++s) {  // between-pass validation (:404-412)
            double y = prm[s * np], x = prm[s * np + 1], f = prm[s * np + rf];
            valid[s] = valid[s] && conv[s] && std::isfinite(y) && std::isfinite(x) && std::isfinite(f) && f > 0;
        }
    }
    std::memcpy(out->params, prm.data(), sizeof(double) * n * np);
    std::memcpy(out->errors, err.data(), sizeof(double) * n * np);
    for (int64_t s = 0; s < n; ++s) {
        out->converged[s] = conv[s];
        out->valid[s] = valid[s];
        out->chisq[s] = chisq[s];
        out->n_iter[s] = niter[s];
        if (out->qfit) out->qfit[s] = diag[s * 6];
        if (out->qfit_expected) out->qfit_expected[s] = diag[s * 6 + 1];
        if (out->qfit_z) out->qfit_z[s] = diag[s * 6 + 2];
        if (out->crowding) out->crowding[s] = diag[s * 6 + 3];
        if (out->spread_model) out->spread_model[s] = diag[s * 6 + 4];
        if (out->spread_model_err) out->spread_model_err[s] = diag[s * 6 + 5];
    }
    if (out->residual) std::memcpy(out->residual, resid.data(), sizeof(double) * npix);
    out->n_passes = n_passes;
    out->n_failed = n_failed;
    out->n_levels = 0;
    out->n_fits = 0;
    out->device_seconds = 0;
    return 0;
}
