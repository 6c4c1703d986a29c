// cpb_lm.cu -- batched per-star Levenberg-Marquardt (CrowdPhot.PSF.fit_star).
//
// Device restatement of
//   _prepare_fit_star_inputs                src/psf/psf_fitting.jl:36-101
//   _accum_circular_gaussian!               :354-451
//   _accum_image_psf!                       :1115-1173
//   _accum_gridded_imagepsf!                :1383-1517
//   lm_irls, damp!, covariance!              src/levenberg_marquardt.jl:64-99, 361-680
//   IRLS weights and scale estimators        :105-355 (k_lm_irls)
// One warp owns one cutout for the whole fit: lanes stride over the cutout's
// pixels, the normal equations are reduced with warp shuffles (every lane
// ends with the same A, b, cost), and every lane runs the identical small
// Cholesky / accept-reject logic, so there is no divergence and no shared
// state between cutouts.  Warps are persistent over a cutout queue.
#include <algorithm>
#include <cstdio>
#include <string>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "cpb_internal.cuh"

namespace cpb {
namespace {

struct LMConst {
    int np, nf;
    int fidx[5];
    int gauss;
    int damping;
    int max_iter;
    int reweighted;
    int irls;         // CPB_LOSS_* (0: plain LM)
    int scale;        // CPB_SCALE_*
    int mscale_max_iter;
    double loss_param, scale_value, mscale_delta, mscale_tol, weight_reset_tol;
    double fixv[5];  // fixed value per model parameter
    double x_tol, f_tol, g_tol;
    double lambda_init, lambda_up, lambda_down, lambda_min, lambda_max, min_diagonal;
};

// Normal equations at the full parameter vector fv (projected onto the free set).
// wv (nullable): per-pixel weights replacing the sanitised inv_var (IRLS);
// res (nullable): receives every pixel's residual model - data.
template <typename TI>
__device__ double lm_accum(const DevPsf& P, const LMConst& L, const TI* __restrict__ pix, const TI* __restrict__ iv,
                           int ny, int nx, int y1, int x1, const double* fv, double* A, double* b,
                           const double* wv = nullptr, double* res = nullptr) {
    const int lane = threadIdx.x & 31;
    double Af[15], bf[5], cost = 0;
#pragma unroll
    for (int q = 0; q < 15; ++q) Af[q] = 0;
#pragma unroll
    for (int q = 0; q < 5; ++q) bf[q] = 0;
    const int npx = ny * nx;
    if (L.gauss) {
        const double gp = -2.772588722239781;
        const double Y = fv[0], X = fv[1], fwhm = fv[2], flux = fv[3], bkg = fv[4];
        const double f2 = fwhm * fwhm;
        const double norm = -(3.141592653589793 * f2 / gp);
        const double amp = flux / norm, gf2 = gp / f2;
        for (int e = lane; e < npx; e += 32) {
            const int i = e % ny, j = e / ny;
            const double dx = (double)(x1 + j) - X, dy = (double)(y1 + i) - Y;
            const double sq = (dx * dx + dy * dy) / f2;
            const double g = exp(gp * sq);
            const double Ag = amp * g;
            const double r = (amp * g + bkg) - (double)pix[e];
            double w = 1.0;
            if (wv) {
                w = wv[e];
            } else if (iv) {
                double v = (double)iv[e];
                w = (isfinite(v) && v > 0) ? v : 0.0;
            }
            if (res) res[e] = r;
            const double wr = w * r;
            cost = wr * r + cost;
            const double gv[5] = {-2 * Ag * gf2 * dy, -2 * Ag * gf2 * dx, -2 * Ag * (1 + gp * sq) / fwhm, g / norm,
                                  1.0};
            int t = 0;
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                bf[q] = wr * gv[q] + bf[q];
#pragma unroll
                for (int pq = 0; pq <= q; ++pq) {
                    Af[t] = (w * gv[pq]) * gv[q] + Af[t];
                    ++t;
                }
            }
        }
    } else {
        const double Y = fv[0], X = fv[1], flux = fv[2], bkg = fv[3];
        StarCoef c;
        c.y = Y;
        c.x = X;
        c.flux = flux;
        c.bkg = bkg;
        grid_corners_dw(P, Y, X, c);
        for (int e = lane; e < npx; e += 32) {
            const int i = e % ny, j = e / ny;
            double s, dY, dX;
            grid_profile<double, double, true>(P, P.data64, c, (double)(y1 + i), (double)(x1 + j), s, dY, dX);
            const double r = (flux * s + bkg) - (double)pix[e];
            double w = 1.0;
            if (wv) {
                w = wv[e];
            } else if (iv) {
                double v = (double)iv[e];
                w = (isfinite(v) && v > 0) ? v : 0.0;
            }
            if (res) res[e] = r;
            const double wr = w * r;
            cost = wr * r + cost;
            const double gv[4] = {flux * dY, flux * dX, s, 1.0};
            int t = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                bf[q] = wr * gv[q] + bf[q];
#pragma unroll
                for (int pq = 0; pq <= q; ++pq) {
                    Af[t] = (w * gv[pq]) * gv[q] + Af[t];
                    ++t;
                }
            }
        }
    }
    cost = warp_sum(cost);
#pragma unroll
    for (int q = 0; q < 5; ++q) bf[q] = warp_sum(bf[q]);
#pragma unroll
    for (int q = 0; q < 15; ++q) Af[q] = warp_sum(Af[q]);
    // packed upper triangle: entry (pq, q), pq <= q, at q*(q+1)/2 + pq
    for (int jq = 0; jq < L.nf; ++jq) {
        b[jq] = bf[L.fidx[jq]];
        for (int iq = 0; iq < L.nf; ++iq) {
            int a = L.fidx[iq], bb = L.fidx[jq];
            int lo = min(a, bb), hi = max(a, bb);
            A[iq + jq * L.nf] = Af[hi * (hi + 1) / 2 + lo];
        }
    }
    return cost;
}

__device__ bool lm_chol_solve(const double* A, int n, const double* b, double* x) {
    double U[25];
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= j; ++i) {
            double s = A[i + j * n];
            for (int k = 0; k < i; ++k) s -= U[k + i * n] * U[k + j * n];
            if (i == j) {
                if (!(s > 0)) return false;
                U[j + j * n] = sqrt(s);
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

// covariance! with the pinv fallback (levenberg_marquardt.jl:366-388).
__device__ void lm_cov(const double* A0, int n, double* cov) {
    double e[5];
    bool ok = true;
    for (int c = 0; c < n && ok; ++c) {
        for (int i = 0; i < n; ++i) e[i] = (i == c) ? 1.0 : 0.0;
        double x[5];
        ok = lm_chol_solve(A0, n, e, x);
        for (int i = 0; i < n; ++i) cov[i + c * n] = x[i];
    }
    if (ok) return;
    // Jacobi pseudo-inverse of the symmetric matrix
    double A[25], V[25];
    for (int i = 0; i < n * n; ++i) A[i] = A0[i];
    for (int i = 0; i < n * n; ++i) V[i] = 0;
    for (int i = 0; i < n; ++i) V[i + i * n] = 1;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
            double s = 0.5 * (A[i + j * n] + A[j + i * n]);
            A[i + j * n] = A[j + i * n] = s;
        }
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) off += A[i + j * n] * A[i + j * n];
        if (off < 1e-300) break;
        for (int pp = 0; pp < n; ++pp)
            for (int q = pp + 1; q < n; ++q) {
                double apq = A[pp + q * n];
                if (apq == 0) continue;
                double tau = (A[q + q * n] - A[pp + pp * n]) / (2 * apq);
                double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1 + tau * tau));
                double c = 1 / sqrt(1 + t * t), s = t * c;
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
    for (int i = 0; i < n; ++i) smax = fmax(smax, fabs(A[i + i * n]));
    double tol = 2.220446049250313e-16 * n * smax;
    for (int i = 0; i < n * n; ++i) cov[i] = 0;
    for (int ev = 0; ev < n; ++ev) {
        double lam = A[ev + ev * n];
        if (!(fabs(lam) > tol)) continue;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) cov[i + j * n] += V[i + ev * n] * V[j + ev * n] / lam;
    }
}

// Per-cutout outputs, device pointers; every one but status may be null.
struct LMOut {
    double* params;   // n x np
    double* cov;      // n x nf x nf
    double *cost, *cost_init, *chisq, *lambda_final;
    uint8_t *converged, *x_converged, *f_converged, *g_converged;
    int32_t* iters;
    int32_t* status;
    double* sigma_final;  // IRLS scale estimate (NaN without IRLS)
};

template <typename TI>
__global__ void __launch_bounds__(256) k_lm(int64_t n_cut, LMConst L, DevPsf P, const int64_t* __restrict__ offs,
                                            const int32_t* __restrict__ cny, const int32_t* __restrict__ cnx,
                                            const int32_t* __restrict__ cy1, const int32_t* __restrict__ cx1,
                                            const TI* __restrict__ pixels, const TI* __restrict__ ivs,
                                            const double* __restrict__ init, LMOut out) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (gridDim.x * (int64_t)blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int np = L.np, nf = L.nf;
    for (int64_t c = warp; c < n_cut; c += nwarps) {
        const int ny = cny[c], nx = cnx[c], y1 = cy1[c], x1 = cx1[c];
        const TI* pix = pixels + offs[c];
        const TI* iv = ivs ? ivs + offs[c] : nullptr;
        const int64_t nobs = (int64_t)ny * nx;
        if (ny <= 0 || nx <= 0) {
            if (lane == 0) out.status[c] = CPB_ERR_ARGUMENT;
            continue;
        }
        // _prepare_fit_star_inputs checks (psf_fitting.jl:61-90) and lm_irls dof (:461-467)
        int bad = 0;
        if (iv) {
            int nvalid = 0;
            for (int64_t e = lane; e < nobs; e += 32) {
                double v = (double)iv[e];
                nvalid += (isfinite(v) && v > 0) ? 1 : 0;
            }
            nvalid = warp_sum(nvalid);
            if (!(nvalid > nf)) bad = 1;
        }
        if (!(nobs - nf > 0)) bad = 1;
        if (bad) {
            if (lane == 0) out.status[c] = CPB_ERR_ARGUMENT;
            continue;
        }
        double fv[5], x[5], xc[5], A[25], b[5], Ac[25], bc[5], Ad[25], d[5], D[5];
        for (int q = 0; q < np; ++q) fv[q] = init[c * np + q];
        for (int q = 0; q < np; ++q) {
            bool fr = false;
            for (int k = 0; k < nf; ++k) fr |= (L.fidx[k] == q);
            if (!fr) fv[q] = L.fixv[q];
        }
        for (int k = 0; k < nf; ++k) x[k] = fv[L.fidx[k]];
        double cost = lm_accum<TI>(P, L, pix, iv, ny, nx, y1, x1, fv, A, b);
        const double cost_init = cost;
        for (int k = 0; k < nf; ++k) D[k] = sqrt(fmax(A[k + k * nf], 1.0e-6));
        double lam = L.lambda_init;
        bool xconv = false, fconv = false, gconv = false, conv = false;
        int iter = 0;
        while (iter < L.max_iter) {
            ++iter;
            double gcos = 0;
            for (int k = 0; k < nf; ++k)
                gcos = nan_max(gcos, fabs(b[k]) / (sqrt(A[k + k * nf] * cost) + 2.220446049250313e-16));
            if (gcos <= L.g_tol) {
                gconv = conv = true;
                break;
            }
            for (int k = 0; k < nf * nf; ++k) Ad[k] = A[k];
            if (L.damping == CPB_DAMP_MARQUARDT)
                for (int k = 0; k < nf; ++k) Ad[k + k * nf] += lam * fmax(Ad[k + k * nf], L.min_diagonal);
            else if (L.damping == CPB_DAMP_LEVENBERG)
                for (int k = 0; k < nf; ++k) Ad[k + k * nf] += lam;
            if (!lm_chol_solve(Ad, nf, b, d)) {
                lam = fmin(lam * L.lambda_up, L.lambda_max);
                continue;
            }
            for (int k = 0; k < nf; ++k) d[k] = -d[k];
            double db = 0, dAd = 0;
            for (int k = 0; k < nf; ++k) db += d[k] * b[k];
            for (int k = 0; k < nf; ++k)
                for (int r = 0; r < nf; ++r) dAd += d[k] * A[k + r * nf] * d[r];
            const double prered = -2 * db - dAd;
            for (int k = 0; k < nf; ++k) xc[k] = x[k] + d[k];
            double fc[5];
            for (int q = 0; q < np; ++q) fc[q] = fv[q];
            for (int k = 0; k < nf; ++k) fc[L.fidx[k]] = xc[k];
            const double cost_c = lm_accum<TI>(P, L, pix, iv, ny, nx, y1, x1, fc, Ac, bc);
            const bool accepted = cost_c < cost;
            const double dcost = cost - cost_c;
            const double ratio = prered > 0 ? dcost / prered : 0.0;
            fconv = fabs(dcost) <= L.f_tol * (fabs(cost) + L.f_tol) && prered <= L.f_tol * (fabs(cost) + L.f_tol) &&
                    0.5 * ratio <= 1;
            double nd = 0, nxv = 0;
            for (int k = 0; k < nf; ++k) {
                nd += (D[k] * d[k]) * (D[k] * d[k]);
                nxv += (D[k] * x[k]) * (D[k] * x[k]);
            }
            xconv = sqrt(nd) <= L.x_tol * (sqrt(nxv) + L.x_tol) && (accepted || fconv);
            if (accepted) {
                cost = cost_c;
                lam = fmax(lam / L.lambda_down, L.lambda_min);
                for (int k = 0; k < nf; ++k) x[k] = xc[k];
                for (int k = 0; k < nf * nf; ++k) A[k] = Ac[k];
                for (int k = 0; k < nf; ++k) b[k] = bc[k];
                for (int q = 0; q < np; ++q) fv[q] = fc[q];
                for (int k = 0; k < nf; ++k) D[k] = fmax(D[k], sqrt(A[k + k * nf]));
                if (xconv || fconv) {
                    conv = true;
                    break;
                }
            } else {
                if (xconv || fconv) {
                    conv = true;
                    break;
                }
                lam = fmin(lam * L.lambda_up, L.lambda_max);
            }
        }
        if (lane == 0) {
            const double dof = (double)(nobs - nf);
            if (out.cov) {
                double cov[25];
                lm_cov(A, nf, cov);
                const double f = L.reweighted ? cost / dof : 1.0;
                for (int k = 0; k < nf * nf; ++k) out.cov[c * nf * nf + k] = cov[k] * f;
            }
            if (out.params)
                for (int q = 0; q < np; ++q) out.params[c * np + q] = fv[q];
            if (out.cost) out.cost[c] = cost;
            if (out.cost_init) out.cost_init[c] = cost_init;
            if (out.chisq) out.chisq[c] = cost / dof;
            if (out.lambda_final) out.lambda_final[c] = lam;
            if (out.converged) out.converged[c] = conv;
            if (out.x_converged) out.x_converged[c] = xconv;
            if (out.f_converged) out.f_converged[c] = fconv;
            if (out.g_converged) out.g_converged[c] = gconv;
            if (out.iters) out.iters[c] = iter;
            if (out.sigma_final) out.sigma_final[c] = __longlong_as_double(0x7ff8000000000000LL);
            out.status[c] = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// IRLS (lm_irls with reweight, levenberg_marquardt.jl:105-355, 611-645)
// ---------------------------------------------------------------------------
// Order-preserving 64-bit key of a double (negative values reversed).
__device__ __forceinline__ unsigned long long dkey(double v) {
    const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
    return (bits >> 63) ? ~bits : (bits | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey_inv(unsigned long long k) {
    const unsigned long long bits = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)bits);
}

// The k-th smallest (0-based) of val(0..n-1), exactly, by one warp: an 8-pass
// radix select on the keys with a 256-bin histogram in the warp's shared memory.
template <class F>
__device__ double warp_kth(F val, int n, int k, unsigned* hist) {
    const int lane = threadIdx.x & 31;
    unsigned long long prefix = 0, mask = 0;
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int t = lane; t < 256; t += 32) hist[t] = 0;
        __syncwarp();
        for (int e = lane; e < n; e += 32) {
            const unsigned long long key = dkey(val(e));
            if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255], 1u);
        }
        __syncwarp();
        unsigned cnt[8], tot = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            cnt[q] = hist[lane * 8 + q];
            tot += cnt[q];
        }
        unsigned incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const unsigned excl = incl - tot;
        const unsigned ball = __ballot_sync(0xffffffffu, (unsigned)k >= excl && (unsigned)k < incl);
        const int owner = ball ? __ffs(ball) - 1 : 31;
        int bin = 0;
        unsigned before = 0;
        if (lane == owner) {
            unsigned acc = excl;
            bin = lane * 8 + 7;
            before = acc;
            for (int q = 0; q < 8; ++q) {
                if ((unsigned)k < acc + cnt[q]) {
                    bin = lane * 8 + q;
                    before = acc;
                    break;
                }
                acc += cnt[q];
            }
        }
        bin = __shfl_sync(0xffffffffu, bin, owner);
        before = __shfl_sync(0xffffffffu, before, owner);
        k -= (int)before;
        prefix |= (unsigned long long)bin << shift;
        mask |= 255ull << shift;
        __syncwarp();
    }
    return dkey_inv(prefix);
}

// Statistics.median: the middle order statistic, or middle(a, b) = a/2 + b/2 of
// the two; NaN when any value is NaN.
template <class F>
__device__ double warp_median(F val, int n, unsigned* hist) {
    const int lane = threadIdx.x & 31;
    bool nan = false;
    for (int e = lane; e < n; e += 32) nan |= isnan(val(e));
    if (__any_sync(0xffffffffu, nan)) return __longlong_as_double(0x7ff8000000000000LL);
    if (n & 1) return warp_kth(val, n, (n - 1) / 2, hist);
    const double a = warp_kth(val, n, n / 2 - 1, hist), b = warp_kth(val, n, n / 2, hist);
    return a / 2 + b / 2;
}

// estimate_scale for MADScale / FixedScale / MScale over the n residuals r.
__device__ double irls_scale(const LMConst& L, const double* r, int n, double fixed_sigma, unsigned* hist) {
    if (L.scale == CPB_SCALE_FIXED || (L.scale == CPB_SCALE_AUTO && fixed_sigma == fixed_sigma))
        return L.scale == CPB_SCALE_FIXED ? L.scale_value : fixed_sigma;
    const double med = warp_median([&](int e) { return r[e]; }, n, hist);
    const double mad = 1.4826 * warp_median([&](int e) { return fabs(r[e] - med); }, n, hist);
    if (L.scale != CPB_SCALE_MSCALE) return mad;
    const int lane = threadIdx.x & 31;
    const double eps = 2.220446049250313e-16;
    double sg = isnan(mad) ? mad : fmax(mad, eps);
    for (int it = 0; it < L.mscale_max_iter; ++it) {
        const double cap = 9 * (sg * sg);
        double chi = 0;
        for (int e = lane; e < n; e += 32) {
            const double r2 = r[e] * r[e];
            chi += r2 < cap ? r2 : cap;
        }
        chi = warp_sum(chi);
        const double sn = sqrt(chi / (n * L.mscale_delta));
        if (fabs(sn - sg) <= L.mscale_tol * fmax(sg, L.mscale_tol)) {
            sg = sn;
            break;
        }
        sg = sn;
    }
    return sg;
}

// weight(loss, r) = psi(r) / (r psi'(0)), 1 near r = 0.
__device__ __forceinline__ double irls_weight(const LMConst& L, double r) {
    if (fabs(r) < 2.220446049250313e-16 * 10) return 1.0;
    const double c = L.loss_param;
    if (L.irls == CPB_LOSS_L2DIST) return (2 * r) / (r * 2.0);
    if (L.irls == CPB_LOSS_HUBER) {
        const double psi = fabs(r) <= c ? r : c * (r > 0 ? 1.0 : -1.0);
        const double psi0 = 0.0 <= c ? 1.0 : 0.0;
        return psi / (r * psi0);
    }
    if (L.irls == CPB_LOSS_LOGITDIST) return tanh(r / 2) / (r * 0.5);  // psi = tanh(r/2), psi'(0) = 1/2
    // TukeyLoss
    double psi = 0.0;
    if (fabs(r) <= c) {
        const double rc2 = (r / c) * (r / c);
        psi = r * ((1 - rc2) * (1 - rc2));
    }
    const double psi0 = 0.0 <= c ? 1.0 : 0.0;
    return psi / (r * psi0);
}

// One warp a cutout, as k_lm, with lm_irls's reweighting: after an accepted,
// unconverged step the scale is estimated from the residuals, every pixel's
// weight becomes base * weight(r / sigma), the normal equations are rebuilt at
// the accepted point and, when the weights moved by weight_reset_tol or more,
// lambda and D restart.  wbuf / rbuf: per-pixel weights and residuals, laid
// out like the cutouts.
template <typename TI>
__global__ void __launch_bounds__(256) k_lm_irls(int64_t n_cut, LMConst L, DevPsf P, const int64_t* __restrict__ offs,
                                                 const int32_t* __restrict__ cny, const int32_t* __restrict__ cnx,
                                                 const int32_t* __restrict__ cy1, const int32_t* __restrict__ cx1,
                                                 const TI* __restrict__ pixels, const TI* __restrict__ ivs,
                                                 const double* __restrict__ init, double* __restrict__ wbuf,
                                                 double* __restrict__ rbuf, LMOut out) {
    __shared__ unsigned hist_all[8][256];
    unsigned* hist = hist_all[(threadIdx.x >> 5) & 7];
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (gridDim.x * (int64_t)blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int np = L.np, nf = L.nf;
    const double eps = 2.220446049250313e-16;
    for (int64_t c = warp; c < n_cut; c += nwarps) {
        const int ny = cny[c], nx = cnx[c], y1 = cy1[c], x1 = cx1[c];
        const TI* pix = pixels + offs[c];
        const TI* iv = ivs ? ivs + offs[c] : nullptr;
        double* wts = wbuf + offs[c];
        double* res = rbuf + offs[c];
        const int64_t nobs = (int64_t)ny * nx;
        if (ny <= 0 || nx <= 0) {
            if (lane == 0) out.status[c] = CPB_ERR_ARGUMENT;
            continue;
        }
        int bad = 0;
        double wsum = 0;
        for (int64_t e = lane; e < nobs; e += 32) {
            double w = 1.0;
            if (iv) {
                const double v = (double)iv[e];
                w = (isfinite(v) && v > 0) ? v : 0.0;
            }
            wts[e] = w;
            wsum += w;
        }
        if (iv) {
            int nvalid = 0;
            for (int64_t e = lane; e < nobs; e += 32) {
                const double v = (double)iv[e];
                nvalid += (isfinite(v) && v > 0) ? 1 : 0;
            }
            nvalid = warp_sum(nvalid);
            if (!(nvalid > nf)) bad = 1;
        }
        if (!(nobs - nf > 0)) bad = 1;
        if (bad) {
            if (lane == 0) out.status[c] = CPB_ERR_ARGUMENT;
            continue;
        }
        // the default scale with weights: FixedScale(sqrt(inv(mean(base_weights))))
        const double fixed_sigma = iv ? sqrt(1.0 / (warp_sum(wsum) / (double)nobs))
                                      : __longlong_as_double(0x7ff8000000000000LL);
        __syncwarp();
        double fv[5], x[5], xc[5], A[25], b[5], Ac[25], bc[5], Ad[25], d[5], D[5];
        for (int q = 0; q < np; ++q) fv[q] = init[c * np + q];
        for (int q = 0; q < np; ++q) {
            bool fr = false;
            for (int k = 0; k < nf; ++k) fr |= (L.fidx[k] == q);
            if (!fr) fv[q] = L.fixv[q];
        }
        for (int k = 0; k < nf; ++k) x[k] = fv[L.fidx[k]];
        double cost = lm_accum<TI>(P, L, pix, iv, ny, nx, y1, x1, fv, A, b, wts, res);
        const double cost_init = cost;
        for (int k = 0; k < nf; ++k) D[k] = sqrt(fmax(A[k + k * nf], 1.0e-6));
        double lam = L.lambda_init;
        double sigma_final = __longlong_as_double(0x7ff8000000000000LL);
        bool xconv = false, fconv = false, gconv = false, conv = false;
        int iter = 0;
        while (iter < L.max_iter) {
            ++iter;
            double gcos = 0;
            for (int k = 0; k < nf; ++k)
                gcos = nan_max(gcos, fabs(b[k]) / (sqrt(A[k + k * nf] * cost) + eps));
            if (gcos <= L.g_tol) {
                gconv = conv = true;
                break;
            }
            for (int k = 0; k < nf * nf; ++k) Ad[k] = A[k];
            if (L.damping == CPB_DAMP_MARQUARDT)
                for (int k = 0; k < nf; ++k) Ad[k + k * nf] += lam * fmax(Ad[k + k * nf], L.min_diagonal);
            else if (L.damping == CPB_DAMP_LEVENBERG)
                for (int k = 0; k < nf; ++k) Ad[k + k * nf] += lam;
            if (!lm_chol_solve(Ad, nf, b, d)) {
                lam = fmin(lam * L.lambda_up, L.lambda_max);
                continue;
            }
            for (int k = 0; k < nf; ++k) d[k] = -d[k];
            double db = 0, dAd = 0;
            for (int k = 0; k < nf; ++k) db += d[k] * b[k];
            for (int k = 0; k < nf; ++k)
                for (int r = 0; r < nf; ++r) dAd += d[k] * A[k + r * nf] * d[r];
            const double prered = -2 * db - dAd;
            for (int k = 0; k < nf; ++k) xc[k] = x[k] + d[k];
            double fc[5];
            for (int q = 0; q < np; ++q) fc[q] = fv[q];
            for (int k = 0; k < nf; ++k) fc[L.fidx[k]] = xc[k];
            const double cost_c = lm_accum<TI>(P, L, pix, iv, ny, nx, y1, x1, fc, Ac, bc, wts, res);
            __syncwarp();
            const bool accepted = cost_c < cost;
            const double dcost = cost - cost_c;
            const double ratio = prered > 0 ? dcost / prered : 0.0;
            fconv = fabs(dcost) <= L.f_tol * (fabs(cost) + L.f_tol) && prered <= L.f_tol * (fabs(cost) + L.f_tol) &&
                    0.5 * ratio <= 1;
            double nd = 0, nxv = 0;
            for (int k = 0; k < nf; ++k) {
                nd += (D[k] * d[k]) * (D[k] * d[k]);
                nxv += (D[k] * x[k]) * (D[k] * x[k]);
            }
            xconv = sqrt(nd) <= L.x_tol * (sqrt(nxv) + L.x_tol) && (accepted || fconv);
            if (accepted) {
                cost = cost_c;
                lam = fmax(lam / L.lambda_down, L.lambda_min);
                for (int k = 0; k < nf; ++k) x[k] = xc[k];
                for (int k = 0; k < nf * nf; ++k) A[k] = Ac[k];
                for (int k = 0; k < nf; ++k) b[k] = bc[k];
                for (int q = 0; q < np; ++q) fv[q] = fc[q];
                for (int k = 0; k < nf; ++k) D[k] = fmax(D[k], sqrt(A[k + k * nf]));
                if (xconv || fconv) {
                    conv = true;
                    break;
                }
                // reweighting from the residuals at the accepted point (:611-645)
                sigma_final = irls_scale(L, res, (int)nobs, fixed_sigma, hist);
                if (sigma_final > eps) {
                    double dw2 = 0, wo2 = 0, wn2 = 0;
                    for (int64_t e = lane; e < nobs; e += 32) {
                        const double old_w = wts[e];
                        double base_w = 1.0;
                        if (iv) {
                            const double v = (double)iv[e];
                            base_w = (isfinite(v) && v > 0) ? v : 0.0;
                        }
                        const double new_w = base_w * irls_weight(L, res[e] / sigma_final);
                        const double dw = new_w - old_w;
                        dw2 = fma(dw, dw, dw2);
                        wo2 = fma(old_w, old_w, wo2);
                        wn2 = fma(new_w, new_w, wn2);
                        wts[e] = new_w;
                    }
                    dw2 = warp_sum(dw2);
                    wo2 = warp_sum(wo2);
                    wn2 = warp_sum(wn2);
                    __syncwarp();
                    cost = lm_accum<TI>(P, L, pix, iv, ny, nx, y1, x1, fv, A, b, wts, res);
                    __syncwarp();
                    const double wchange = sqrt(dw2) / fmax(fmax(sqrt(wo2), sqrt(wn2)), eps);
                    if (wchange >= L.weight_reset_tol) {
                        lam = L.lambda_init;
                        for (int k = 0; k < nf; ++k) D[k] = sqrt(fmax(A[k + k * nf], 1.0e-6));
                    }
                }
            } else {
                if (xconv || fconv) {
                    conv = true;
                    break;
                }
                lam = fmin(lam * L.lambda_up, L.lambda_max);
            }
        }
        if (lane == 0) {
            const double dof = (double)(nobs - nf);
            if (out.cov) {
                double cov[25];
                lm_cov(A, nf, cov);
                const double f = L.reweighted ? cost / dof : 1.0;
                for (int k = 0; k < nf * nf; ++k) out.cov[c * nf * nf + k] = cov[k] * f;
            }
            const double s2 = cost / dof;
            const bool scaled = !iv && !isnan(sigma_final) && sigma_final > eps;
            if (out.params)
                for (int q = 0; q < np; ++q) out.params[c * np + q] = fv[q];
            if (out.cost) out.cost[c] = cost;
            if (out.cost_init) out.cost_init[c] = cost_init;
            if (out.chisq) out.chisq[c] = scaled ? s2 / (sigma_final * sigma_final) : s2;
            if (out.lambda_final) out.lambda_final[c] = lam;
            if (out.converged) out.converged[c] = conv;
            if (out.x_converged) out.x_converged[c] = xconv;
            if (out.f_converged) out.f_converged[c] = fconv;
            if (out.g_converged) out.g_converged[c] = gconv;
            if (out.iters) out.iters[c] = iter;
            if (out.sigma_final) out.sigma_final[c] = sigma_final;
            out.status[c] = 0;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Fast form: compile-time parameter counts (every small matrix in registers),
// single-node image PSFs read through the edge-padded polyphase copy (the 16
// stencil taps of the 32 lanes' pixels -- consecutive cutout rows -- are
// adjacent doubles, staged in shared memory), only the cutout rectangle that
// can reach the ePSF grid evaluated in full, and a device work queue over the
// cutouts.  Arithmetic per pixel is corner_eval's (psf_fitting.jl:1233-1321
// restated); only the order of the per-lane sums differs.
// ---------------------------------------------------------------------------
template <int NF>
__device__ __forceinline__ bool chol_solve_t(const double* A, const double* b, double* x) {
    double U[NF * NF];
#pragma unroll
    for (int j = 0; j < NF; ++j)
#pragma unroll
        for (int i = 0; i <= j; ++i) {
            double s = A[i + j * NF];
#pragma unroll
            for (int k = 0; k < i; ++k) s -= U[k + i * NF] * U[k + j * NF];
            if (i == j) {
                if (!(s > 0)) return false;
                U[j + j * NF] = sqrt(s);
            } else {
                U[i + j * NF] = s / U[i + i * NF];
            }
        }
    double y[NF];
#pragma unroll
    for (int i = 0; i < NF; ++i) {
        double s = b[i];
#pragma unroll
        for (int k = 0; k < i; ++k) s -= U[k + i * NF] * y[k];
        y[i] = s / U[i + i * NF];
    }
#pragma unroll
    for (int i = NF - 1; i >= 0; --i) {
        double s = y[i];
#pragma unroll
        for (int k = i + 1; k < NF; ++k) s -= U[i + k * NF] * x[k];
        x[i] = s / U[i + i * NF];
    }
    return true;
}

// v[idx] for a register array v and a runtime index, without local memory.
template <int N>
__device__ __forceinline__ double pick(const double* v, int idx) {
    double r = 0;
#pragma unroll
    for (int q = 0; q < N; ++q) r = (q == idx) ? v[q] : r;
    return r;
}

// Stencil row / column taps of one axis in the polyphase copy: with the 0-based
// sample index i0 of the first tap, the four taps i0..i0+3 live at
// (i % is) * pstride + (i / is) * qstride.
__device__ __forceinline__ void pp_taps(int i0, int is, float inv_is, int pstride, int qstride, int* t) {
    int q = __float2int_rz(__int2float_rn(i0) * inv_is);
    int r = i0 - q * is;
    if (r < 0) {
        r += is;
        --q;
    } else if (r >= is) {
        r -= is;
        ++q;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        t[k] = r * pstride + q * qstride;
        if (++r == is) {
            r = 0;
            ++q;
        }
    }
}

struct PPNode {
    const double* pp;   // this node's edge-padded polyphase block (DevNode::lpoff)
    DevNode nd;
    int plane;          // LPY * LPX
    float inv_isy, inv_isx;
};

// Stencil offsets of the previous pixel a lane evaluated (ly = lx = 0: none).
struct TapCursor {
    int ly, lx;
    int ry[4], cx[4];
};

// Single-node image profile and its derivatives in the detector frame:
// s, dsdY = -sy * dp/dv, dsdX = -sx * dp/du (grid_profile with weights (1, 0, 0, 0)).
// pp: the node's edge-padded polyphase samples (shared or global memory), so the
// clamped stencils at the grid's border need no special case.  (di, dj): how far
// the cutout row / column moved since the lane's previous pixel; when the
// stencil origin moved by whole oversampling periods the cached tap offsets are
// advanced instead of recomputed.
__device__ __forceinline__ void pp_profile(const PPNode& N, const double* pp, TapCursor& T, int di, int dj, double Y,
                                           double X, double py, double px, double& s, double& dY, double& dX) {
    const DevNode& nd = N.nd;
    const double u = nd.sx * (px - X) + nd.ox;
    const double v = nd.sy * (py - Y) + nd.oy;
    const int nyd = nd.ny, nxd = nd.nx;
    // NaN and infinite u, v fail these range tests, as isfinite would
    const bool inb = u >= 1.0 && u <= (double)nxd && v >= 1.0 && v <= (double)nyd;
    if (!inb) {
        s = nd.fill;
        dY = 0.0;
        dX = 0.0;
        T.ly = T.lx = 0;
        return;
    }
    const int lx = clampi((int)floor(u), 1, nxd - 1);
    const int ly = clampi((int)floor(v), 1, nyd - 1);
    const double du = u - (double)lx, dv = v - (double)ly;
    if (T.ly != 0 && ly == T.ly + nd.isy * di) {
#pragma unroll
        for (int k = 0; k < 4; ++k) T.ry[k] += di;
    } else {
        pp_taps(ly - 1, nd.isy, N.inv_isy, N.plane, 1, T.ry);  // padded index of sample ly - 2
    }
    if (T.lx != 0 && lx == T.lx + nd.isx * dj) {
#pragma unroll
        for (int k = 0; k < 4; ++k) T.cx[k] += dj * nd.LPY;
    } else {
        pp_taps(lx - 1, nd.isx, N.inv_isx, nd.isy * N.plane, nd.LPY, T.cx);
    }
    T.ly = ly;
    T.lx = lx;
    double row[4], drow[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const double* q = pp + T.ry[r];
        const double a = q[T.cx[0]], b = q[T.cx[1]], c = q[T.cx[2]], e = q[T.cx[3]];
        const double k1 = (c - a) / 2;
        const double k4 = c - b - k1;
        const double k2 = 3 * k4 - (e - b) / 2 + k1;
        const double k3 = k4 - k2;
        row[r] = du * (du * (du * k3 + k2) + k1) + b;
        drow[r] = du * (3 * du * k3 + 2 * k2) + k1;
    }
    const double v1 = (row[2] - row[0]) / 2;
    const double v4 = row[2] - row[1] - v1;
    const double v2 = 3 * v4 - (row[3] - row[1]) / 2 + v1;
    const double v3 = v4 - v2;
    const double pv = dv * (dv * (dv * v3 + v2) + v1) + row[1];
    const double pdv = dv * (3 * dv * v3 + 2 * v2) + v1;
    const double u1 = (drow[2] - drow[0]) / 2;
    const double u4 = drow[2] - drow[1] - u1;
    const double u2 = 3 * u4 - (drow[3] - drow[1]) / 2 + u1;
    const double u3 = u4 - u2;
    const double pdu = dv * (dv * (dv * u3 + u2) + u1) + drow[1];
    s = pv;
    dY = -(nd.sy * pdv);
    dX = -(nd.sx * pdu);
}

// A cutout is fitted by a team of WPC warps (1: one warp a cutout, the
// throughput form for large batches; 4: a 128-thread team, the latency form for
// batches too small to fill the GPU).  Teams synchronise on their own named
// barrier (1 + team index; barrier 0 is __syncthreads).
template <int WPC>
__device__ __forceinline__ void team_sync() {
    if (WPC == 1) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)(threadIdx.x / (32 * WPC))), "r"(32 * WPC) : "memory");
    }
}

// Sums of K per-thread values over the team, in a fixed order (warp sums, then
// the team's warps in index order); every thread of the team receives them.
// red: the team's K * WPC doubles of shared memory.
template <int WPC, int K>
__device__ __forceinline__ void team_sum(double (&v)[K], double* red) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    if (WPC == 1) return;
    const int lane = threadIdx.x & 31, w = (threadIdx.x >> 5) % WPC;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) red[w * K + k] = v[k];
    team_sync<WPC>();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double t = red[k];
#pragma unroll
        for (int q = 1; q < WPC; ++q) t += red[q * K + k];
        v[k] = t;
    }
}

// Normal equations of one cutout at the full parameter vector fv, projected onto
// the free set (A: NF x NF column-major, b: NF); every thread of the team returns
// the same cost.  (qs, rs): the column / row step of a 32 * WPC pixel stride;
// red: the team's reduction scratch (WPC * (1 + NF + NF (NF + 1) / 2) doubles).
template <typename TI, int NP, int NF, int WPC>
__device__ double lm_accum_t(const PPNode& N, const double* pp, const LMConst& L, const TI* __restrict__ pix,
                             const TI* __restrict__ iv, int ny, int nx, int y1, int x1, int qs, int rs,
                             const double* fv, double* A, double* b, double* red) {
    constexpr int NT = NP * (NP + 1) / 2;
    constexpr int TS = 32 * WPC;  // team size = pixel stride
    const int lane = threadIdx.x % TS;
    const int q32 = qs, r32 = rs;
    double Af[NT], bf[NP], cost = 0;
#pragma unroll
    for (int q = 0; q < NT; ++q) Af[q] = 0;
#pragma unroll
    for (int q = 0; q < NP; ++q) bf[q] = 0;
    const int npx = ny * nx;
    // one pixel's contribution: cost, b and the upper triangle of A
    auto acc = [&](int e, double mval, const double* gv) {
        const double r = mval - (double)pix[e];
        double w = 1.0;
        if (iv) {
            const double vv = (double)iv[e];
            w = (isfinite(vv) && vv > 0) ? vv : 0.0;
        }
        const double wr = w * r;
        cost = wr * r + cost;
        int t = 0;
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            bf[q] = wr * gv[q] + bf[q];
#pragma unroll
            for (int pq = 0; pq <= q; ++pq) {
                Af[t] = (w * gv[pq]) * gv[q] + Af[t];
                ++t;
            }
        }
    };
    if (NP == 5) {  // CircularGaussianPSF (parametric_models.jl:79-115)
        const double gp = -2.772588722239781;
        const double Y = fv[0], X = fv[1], fwhm = fv[2], flux = fv[3], bkg = fv[NP - 1];
        const double f2 = fwhm * fwhm;
        const double norm = -(3.141592653589793 * f2 / gp);
        const double amp = flux / norm, gf2 = gp / f2;
        int i = lane % ny, j = lane / ny;
        for (int e = lane; e < npx; e += TS) {
            const double py = (double)(y1 + i), px = (double)(x1 + j);
            const double dx = px - X, dy = py - Y;
            const double sq = (dx * dx + dy * dy) / f2;
            const double g = exp(gp * sq);
            const double Ag = amp * g;
            double gv[NP];
            gv[0] = -2 * Ag * gf2 * dy;
            gv[1] = -2 * Ag * gf2 * dx;
            gv[2] = -2 * Ag * (1 + gp * sq) / fwhm;
            gv[3] = g / norm;
            gv[NP - 1] = 1.0;
            acc(e, amp * g + bkg, gv);
            i += r32;
            j += q32;
            if (i >= ny) {
                i -= ny;
                ++j;
            }
        }
    } else {
        const DevNode& nd = N.nd;
        const double Y = fv[0], X = fv[1], flux = fv[2], bkg = fv[3];
        // Cutout pixels outside [ilo, ihi] x [jlo, jhi] are at least one pixel
        // (>= one grid sample) beyond the grid, so their profile is the fill
        // value with zero derivatives; the rectangle is evaluated in full.
        int ilo = 0, ihi = ny - 1, jlo = 0, jhi = nx - 1;
        if (isfinite(Y) && isfinite(X)) {
            const double ya = Y - (double)y1 + (1.0 - nd.oy) / nd.sy;
            const double yb = Y - (double)y1 + ((double)nd.ny - nd.oy) / nd.sy;
            const double xa = X - (double)x1 + (1.0 - nd.ox) / nd.sx;
            const double xb = X - (double)x1 + ((double)nd.nx - nd.ox) / nd.sx;
            ilo = (int)fmin(fmax(0.0, floor(ya) - 1.0), (double)ny);
            ihi = (int)fmax(fmin((double)(ny - 1), ceil(yb) + 1.0), -1.0);
            jlo = (int)fmin(fmax(0.0, floor(xa) - 1.0), (double)nx);
            jhi = (int)fmax(fmin((double)(nx - 1), ceil(xb) + 1.0), -1.0);
        }
        const int ni = ihi - ilo + 1, nj = jhi - jlo + 1;
        if (ni > 0 && nj > 0) {
            const int nr = ni * nj, rq = TS / ni, rr = TS % ni;
            int ii = lane % ni, jj = lane / ni, di = 0, dj = 0;
            TapCursor T;
            T.ly = T.lx = 0;
            for (int k = lane; k < nr; k += TS) {
                const int i = ilo + ii, j = jlo + jj;
                double s, dY, dX;
                pp_profile(N, pp, T, di, dj, Y, X, (double)(y1 + i), (double)(x1 + j), s, dY, dX);
                const double gv[NP] = {flux * dY, flux * dX, s, 1.0};
                acc(i + j * ny, flux * s + bkg, gv);
                ii += rr;
                jj += rq;
                di = rr;
                dj = rq;
                if (ii >= ni) {
                    ii -= ni;
                    ++jj;
                    di -= ni;
                    ++dj;
                }
            }
        }
        if (ni < ny || nj < nx) {
            const double s = nd.fill, dY = 0.0, dX = 0.0;
            const double gv[NP] = {flux * dY, flux * dX, s, 1.0};
            const double mval = flux * s + bkg;
            int i = lane % ny, j = lane / ny;
            for (int e = lane; e < npx; e += TS) {
                if (!(i >= ilo && i <= ihi && j >= jlo && j <= jhi)) acc(e, mval, gv);
                i += r32;
                j += q32;
                if (i >= ny) {
                    i -= ny;
                    ++j;
                }
            }
        }
    }
    // project onto the free set, then reduce only what the solve needs
    double Ap[NF * (NF + 1) / 2], bp[NF];
    {
        int t = 0;
#pragma unroll
        for (int jq = 0; jq < NF; ++jq) {
            bp[jq] = pick<NP>(bf, L.fidx[jq]);
#pragma unroll
            for (int iq = 0; iq <= jq; ++iq) {
                const int a = L.fidx[iq], c = L.fidx[jq];
                const int lo = min(a, c), hi = max(a, c);
                Ap[t++] = pick<NT>(Af, hi * (hi + 1) / 2 + lo);
            }
        }
    }
    constexpr int KR = 1 + NF + NF * (NF + 1) / 2;
    double v[KR];
    v[0] = cost;
#pragma unroll
    for (int q = 0; q < NF; ++q) v[1 + q] = bp[q];
#pragma unroll
    for (int t = 0; t < NF * (NF + 1) / 2; ++t) v[1 + NF + t] = Ap[t];
    team_sum<WPC, KR>(v, red);
#pragma unroll
    for (int q = 0; q < NF; ++q) b[q] = v[1 + q];
    {
        int t = 0;
#pragma unroll
        for (int jq = 0; jq < NF; ++jq)
#pragma unroll
            for (int iq = 0; iq <= jq; ++iq) {
                const double s = v[1 + NF + t++];
                A[iq + jq * NF] = s;
                A[jq + iq * NF] = s;
            }
    }
    return v[0];
}

// covariance! (levenberg_marquardt.jl:366-388) for compile-time NF; the pinv
// fallback is the general one.
template <int NF>
__device__ void lm_cov_t(const double* A, double* cov) {
    double e[NF], x[NF];
    bool ok = true;
#pragma unroll
    for (int c = 0; c < NF; ++c) {
#pragma unroll
        for (int i = 0; i < NF; ++i) e[i] = (i == c) ? 1.0 : 0.0;
        ok = ok && chol_solve_t<NF>(A, e, x);
#pragma unroll
        for (int i = 0; i < NF; ++i) cov[i + c * NF] = x[i];
    }
    if (!ok) lm_cov(A, NF, cov);
}

// LM bookkeeping of one cutout, kept in shared memory between normal-equation
// passes so that none of it occupies registers during the pixel loop.
template <int NP, int NF>
struct LMState {
    double fv[NP], fc[NP];       // accepted / candidate full parameter vectors
    double x[NF], xc[NF], d[NF], D[NF], b[NF], A[NF * NF];
    double cost, cost_init, lam, prered;
    int iter, phase;             // phase 0: the initial pass is pending
    int conv, xconv, fconv, gconv;
};

// Consumes one normal-equation pass (cost_c, Ac, bc at S.fc) and prepares the
// next candidate; returns true when the fit is over.  Every thread of the team
// computes the same values; its first thread (lane 0) stores them.  lm_irls,
// levenberg_marquardt.jl:478-680.
template <int NP, int NF, int WPC>
__device__ __forceinline__ bool lm_step(LMState<NP, NF>& S, const LMConst& L, double cost_c, const double* Ac,
                                        const double* bc, int lane) {
    double fv[NP], x[NF], A[NF * NF], b[NF], D[NF];
    double cost, lam = S.lam;
    int iter = S.iter;
    int conv = S.conv, xconv = S.xconv, fconv = S.fconv, gconv = S.gconv;
    bool done = false;
    if (S.phase == 0) {
#pragma unroll
        for (int q = 0; q < NP; ++q) fv[q] = S.fc[q];
#pragma unroll
        for (int k = 0; k < NF; ++k) x[k] = pick<NP>(fv, L.fidx[k]);
#pragma unroll
        for (int k = 0; k < NF * NF; ++k) A[k] = Ac[k];
#pragma unroll
        for (int k = 0; k < NF; ++k) b[k] = bc[k];
        cost = cost_c;
        if (lane == 0) S.cost_init = cost_c;
#pragma unroll
        for (int k = 0; k < NF; ++k) D[k] = sqrt(fmax(A[k + k * NF], 1.0e-6));
    } else {
        cost = S.cost;
        double d[NF], xc[NF];
#pragma unroll
        for (int k = 0; k < NF; ++k) {
            x[k] = S.x[k];
            d[k] = S.d[k];
            xc[k] = S.xc[k];
            D[k] = S.D[k];
            b[k] = S.b[k];
        }
#pragma unroll
        for (int k = 0; k < NF * NF; ++k) A[k] = S.A[k];
#pragma unroll
        for (int q = 0; q < NP; ++q) fv[q] = S.fv[q];
        const double prered = S.prered;
        const bool accepted = cost_c < cost;
        const double dcost = cost - cost_c;
        const double ratio = prered > 0 ? dcost / prered : 0.0;
        fconv = fabs(dcost) <= L.f_tol * (fabs(cost) + L.f_tol) && prered <= L.f_tol * (fabs(cost) + L.f_tol) &&
                0.5 * ratio <= 1;
        double nd = 0, nxv = 0;
#pragma unroll
        for (int k = 0; k < NF; ++k) {
            nd += (D[k] * d[k]) * (D[k] * d[k]);
            nxv += (D[k] * x[k]) * (D[k] * x[k]);
        }
        xconv = sqrt(nd) <= L.x_tol * (sqrt(nxv) + L.x_tol) && (accepted || fconv);
        if (accepted) {
            cost = cost_c;
            lam = fmax(lam / L.lambda_down, L.lambda_min);
#pragma unroll
            for (int k = 0; k < NF; ++k) x[k] = xc[k];
#pragma unroll
            for (int k = 0; k < NF * NF; ++k) A[k] = Ac[k];
#pragma unroll
            for (int k = 0; k < NF; ++k) b[k] = bc[k];
#pragma unroll
            for (int q = 0; q < NP; ++q) fv[q] = S.fc[q];
#pragma unroll
            for (int k = 0; k < NF; ++k) D[k] = fmax(D[k], sqrt(A[k + k * NF]));
            if (xconv || fconv) conv = 1, done = true;
        } else {
            if (xconv || fconv) conv = 1, done = true;
            else lam = fmin(lam * L.lambda_up, L.lambda_max);
        }
    }
    // next candidate (the head of the lm_irls loop)
    double d[NF], xc[NF], fc[NP], prered = 0;
    while (!done) {
        if (iter >= L.max_iter) {
            done = true;
            break;
        }
        ++iter;
        double gcos = 0;
#pragma unroll
        for (int k = 0; k < NF; ++k)
            gcos = nan_max(gcos, fabs(b[k]) / (sqrt(A[k + k * NF] * cost) + 2.220446049250313e-16));
        if (gcos <= L.g_tol) {
            gconv = conv = 1;
            done = true;
            break;
        }
        double Ad[NF * NF];
#pragma unroll
        for (int k = 0; k < NF * NF; ++k) Ad[k] = A[k];
        if (L.damping == CPB_DAMP_MARQUARDT) {
#pragma unroll
            for (int k = 0; k < NF; ++k) Ad[k + k * NF] += lam * fmax(Ad[k + k * NF], L.min_diagonal);
        } else if (L.damping == CPB_DAMP_LEVENBERG) {
#pragma unroll
            for (int k = 0; k < NF; ++k) Ad[k + k * NF] += lam;
        }
        if (!chol_solve_t<NF>(Ad, b, d)) {
            lam = fmin(lam * L.lambda_up, L.lambda_max);
            continue;
        }
#pragma unroll
        for (int k = 0; k < NF; ++k) d[k] = -d[k];
        double db = 0, dAd = 0;
#pragma unroll
        for (int k = 0; k < NF; ++k) db += d[k] * b[k];
#pragma unroll
        for (int k = 0; k < NF; ++k)
#pragma unroll
            for (int r = 0; r < NF; ++r) dAd += d[k] * A[k + r * NF] * d[r];
        prered = -2 * db - dAd;
#pragma unroll
        for (int k = 0; k < NF; ++k) xc[k] = x[k] + d[k];
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            double vq = fv[q];
#pragma unroll
            for (int k = 0; k < NF; ++k) vq = (L.fidx[k] == q) ? xc[k] : vq;
            fc[q] = vq;
        }
        break;
    }
    team_sync<WPC>();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NP; ++q) S.fv[q] = fv[q];
#pragma unroll
        for (int k = 0; k < NF; ++k) {
            S.x[k] = x[k];
            S.D[k] = D[k];
            S.b[k] = b[k];
        }
#pragma unroll
        for (int k = 0; k < NF * NF; ++k) S.A[k] = A[k];
        if (!done) {
#pragma unroll
            for (int k = 0; k < NF; ++k) {
                S.d[k] = d[k];
                S.xc[k] = xc[k];
            }
#pragma unroll
            for (int q = 0; q < NP; ++q) S.fc[q] = fc[q];
            S.prered = prered;
        }
        S.cost = cost;
        S.lam = lam;
        S.iter = iter;
        S.phase = 1;
        S.conv = conv;
        S.xconv = xconv;
        S.fconv = fconv;
        S.gconv = gconv;
    }
    team_sync<WPC>();
    return done;
}

constexpr int kLMThreads = 256;

// fit_star of one cutout by a team (pixels pix / weights iv, column-major
// ny x nx whose first pixel is image pixel (y1, x1); init: the NP model
// parameters, fixed ones replaced by L.fixv).  Returns 0 with the result in S,
// or CPB_ERR_ARGUMENT when the inputs fail _prepare_fit_star_inputs's checks
// (psf_fitting.jl:61-90) or lm_irls's dof test (:461-467).
template <typename TI, int NP, int NF, int WPC>
__device__ int lm_team_fit(const PPNode& N, const double* pp, const LMConst& L, const TI* __restrict__ pix,
                           const TI* __restrict__ iv, int ny, int nx, int y1, int x1, const double* init,
                           LMState<NP, NF>& S, double* red, int lane) {
    constexpr int TS = 32 * WPC;
    const int64_t nobs = (int64_t)ny * nx;
    if (ny <= 0 || nx <= 0) return CPB_ERR_ARGUMENT;
    bool bad = !(nobs - NF > 0);
    if (iv) {
        double nv[1] = {0.0};
        for (int64_t e = lane; e < nobs; e += TS) {
            const double v = (double)iv[e];
            nv[0] += (isfinite(v) && v > 0) ? 1.0 : 0.0;
        }
        team_sum<WPC, 1>(nv, red);
        team_sync<WPC>();  // red is reused by the first normal-equation pass
        bad = bad || !((int)nv[0] > NF);
    }
    if (bad) return CPB_ERR_ARGUMENT;
    const int qs = TS / ny, rs = TS % ny;
    team_sync<WPC>();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            bool fr = false;
#pragma unroll
            for (int k = 0; k < NF; ++k) fr |= (L.fidx[k] == q);
            S.fc[q] = fr ? init[q] : L.fixv[q];
        }
        S.iter = 0;
        S.phase = 0;
        S.lam = L.lambda_init;
        S.conv = S.xconv = S.fconv = S.gconv = 0;
    }
    team_sync<WPC>();
    for (;;) {
        double fc[NP], Ac[NF * NF], bc[NF];
#pragma unroll
        for (int q = 0; q < NP; ++q) fc[q] = S.fc[q];
        const double cost_c = lm_accum_t<TI, NP, NF, WPC>(N, pp, L, pix, iv, ny, nx, y1, x1, qs, rs, fc, Ac, bc, red);
        if (lm_step<NP, NF, WPC>(S, L, cost_c, Ac, bc, lane)) break;
    }
    return 0;
}

template <typename TI, int NP, int NF, bool SMEM, int WPC>
__global__ void __launch_bounds__(kLMThreads, 2) k_lm_t(int64_t n_cut, LMConst L, PPNode N,
                                             const int64_t* __restrict__ offs, const int32_t* __restrict__ cny,
                                             const int32_t* __restrict__ cnx, const int32_t* __restrict__ cy1,
                                             const int32_t* __restrict__ cx1, const TI* __restrict__ pixels,
                                             const TI* __restrict__ ivs, const double* __restrict__ init, LMOut out,
                                             unsigned long long* __restrict__ queue) {
    constexpr int TS = 32 * WPC;
    constexpr int KR = 1 + NF + NF * (NF + 1) / 2;
    __shared__ LMState<NP, NF> states[kLMThreads / TS];
    __shared__ double red_all[(kLMThreads / 32) * KR];
    __shared__ unsigned long long cut_sh[kLMThreads / TS];
    extern __shared__ double node_smem[];
    const int team = threadIdx.x / TS;
    LMState<NP, NF>& S = states[team];
    double* red = red_all + team * WPC * KR;
    const int lane = threadIdx.x % TS;  // index within the team (lane 0 stores the team's state)
    // the node's polyphase samples, staged once per (persistent) block (plain
    // loads: a 1-D bulk asynchronous copy measured 4.5 % slower for the whole kernel)
    const double* pp = N.pp;
    if (SMEM && NP == 4) {
        const int nel = N.plane * N.nd.isy * N.nd.isx;
        for (int k = threadIdx.x; k < nel; k += blockDim.x) node_smem[k] = N.pp[k];
        __syncthreads();
        pp = node_smem;
    }
    for (;;) {
        unsigned long long cc = 0;
        if (WPC == 1) {
            if (lane == 0) cc = atomicAdd(queue, 1ull);
            cc = __shfl_sync(0xffffffffu, cc, 0);
        } else {
            if (lane == 0) cut_sh[team] = atomicAdd(queue, 1ull);
            team_sync<WPC>();
            cc = cut_sh[team];
        }
        if (cc >= (unsigned long long)n_cut) return;
        const int64_t c = (int64_t)cc;
        const int ny = cny[c], nx = cnx[c];
        const int64_t o = (ny > 0 && nx > 0) ? offs[c] : 0;
        const int st = lm_team_fit<TI, NP, NF, WPC>(N, pp, L, pixels + o, ivs ? ivs + o : nullptr, ny, nx, cy1[c],
                                                    cx1[c], init + c * NP, S, red, lane);
        if (st != 0) {
            if (lane == 0) out.status[c] = st;
            team_sync<WPC>();
            continue;
        }
        if (lane == 0) {
            const double dof = (double)((int64_t)ny * nx - NF);
            const double cost = S.cost;
            if (out.cov) {
                double cov[NF * NF];
                lm_cov_t<NF>(S.A, cov);
                const double f = L.reweighted ? cost / dof : 1.0;
#pragma unroll
                for (int k = 0; k < NF * NF; ++k) out.cov[c * NF * NF + k] = cov[k] * f;
            }
            if (out.params)
#pragma unroll
                for (int q = 0; q < NP; ++q) out.params[c * NP + q] = S.fv[q];
            if (out.cost) out.cost[c] = cost;
            if (out.cost_init) out.cost_init[c] = S.cost_init;
            if (out.chisq) out.chisq[c] = cost / dof;
            if (out.lambda_final) out.lambda_final[c] = S.lam;
            if (out.converged) out.converged[c] = S.conv;
            if (out.x_converged) out.x_converged[c] = S.xconv;
            if (out.f_converged) out.f_converged[c] = S.fconv;
            if (out.g_converged) out.g_converged[c] = S.gconv;
            if (out.iters) out.iters[c] = S.iter;
            if (out.sigma_final) out.sigma_final[c] = __longlong_as_double(0x7ff8000000000000LL);
            out.status[c] = 0;
        }
        team_sync<WPC>();
    }
}

// ---------------------------------------------------------------------------
// fit_all_stars as one dependency-driven launch per pass
// ---------------------------------------------------------------------------
// A star may be fitted as soon as every brighter star whose box meets its own
// has been subtracted; stars that are ready together have disjoint boxes.  One
// persistent launch per pass walks that order: 128-thread teams take ready
// stars from a device queue (position indices, filled in the order they become
// ready), add the star's previous model back (passes 2+), copy its cutout, fit
// it (lm_team_fit), update the star's state, subtract the new model, keep a
// snapshot of its box for the diagnostics on the last pass, and release the
// stars that waited for it.  Each pixel still sees its adds and subtracts in
// brightness order, so the result is the one-star-at-a-time one, but a slow
// fit only holds back the stars that overlap it.  The residual image is read
// and written around L1 (ld/st.cg): other SMs change it between uses.
constexpr long long kDagSpinLimit = 1ll << 26;  // default: ~64 M polls of >= 64 ns before a team gives up
// Warps of one team: 4 measured fastest on the 2048^2 field (k_mp_dag 34.6 ms for
// three passes, against 58.2 ms with 1 and 41.0 ms with 8).
constexpr int kDagWarps = 4;

template <typename TIV, int NP, int NF, bool SMEM>
__global__ void __launch_bounds__(kLMThreads, 2) k_mp_dag(LMConst L, PPNode N, DevPsf P, DagArgs A) {
    constexpr int WPC = kDagWarps, TS = 32 * kDagWarps;
    constexpr int KR = 1 + NF + NF * (NF + 1) / 2;
    __shared__ LMState<NP, NF> states[kLMThreads / TS];
    __shared__ double red_all[(kLMThreads / 32) * KR];
    __shared__ int pos_sh[kLMThreads / TS];
    extern __shared__ double node_smem[];
    const int team = threadIdx.x / TS;
    LMState<NP, NF>& S = states[team];
    double* red = red_all + team * WPC * KR;
    const int lane = threadIdx.x % TS;
    const int gteam = blockIdx.x * (kLMThreads / TS) + team;
    double* cpix = A.cpix + (int64_t)gteam * A.box_max;
    double* civ = A.civ ? A.civ + (int64_t)gteam * A.box_max : nullptr;
    const TIV* ivimg = (const TIV*)A.iv;
    const double* pp = N.pp;
    if (SMEM && NP == 4) {  // the node's polyphase samples, staged once per block
        const int nel = N.plane * N.nd.isy * N.nd.isx;
        for (int k = threadIdx.x; k < nel; k += blockDim.x) node_smem[k] = N.pp[k];
        __syncthreads();
        pp = node_smem;
    }
    int* head = A.counters;
    int* tail = A.counters + 1;
    int* errf = A.counters + 2;
    const int np = A.M.np;
    for (;;) {
        // claim the next queue slot and wait (bounded) until a ready star fills it
        if (lane == 0) {
            int k = -2;
            const int h = atomicAdd(head, 1);
            if (h < A.npos) {
                for (long long it = 0;; ++it) {
                    k = ((volatile int32_t*)A.queue)[h];
                    if (k >= 0) break;
                    if (it > A.spin_limit || ((volatile int*)errf)[0]) {
                        atomicExch(errf, 1);
                        k = -2;
                        break;
                    }
                    __nanosleep(64);
                }
            }
            __threadfence();
            pos_sh[team] = k;
        }
        team_sync<WPC>();
        const int k = pos_sh[team];
        if (k < 0) return;
        const int4 b = A.box[k];
        const int nb = b.z * b.w;
        const double* pin = A.pin + (int64_t)k * np;
        // passes 2+: the previous model back in (:360-365), and the cutout
        for (int e = lane; e < nb; e += TS) {
            const int i = b.x + e % b.z, j = b.y + e / b.z;
            const int64_t q = (i - 1) + (int64_t)(j - 1) * A.ny;
            double r = __ldcg(A.resid + q);
            if (A.pass > 1) {
                r = r + mp_model(P, A.M, pin, i, j);
                __stcg(A.resid + q, r);
            }
            cpix[e] = r;
            if (civ) civ[e] = (double)ivimg[q];
        }
        team_sync<WPC>();
        const int st = lm_team_fit<double, NP, NF, WPC>(N, pp, L, cpix, civ, b.z, b.w, b.x, b.y, pin, S, red, lane);
        // bookkeeping (:373-401)
        const int64_t s = A.idx[k];
        double* ps = A.psub + (int64_t)k * np;
        if (lane == 0) {
            if (st != 0) {
                A.valid[s] = 0;
                atomicAdd(A.n_failed, 1);
                A.flag[k] = A.pass > 1 ? 1 : 0;
                for (int q = 0; q < np; ++q) ps[q] = pin[q];
            } else {
                const double dof = (double)((int64_t)nb - NF);
                double cov[NF * NF];
                lm_cov_t<NF>(S.A, cov);
                const double f = L.reweighted ? S.cost / dof : 1.0;
                for (int q = 0; q < np; ++q) {
                    A.prm[s * np + q] = S.fv[q];
                    ps[q] = S.fv[q];
                }
                for (int a = 0; a < NF; ++a) A.err[s * np + A.F.idx[a]] = sqrt(fmax(0.0, cov[a + a * NF] * f));
                A.conv[s] = S.conv;
                A.chisq[s] = S.cost / dof;
                A.niter[s] += S.iter;
                A.flag[k] = 2;
            }
        }
        team_sync<WPC>();
        // subtract_star! of the new (or, undoing the add-back, the previous) model
        if (!(st != 0 && A.pass == 1)) {
            double pr[NP];
#pragma unroll
            for (int q = 0; q < NP; ++q) pr[q] = ps[q];
            for (int e = lane; e < nb; e += TS) {
                const int i = b.x + e % b.z, j = b.y + e / b.z;
                const int64_t q = (i - 1) + (int64_t)(j - 1) * A.ny;
                const double r = __ldcg(A.resid + q) - mp_model(P, A.M, pr, i, j);
                __stcg(A.resid + q, r);
                if (A.snap) A.snap[A.snap_off[k] + e] = r;
            }
        } else if (A.snap) {
            for (int e = lane; e < nb; e += TS) {
                const int i = b.x + e % b.z, j = b.y + e / b.z;
                A.snap[A.snap_off[k] + e] = __ldcg(A.resid + (i - 1) + (int64_t)(j - 1) * A.ny);
            }
        }
        __threadfence();
        team_sync<WPC>();
        // release the stars that waited for this one (their chain depth first)
        if (lane == 0) {
            const int lv = ((volatile int32_t*)A.plevel)[k];
            atomicMax(A.counters + 3, lv);
            for (int q = A.succ_start[k]; q < A.succ_start[k + 1]; ++q) atomicMax(&A.plevel[A.succ_list[q]], lv + 1);
            __threadfence();
            for (int q = A.succ_start[k]; q < A.succ_start[k + 1]; ++q) {
                const int u = A.succ_list[q];
                if (atomicSub(&A.indeg[u], 1) == 1) {
                    const int t = atomicAdd(tail, 1);
                    atomicExch(&A.queue[t], u);
                }
            }
        }
        team_sync<WPC>();
    }
}

}  // namespace

void* scratch(cpb_ctx* ctx, const char* name, size_t bytes);

namespace {

LMConst lm_const(const cpb_psf* psf, const cpb_lm_params* P, bool have_iv) {
    if (P->precision != CPB_PREC_FP64) throw ArgError{"only the FP64 precision form is built for fit_star"};
    LMConst L{};
    L.gauss = psf->dev.kind == CPB_PSF_CIRCULAR_GAUSSIAN;
    L.np = L.gauss ? 5 : 4;
    const int bits_g[5] = {CPB_FREE_Y, CPB_FREE_X, CPB_FREE_FWHM, CPB_FREE_FLUX, CPB_FREE_BKG};
    const int bits_i[4] = {CPB_FREE_Y, CPB_FREE_X, CPB_FREE_FLUX, CPB_FREE_BKG};
    const double fix_g[5] = {P->fixed_y, P->fixed_x, P->fixed_fwhm, P->fixed_flux, P->fixed_bkg};
    const double fix_i[4] = {P->fixed_y, P->fixed_x, P->fixed_flux, P->fixed_bkg};
    L.nf = 0;
    for (int q = 0; q < L.np; ++q) {
        L.fixv[q] = L.gauss ? fix_g[q] : fix_i[q];
        if (P->free_mask & (L.gauss ? bits_g[q] : bits_i[q])) L.fidx[L.nf++] = q;
    }
    if (L.nf == 0) throw ArgError{"all model parameters are fixed; nothing to fit"};
    L.damping = P->damping;
    L.max_iter = P->max_iter;
    if (!(P->weight_reset_tol >= 0) && P->reweight != CPB_LOSS_NONE)
        throw ArgError{"`weight_reset_tol` must be non-negative"};
    if (P->reweight < CPB_LOSS_NONE || P->reweight > CPB_LOSS_LOGITDIST) throw ArgError{"unknown IRLS loss"};
    if (P->scale_estimator < CPB_SCALE_AUTO || P->scale_estimator > CPB_SCALE_MSCALE)
        throw ArgError{"unknown IRLS scale estimator"};
    L.irls = P->reweight;
    L.scale = P->scale_estimator;
    L.loss_param = P->loss_param;
    L.scale_value = P->scale_value;
    L.mscale_delta = P->mscale_delta;
    L.mscale_tol = P->mscale_tol;
    L.mscale_max_iter = P->mscale_max_iter;
    L.weight_reset_tol = P->weight_reset_tol;
    // covariance_estimator default (:647-653): known weights only without IRLS
    L.reweighted = P->covariance == CPB_COV_REWEIGHTED ||
                   (P->covariance == CPB_COV_AUTO && (!have_iv || P->reweight != CPB_LOSS_NONE));
    L.x_tol = P->x_tol;
    L.f_tol = P->f_tol;
    L.g_tol = P->g_tol;
    L.lambda_init = P->lambda_init;
    L.lambda_up = P->lambda_up;
    L.lambda_down = P->lambda_down;
    L.lambda_min = P->lambda_min;
    L.lambda_max = P->lambda_max;
    L.min_diagonal = P->min_diagonal;
    return L;
}

// One launch of k_lm over device-resident cutouts; `pix_elems` (the cutout
// pixels in total, for the instrumentation's byte count) may be 0.
// Launch configuration: persistent blocks per SM (1 or 2; 0 = 2) and whether the
// node's samples may be staged in shared memory (-1 = when they fit).  `queue`
// (nullable) is the work-queue counter to use instead of the context's scratch
// one; `st` (nullable) the stream instead of the context's.
struct LMConfig {
    int blocks_per_sm = 0;
    int smem_node = -1;
    int team_warps = 0;  // warps a cutout: 0 = by batch size (1 or 4), else 1 or 4
    bool queue_zeroed = false;  // `queue` is already zero (no reset launch)
    unsigned long long* queue = nullptr;
    cudaStream_t stream = nullptr;
};

void launch_lm(cpb_ctx* ctx, const cpb_psf* psf, const LMConst& L, int64_t n_cut, const int64_t* d_off,
               const int32_t* d_ny, const int32_t* d_nx, const int32_t* d_y1, const int32_t* d_x1, const void* d_pix,
               int32_t eltype, const void* d_iv, const double* d_init, const LMOut& o, int64_t pix_elems,
               const LMConfig& cfg = LMConfig()) {
    const size_t esz = eltype == CPB_F64 ? 8 : 4;
    const double bytes = (double)pix_elems * esz * (d_iv ? 2 : 1) + (double)n_cut * (8 + 16 + 8 * L.np) +
                         (double)n_cut * (8 * L.np + (o.cov ? 8 * L.nf * L.nf : 0) + 4 * 8 + 4 + 4 + 4);
    cudaStream_t st = cfg.stream ? cfg.stream : ctx->stream;
    const bool gauss = psf->dev.kind == CPB_PSF_CIRCULAR_GAUSSIAN;
    if (L.irls != CPB_LOSS_NONE) {
        if (pix_elems <= 0) throw ArgError{"IRLS reweighting needs the cutouts' total pixel count"};
        double* wbuf = (double*)scratch(ctx, "lm_irls_w", sizeof(double) * (size_t)pix_elems);
        double* rbuf = (double*)scratch(ctx, "lm_irls_r", sizeof(double) * (size_t)pix_elems);
        const unsigned blocks = (unsigned)std::min<int64_t>((n_cut * 32 + 255) / 256, (int64_t)ctx->n_sm * 16);
        KernelScope ks_(ctx, "k_lm_irls", bytes);
        if (eltype == CPB_F64)
            k_lm_irls<double><<<blocks, 256, 0, st>>>(n_cut, L, psf->dev, d_off, d_ny, d_nx, d_y1, d_x1,
                                                      (const double*)d_pix, (const double*)d_iv, d_init, wbuf, rbuf, o);
        else
            k_lm_irls<float><<<blocks, 256, 0, st>>>(n_cut, L, psf->dev, d_off, d_ny, d_nx, d_y1, d_x1,
                                                     (const float*)d_pix, (const float*)d_iv, d_init, wbuf, rbuf, o);
        check(cudaGetLastError(), "k_lm_irls");
        return;
    }
    if (gauss || psf->dev.n_nodes == 1) {
        // fast form: compile-time parameter counts, polyphase taps, work queue
        PPNode N{};
        if (!gauss) {
            N.nd = psf->h_nodes[0];
            N.pp = psf->dev.lpp64 + N.nd.lpoff;
            N.plane = N.nd.LPY * N.nd.LPX;
            N.inv_isy = 1.0f / (float)N.nd.isy;
            N.inv_isx = 1.0f / (float)N.nd.isx;
        }
        auto* queue = cfg.queue ? cfg.queue
                                : (unsigned long long*)scratch(ctx, "lm_queue", sizeof(unsigned long long));
        if (!(cfg.queue && cfg.queue_zeroed)) check(cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st), "memset");
        // two persistent 256-thread blocks an SM (128 registers a thread); the
        // node's samples go to shared memory when two copies fit an SM
        const size_t node_bytes = gauss ? 0 : sizeof(double) * (size_t)N.plane * N.nd.isy * N.nd.isx;
        const bool smem = !gauss && node_bytes <= 100 * 1024 && cfg.smem_node != 0;
        const int per_sm = cfg.blocks_per_sm == 1 ? 1 : 2;
        // one warp a cutout while the batch fills the GPU's warps; a batch too
        // small for that (the late batches of fit_all_stars) gets 128-thread
        // teams, which cut each LM iteration's latency instead
        const int64_t warps_total = (int64_t)ctx->n_sm * per_sm * (kLMThreads / 32);
        const int wpc = cfg.team_warps == 4 || cfg.team_warps == 1 ? cfg.team_warps
                                                                  : (n_cut * 4 <= warps_total ? 4 : 1);
        const unsigned blocks = (unsigned)std::min<int64_t>((n_cut * 32 * wpc + kLMThreads - 1) / kLMThreads,
                                                            (int64_t)ctx->n_sm * per_sm);
        KernelScope ks_(ctx, "k_lm", bytes);
#define CPB_LM_LAUNCH_W(TI, NP, NF, W)                                                                             \
    do {                                                                                                          \
        if (smem) {                                                                                               \
            check(cudaFuncSetAttribute(k_lm_t<TI, NP, NF, true, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                       (int)node_bytes),                                                         \
                  "smem attribute");                                                                             \
            k_lm_t<TI, NP, NF, true, W><<<blocks, kLMThreads, node_bytes, st>>>(                                  \
                n_cut, L, N, d_off, d_ny, d_nx, d_y1, d_x1, (const TI*)d_pix, (const TI*)d_iv, d_init, o, queue); \
        } else {                                                                                                  \
            k_lm_t<TI, NP, NF, false, W><<<blocks, kLMThreads, 0, st>>>(                                          \
                n_cut, L, N, d_off, d_ny, d_nx, d_y1, d_x1, (const TI*)d_pix, (const TI*)d_iv, d_init, o, queue); \
        }                                                                                                         \
    } while (0)
#define CPB_LM_LAUNCH(TI, NP, NF)             \
    do {                                      \
        if (wpc == 4)                         \
            CPB_LM_LAUNCH_W(TI, NP, NF, 4);   \
        else                                  \
            CPB_LM_LAUNCH_W(TI, NP, NF, 1);   \
    } while (0)
#define CPB_LM_NF(TI, NP)                          \
    switch (L.nf) {                                \
        case 1: CPB_LM_LAUNCH(TI, NP, 1); break;   \
        case 2: CPB_LM_LAUNCH(TI, NP, 2); break;   \
        case 3: CPB_LM_LAUNCH(TI, NP, 3); break;   \
        case 4: CPB_LM_LAUNCH(TI, NP, 4); break;   \
        default: CPB_LM_LAUNCH(TI, NP, NP); break; \
    }
        if (eltype == CPB_F64) {
            if (gauss) {
                CPB_LM_NF(double, 5)
            } else {
                CPB_LM_NF(double, 4)
            }
        } else {
            if (gauss) {
                CPB_LM_NF(float, 5)
            } else {
                CPB_LM_NF(float, 4)
            }
        }
#undef CPB_LM_NF
#undef CPB_LM_LAUNCH
#undef CPB_LM_LAUNCH_W
        check(cudaGetLastError(), "k_lm");
        return;
    }
    const unsigned blocks = (unsigned)std::min<int64_t>((n_cut * 32 + 255) / 256, (int64_t)ctx->n_sm * 16);
    KernelScope ks_(ctx, "k_lm", bytes);
    if (eltype == CPB_F64)
        k_lm<double><<<blocks, 256, 0, st>>>(n_cut, L, psf->dev, d_off, d_ny, d_nx, d_y1, d_x1,
                                             (const double*)d_pix, (const double*)d_iv, d_init, o);
    else
        k_lm<float><<<blocks, 256, 0, st>>>(n_cut, L, psf->dev, d_off, d_ny, d_nx, d_y1, d_x1, (const float*)d_pix,
                                            (const float*)d_iv, d_init, o);
    check(cudaGetLastError(), "k_lm");
}

}  // namespace

// ---------------------------------------------------------------------------
// A bound batch over fixed device buffers (CUDA-graph capture and tuning)
// ---------------------------------------------------------------------------
struct LMBatch {
    const cpb_psf* psf;
    LMConst L;
    int64_t n_cut;
    const int64_t* off;
    const int32_t *ny, *nx, *y1, *x1;
    const void* pix;
    int32_t eltype;
    const void* iv;
    const double* init;
    LMOut o;
    int64_t pix_elems;
    unsigned long long* queue = nullptr;  // owned
};

LMBatch* lm_batch_create(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* P, int64_t n_cut,
                         const int64_t* d_off, const int32_t* d_ny, const int32_t* d_nx, const int32_t* d_y1,
                         const int32_t* d_x1, const void* d_pix, int32_t eltype, const void* d_iv,
                         const double* d_init, int64_t total_pixels, const cpb_lm_result* out) {
    if (eltype != CPB_F32 && eltype != CPB_F64) throw ArgError{"unsupported pixel eltype"};
    if (n_cut > 0 && (!d_off || !d_ny || !d_nx || !d_y1 || !d_x1 || !d_pix || !d_init || !out || !out->status))
        throw ArgError{"null argument"};
    const LMConst Lc = lm_const(psf, P, d_iv != nullptr);
    if (Lc.irls != CPB_LOSS_NONE) throw ArgError{"IRLS reweighting is not supported in a bound fit_star batch"};
    auto* b = new LMBatch();
    b->psf = psf;
    b->L = Lc;
    b->n_cut = n_cut;
    b->off = d_off;
    b->ny = d_ny;
    b->nx = d_nx;
    b->y1 = d_y1;
    b->x1 = d_x1;
    b->pix = d_pix;
    b->eltype = eltype;
    b->iv = d_iv;
    b->init = d_init;
    if (out)
        b->o = LMOut{out->params, out->cov, out->cost, out->cost_init, out->chisq, out->lambda_final, out->converged,
                     out->x_converged, out->f_converged, out->g_converged, out->iterations, out->status, out->sigma_final};
    b->pix_elems = total_pixels;
    if (cudaMalloc(&b->queue, sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        throw OomError{"device memory exhausted allocating the fit_star work queue"};
    }
    return b;
}

void lm_batch_enqueue(cpb_ctx* ctx, LMBatch* b, cudaStream_t st, int blocks_per_sm, int smem_node) {
    if (b->n_cut <= 0) return;
    LMConfig cfg;
    cfg.blocks_per_sm = blocks_per_sm;
    cfg.smem_node = smem_node;
    cfg.queue = b->queue;
    cfg.stream = st;
    launch_lm(ctx, b->psf, b->L, b->n_cut, b->off, b->ny, b->nx, b->y1, b->x1, b->pix, b->eltype, b->iv, b->init,
              b->o, b->pix_elems, cfg);
}

bool lm_batch_smem_possible(const LMBatch* b) {
    const cpb_psf* psf = b->psf;
    if (psf->dev.kind == CPB_PSF_CIRCULAR_GAUSSIAN || psf->dev.n_nodes != 1) return false;
    const DevNode& nd = psf->h_nodes[0];
    return sizeof(double) * (size_t)nd.LPY * nd.LPX * nd.isy * nd.isx <= 100 * 1024;
}

int64_t lm_batch_size(const LMBatch* b) { return b->n_cut; }

// Tuning signature: what the best launch shape depends on.
std::string lm_batch_signature(const LMBatch* b) {
    char buf[160];
    std::snprintf(buf, sizeof(buf), "fit_star psf%d nodes%d el%d np%d nf%d iv%d n2^%d px/cut%lld", b->psf->dev.kind,
                  b->psf->dev.n_nodes, b->eltype, b->L.np, b->L.nf, b->iv ? 1 : 0,
                  (int)std::log2((double)std::max<int64_t>(b->n_cut, 1)),
                  (long long)(b->pix_elems / std::max<int64_t>(b->n_cut, 1) / 64 * 64));
    return buf;
}

void lm_batch_destroy(LMBatch* b) {
    if (!b) return;
    cudaFree(b->queue);
    delete b;
}

int fit_lm_batch(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* P, int64_t n_cut, const int64_t* offsets,
                 const int32_t* ny, const int32_t* nx, const int32_t* y_origin, const int32_t* x_origin,
                 const void* pixels, int32_t eltype, const void* inv_var, const double* init, cpb_lm_result* out) {
    NvtxRange nv_("cpb:fit_star_batch");
    if (eltype != CPB_F32 && eltype != CPB_F64) throw ArgError{"unsupported pixel eltype"};
    const LMConst L = lm_const(psf, P, inv_var != nullptr);
    if (n_cut <= 0) return 0;
    cudaStream_t st = ctx->stream;
    int64_t total = 0;
    for (int64_t c = 0; c < n_cut; ++c) {
        if (ny[c] <= 0 || nx[c] <= 0) throw ArgError{"cutout dimensions must be positive"};
        if (offsets[c] < 0) throw ArgError{"cutout offsets must be non-negative"};
        total = std::max<int64_t>(total, offsets[c] + (int64_t)ny[c] * nx[c]);
    }
    const size_t esz = eltype == CPB_F64 ? 8 : 4;
    auto up = [&](const char* name, const void* h, size_t bytes) {
        void* d = scratch(ctx, name, std::max<size_t>(bytes, 8));
        check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st), "h2d");
        return d;
    };
    check(cudaEventRecord(ctx->ev0, st), "event");
    const int64_t* d_off = (const int64_t*)up("lm_off", offsets, sizeof(int64_t) * n_cut);
    const int32_t* d_ny = (const int32_t*)up("lm_ny", ny, sizeof(int32_t) * n_cut);
    const int32_t* d_nx = (const int32_t*)up("lm_nx", nx, sizeof(int32_t) * n_cut);
    const int32_t* d_y1 = (const int32_t*)up("lm_y1", y_origin, sizeof(int32_t) * n_cut);
    const int32_t* d_x1 = (const int32_t*)up("lm_x1", x_origin, sizeof(int32_t) * n_cut);
    const double* d_init = (const double*)up("lm_init", init, sizeof(double) * n_cut * L.np);
    char* d_pix = (char*)scratch(ctx, "lm_pix", std::max<size_t>(esz * total, 8));
    char* d_iv = inv_var ? (char*)scratch(ctx, "lm_iv", std::max<size_t>(esz * total, 8)) : nullptr;
    // device outputs: one block, carved in the order of the host fields
    const size_t nd = (size_t)n_cut * (L.np + (out->cov ? L.nf * L.nf : 0) + 4);
    double* dd = (double*)scratch(ctx, "lm_out_f64", sizeof(double) * nd);
    uint8_t* du = (uint8_t*)scratch(ctx, "lm_out_u8", (size_t)n_cut * 4);
    int32_t* di = (int32_t*)scratch(ctx, "lm_out_i32", sizeof(int32_t) * n_cut * 2);
    LMOut o;
    o.params = dd;
    o.cov = out->cov ? dd + n_cut * L.np : nullptr;
    double* sc = dd + n_cut * L.np + (out->cov ? n_cut * L.nf * L.nf : 0);
    o.cost = sc;
    o.cost_init = sc + n_cut;
    o.chisq = sc + 2 * n_cut;
    o.lambda_final = sc + 3 * n_cut;
    o.converged = du;
    o.x_converged = du + n_cut;
    o.f_converged = du + 2 * n_cut;
    o.g_converged = du + 3 * n_cut;
    o.iters = di;
    o.status = di + n_cut;
    o.sigma_final = out->sigma_final ? (double*)scratch(ctx, "lm_out_sigma", sizeof(double) * n_cut) : nullptr;
    // Pixels and weights: when the cutouts are packed in order they go up in
    // chunks on the copy stream, and chunk k is fitted while chunk k + 1 is in
    // flight; otherwise in one piece.
    bool ordered = true;
    for (int64_t c = 1; c < n_cut && ordered; ++c)
        ordered = offsets[c] >= offsets[c - 1] + (int64_t)ny[c - 1] * nx[c - 1];
    const int64_t bytes_all = (int64_t)esz * total * (inv_var ? 2 : 1);
    // (IRLS keeps one launch: its weight / residual scratch is laid out like the whole batch)
    const int K = ordered && L.irls == CPB_LOSS_NONE
                      ? (int)std::min<int64_t>({(int64_t)8, n_cut, std::max<int64_t>(1, bytes_all >> 25)})
                      : 1;
    for (int k = 0; k < K; ++k) {
        const int64_t c0 = n_cut * k / K, c1 = n_cut * (k + 1) / K;
        if (c1 <= c0) continue;
        const int64_t e0 = K == 1 ? 0 : offsets[c0];
        const int64_t e1 = K == 1 ? total : offsets[c1 - 1] + (int64_t)ny[c1 - 1] * nx[c1 - 1];
        cudaStream_t cs = ctx->copy_stream;
        check(cudaMemcpyAsync(d_pix + esz * e0, (const char*)pixels + esz * e0, esz * (e1 - e0),
                              cudaMemcpyHostToDevice, cs), "h2d pixels");
        if (inv_var)
            check(cudaMemcpyAsync(d_iv + esz * e0, (const char*)inv_var + esz * e0, esz * (e1 - e0),
                                  cudaMemcpyHostToDevice, cs), "h2d inv_var");
        cudaEvent_t ev = ctx->copy_ev[k % cpb_ctx::kCopyEvents];
        check(cudaEventRecord(ev, cs), "event");
        check(cudaStreamWaitEvent(st, ev, 0), "wait");
        LMOut ok = o;
        ok.params += c0 * L.np;
        if (ok.cov) ok.cov += c0 * L.nf * L.nf;
        ok.cost += c0;
        ok.cost_init += c0;
        ok.chisq += c0;
        ok.lambda_final += c0;
        ok.converged += c0;
        ok.x_converged += c0;
        ok.f_converged += c0;
        ok.g_converged += c0;
        ok.iters += c0;
        ok.status += c0;
        if (ok.sigma_final) ok.sigma_final += c0;
        launch_lm(ctx, psf, L, c1 - c0, d_off + c0, d_ny + c0, d_nx + c0, d_y1 + c0, d_x1 + c0, d_pix, eltype,
                  d_iv, d_init + c0 * L.np, ok, e1 - e0);
    }
    check(cudaEventRecord(ctx->ev1, st), "event");
    auto down = [&](void* h, const void* d, size_t bytes) {
        if (h) check(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st), "d2h");
    };
    down(out->params, o.params, sizeof(double) * n_cut * L.np);
    down(out->cov, o.cov, sizeof(double) * n_cut * L.nf * L.nf);
    double* hs[4] = {out->cost, out->cost_init, out->chisq, out->lambda_final};
    for (int k = 0; k < 4; ++k) down(hs[k], sc + k * n_cut, sizeof(double) * n_cut);
    uint8_t* hf[4] = {out->converged, out->x_converged, out->f_converged, out->g_converged};
    for (int k = 0; k < 4; ++k) down(hf[k], du + k * n_cut, (size_t)n_cut);
    down(out->iterations, o.iters, sizeof(int32_t) * n_cut);
    down(out->status, o.status, sizeof(int32_t) * n_cut);
    down(out->sigma_final, o.sigma_final, sizeof(double) * n_cut);
    check(cudaStreamSynchronize(st), "sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    out->device_seconds = ms * 1e-3;
    return 0;
}

void lm_enqueue_device(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* P, int64_t n_cut, const int64_t* d_off,
                       const int32_t* d_ny, const int32_t* d_nx, const int32_t* d_y1, const int32_t* d_x1,
                       const void* d_pix, int32_t eltype, const void* d_iv, const double* d_init, int64_t total_pixels,
                       const cpb_lm_result* out, int team_warps, unsigned long long* zeroed_queue) {
    const LMConst L = lm_const(psf, P, d_iv != nullptr);
    if (n_cut <= 0) return;
    LMOut o{out->params, out->cov, out->cost, out->cost_init, out->chisq, out->lambda_final, out->converged,
            out->x_converged, out->f_converged, out->g_converged, out->iterations, out->status, out->sigma_final};
    LMConfig cfg;
    cfg.team_warps = team_warps;
    cfg.queue = zeroed_queue;
    cfg.queue_zeroed = zeroed_queue != nullptr;
    launch_lm(ctx, psf, L, n_cut, d_off, d_ny, d_nx, d_y1, d_x1, d_pix, eltype, d_iv, d_init, o, total_pixels, cfg);
}

int fit_lm_batch_device(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* P, int64_t n_cut,
                        const int64_t* d_off, const int32_t* d_ny, const int32_t* d_nx, const int32_t* d_y1,
                        const int32_t* d_x1, const void* d_pix, int32_t eltype, const void* d_iv,
                        const double* d_init, int64_t total_pixels, cpb_lm_result* out) {
    if (eltype != CPB_F32 && eltype != CPB_F64) throw ArgError{"unsupported pixel eltype"};
    const LMConst L = lm_const(psf, P, d_iv != nullptr);
    if (n_cut <= 0) return 0;
    LMOut o{out->params, out->cov, out->cost, out->cost_init, out->chisq, out->lambda_final, out->converged,
            out->x_converged, out->f_converged, out->g_converged, out->iterations, out->status, out->sigma_final};
    cudaStream_t st = ctx->stream;
    check(cudaEventRecord(ctx->ev0, st), "event");
    launch_lm(ctx, psf, L, n_cut, d_off, d_ny, d_nx, d_y1, d_x1, d_pix, eltype, d_iv, d_init, o, total_pixels);
    check(cudaEventRecord(ctx->ev1, st), "event");
    check(cudaStreamSynchronize(st), "sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    out->device_seconds = ms * 1e-3;
    return 0;
}


bool mp_dag_supported(const cpb_psf* psf, const cpb_lm_params* P) {
    const bool gauss = psf->dev.kind == CPB_PSF_CIRCULAR_GAUSSIAN;
    return (gauss || psf->dev.n_nodes == 1) && P->reweight == CPB_LOSS_NONE && P->precision == CPB_PREC_FP64;
}

int mp_dag_teams(cpb_ctx* ctx) { return ctx->n_sm * 2 * (kLMThreads / (32 * kDagWarps)); }

void mp_dag_launch(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* P, int32_t iv_eltype,
                   const DagArgs& A_in) {
    DagArgs A = A_in;
    A.spin_limit = ctx->wait_limit > 0 ? (long long)ctx->wait_limit : kDagSpinLimit;
    const LMConst L = lm_const(psf, P, A.iv != nullptr);
    cudaStream_t st = ctx->stream;
    const bool gauss = psf->dev.kind == CPB_PSF_CIRCULAR_GAUSSIAN;
    PPNode N{};
    if (!gauss) {
        N.nd = psf->h_nodes[0];
        N.pp = psf->dev.lpp64 + N.nd.lpoff;
        N.plane = N.nd.LPY * N.nd.LPX;
        N.inv_isy = 1.0f / (float)N.nd.isy;
        N.inv_isx = 1.0f / (float)N.nd.isx;
    }
    const size_t node_bytes = gauss ? 0 : sizeof(double) * (size_t)N.plane * N.nd.isy * N.nd.isx;
    const bool smem = !gauss && node_bytes <= 100 * 1024;
    const unsigned blocks = (unsigned)(ctx->n_sm * 2);  // persistent: every team resident
    KernelScope ks_(ctx, "k_mp_dag", 0.0);
#define CPB_DAG(TIV, NP, NF)                                                                                    \
    do {                                                                                                        \
        if (smem) {                                                                                             \
            check(cudaFuncSetAttribute(k_mp_dag<TIV, NP, NF, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                       (int)node_bytes),                                                       \
                  "smem attribute");                                                                           \
            k_mp_dag<TIV, NP, NF, true><<<blocks, kLMThreads, node_bytes, st>>>(L, N, psf->dev, A);             \
        } else {                                                                                                \
            k_mp_dag<TIV, NP, NF, false><<<blocks, kLMThreads, 0, st>>>(L, N, psf->dev, A);                     \
        }                                                                                                       \
    } while (0)
#define CPB_DAG_NF(TIV, NP)                     \
    switch (L.nf) {                             \
        case 1: CPB_DAG(TIV, NP, 1); break;     \
        case 2: CPB_DAG(TIV, NP, 2); break;     \
        case 3: CPB_DAG(TIV, NP, 3); break;     \
        case 4: CPB_DAG(TIV, NP, 4); break;     \
        default: CPB_DAG(TIV, NP, NP); break;   \
    }
    if (iv_eltype == CPB_F64) {
        if (gauss) {
            CPB_DAG_NF(double, 5)
        } else {
            CPB_DAG_NF(double, 4)
        }
    } else {
        if (gauss) {
            CPB_DAG_NF(float, 5)
        } else {
            CPB_DAG_NF(float, 4)
        }
    }
#undef CPB_DAG_NF
#undef CPB_DAG
    check(cudaGetLastError(), "k_mp_dag");
}

}  // namespace cpb
