// cpb_groups.cu -- many small simultaneous fits in one persistent launch.
//
// A "group" is a small field holding a blend of a few stars; each group is an
// independent fit_all_stars_simultaneous call
// (src/photometry/psf_photometry_simultaneous.jl:953-1431).  One thread
// block owns one group for the whole fit and keeps every working array of it
// in shared memory:
//
//   * the union U of the stars' fit-box pixels (_touched_pixels, :329-335),
//     sorted in the group image's column-major order, with data_work, w, the
//     weighted residual and the LSQR u vector per pixel of U -- the reference's
//     npix-long vectors are zero outside U, so nothing else is kept;
//   * per pixel of U, bit masks of the (Morton-ordered) active stars whose fit
//     box and model box contain it.  J v, the renders and the frozen-star
//     subtraction are gathers over those bits in ascending (Morton) order,
//     which is the order in which the reference's scatter-adds reach the pixel
//     (apply_J! :95-137, _render_model! :545-673, _freeze_star! :739-754);
//   * the stamp derivatives V (StampDerivatives, :19-43) with, per stamp
//     entry, its index in U (0 = unusable entry, as the reference's pixel 0);
//   * per star the solver state (theta, colnorm, D, b, LSQR x / v / w).
//
// Renders are evaluated only on U: the residual, cost and data_work are read
// only there (_residual_cost! :675-684, _cost! :686-693), so values of the
// model boxes outside U never influence the fit.  The final residual image
// and the diagnostics evaluate the full model boxes.  Blocks take groups from
// a device work queue (an atomic counter), so groups of uneven size share the
// GPU without a host round trip.  All reductions use a fixed order (results
// are bitwise reproducible run to run); the host never reads anything back
// until the batch is done.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "cpb_internal.cuh"
#include "cpb_linalg.cuh"

namespace cpb {

namespace {

constexpr double kEpsG = 2.220446049250313e-16;
constexpr int kMaxGroupStars = 64;
constexpr int kNoU = 0x7fffffff;

struct GroupConst {
    int p;
    int gc[3];     // grad_col of free parameter k (1 = dy, 2 = dx, 3 = dflux)
    int ky, kx;    // position of y / x in the free list, -1 if fixed
    double fixed_y, fixed_x, fixed_flux, fixed_bkg;
    int R, S, S2;  // fit box
    int mR;        // model radius (scalar model_rad)
    int nmax;      // star capacity of the shared-memory layout
    int umax;      // union-pixel capacity
    int keyn;      // power-of-two key buffer for the union sort (>= nmax * S2)
    int max_iter, max_trials, itmax;
    double linear_tol, max_step, x_tol, f_tol, g_tol;
    double lambda_init, lambda_up, lambda_down, lambda_min, lambda_max;
    int eltype;
    int reweighted;
    double fit_rad;
    // spread_model: on when requested and its disk width is NaN (derived per
    // group) or finite and positive; the disk table length and the fit box
    // capacity ((2 R + 2)^2 pixels)
    int sp_on, sp_tab, sp_box;
    double sp_param;     // spread_model_fwhm (NaN: _spread_fwhm of the group's first star)
    double sp_psf_fwhm;  // the PSF object's own FWHM, which _spread_fwhm renders
};

struct GroupIn {
    const int64_t* pix_off;
    const int32_t* ny;
    const int32_t* nx;
    const void* pix;
    const void* iv;   // nullable
    const void* bkg;  // nullable
    const int64_t* star_off;
    const double *y0, *x0, *f0;
};

struct GroupOut {
    double *y, *x, *flux, *y_err, *x_err, *flux_err;
    uint8_t *converged, *valid;
    int32_t* n_iter;
    double *chisq, *qfit, *qfit_expected, *qfit_z, *crowding;
    double* residual;
    int32_t *n_passes, *n_failed, *status, *error_kind, *n_active, *n_union, *n_trials, *n_lsqr;
    double *spread, *spread_err;
    double* sp_rw;          // per star: residual and weight over its box, 2 sp_box doubles (spread_model)
    const double* sp_rule;  // kSpreadRuleLen doubles (spread_rule)
};

// Byte offsets of the shared-memory layout (same computation on host and device).
struct Layout {
    size_t coef, coefc, theta, delta, dsc, cn, D, bsc, xl, vt, wl;
    size_t ay, ax, act, frozen, live, conv, newf;
    size_t V, uidx;
    size_t dw, w, wr, u, upix, fmask, mmask;
    size_t total;
};

__host__ __device__ inline size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

template <typename MaskT>
__host__ __device__ inline Layout make_layout(int nmax, int S2, int umax, int keyn) {
    Layout L;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        size_t at = o;
        o = align16(o + bytes);
        return at;
    };
    const size_t np = (size_t)3 * nmax;
    L.coef = take(sizeof(StarCoef) * nmax);
    L.coefc = take(sizeof(StarCoef) * nmax);
    L.theta = take(8 * np);
    L.delta = take(8 * np);
    L.dsc = take(8 * np);
    L.cn = take(8 * np);
    L.D = take(8 * np);
    L.bsc = take(8 * np);
    L.xl = take(8 * np);
    L.vt = take(8 * np);
    L.wl = take(8 * np);
    L.ay = take(4 * nmax);
    L.ax = take(4 * nmax);
    L.act = take(4 * nmax);
    L.frozen = take(4 * nmax);
    L.live = take(nmax);
    L.conv = take(nmax);
    L.newf = take(nmax);
    // V doubles as the key buffer of the union sort (keyn int32 <= 3 * 8 * nmax * S2 bytes)
    size_t vbytes = (size_t)24 * nmax * S2;
    if (vbytes < (size_t)4 * keyn) vbytes = (size_t)4 * keyn;
    L.V = take(vbytes);
    L.uidx = take((size_t)4 * nmax * S2);
    L.dw = take((size_t)8 * umax);
    L.w = take((size_t)8 * umax);
    L.wr = take((size_t)8 * umax);
    L.u = take((size_t)8 * umax);
    L.upix = take((size_t)4 * umax);
    L.fmask = take(sizeof(MaskT) * umax);
    L.mmask = take(sizeof(MaskT) * umax);
    L.total = o;
    return L;
}

__device__ __forceinline__ uint64_t spread_bits(uint64_t v) {
    v &= 0x00000000ffffffffULL;
    v = (v | (v << 16)) & 0x0000ffff0000ffffULL;
    v = (v | (v << 8)) & 0x00ff00ff00ff00ffULL;
    v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0fULL;
    v = (v | (v << 2)) & 0x3333333333333333ULL;
    v = (v | (v << 1)) & 0x5555555555555555ULL;
    return v;
}

// Block-wide sum / max whose result every thread receives.  `buf` alternates
// between two 32-entry halves so that consecutive reductions need one barrier each.
template <int NT>
__device__ __forceinline__ double block_allsum(double v, double* sh, int& flip) {
    double* b = sh + 32 * (flip & 1);
    ++flip;
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) b[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
#pragma unroll
    for (int k = 0; k < NT / 32; ++k) r += b[k];
    return r;
}
template <int NT>
__device__ __forceinline__ double block_allmax(double v, double* sh, int& flip) {
    double* b = sh + 32 * (flip & 1);
    ++flip;
    v = warp_max(v);
    if ((threadIdx.x & 31) == 0) b[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
#pragma unroll
    for (int k = 0; k < NT / 32; ++k) r = nan_max(r, b[k]);
    return r;
}

template <typename MaskT>
__device__ __forceinline__ int next_bit(MaskT& m) {
    int a;
    if (sizeof(MaskT) == 8) a = __ffsll((long long)m) - 1;
    else a = __ffs((int)m) - 1;
    m &= m - 1;
    return a;
}

// Per-group view of the inputs.
struct GView {
    GroupIn in;
    int eltype;
    int64_t off;
    int ny, nx;
    __device__ double ld(const void* p, int64_t q) const {
        return eltype == CPB_F64 ? ((const double*)p)[off + q] : (double)((const float*)p)[off + q];
    }
    // sanitised data (image - background; non-finite -> 0) and weight (:1056-1084)
    __device__ void data_w(int64_t q, double& d, double& w) const {
        d = ld(in.pix, q) - (in.bkg ? ld(in.bkg, q) : 0.0);
        if (in.iv) {
            const double v = ld(in.iv, q);
            w = (isfinite(v) && v > 0) ? v : 0.0;
        } else {
            w = 1.0;
        }
        if (!isfinite(d)) {
            d = 0.0;
            w = 0.0;
        }
    }
};

__device__ __forceinline__ double psf_value(const DevPsf& P, const StarCoef& c, int gy, int gx) {
    return model_value<double, double>(P, P.data64, c, (double)gy, (double)gx);
}
__device__ __forceinline__ void psf_grad(const DevPsf& P, const StarCoef& c, int gy, int gx, double* g) {
    model_grad<double, double>(P, P.data64, c, (double)gy, (double)gx, g);
}

template <int NT, typename MaskT>
struct GroupFit {
    const GroupConst& C;
    const DevPsf& P;
    const GroupOut& O;
    GView G;
    char* smem;
    Layout L;
    double* sh;       // 64 doubles of reduction scratch
    int flip = 0;
    int n_act = 0, nU = 0;

    __device__ StarCoef* coef() const { return (StarCoef*)(smem + L.coef); }
    __device__ StarCoef* coefc() const { return (StarCoef*)(smem + L.coefc); }
    __device__ double* dp(size_t o) const { return (double*)(smem + o); }
    __device__ int32_t* ip(size_t o) const { return (int32_t*)(smem + o); }
    __device__ uint8_t* bp(size_t o) const { return (uint8_t*)(smem + o); }
    __device__ MaskT* mp(size_t o) const { return (MaskT*)(smem + o); }

    // model_from_vector (psf_fitting.jl:23-26) for active slot a at theta (+ delta).
    __device__ void make_coef(int a, const double* th, const double* dl, StarCoef& c) const {
        c.y = C.fixed_y;
        c.x = C.fixed_x;
        c.flux = C.fixed_flux;
        c.bkg = C.fixed_bkg;
        for (int k = 0; k < C.p; ++k) {
            double v = th[a * C.p + k];
            if (dl) v = v + dl[a * C.p + k];
            if (C.gc[k] == 1) c.y = v;
            else if (C.gc[k] == 2) c.x = v;
            else c.flux = v;
        }
        grid_corners_dw(P, c.y, c.x, c);
    }
    __device__ double mval(const StarCoef& c, int gy, int gx) const { return psf_value(P, c, gy, gx); }
    __device__ void uxy(int u, int& gy, int& gx) const {
        const int q = ip(L.upix)[u];
        gy = q % G.ny + 1;
        gx = q / G.ny + 1;
    }

    // coef[a] for every active slot at theta (+ delta into coefc).
    __device__ void coefs(bool cand) {
        const double* th = dp(L.theta);
        for (int a = threadIdx.x; a < n_act; a += NT) {
            StarCoef c;
            make_coef(a, th, cand ? dp(L.delta) : nullptr, c);
            (cand ? coefc() : coef())[a] = c;
        }
        __syncthreads();
    }

    // _fill_stamps! (:342-543) for the live stars (all when `all`); with `gram`
    // the per-star p x p Gram block of the raw columns is written instead of V
    // (errors pass, :1302-1329).  One warp per star.
    __device__ void fill(bool all, double* gram) {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const int p = C.p, S = C.S, S2 = C.S2, R = C.R;
        double* V = dp(L.V);
        const int32_t* ui = ip(L.uidx);
        const double* w = dp(L.w);
        double* cn = dp(L.cn);
        const uint8_t* live = bp(L.live);
        const StarCoef* cf = coef();
        for (int a = wid; a < n_act; a += NT / 32) {
            if (!all && !live[a]) continue;
            const StarCoef c = cf[a];
            const int ay = ip(L.ay)[a], ax = ip(L.ax)[a];
            double s0 = 0, s1 = 0, s2 = 0, g01 = 0, g02 = 0, g12 = 0;
            for (int m = lane; m < S2; m += 32) {
                const int u = ui[a * S2 + m];
                if (u == kNoU) continue;
                const int gy = ay + (m % S) - R, gx = ax + (m / S) - R;
                double g[3];
                psf_grad(P, c, gy, gx, g);
                const double swv = sqrt(w[u]);
                double r[3] = {0, 0, 0};
                for (int k = 0; k < p; ++k) r[k] = swv * g[C.gc[k] - 1];
                if (!gram)
                    for (int k = 0; k < p; ++k) V[(a * S2 + m) * p + k] = r[k];
                s0 += r[0] * r[0];
                s1 += r[1] * r[1];
                s2 += r[2] * r[2];
                g01 += r[0] * r[1];
                g02 += r[0] * r[2];
                g12 += r[1] * r[2];
            }
            s0 = warp_sum(s0);
            s1 = warp_sum(s1);
            s2 = warp_sum(s2);
            if (gram) {
                g01 = warp_sum(g01);
                g02 = warp_sum(g02);
                g12 = warp_sum(g12);
                if (lane == 0) {
                    double* gr = gram + a * 6;
                    gr[0] = s0;
                    gr[1] = g01;
                    gr[2] = g02;
                    gr[3] = s1;
                    gr[4] = g12;
                    gr[5] = s2;
                }
                continue;
            }
            const double ss[3] = {s0, s1, s2};
            double inv[3];
            for (int k = 0; k < p; ++k) {
                double cv = sqrt(ss[k]);
                cv = cv < kEpsG ? kEpsG : cv;
                inv[k] = 1.0 / cv;
                if (lane == 0) cn[a * p + k] = cv;
            }
            for (int m = lane; m < S2; m += 32) {
                if (ui[a * S2 + m] == kNoU) continue;
                for (int k = 0; k < p; ++k) V[(a * S2 + m) * p + k] *= inv[k];
            }
        }
        __syncthreads();
    }

    // Model render on U for the stars in `sel` (bit a = active slot a):
    // mode 0: weighted residual wr = sqrt(w) (model - data_work) and its cost;
    // mode 1: candidate cost sum w (model - data_work)^2 at coefc;
    // mode 2: data_work -= model (frozen-star subtraction).
    __device__ double render(int mode, MaskT sel) {
        const StarCoef* cf = mode == 1 ? coefc() : coef();
        const MaskT* mm = mp(L.mmask);
        double* dw = dp(L.dw);
        const double* w = dp(L.w);
        double* wr = dp(L.wr);
        double part = 0.0;
        for (int u = threadIdx.x; u < nU; u += NT) {
            int gy, gx;
            uxy(u, gy, gx);
            MaskT m = mm[u] & sel;
            if (mode == 2) {
                double d = dw[u];
                while (m) d -= mval(cf[next_bit(m)], gy, gx);
                dw[u] = d;
                continue;
            }
            double acc = 0.0;
            while (m) acc += mval(cf[next_bit(m)], gy, gx);
            const double r = acc - dw[u];
            if (mode == 0) {
                const double v = sqrt(w[u]) * r;
                wr[u] = v;
                part += v * v;
            } else {
                part += w[u] * r * r;
            }
        }
        if (mode == 2) {
            __syncthreads();
            return 0.0;
        }
        return block_allsum<NT>(part, sh, flip);
    }

    // z = J^T src * scale for the live stars (apply_JT!, :55-85), one warp per
    // star.  LSQR form: v_new = z - beta v_old / alpha, returns ||v_new||^2.
    __device__ double jt(const double* src, double scale, bool lsqr, double beta, double inv_alpha, double* z) {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const int p = C.p, S2 = C.S2;
        const double* V = dp(L.V);
        const int32_t* ui = ip(L.uidx);
        const uint8_t* live = bp(L.live);
        double part = 0.0;
        for (int a = wid; a < n_act; a += NT / 32) {
            if (!live[a]) continue;
            double z0 = 0, z1 = 0, z2 = 0;
            for (int m = lane; m < S2; m += 32) {
                const int u = ui[a * S2 + m];
                if (u == kNoU) continue;
                const double uv = lsqr ? src[u] * scale : src[u];
                const double* v = V + (a * S2 + m) * p;
                z0 += v[0] * uv;
                if (p > 1) z1 += v[1] * uv;
                if (p > 2) z2 += v[2] * uv;
            }
            z0 = warp_sum(z0);
            z1 = warp_sum(z1);
            z2 = warp_sum(z2);
            if (lane == 0) {
                for (int k = 0; k < p; ++k) {
                    double val = k == 0 ? z0 : (k == 1 ? z1 : z2);
                    if (lsqr) {
                        val = val - beta * (z[a * p + k] * inv_alpha);
                        part += val * val;
                    }
                    z[a * p + k] = val;
                }
            }
        }
        if (!lsqr) {
            __syncthreads();
            return 0.0;
        }
        return block_allsum<NT>(part, sh, flip);
    }

    // u_new = J v / alpha - alpha u_old (apply_J!, :95-137, gathered per pixel of
    // U in Morton order); u_old = src * uscale.  Returns ||u_new||^2.
    __device__ double jv(const double* src, double uscale, double alpha, double inv_alpha, MaskT live_bits) {
        const int p = C.p, S = C.S, S2 = C.S2, R = C.R;
        const double* V = dp(L.V);
        const double* vt = dp(L.vt);
        const MaskT* fm = mp(L.fmask);
        const int32_t* ay = ip(L.ay);
        const int32_t* ax = ip(L.ax);
        double* uu = dp(L.u);
        double part = 0.0;
        for (int u = threadIdx.x; u < nU; u += NT) {
            int gy, gx;
            uxy(u, gy, gx);
            MaskT m = fm[u] & live_bits;
            double acc = 0.0;
            while (m) {
                const int a = next_bit(m);
                const int mi = (gy - ay[a] + R) + (gx - ax[a] + R) * S;
                const double* v = V + (a * S2 + mi) * p;
                double t = v[0] * (vt[a * p] * inv_alpha);
                if (p > 1) t += v[1] * (vt[a * p + 1] * inv_alpha);
                if (p > 2) t += v[2] * (vt[a * p + 2] * inv_alpha);
                acc += t;
            }
            const double un = acc - alpha * (src[u] * uscale);
            uu[u] = un;
            part += un * un;
        }
        return block_allsum<NT>(part, sh, flip);
    }

    // Damped LSQR (Paige & Saunders 1982, Krylov.jl 0.10 stopping rules) on
    // min ||J d + r||^2 + lambda ||d||^2, right-hand side -wr, zero start.
    // Returns the iterations run.
    __device__ int lsqr(double cost, double lam, MaskT live_bits) {
        const int n = n_act * C.p;
        double* xl = dp(L.xl);
        double* vt = dp(L.vt);
        double* wl = dp(L.wl);
        const double* bsc = dp(L.bsc);
        const double beta1 = sqrt(cost);
        for (int i = threadIdx.x; i < n; i += NT) xl[i] = 0.0;
        if (beta1 == 0.0) {
            __syncthreads();
            return 0;
        }
        const double inv_b1 = 1.0 / beta1;
        // v1 = A'u1 = -b / beta1 (the gradient pass already holds A'r)
        double part = 0.0;
        for (int i = threadIdx.x; i < n; i += NT) {
            const double v = -(bsc[i] * inv_b1);
            vt[i] = v;
            part += v * v;
        }
        const double a2 = block_allsum<NT>(part, sh, flip);
        double alpha = sqrt(a2);
        if (alpha == 0.0) return 0;
        double inv_alpha = 1.0 / alpha;
        {
            const double t = (alpha * beta1) / (alpha * beta1);
            if (t <= 1.4901161193847656e-08 || 1.0 + t <= 1.0) return 0;
        }
        part = 0.0;
        for (int i = threadIdx.x; i < n; i += NT) {
            const double v = vt[i] * inv_alpha;
            wl[i] = v;
            part += v * v;
        }
        double wnorm2 = block_allsum<NT>(part, sh, flip);
        const double lambda = sqrt(lam);
        double Anorm2 = a2, dNorm2 = 0, xNorm2 = 0, c2 = -1, s2 = 0, z = 0, xENorm2 = 0, res2 = 0;
        double rhobar = alpha, phibar = beta1, inv_beta = inv_b1, beta = beta1;
        double err_vec[5] = {0, 0, 0, 0, 0};
        const double atol = C.linear_tol, btol = C.linear_tol;
        const double axtol = 1.4901161193847656e-08, etol = axtol, ctol = axtol;
        int iter = 0;
        for (int it = 0; it < C.itmax; ++it) {
            // beta u = A v - alpha u
            const double b2 = jv(it == 0 ? dp(L.wr) : dp(L.u), (it == 0 ? -1.0 : 1.0) * inv_beta, alpha, inv_alpha,
                                 live_bits);
            beta = sqrt(b2);
            if (beta != 0.0) {
                inv_beta = 1.0 / beta;
                Anorm2 = Anorm2 + alpha * alpha + beta * beta;
                if (lambda > 0) Anorm2 += lambda * lambda;
                // alpha v = A'u - beta v
                const double an2 = jt(dp(L.u), inv_beta, true, beta, inv_alpha, vt);
                alpha = sqrt(an2);
                inv_alpha = alpha != 0.0 ? 1.0 / alpha : 0.0;
            }
            double c1, s1, rhobar1;
            sym_givens(rhobar, lambda, c1, s1, rhobar1);
            const double psi = s1 * phibar;
            phibar = c1 * phibar;
            double c, s, rho;
            sym_givens(rhobar1, beta, c, s, rho);
            const double phi = c * phibar;
            phibar = s * phibar;
            const double theta = s * alpha;
            const double sigma = phi / rho, tr = -theta / rho;
            part = 0.0;
            for (int i = threadIdx.x; i < n; i += NT) {
                const double wi = wl[i];
                xl[i] = xl[i] + sigma * wi;
                const double wn = vt[i] * inv_alpha + tr * wi;
                wl[i] = wn;
                part += wn * wn;
            }
            const double wn2 = block_allsum<NT>(part, sh, flip);
            iter += 1;
            xENorm2 = xENorm2 + phi * phi;
            err_vec[iter % 5] = phi;
            double err_lbnd = 0;
            if (iter >= 5) {
                double e2 = 0;
                for (int k = 0; k < 5; ++k) e2 += err_vec[k] * err_vec[k];
                err_lbnd = sqrt(e2);
            }
            const double tau = s * phi;
            dNorm2 = dNorm2 + wnorm2 / (rho * rho);
            const double delta = s2 * rho;
            const double gambar = -c2 * rho;
            const double rhs = phi - delta * z;
            const double zbar = rhs / gambar;
            const double xNorm = sqrt(xNorm2 + zbar * zbar);
            double gamma;
            sym_givens(gambar, theta, c2, s2, gamma);
            z = rhs / gamma;
            xNorm2 = xNorm2 + z * z;
            const double Anorm = sqrt(Anorm2);
            const double Acond = Anorm * sqrt(dNorm2);
            const double res1 = phibar * phibar;
            res2 = res2 + psi * psi;
            const double rNorm = sqrt(res1 + res2);
            const double ArNorm = alpha * fabs(tau);
            const double test1 = rNorm / beta1;
            const double test2 = ArNorm / (Anorm * rNorm);
            const double test3 = 1.0 / Acond;
            const double t1 = test1 / (1.0 + Anorm * xNorm / beta1);
            const double rNormtol = btol + axtol * Anorm * xNorm / beta1;
            const bool ill = (1.0 + test3 <= 1.0) || (test3 <= ctol);
            const bool zr = (1.0 + t1 <= 1.0) || (test1 <= rNormtol);
            const bool fwd = iter >= 5 && err_lbnd <= etol * sqrt(xENorm2);
            const bool solved = (1.0 + test2 <= 1.0) || (test2 <= axtol) || (ArNorm <= atol) || zr || fwd;
            rhobar = -c * alpha;
            wnorm2 = wn2;
            if (solved || ill || iter >= C.itmax) break;
        }
        return iter;
    }
};

template <int NT, typename MaskT>
__global__ void __launch_bounds__(NT) k_groups(GroupConst C, DevPsf P, GroupIn in, GroupOut O,
                                               const int32_t* __restrict__ glist, int nlist, int* queue) {
    extern __shared__ __align__(16) char smem[];
    __shared__ double sh[64];
    __shared__ int s_g;
    __shared__ double s_gram[kMaxGroupStars * 6];
    __shared__ uint64_t s_key[kMaxGroupStars];
    __shared__ int s_ay0[kMaxGroupStars], s_ax0[kMaxGroupStars];
    __shared__ uint8_t s_ok[kMaxGroupStars];
    const double NaN = __longlong_as_double(0x7ff8000000000000LL);
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    GroupFit<NT, MaskT> F{C, P, O};
    F.smem = smem;
    F.L = make_layout<MaskT>(C.nmax, C.S2, C.umax, C.keyn);
    F.sh = sh;
    F.G.in = in;
    F.G.eltype = C.eltype;
    const int p = C.p, S = C.S, S2 = C.S2, R = C.R;
    for (;;) {
        if (tid == 0) s_g = atomicAdd(queue, 1);
        __syncthreads();
        const int li = s_g;
        __syncthreads();
        if (li >= nlist) break;
        const int g = glist[li];
        const int64_t soff = in.star_off[g];
        const int ng = (int)(in.star_off[g + 1] - soff);
        F.G.off = in.pix_off[g];
        F.G.ny = in.ny[g];
        F.G.nx = in.nx[g];
        const int ny = F.G.ny, nx = F.G.nx;
        const int64_t npix = (int64_t)ny * nx;
        const double* y0 = in.y0 + soff;
        const double* x0 = in.x0 + soff;
        const double* f0 = in.f0 + soff;
        // outputs that hold the catalogue (failed / empty groups, inactive stars)
        auto write_catalogue = [&](int i) {
            const int64_t o = soff + i;
            O.y[o] = y0[i];
            O.x[o] = x0[i];
            O.flux[o] = f0[i];
            O.y_err[o] = NaN;
            O.x_err[o] = NaN;
            O.flux_err[o] = NaN;
            O.converged[o] = 0;
            O.valid[o] = 0;
            O.n_iter[o] = 0;
            if (O.chisq) O.chisq[o] = 0.0;
            if (O.qfit) O.qfit[o] = NaN;
            if (O.qfit_expected) O.qfit_expected[o] = NaN;
            if (O.qfit_z) O.qfit_z[o] = NaN;
            if (O.crowding) O.crowding[o] = NaN;
            if (O.spread) O.spread[o] = NaN;
            if (O.spread_err) O.spread_err[o] = NaN;
        };
        auto fixed_fix = [&](int64_t o) {  // fixed parameters take the fixed values, error 0
            bool fy = false, fx = false, ff = false;
            for (int k = 0; k < p; ++k) {
                fy |= C.gc[k] == 1;
                fx |= C.gc[k] == 2;
                ff |= C.gc[k] == 3;
            }
            if (!fy) {
                O.y[o] = C.fixed_y;
                O.y_err[o] = 0.0;
            }
            if (!fx) {
                O.x[o] = C.fixed_x;
                O.x_err[o] = 0.0;
            }
            if (!ff) {
                O.flux[o] = C.fixed_flux;
                O.flux_err[o] = 0.0;
            }
        };
        auto zero_residual = [&]() {
            if (O.residual)
                for (int64_t q = tid; q < npix; q += NT) O.residual[F.G.off + q] = 0.0;
        };
        auto group_stats = [&](int passes, int failed, int status, int kind, int nact, int nun, int ntr, int nls) {
            if (tid != 0) return;
            O.n_passes[g] = passes;
            O.n_failed[g] = failed;
            O.status[g] = status;
            if (O.error_kind) O.error_kind[g] = kind;
            if (O.n_active) O.n_active[g] = nact;
            if (O.n_union) O.n_union[g] = nun;
            if (O.n_trials) O.n_trials[g] = ntr;
            if (O.n_lsqr) O.n_lsqr[g] = nls;
        };
        auto fail_group = [&](int kind) {
            for (int i = tid; i < ng; i += NT) {
                write_catalogue(i);
                fixed_fix(soff + i);
            }
            zero_residual();
            group_stats(0, ng, CPB_ERR_ARGUMENT, kind, 0, 0, 0, 0);
            __syncthreads();
        };
        if (ng == 0) {
            zero_residual();
            group_stats(0, 0, 0, 0, 0, 0, 0, 0);
            __syncthreads();
            continue;
        }
        if (ng > C.nmax || ng > kMaxGroupStars) {  // the host routes such groups elsewhere
            group_stats(0, ng, CPB_ERR_INTERNAL, 0, 0, 0, 0, 0);
            __syncthreads();
            continue;
        }
        // ---- non-finite data without inv_var is an ArgumentError (:1065-1072)
        if (!in.iv) {
            int bad = 0;
            for (int64_t q = tid; q < npix; q += NT) {
                const double d = F.G.ld(in.pix, q) - (in.bkg ? F.G.ld(in.bkg, q) : 0.0);
                bad |= !isfinite(d);
            }
            if (__syncthreads_or(bad)) {
                fail_group(1);
                continue;
            }
        }
        // ---- anchors and usable stamps (_build_stamps!, :245-323)
        for (int i = wid; i < ng; i += NT / 32) {
            const double yy = y0[i], xx = x0[i];
            const bool fin = isfinite(yy) && isfinite(xx) && fabs(yy) < 1e9 && fabs(xx) < 1e9;
            const int ay = fin ? (int)rint(yy) : 0, ax = fin ? (int)rint(xx) : 0;
            int any = 0;
            if (fin)
                for (int m = lane; m < S2; m += 32) {
                    const int gy = ay + (m % S) - R, gx = ax + (m / S) - R;
                    if (gy >= 1 && gy <= ny && gx >= 1 && gx <= nx) {
                        double d, w;
                        F.G.data_w((gy - 1) + (int64_t)(gx - 1) * ny, d, w);
                        any |= w > 0;
                    }
                }
            any = __any_sync(0xffffffffu, any);
            if (lane == 0) {
                s_ok[i] = (any && fin && isfinite(f0[i])) ? 1 : 0;
                s_ay0[i] = ay;
                s_ax0[i] = ax;
                s_key[i] = (ay >= 0 && ax >= 0) ? (spread_bits((uint64_t)ay) | (spread_bits((uint64_t)ax) << 1)) : 0;
            }
        }
        __syncthreads();
        // active set in stable Morton order (:306); negative anchors fail (Morton key of a negative Int)
        int* act = F.ip(F.L.act);
        {
            int nok = 0, neg = 0;
            for (int j = 0; j < ng; ++j) {
                nok += s_ok[j];
                neg |= s_ok[j] && (s_ay0[j] < 0 || s_ax0[j] < 0);
            }
            F.n_act = nok;
            if (neg) {
                fail_group(2);
                continue;
            }
            if (tid < ng && s_ok[tid]) {
                const uint64_t k = s_key[tid];
                int rank = 0;
                for (int j = 0; j < ng; ++j)
                    rank += s_ok[j] && (s_key[j] < k || (s_key[j] == k && j < tid));
                act[rank] = tid;
            }
        }
        const int n_act = F.n_act;
        if (n_act == 0) {  // _empty_simultaneous_result (:1433-1445)
            for (int i = tid; i < ng; i += NT) {
                write_catalogue(i);
                fixed_fix(soff + i);
            }
            zero_residual();
            group_stats(0, ng, 0, 0, 0, 0, 0, 0);
            __syncthreads();
            continue;
        }
        __syncthreads();
        int32_t* ay = F.ip(F.L.ay);
        int32_t* ax = F.ip(F.L.ax);
        double* theta = F.dp(F.L.theta);
        uint8_t* live = F.bp(F.L.live);
        uint8_t* conv = F.bp(F.L.conv);
        uint8_t* newf = F.bp(F.L.newf);
        int32_t* frozen = F.ip(F.L.frozen);
        double* cn = F.dp(F.L.cn);
        double* D = F.dp(F.L.D);
        double* bsc = F.dp(F.L.bsc);
        double* delta = F.dp(F.L.delta);
        double* dsc = F.dp(F.L.dsc);
        for (int a = tid; a < n_act; a += NT) {
            const int i = act[a];
            ay[a] = s_ay0[i];
            ax[a] = s_ax0[i];
            for (int k = 0; k < p; ++k)
                theta[a * p + k] = C.gc[k] == 1 ? y0[i] : (C.gc[k] == 2 ? x0[i] : f0[i]);
            live[a] = 1;
            conv[a] = 0;
            newf[a] = 0;
            frozen[a] = 0;
            for (int k = 0; k < p; ++k) cn[a * p + k] = 0.0;
        }
        // ---- union of usable stamp pixels (_touched_pixels, :329-335): sort the
        // entries' pixel indices (bitonic, in the V region) and drop duplicates
        int32_t* keys = F.ip(F.L.V);
        const int ne = n_act * S2;
        int kn = 2;
        while (kn < ne) kn <<= 1;
        for (int e = tid; e < kn; e += NT) {
            int key = kNoU;
            if (e < ne) {
                const int a = e / S2, m = e % S2;
                const int gy = s_ay0[act[a]] + (m % S) - R, gx = s_ax0[act[a]] + (m / S) - R;
                if (gy >= 1 && gy <= ny && gx >= 1 && gx <= nx) {
                    const int q = (gy - 1) + (gx - 1) * ny;
                    double d, w;
                    F.G.data_w(q, d, w);
                    if (w > 0) key = q;
                }
            }
            keys[e] = key;
        }
        __syncthreads();
        for (int k = 2; k <= kn; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = tid; i < kn; i += NT) {
                    const int l = i ^ j;
                    if (l > i) {
                        const int ki = keys[i], kl = keys[l];
                        const bool up = (i & k) == 0;
                        if ((ki > kl) == up) {
                            keys[i] = kl;
                            keys[l] = ki;
                        }
                    }
                }
                __syncthreads();
            }
        // compaction of the distinct keys (chunked block scan)
        int32_t* upix = F.ip(F.L.upix);
        {
            const int per = (kn + NT - 1) / NT;
            const int b0 = min(tid * per, kn), b1 = min(b0 + per, kn);
            int cnt = 0;
            for (int e = b0; e < b1; ++e) cnt += keys[e] != kNoU && (e == 0 || keys[e] != keys[e - 1]);
            // exclusive scan of cnt over the block
            int incl = cnt;
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            __shared__ int s_wsum[32];
            if (lane == 31) s_wsum[wid] = incl;
            __syncthreads();
            int wbase = 0, tot = 0;
            for (int k = 0; k < NT / 32; ++k) {
                if (k < wid) wbase += s_wsum[k];
                tot += s_wsum[k];
            }
            int pos = wbase + incl - cnt;
            for (int e = b0; e < b1; ++e)
                if (keys[e] != kNoU && (e == 0 || keys[e] != keys[e - 1]) && pos < C.umax) upix[pos++] = keys[e];
            F.nU = min(tot, C.umax);
        }
        __syncthreads();
        const int nU = F.nU;
        // per stamp entry: its position in U (binary search), kNoU when unusable
        int32_t* uidx = F.ip(F.L.uidx);
        for (int e = tid; e < ne; e += NT) {
            const int a = e / S2, m = e % S2;
            const int gy = ay[a] + (m % S) - R, gx = ax[a] + (m / S) - R;
            int r = kNoU;
            if (gy >= 1 && gy <= ny && gx >= 1 && gx <= nx) {
                const int q = (gy - 1) + (gx - 1) * ny;
                int lo = 0, hi = nU;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (upix[mid] < q) lo = mid + 1;
                    else hi = mid;
                }
                if (lo < nU && upix[lo] == q) r = lo;
            }
            uidx[e] = r;
        }
        // per pixel of U: data_work, w and the star masks
        {
            double* dw = F.dp(F.L.dw);
            double* wv = F.dp(F.L.w);
            MaskT* fm = F.mp(F.L.fmask);
            MaskT* mm = F.mp(F.L.mmask);
            for (int u = tid; u < nU; u += NT) {
                const int q = upix[u];
                double d, w;
                F.G.data_w(q, d, w);
                dw[u] = d;
                wv[u] = w;
                const int gy = q % ny + 1, gx = q / ny + 1;
                MaskT f = 0, mo = 0;
                for (int a = 0; a < n_act; ++a) {
                    const int dy = abs(gy - ay[a]), dx = abs(gx - ax[a]);
                    if (dy <= R && dx <= R) f |= (MaskT)1 << a;
                    if (dy <= C.mR && dx <= C.mR) mo |= (MaskT)1 << a;
                }
                fm[u] = f;
                mm[u] = mo;
            }
        }
        const MaskT all_bits = n_act >= (int)(8 * sizeof(MaskT)) ? ~(MaskT)0 : (((MaskT)1 << n_act) - 1);
        MaskT live_bits = all_bits;
        const int n = n_act * p;
        const double dof = (double)max(nU - n, 1);
        __syncthreads();

        // ---- initial fill and cost (:1171-1178)
        F.coefs(false);
        F.fill(false, nullptr);
        double cost = F.render(0, live_bits);
        for (int i = tid; i < n; i += NT) D[i] = cn[i];
        bool fresh = true;
        double lam = C.lambda_init;
        int n_run = 0, n_trials = 0, n_lsqr = 0;
        // ---- outer loop (:1186-1284)
        for (int iter = 1; iter <= C.max_iter; ++iter) {
            if (!fresh) {
                F.coefs(false);
                F.fill(false, nullptr);
                cost = F.render(0, live_bits);
            }
            fresh = false;
            for (int i = tid; i < n; i += NT) bsc[i] = 0.0;
            __syncthreads();
            F.jt(F.dp(F.L.wr), 1.0, false, 0.0, 0.0, bsc);
            // global gradient cosine (:1199-1213)
            const double C_r = cost / dof;
            double gmax = 0.0;
            for (int i = tid; i < n; i += NT) {
                const double bt = cn[i] * bsc[i], Aii = cn[i] * cn[i];
                gmax = nan_max(gmax, fabs(bt) / (sqrt(Aii * C_r) + kEpsG));
            }
            const double gnorm = block_allmax<NT>(gmax, sh, F.flip);
            if (gnorm <= C.g_tol) {
                for (int a = tid; a < n_act; a += NT)
                    if (live[a]) {
                        live[a] = 0;
                        frozen[a] = iter - 1;
                        conv[a] = 1;
                    }
                live_bits = 0;
                n_run = iter - 1;
                __syncthreads();
                break;
            }
            bool accepted = false, f_conv = false;
            for (int trial = 1; trial <= C.max_trials; ++trial) {
                ++n_trials;
                n_lsqr += F.lsqr(cost, lam, live_bits);
                // delta = x / colnorm, position step cap (:700-716), delta_scaled
                const double* xl = F.dp(F.L.xl);
                for (int a = tid; a < n_act; a += NT) {
                    double d[3];
                    for (int k = 0; k < p; ++k) d[k] = xl[a * p + k] / cn[a * p + k];
                    if (C.ky >= 0 || C.kx >= 0) {
                        const double dy = C.ky < 0 ? 0.0 : d[C.ky];
                        const double dx = C.kx < 0 ? 0.0 : d[C.kx];
                        const double len = sqrt(dy * dy + dx * dx);
                        if (len > C.max_step) {
                            const double scl = C.max_step / len;
                            if (C.ky >= 0) d[C.ky] *= scl;
                            if (C.kx >= 0) d[C.kx] *= scl;
                        }
                    }
                    for (int k = 0; k < p; ++k) {
                        delta[a * p + k] = d[k];
                        dsc[a * p + k] = cn[a * p + k] * d[k];
                    }
                }
                __syncthreads();
                F.coefs(true);
                const double cost_cand = F.render(1, live_bits);
                f_conv = (cost_cand < cost) && ((cost - cost_cand) / cost <= C.f_tol);
                if (cost_cand < cost) {
                    accepted = true;
                    lam = fmax(lam / C.lambda_down, C.lambda_min);
                    // accepted step (:1245-1251) and per-star freeze tests (:1265-1283)
                    int nf = 0;
                    for (int a = tid; a < n_act; a += NT) {
                        for (int k = 0; k < p; ++k) {
                            const int i = a * p + k;
                            theta[i] = theta[i] + delta[i];
                            D[i] = fmax(D[i], cn[i]);
                        }
                        newf[a] = 0;
                        if (!live[a] || f_conv) continue;
                        double num = 0, xn = 0, gn = 0;
                        for (int k = 0; k < p; ++k) {
                            const int i = a * p + k;
                            const double v = (D[i] / cn[i]) * dsc[i];
                            num += v * v;
                            const double xv = D[i] * theta[i];
                            xn += xv * xv;
                            const double bt = cn[i] * bsc[i], Aii = cn[i] * cn[i];
                            gn = nan_max(gn, fabs(bt) / (sqrt(Aii * C_r) + kEpsG));
                        }
                        const bool xt = sqrt(num) <= C.x_tol * (sqrt(xn) + C.x_tol);
                        const bool gt = gn <= C.g_tol;
                        if (xt || gt) {
                            live[a] = 0;
                            newf[a] = 1;
                            frozen[a] = iter;
                            conv[a] = 1;
                            nf = 1;
                        }
                    }
                    cost = cost_cand;
                    if (__syncthreads_or(nf)) {
                        MaskT nb = 0;
                        for (int a = 0; a < n_act; ++a)
                            if (newf[a]) nb |= (MaskT)1 << a;
                        live_bits &= ~nb;
                        F.coefs(false);
                        F.render(2, nb);  // _freeze_star! in Morton order
                    }
                    break;
                }
                lam = fmin(lam * C.lambda_up, C.lambda_max);
            }
            n_run = iter;
            if (f_conv) {
                for (int a = tid; a < n_act; a += NT)
                    if (live[a]) {
                        live[a] = 0;
                        frozen[a] = iter;
                        conv[a] = 1;
                    }
                live_bits = 0;
                __syncthreads();
                break;
            }
            if (accepted && live_bits == 0) break;
        }
        __syncthreads();
        // ---- errors at the final theta, every active star (:1302-1329)
        F.coefs(false);
        F.fill(true, s_gram);
        const StarCoef* cf = F.coef();
        double* err = F.dp(F.L.delta);  // reuse: per-star errors
        for (int a = tid; a < n_act; a += NT) {
            double A[9], inv[9];
            const double* gr = s_gram + a * 6;
            const double gfull[3][3] = {{gr[0], gr[1], gr[2]}, {gr[1], gr[3], gr[4]}, {gr[2], gr[4], gr[5]}};
            for (int k = 0; k < p; ++k)
                for (int l = 0; l < p; ++l) A[k + l * p] = gfull[k][l];
            double tr = 0;
            for (int k = 0; k < p; ++k) tr += A[k + k * p];
            for (int k = 0; k < p; ++k) A[k + k * p] += 1.0e-12 * tr;
            if (!chol_inv_small(A, p, inv)) pinv_small(A, p, inv);
            const double fsc = C.reweighted ? cost / dof : 1.0;
            for (int k = 0; k < p; ++k) err[a * p + k] = sqrt(fmax(0.0, inv[k + k * p] * fsc));
        }
        __syncthreads();
        // ---- outputs in catalogue order (:1289-1337, :1404-1430)
        for (int i = tid; i < ng; i += NT) {
            write_catalogue(i);
            fixed_fix(soff + i);
        }
        __syncthreads();
        for (int a = tid; a < n_act; a += NT) {
            const int64_t o = soff + act[a];
            for (int k = 0; k < p; ++k) {
                const double v = theta[a * p + k], e = err[a * p + k];
                if (C.gc[k] == 1) {
                    O.y[o] = v;
                    O.y_err[o] = e;
                } else if (C.gc[k] == 2) {
                    O.x[o] = v;
                    O.x_err[o] = e;
                } else {
                    O.flux[o] = v;
                    O.flux_err[o] = e;
                }
            }
            const StarCoef& c = cf[a];
            O.valid[o] = (isfinite(c.y) && isfinite(c.x) && isfinite(c.flux) && c.flux > 0) ? 1 : 0;
            O.converged[o] = conv[a];
            O.n_iter[o] = live[a] ? n_run : frozen[a];
        }
        // ---- final residual against the original data (:1344-1356), every active star
        if (O.residual) {
            for (int64_t q = tid; q < npix; q += NT) {
                const int gy = (int)(q % ny) + 1, gx = (int)(q / ny) + 1;
                double acc = 0.0;
                for (int a = 0; a < n_act; ++a)
                    if (abs(gy - ay[a]) <= C.mR && abs(gx - ax[a]) <= C.mR) acc += F.mval(cf[a], gy, gx);
                double d, w;
                F.G.data_w(q, d, w);
                O.residual[F.G.off + q] = d - acc;
            }
        }
        // ---- chisq and the qfit / crowding diagnostics (:1358-1397,
        // psf_photometry_diagnostics.jl:154-231), one warp per valid star; with
        // spread_model on, each box pixel's residual and weight also go to the
        // star's planes for k_group_spread
        for (int a = wid; a < n_act; a += NT / 32) {
            const StarCoef c = cf[a];
            const int64_t o = soff + act[a];
            if (!(isfinite(c.y) && isfinite(c.x) && isfinite(c.flux) && c.flux > 0)) continue;
            const int ylo = max((int)floor(c.y - C.fit_rad), 1), yhi = min((int)ceil(c.y + C.fit_rad), ny);
            const int xlo = max((int)floor(c.x - C.fit_rad), 1), xhi = min((int)ceil(c.x + C.fit_rad), nx);
            double num = 0, qv = 0, ncl = 0, ndi = 0, den = 0, ss = 0, ss2 = 0;
            int ng_ = 0, ngi = 0;
            const int h = yhi - ylo + 1, wd = xhi - xlo + 1;
            const double inv_flux = 1.0 / c.flux;
            double* rw = C.sp_on ? O.sp_rw + (size_t)o * 2 * C.sp_box : nullptr;
            if (h > 0 && wd > 0)
                for (int e = lane; e < h * wd; e += 32) {
                    const int gy = ylo + e % h, gx = xlo + e / h;
                    const int64_t q = (gy - 1) + (int64_t)(gx - 1) * ny;
                    double acc = 0.0;
                    for (int b = 0; b < n_act; ++b)
                        if (abs(gy - ay[b]) <= C.mR && abs(gx - ax[b]) <= C.mR) acc += F.mval(cf[b], gy, gx);
                    double d, wsan;
                    F.G.data_w(q, d, wsan);
                    const double r = d - acc;
                    const double wp = in.iv ? F.G.ld(in.iv, q) : 1.0;
                    if (rw) {
                        rw[e] = r;
                        rw[C.sp_box + e] = (isfinite(wp) && wp > 0) ? wp : 0.0;
                    }
                    if (isfinite(wp) && wp > 0) {
                        num += wp * (r * r);
                        ng_ += 1;
                        const double mv = F.mval(c, gy, gx);
                        qv += fabs(r);
                        const double Pp = (mv - c.bkg) * inv_flux;
                        const double wP = wp * Pp;
                        ncl += wP * (r + mv - c.bkg);
                        const double im = F.G.ld(in.pix, q) - (in.bkg ? F.G.ld(in.bkg, q) : 0.0);
                        ndi += wP * (im - c.bkg);
                        den += wP * Pp;
                        if (in.iv) {
                            const double si = 1.0 / sqrt(wp);
                            ss += si;
                            ss2 += si * si;
                            ngi += 1;
                        }
                    }
                }
            num = warp_sum(num);
            qv = warp_sum(qv);
            ncl = warp_sum(ncl);
            ndi = warp_sum(ndi);
            den = warp_sum(den);
            ss = warp_sum(ss);
            ss2 = warp_sum(ss2);
            ng_ = warp_sum(ng_);
            ngi = warp_sum(ngi);
            if (lane == 0) {
                if (O.chisq) O.chisq[o] = (ng_ - p > 0) ? num / (double)(ng_ - p) : 0.0;
                if (O.qfit) O.qfit[o] = qv * inv_flux;
                if (O.crowding) O.crowding[o] = (den > 0 && ncl > 0 && ndi > 0) ? 2.5 * log10(ndi / ncl) : NaN;
                if (in.iv) {
                    if (O.qfit_expected) O.qfit_expected[o] = sqrt(2.0 / 3.141592653589793) * ss * inv_flux;
                    if (O.qfit_z) {
                        if (ss2 > 0 && ngi > p) {
                            const double dfac = sqrt(1.0 - (double)p / (double)ngi);
                            O.qfit_z[o] = (qv - sqrt(2.0 / 3.141592653589793) * dfac * ss) /
                                          (sqrt((1.0 - 2.0 / 3.141592653589793) * ss2) * dfac);
                        }
                    }
                }
            }
        }
        group_stats(n_run, ng - n_act, 0, 0, n_act, nU, n_trials, n_lsqr);
        __syncthreads();
    }
}

// spread_model of the kernel-fitted groups (_star_diagnostics!,
// psf_photometry_diagnostics.jl:200-231, with the disk of
// psf_photometry_simultaneous.jl:1361-1365), after k_groups: one block per group
// (grid-stride over the group list), one warp per valid star.  The block builds
// the group's disk into shared memory, its width from the first catalogue
// star's final parameters; each warp renders its star's model stamp over the
// fit box and correlates it with the disk one component at a time (x pass, then
// the y pass added into the correlated stamp), all in its own 3 sp_box doubles
// of shared memory, and sums against the residual and weight planes k_groups
// saved for the star.  Kept out of k_groups so that the fit's register
// allocation does not carry it.
__global__ void __launch_bounds__(128) k_group_spread(GroupConst C, DevPsf P, GroupIn in, GroupOut O,
                                                      const int32_t* __restrict__ glist, int nlist) {
    extern __shared__ __align__(16) double sm[];
    __shared__ double red[2 * 4 + 1];
    const double NaN = __longlong_as_double(0x7ff8000000000000LL);
    const int kh = C.R, box = C.sp_box, n = 2 * kh + 1;
    const int nw = blockDim.x >> 5, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double* tab = sm;
    double* pan = tab + ((C.sp_tab + 1) & ~1);
    double* M = pan + (7 + kh) * kSpreadGL + (size_t)wid * 3 * box;  // the warp's model stamp
    double* T = M + box;                                             // one component's x pass
    double* Gs = T + box;                                            // the disk-correlated stamp
    DevPsf Ps = P;
    Ps.fwhm = C.sp_psf_fwhm;  // _spread_fwhm renders the PSF object's own width
    for (int li = blockIdx.x; li < nlist; li += gridDim.x) {
        const int g = glist[li];
        const int64_t soff = in.star_off[g];
        const int ng = (int)(in.star_off[g + 1] - soff);
        int any = 0;
        for (int i = threadIdx.x; i < ng; i += blockDim.x) any |= O.valid[soff + i];
        if (!__syncthreads_or(any)) continue;  // also: the previous group's disk is no longer read
        spread_disk_block(Ps, C.sp_param, kh, O.y[soff], O.x[soff], O.sp_rule, tab, red, pan);
        if (!spread_tab_on(tab)) continue;
        const SpreadDev D = spread_dev(tab, kh);
        const int ny = in.ny[g], nx = in.nx[g];
        for (int i = wid; i < ng; i += nw) {
            const int64_t o = soff + i;
            if (!O.valid[o]) continue;
            StarCoef c;
            c.y = O.y[o];
            c.x = O.x[o];
            c.flux = O.flux[o];
            c.bkg = C.fixed_bkg;
            grid_corners_dw(P, c.y, c.x, c);
            const int ylo = max((int)floor(c.y - C.fit_rad), 1), yhi = min((int)ceil(c.y + C.fit_rad), ny);
            const int xlo = max((int)floor(c.x - C.fit_rad), 1), xhi = min((int)ceil(c.x + C.fit_rad), nx);
            const int h = yhi - ylo + 1, wd = xhi - xlo + 1, nb = h * wd;
            if (h <= 0 || wd <= 0 || nb > box) continue;
            const double* Rr = O.sp_rw + (size_t)o * 2 * box;
            const double* Wt = Rr + box;
            __syncwarp();  // the warp's previous stamp is no longer read
            for (int e = lane; e < nb; e += 32) {
                M[e] = psf_value(P, c, ylo + e % h, xlo + e / h);
                Gs[e] = 0.0;
            }
            for (int cc = 0; cc < 6; ++cc) {
                const int L = D.L[cc];
                const double* I = D.I + cc * n + kh;
                __syncwarp();
                for (int e = lane; e < nb; e += 32) {  // x pass
                    const int r = e % h, col = e / h;
                    const int q0 = max(-L, -col), q1 = min(L, wd - 1 - col);
                    double t = 0.0;
                    for (int q = q0; q <= q1; ++q) t += I[q] * M[r + (col + q) * h];
                    T[e] = t;
                }
                __syncwarp();
                for (int e = lane; e < nb; e += 32) {  // y pass
                    const int r = e % h, col = e / h;
                    const int p0 = max(-L, -r), p1 = min(L, h - 1 - r);
                    double t = 0.0;
                    for (int p = p0; p <= p1; ++p) t += I[p] * T[r + p + col * h];
                    Gs[e] += D.alpha[cc] * t;
                }
            }
            __syncwarp();
            const double inv_flux = 1.0 / c.flux;
            double Sp = 0, Sq = 0, Sp0 = 0, Sq0 = 0, SqG = 0;
            for (int e = lane; e < nb; e += 32) {
                const double wp = Wt[e];
                if (wp > 0) {
                    const double mv = M[e];
                    const double Pp = (mv - c.bkg) * inv_flux;
                    const double wP = wp * Pp;
                    const double p_i = Rr[e] + mv - c.bkg;
                    const double g_i = (Gs[e] - c.bkg) * inv_flux;
                    Sp += wP * p_i;
                    Sq += wp * g_i * p_i;
                    Sp0 += wP * Pp;
                    Sq0 += wp * Pp * g_i;
                    SqG += wp * g_i * g_i;
                }
            }
            Sp = warp_sum(Sp);
            Sq = warp_sum(Sq);
            Sp0 = warp_sum(Sp0);
            Sq0 = warp_sum(Sq0);
            SqG = warp_sum(SqG);
            if (lane == 0 && Sp > 0) {
                if (O.spread) O.spread[o] = Sq / Sp - Sq0 / Sp0;
                if (O.spread_err)
                    O.spread_err[o] =
                        in.iv ? sqrt(fmax(0.0, Sp * Sp * SqG + Sq * Sq * Sp0 - 2 * Sq * Sp * Sq0)) / (Sp * Sp) : NaN;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
inline int next_pow2(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// Groups are launched in buckets of star count, each launch with a
// shared-memory layout sized for its largest group.  Measured on the B200 with
// the blended-group workload (2-12 stars), one launch over all groups (20,000
// groups: 56 ms) beats four launches by size class (65 ms): the class
// launches run one after another and each fills the GPU less.  So groups up to
// 32 stars share one bucket; larger ones (up to 64) get a second.
constexpr int kBucketEdges[] = {32, 64};
constexpr int kNumBuckets = sizeof(kBucketEdges) / sizeof(int);

struct Bucket {
    std::vector<int32_t> groups;
    int nmax = 1, umax = 1, keyn = 2;
    bool wide = false;
    size_t smem = 0;
    GroupConst C{};
    int threads = 256;  // default block size
};

struct GroupPlan {
    std::vector<Bucket> buckets;  // non-empty buckets only
    std::vector<int32_t> routed_groups;
    int64_t n_kernel = 0;
};

// Everything a launch needs, derived once from the arguments.
struct GroupSetup {
    GroupConst C{};
    DevPsf dp{};
    GroupPlan plan;
    GroupIn gin{};
    GroupOut go{};
    std::vector<int64_t> h_off, h_soff;
    std::vector<int32_t> h_ny, h_nx;
    int64_t total_pixels = 0;
    int32_t eltype = CPB_F64;
    int sp_nw = 0;        // spread_model: warps a k_group_spread block (0: off)
    size_t sp_smem = 0;   // its dynamic shared memory
    int64_t n_stars = 0;  // catalogue length (sizes the residual / weight planes)
};

constexpr size_t kStaticSmem = 8 * 1024;  // the kernel's static shared arrays, rounded up

template <typename MaskT>
size_t layout_bytes(int nmax, int S2, int umax, int keyn) {
    return make_layout<MaskT>(nmax, S2, umax, keyn).total;
}

// Argument checks (the reference's, :984-1051), constants, group metadata on
// the host and the shared-memory plan: which groups one block can hold.
void setup_groups(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* P, int64_t G, const int64_t* d_off,
                  const int32_t* d_ny, const int32_t* d_nx, const void* d_pix, int32_t eltype, const void* d_iv,
                  const void* d_bkg, const int64_t* d_soff, const double* d_y0, const double* d_x0,
                  const double* d_f0, int64_t total_pixels, const cpb_group_result* out, const int64_t* h_off_opt,
                  const int32_t* h_ny_opt, const int32_t* h_nx_opt, const int64_t* h_soff_opt, GroupSetup& su) {
    cudaStream_t st = ctx->stream;
    // argument checks in the reference's order (:984-997), shared by every group
    if (!(P->max_iter > 0)) throw ArgError{"max_iter must be positive"};
    if (!(P->inner_iterations > 0)) throw ArgError{"inner_iterations must be positive"};
    if (!(P->linear_tol > 0)) throw ArgError{"linear_tol must be positive"};
    if (!(P->max_trials > 0)) throw ArgError{"max_trials must be positive"};
    if (!P->model_rad_auto && !(P->model_rad > 0)) throw ArgError{"model_rad must be :auto or a positive real"};
    const double model_rad_max = P->model_rad_max < 0 ? 10 * P->fit_rad : P->model_rad_max;
    if (!(model_rad_max >= P->fit_rad)) throw ArgError{"model_rad_max must be >= fit_rad"};
    if (!(P->model_rad_nsigma > 0)) throw ArgError{"model_rad_nsigma must be positive"};
    if (P->solver != CPB_SOLVER_LSQR && P->solver != CPB_SOLVER_LSMR) throw ArgError{"solver must be :lsqr or :lsmr"};
    if (P->damping == CPB_DAMP_LEVENBERG)
        throw ArgError{
            "LevenbergDamping is not supported by fit_all_stars_simultaneous: it conflicts with the "
            "column-equilibrated x_tol scaling. Use MarquardtDamping."};
    if (!(P->fit_rad > 0)) throw ArgError{"fit_rad must be positive"};
    if (eltype != CPB_F32 && eltype != CPB_F64) throw ArgError{"unsupported image eltype"};
    if (P->model_rad_auto && !d_iv)
        throw ArgError{
            "model_rad=:auto requires inv_var (it needs a noise scale); pass inv_var or an explicit scalar model_rad"};
    if (G < 0) throw ArgError{"n_groups must be >= 0"};
    if (!out->y || !out->x || !out->flux || !out->y_err || !out->x_err || !out->flux_err || !out->converged ||
        !out->valid || !out->n_iter || !out->n_passes || !out->n_failed || !out->status)
        throw ArgError{"null output array"};
    GroupConst& C = su.C;
    C.p = 0;
    if (P->free_mask & CPB_FREE_Y) C.gc[C.p++] = 1;
    if (P->free_mask & CPB_FREE_X) C.gc[C.p++] = 2;
    if (P->free_mask & CPB_FREE_FLUX) C.gc[C.p++] = 3;
    if (P->free_mask & ~(CPB_FREE_Y | CPB_FREE_X | CPB_FREE_FLUX))
        throw ArgError{
            "fit_all_stars_simultaneous fits only (y, x, flux) per star. Fix `bkg` (subtract the background first "
            "and pass `fixed = (; bkg = zero(eltype(image)))`), and fix all shape parameters."};
    if (C.p == 0) throw ArgError{"all model parameters are fixed; nothing to fit"};
    C.ky = C.kx = -1;
    for (int k = 0; k < C.p; ++k) {
        if (C.gc[k] == 1) C.ky = k;
        if (C.gc[k] == 2) C.kx = k;
    }
    for (int k = C.p; k < 3; ++k) C.gc[k] = 3;
    C.fixed_y = P->fixed_y;
    C.fixed_x = P->fixed_x;
    C.fixed_flux = P->fixed_flux;
    C.fixed_bkg = P->fixed_bkg;
    C.R = (int)std::ceil(P->fit_rad);
    C.S = 2 * C.R + 1;
    C.S2 = C.S * C.S;
    {
        const int R_cap = (int)std::ceil(std::max(P->model_rad, P->fit_rad));
        C.mR = std::min(std::max((int)std::ceil(P->model_rad), C.R), R_cap);
    }
    C.max_iter = P->max_iter;
    C.max_trials = P->max_trials;
    C.itmax = P->inner_iterations;
    C.linear_tol = P->linear_tol;
    C.max_step = P->max_step;
    C.x_tol = P->x_tol;
    C.f_tol = P->f_tol;
    C.g_tol = P->g_tol;
    C.lambda_init = P->lambda_init;
    C.lambda_up = P->lambda_up;
    C.lambda_down = P->lambda_down;
    C.lambda_min = P->lambda_min;
    C.lambda_max = P->lambda_max;
    C.eltype = eltype;
    C.reweighted = (P->covariance == CPB_COV_REWEIGHTED || (P->covariance == CPB_COV_AUTO && d_iv == nullptr)) ? 1 : 0;
    C.fit_rad = P->fit_rad;
    {
        const double spp = P->spread_model_fwhm;
        C.sp_on = (out->spread_model || out->spread_model_err) && (std::isnan(spp) || (std::isfinite(spp) && spp > 0));
        C.sp_tab = spread_tab_len(C.R);
        C.sp_box = (2 * C.R + 2) * (2 * C.R + 2);
        C.sp_param = spp;
        C.sp_psf_fwhm = psf->dev.fwhm;
    }
    su.dp = psf->dev;
    su.dp.fwhm = P->fixed_fwhm;

    su.total_pixels = total_pixels;
    su.eltype = eltype;
    su.gin = GroupIn{d_off, d_ny, d_nx, d_pix, d_iv, d_bkg, d_soff, d_y0, d_x0, d_f0};
    su.go = GroupOut{out->y, out->x, out->flux, out->y_err, out->x_err, out->flux_err, out->converged, out->valid,
                     out->n_iter, out->chisq, out->qfit, out->qfit_expected, out->qfit_z, out->crowding,
                     out->residual, out->n_passes, out->n_failed, out->status, out->error_kind, out->n_active,
                     out->n_union, out->n_trials, out->n_lsqr_iters, out->spread_model, out->spread_model_err,
                     nullptr, nullptr};
    if (G == 0) return;
    // group sizes on the host (plan the shared-memory layout, route oversized groups)
    std::vector<int64_t>& h_off = su.h_off;
    std::vector<int64_t>& h_soff = su.h_soff;
    std::vector<int32_t>& h_ny = su.h_ny;
    std::vector<int32_t>& h_nx = su.h_nx;
    h_off.resize(G);
    h_soff.resize(G + 1);
    h_ny.resize(G);
    h_nx.resize(G);
    if (h_off_opt) {
        std::memcpy(h_off.data(), h_off_opt, sizeof(int64_t) * G);
        std::memcpy(h_soff.data(), h_soff_opt, sizeof(int64_t) * (G + 1));
        std::memcpy(h_ny.data(), h_ny_opt, sizeof(int32_t) * G);
        std::memcpy(h_nx.data(), h_nx_opt, sizeof(int32_t) * G);
    } else {
        check(cudaMemcpyAsync(h_off.data(), d_off, sizeof(int64_t) * G, cudaMemcpyDeviceToHost, st), "d2h");
        check(cudaMemcpyAsync(h_soff.data(), d_soff, sizeof(int64_t) * (G + 1), cudaMemcpyDeviceToHost, st), "d2h");
        check(cudaMemcpyAsync(h_ny.data(), d_ny, sizeof(int32_t) * G, cudaMemcpyDeviceToHost, st), "d2h");
        check(cudaMemcpyAsync(h_nx.data(), d_nx, sizeof(int32_t) * G, cudaMemcpyDeviceToHost, st), "d2h");
        check(cudaStreamSynchronize(st), "sync");
    }
    for (int64_t g = 0; g < G; ++g) {
        if (h_ny[g] <= 0 || h_nx[g] <= 0 || (int64_t)h_ny[g] * h_nx[g] >= (1LL << 31))
            throw ArgError{"group image size out of range"};
        if (h_soff[g + 1] < h_soff[g]) throw ArgError{"star_offsets must be non-decreasing"};
        if (out->residual && h_off[g] + (int64_t)h_ny[g] * h_nx[g] > total_pixels)
            throw ArgError{"total_pixels is smaller than the pixels the groups span"};
    }
    int smem_optin = 0, smem_sm = 0;
    check(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device), "attr");
    check(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device), "attr");
    const size_t cap = (size_t)smem_optin - kStaticSmem;
    su.n_stars = h_soff[G];
    if (C.sp_on) {
        // k_group_spread: the disk table and one panel of the quadrature, then
        // 3 sp_box doubles a warp; up to 4 warps within 96 KB, else fewer; a fit
        // box beyond shared memory even for one warp leaves spread_model NaN
        const size_t fixed = ((size_t)((C.sp_tab + 1) & ~1) + (size_t)(7 + C.R) * kSpreadGL) * sizeof(double);
        const size_t per_warp = (size_t)3 * C.sp_box * sizeof(double);
        int nw = 4;
        while (nw > 1 && fixed + nw * per_warp > 96 * 1024) --nw;
        if (fixed + nw * per_warp > cap) C.sp_on = 0;
        su.sp_nw = C.sp_on ? nw : 0;
        su.sp_smem = fixed + nw * per_warp;
    }
    GroupPlan& plan = su.plan;
    auto need_of = [&](int ng, int um, int kn) {
        return ng > 32 ? layout_bytes<uint64_t>(std::max(ng, 1), C.S2, std::max(um, 1), kn)
                       : layout_bytes<uint32_t>(std::max(ng, 1), C.S2, std::max(um, 1), kn);
    };
    // a group runs in the kernel when it has <= 64 stars and its own layout fits;
    // the kernel computes in FP64 with LSQR and one scalar model radius, so
    // solver = :lsmr, model_rad = :auto or the mixed form route every group to
    // the full-field fit
    const bool route_all = P->solver == CPB_SOLVER_LSMR || P->model_rad_auto || P->precision != CPB_PREC_FP64;
    std::vector<Bucket> bk(kNumBuckets);
    for (int64_t g = 0; g < G; ++g) {
        const int ng = (int)(h_soff[g + 1] - h_soff[g]);
        const int um = (int)std::min<int64_t>((int64_t)ng * C.S2, (int64_t)h_ny[g] * h_nx[g]);
        const int kn = next_pow2(std::max(ng * C.S2, 2));
        if (route_all || ng > kMaxGroupStars || need_of(ng, um, kn) > cap) {
            plan.routed_groups.push_back((int32_t)g);
            continue;
        }
        int b = 0;
        while (kBucketEdges[b] < ng) ++b;
        Bucket& B = bk[b];
        // the bucket's layout must still fit with this group's sizes folded in
        const int nm2 = std::max(B.nmax, ng), um2 = std::max(B.umax, um), kn2 = std::max(B.keyn, kn);
        if (need_of(nm2, um2, kn2) > cap) {
            plan.routed_groups.push_back((int32_t)g);
            continue;
        }
        B.groups.push_back((int32_t)g);
        B.nmax = nm2;
        B.umax = um2;
        B.keyn = kn2;
    }
    std::sort(plan.routed_groups.begin(), plan.routed_groups.end());
    for (Bucket& B : bk) {
        if (B.groups.empty()) continue;
        B.wide = B.nmax > 32;
        B.smem = need_of(B.nmax, B.umax, B.keyn);
        B.C = C;
        B.C.nmax = B.nmax;
        B.C.umax = B.umax;
        B.C.keyn = B.keyn;
        // default block size: about 512 threads an SM (the kernel's register budget
        // allows 512 threads of 128 registers), in as many blocks as shared memory holds
        const int by_smem = std::max(1, (int)((size_t)smem_sm / (B.smem + kStaticSmem + 1024)));
        const int blocks = std::min(by_smem, 8);
        B.threads = blocks >= 8 ? 64 : (blocks >= 4 ? 128 : 256);
        plan.n_kernel += (int64_t)B.groups.size();
        plan.buckets.push_back(std::move(B));
    }
}

template <int NT, typename MaskT>
void* group_kernel() {
    return (void*)k_groups<NT, MaskT>;
}

void* group_kernel_for(int threads, bool wide) {
    if (threads == 64) return wide ? group_kernel<64, uint64_t>() : group_kernel<64, uint32_t>();
    if (threads == 128) return wide ? group_kernel<128, uint64_t>() : group_kernel<128, uint32_t>();
    return wide ? group_kernel<256, uint64_t>() : group_kernel<256, uint32_t>();
}

inline int valid_threads(int t) { return t == 64 ? 64 : (t == 128 ? 128 : 256); }

// Resident blocks per SM of the group kernel for this bucket and block size.
int group_occupancy(const Bucket& B, int threads) {
    threads = valid_threads(threads);
    void* kfn = group_kernel_for(threads, B.wide);
    check(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B.smem), "smem attr");
    int per_sm = 0;
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads, B.smem), "occupancy");
    return std::max(per_sm, 1);
}

// One launch of the group kernel over one bucket's groups: resets the work
// queue and starts min(groups, SMs x blocks_per_sm) persistent blocks.
// threads: 64, 128 or 256 (<= 0: the bucket's default); blocks_per_sm <= 0
// means the occupancy limit.
void launch_bucket(cpb_ctx* ctx, cudaStream_t st, const GroupSetup& su, const Bucket& B, const int32_t* d_list,
                   int* d_queue, int threads, int blocks_per_sm) {
    const int64_t nk = (int64_t)B.groups.size();
    if (nk <= 0) return;
    threads = valid_threads(threads <= 0 ? B.threads : threads);
    const int occ = group_occupancy(B, threads);
    const int per_sm = blocks_per_sm <= 0 ? occ : std::min(blocks_per_sm, occ);
    const int64_t grid = std::min<int64_t>(nk, (int64_t)ctx->n_sm * per_sm);
    check(cudaMemsetAsync(d_queue, 0, sizeof(int), st), "memset");
    KernelScope ks_(ctx, "k_groups",
                    (double)su.total_pixels * (su.eltype == CPB_F64 ? 8 : 4) * (su.gin.iv ? 2 : 1) * nk /
                        std::max<int64_t>(su.plan.n_kernel, 1));
    const size_t smem = B.smem;
#define CPB_GROUPS_LAUNCH(NTV)                                                                                      \
    do {                                                                                                            \
        if (B.wide)                                                                                                 \
            k_groups<NTV, uint64_t><<<(unsigned)grid, NTV, smem, st>>>(B.C, su.dp, su.gin, su.go, d_list, (int)nk, \
                                                                       d_queue);                                   \
        else                                                                                                        \
            k_groups<NTV, uint32_t><<<(unsigned)grid, NTV, smem, st>>>(B.C, su.dp, su.gin, su.go, d_list, (int)nk, \
                                                                       d_queue);                                   \
    } while (0)
    if (threads == 64) CPB_GROUPS_LAUNCH(64);
    else if (threads == 128) CPB_GROUPS_LAUNCH(128);
    else CPB_GROUPS_LAUNCH(256);
#undef CPB_GROUPS_LAUNCH
    check(cudaGetLastError(), "k_groups");
}

// k_group_spread over the kernel-fitted groups (after their bucket launches).
void launch_spread(cpb_ctx* ctx, cudaStream_t st, const GroupSetup& su, const int32_t* d_list, int64_t nk) {
    if (!su.C.sp_on || nk <= 0) return;
    const int threads = 32 * su.sp_nw;
    check(cudaFuncSetAttribute(k_group_spread, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)su.sp_smem),
          "smem attr");
    int per_sm = 0;
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_group_spread, threads, su.sp_smem), "occupancy");
    const int64_t grid = std::min<int64_t>(nk, (int64_t)ctx->n_sm * std::max(per_sm, 1));
    KernelScope ks_(ctx, "k_group_spread", 0.0);
    k_group_spread<<<(unsigned)grid, threads, su.sp_smem, st>>>(su.C, su.dp, su.gin, su.go, d_list, (int)nk);
    check(cudaGetLastError(), "k_group_spread");
}

}  // namespace

int fit_groups_dev(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* P, int64_t G, const int64_t* d_off,
                   const int32_t* d_ny, const int32_t* d_nx, const void* d_pix, int32_t eltype, const void* d_iv,
                   const void* d_bkg, const int64_t* d_soff, const double* d_y0, const double* d_x0,
                   const double* d_f0, int64_t total_pixels, cpb_group_result* out, const int64_t* h_off_opt,
                   const int32_t* h_ny_opt, const int32_t* h_nx_opt, const int64_t* h_soff_opt) {
    NvtxRange nv_("cpb:group_batch");
    cudaStream_t st = ctx->stream;
    GroupSetup su;
    setup_groups(ctx, psf, P, G, d_off, d_ny, d_nx, d_pix, eltype, d_iv, d_bkg, d_soff, d_y0, d_x0, d_f0,
                 total_pixels, out, h_off_opt, h_ny_opt, h_nx_opt, h_soff_opt, su);
    out->n_kernel_groups = 0;
    out->n_routed_groups = 0;
    out->device_seconds = 0;
    if (G == 0) return 0;
    const GroupPlan& plan = su.plan;
    const std::vector<int64_t>& h_off = su.h_off;
    const std::vector<int64_t>& h_soff = su.h_soff;
    const std::vector<int32_t>& h_ny = su.h_ny;
    const std::vector<int32_t>& h_nx = su.h_nx;
    check(cudaEventRecord(ctx->ev0, st), "event");
    const int64_t nk = plan.n_kernel;
    if (nk > 0) {
        // every bucket's group list back to back, one queue counter per bucket
        std::vector<int32_t> lists;
        for (const Bucket& B : plan.buckets) lists.insert(lists.end(), B.groups.begin(), B.groups.end());
        if (su.C.sp_on) {
            double h_rule[kSpreadRuleLen];
            spread_rule(h_rule);
            auto* d_rule = (double*)scratch(ctx, "grp_sp_rule", sizeof(h_rule));
            check(cudaMemcpyAsync(d_rule, h_rule, sizeof(h_rule), cudaMemcpyHostToDevice, st), "h2d");
            su.go.sp_rule = d_rule;
            su.go.sp_rw = (double*)scratch(ctx, "grp_sp_rw", sizeof(double) * 2 * su.C.sp_box * su.n_stars);
        }
        int32_t* d_list = (int32_t*)scratch(ctx, "grp_list", sizeof(int32_t) * nk);
        int* d_queue = (int*)scratch(ctx, "grp_queue", sizeof(int) * plan.buckets.size());
        check(cudaMemcpyAsync(d_list, lists.data(), sizeof(int32_t) * nk, cudaMemcpyHostToDevice, st), "h2d");
        int64_t at = 0;
        for (size_t b = 0; b < plan.buckets.size(); ++b) {
            launch_bucket(ctx, st, su, plan.buckets[b], d_list + at, d_queue + b, 0, 0);
            at += (int64_t)plan.buckets[b].groups.size();
        }
        launch_spread(ctx, st, su, d_list, nk);
    }
    check(cudaEventRecord(ctx->ev1, st), "event");
    check(cudaStreamSynchronize(st), "sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    out->device_seconds = ms * 1e-3;
    out->n_kernel_groups = nk;
    out->n_routed_groups = (int64_t)plan.routed_groups.size();
    // groups too large for one block: the full-field path, one at a time
    for (int32_t g : plan.routed_groups) {
        const int64_t s0 = h_soff[g], ng = h_soff[g + 1] - h_soff[g];
        const int ny = h_ny[g], nx = h_nx[g];
        const size_t esz = eltype == CPB_F64 ? 8 : 4;
        const int64_t off = h_off[g];
        std::vector<double> y(ng), x(ng), f(ng), b(ng), ey(ng), ex(ng), ef(ng), eb(ng), chi(ng), q1(ng), q2(ng),
            q3(ng), cr(ng), sm(ng), sme(ng);
        std::vector<uint8_t> cv(ng), va(ng);
        std::vector<int32_t> it(ng);
        std::vector<double> res(out->residual ? (size_t)ny * nx : 0);
        cpb_sim_result r{};
        r.y = y.data();
        r.x = x.data();
        r.flux = f.data();
        r.bkg = b.data();
        r.y_err = ey.data();
        r.x_err = ex.data();
        r.flux_err = ef.data();
        r.bkg_err = eb.data();
        r.converged = cv.data();
        r.valid = va.data();
        r.chisq = chi.data();
        r.qfit = q1.data();
        r.qfit_expected = q2.data();
        r.qfit_z = q3.data();
        r.crowding = cr.data();
        r.spread_model = sm.data();
        r.spread_model_err = sme.data();
        r.n_iter = it.data();
        r.residual = out->residual ? res.data() : nullptr;
        int32_t status = 0, kind = 0;
        try {
            fit_simultaneous_dev(ctx, psf, P, (const char*)d_pix + esz * off, eltype, ny, nx,
                                 d_iv ? (const char*)d_iv + esz * off : nullptr,
                                 d_bkg ? (const char*)d_bkg + esz * off : nullptr, ng, d_y0 + s0, d_x0 + s0,
                                 d_f0 + s0, &r);
        } catch (const ArgError& e) {
            status = CPB_ERR_ARGUMENT;
            kind = e.msg.find("non-finite") != std::string::npos ? 1 : 2;
            std::vector<double> hy(ng), hx(ng), hf(ng);
            if (ng > 0) {
                // on the context's stream (non-blocking: a legacy-stream copy would not
                // wait for the catalogue's upload)
                check(cudaMemcpyAsync(hy.data(), d_y0 + s0, 8 * ng, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
                check(cudaMemcpyAsync(hx.data(), d_x0 + s0, 8 * ng, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
                check(cudaMemcpyAsync(hf.data(), d_f0 + s0, 8 * ng, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
                check(cudaStreamSynchronize(ctx->stream), "d2h");
            }
            const double NaN = std::numeric_limits<double>::quiet_NaN();
            for (int64_t i = 0; i < ng; ++i) {
                y[i] = (P->free_mask & CPB_FREE_Y) ? hy[i] : P->fixed_y;
                x[i] = (P->free_mask & CPB_FREE_X) ? hx[i] : P->fixed_x;
                f[i] = (P->free_mask & CPB_FREE_FLUX) ? hf[i] : P->fixed_flux;
                ey[i] = (P->free_mask & CPB_FREE_Y) ? NaN : 0.0;
                ex[i] = (P->free_mask & CPB_FREE_X) ? NaN : 0.0;
                ef[i] = (P->free_mask & CPB_FREE_FLUX) ? NaN : 0.0;
                cv[i] = 0;
                va[i] = 0;
                it[i] = 0;
                chi[i] = 0.0;
                q1[i] = q2[i] = q3[i] = cr[i] = sm[i] = sme[i] = NaN;
            }
            std::fill(res.begin(), res.end(), 0.0);
            r.n_passes = 0;
            r.n_failed = (int32_t)ng;
            r.n_active = 0;
            r.n_union = 0;
            r.n_trials = 0;
            r.n_lsqr_iters = 0;
        }
        auto up = [&](void* dst, const void* src, size_t bytes) {
            if (dst && bytes) check(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice), "h2d routed group");
        };
        up(out->y + s0, y.data(), 8 * ng);
        up(out->x + s0, x.data(), 8 * ng);
        up(out->flux + s0, f.data(), 8 * ng);
        up(out->y_err + s0, ey.data(), 8 * ng);
        up(out->x_err + s0, ex.data(), 8 * ng);
        up(out->flux_err + s0, ef.data(), 8 * ng);
        up(out->converged + s0, cv.data(), ng);
        up(out->valid + s0, va.data(), ng);
        up(out->n_iter + s0, it.data(), 4 * ng);
        if (out->chisq) up(out->chisq + s0, chi.data(), 8 * ng);
        if (out->qfit) up(out->qfit + s0, q1.data(), 8 * ng);
        if (out->qfit_expected) up(out->qfit_expected + s0, q2.data(), 8 * ng);
        if (out->qfit_z) up(out->qfit_z + s0, q3.data(), 8 * ng);
        if (out->crowding) up(out->crowding + s0, cr.data(), 8 * ng);
        if (out->spread_model) up(out->spread_model + s0, sm.data(), 8 * ng);
        if (out->spread_model_err) up(out->spread_model_err + s0, sme.data(), 8 * ng);
        if (out->residual) up(out->residual + off, res.data(), 8 * res.size());
        const int32_t na = (int32_t)r.n_active, nu = (int32_t)r.n_union, ntr = (int32_t)r.n_trials,
                      nls = (int32_t)r.n_lsqr_iters;
        up(out->n_passes + g, &r.n_passes, 4);
        up(out->n_failed + g, &r.n_failed, 4);
        up(out->status + g, &status, 4);
        if (out->error_kind) up(out->error_kind + g, &kind, 4);
        if (out->n_active) up(out->n_active + g, &na, 4);
        if (out->n_union) up(out->n_union + g, &nu, 4);
        if (out->n_trials) up(out->n_trials + g, &ntr, 4);
        if (out->n_lsqr_iters) up(out->n_lsqr_iters + g, &nls, 4);
        out->device_seconds += r.device_seconds;
    }
    return 0;
}


// ---------------------------------------------------------------------------
// A bound batch over fixed device buffers (CUDA-graph capture and tuning)
// ---------------------------------------------------------------------------
struct GroupBatch {
    GroupSetup su;
    int32_t* d_list = nullptr;  // owned: every bucket's groups back to back
    int* d_queue = nullptr;     // owned: one counter per bucket
    std::vector<int64_t> at;    // first list entry of each bucket
    std::vector<int> threads;   // chosen block size per bucket
    double* sp_buf = nullptr;   // owned: spread_model rule and the stars' residual / weight planes
};

GroupBatch* group_batch_create(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* P, int64_t G,
                               const int64_t* d_off, const int32_t* d_ny, const int32_t* d_nx, const void* d_pix,
                               int32_t eltype, const void* d_iv, const void* d_bkg, const int64_t* d_soff,
                               const double* d_y0, const double* d_x0, const double* d_f0, int64_t total_pixels,
                               const cpb_group_result* out) {
    if (G > 0 && (!d_off || !d_ny || !d_nx || !d_pix || !d_soff || !d_y0 || !d_x0 || !d_f0 || !out))
        throw ArgError{"null argument"};
    auto* b = new GroupBatch();
    try {
        if (G > 0)
            setup_groups(ctx, psf, P, G, d_off, d_ny, d_nx, d_pix, eltype, d_iv, d_bkg, d_soff, d_y0, d_x0, d_f0,
                         total_pixels, out, nullptr, nullptr, nullptr, nullptr, b->su);
        const GroupPlan& plan = b->su.plan;
        if (!plan.routed_groups.empty() &&
            (P->solver == CPB_SOLVER_LSMR || P->model_rad_auto || P->precision != CPB_PREC_FP64))
            throw ArgError{"groups with solver :lsmr, model_rad = :auto or mixed precision are fitted one by one "
                           "by the full-field fit; use cpb_fit_simultaneous_batch instead of a captured batch"};
        if (!plan.routed_groups.empty())
            throw ArgError{"group " + std::to_string(plan.routed_groups[0]) +
                           " is too large for one thread block (more than 64 stars, or a working set beyond shared "
                           "memory); fit it with cpb_fit_simultaneous_batch instead of a captured batch"};
        std::vector<int32_t> lists;
        for (const Bucket& B : plan.buckets) {
            b->at.push_back((int64_t)lists.size());
            b->threads.push_back(B.threads);
            lists.insert(lists.end(), B.groups.begin(), B.groups.end());
        }
        if (cudaMalloc(&b->d_list, sizeof(int32_t) * std::max<size_t>(lists.size(), 1)) != cudaSuccess ||
            cudaMalloc(&b->d_queue, sizeof(int) * std::max<size_t>(plan.buckets.size(), 1)) != cudaSuccess) {
            cudaGetLastError();
            throw OomError{"device memory exhausted allocating the group work queues"};
        }
        if (!lists.empty())
            check(cudaMemcpy(b->d_list, lists.data(), sizeof(int32_t) * lists.size(), cudaMemcpyHostToDevice),
                  "h2d");
        GroupSetup& su = b->su;
        if (su.C.sp_on && !plan.buckets.empty()) {
            const size_t n_rule = kSpreadRuleLen, n_rw = (size_t)2 * su.C.sp_box * su.n_stars;
            if (cudaMalloc(&b->sp_buf, sizeof(double) * (n_rule + n_rw)) != cudaSuccess) {
                cudaGetLastError();
                throw OomError{"device memory exhausted allocating the spread_model planes"};
            }
            double h_rule[kSpreadRuleLen];
            spread_rule(h_rule);
            check(cudaMemcpy(b->sp_buf, h_rule, sizeof(h_rule), cudaMemcpyHostToDevice), "h2d");
            su.go.sp_rule = b->sp_buf;
            su.go.sp_rw = b->sp_buf + n_rule;
        }
    } catch (...) {
        cudaFree(b->sp_buf);
        cudaFree(b->d_list);
        cudaFree(b->d_queue);
        delete b;
        throw;
    }
    return b;
}

int group_batch_buckets(const GroupBatch* b) { return (int)b->su.plan.buckets.size(); }

// bucket < 0: every bucket, each with its chosen block size; threads <= 0: the chosen one.
void group_batch_enqueue(cpb_ctx* ctx, GroupBatch* b, cudaStream_t st, int bucket, int threads) {
    const auto& bks = b->su.plan.buckets;
    for (int k = 0; k < (int)bks.size(); ++k) {
        if (bucket >= 0 && k != bucket) continue;
        launch_bucket(ctx, st, b->su, bks[k], b->d_list + b->at[k], b->d_queue + k,
                      threads > 0 ? threads : b->threads[k], 0);
    }
    if (bucket < 0) launch_spread(ctx, st, b->su, b->d_list, group_batch_size(b));
}

void group_batch_set_threads(GroupBatch* b, int bucket, int threads) { b->threads[bucket] = valid_threads(threads); }
int group_batch_threads(const GroupBatch* b, int bucket) { return b->threads[bucket]; }
int group_batch_occupancy(GroupBatch* b, int bucket, int threads) {
    return group_occupancy(b->su.plan.buckets[bucket], threads);
}
int64_t group_batch_size(const GroupBatch* b) { return b->su.plan.n_kernel; }

// Tuning signature of one bucket: what its best block size depends on.
std::string group_batch_signature(const GroupBatch* b, int bucket) {
    const GroupSetup& su = b->su;
    const Bucket& B = su.plan.buckets[bucket];
    char buf[256];
    std::snprintf(buf, sizeof(buf), "groups psf%d nodes%d el%d p%d S2_%d mR%d nmax%d umax%d G2^%d", su.dp.kind,
                  su.dp.n_nodes, su.eltype, su.C.p, su.C.S2, su.C.mR, B.nmax, B.umax,
                  (int)std::log2((double)std::max<size_t>(B.groups.size(), 1)));
    return buf;
}

void group_batch_destroy(GroupBatch* b) {
    if (!b) return;
    cudaFree(b->sp_buf);
    cudaFree(b->d_list);
    cudaFree(b->d_queue);
    delete b;
}

}  // namespace cpb
