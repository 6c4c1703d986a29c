// cpb_multipass.cu -- CrowdPhot.fit_all_stars (sequential multi-pass photometry).
//
// Restates src/photometry/psf_photometry_single.jl:267-469.  Each pass visits
// the valid stars brightest first; a star is added back into the running
// residual image (passes 2+), fitted with fit_star on its +-fit_rad box and
// subtracted with its new model.  The only coupling between two stars of a
// pass is the pixels their boxes share, and the boxes are fixed when the pass
// starts (a star's box comes from its parameters before it is refitted), so
// the visit order is replaced by batches: star s goes into batch
// 1 + max{batch(t) : t earlier than s and box(t) meets box(s)}.  Stars of one
// batch have pairwise disjoint boxes, every star they depend on is in an
// earlier batch, and each pixel sees its adds and subtracts in the reference's
// order -- so the result is the sequential one, while each batch is one
// add-back launch, one cutout gather, one batched LM launch (the fit_star
// kernel of cpb_lm.cu), one bookkeeping launch and one subtract launch.  The
// per-star state lives on the device for the whole pass; the host plans a pass
// (brightness order, boxes, batches) from the state read back once per pass.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <unordered_map>
#include <vector>

#include "cpb_internal.cuh"

namespace cpb {
namespace {

struct MPFree {
    int idx[5];  // the free parameters' rows
};

struct MPConst {
    int np;           // model parameters per star (4 image PSFs, 5 Gaussian)
    int gauss;
    int ry, rx, rf, rb, rw;  // rows of y, x, flux, bkg, fwhm (-1: none)
};

// The star's model at pixel (i, j) from its parameter row.
__device__ __forceinline__ double mp_model(const DevPsf& P, const MPConst& M, const double* pr, int i, int j) {
    StarCoef c;
    c.y = pr[M.ry];
    c.x = pr[M.rx];
    c.flux = pr[M.rf];
    c.bkg = pr[M.rb];
    if (M.gauss) {
        DevPsf Pj = P;
        Pj.fwhm = pr[M.rw];
        double a, b, e;
        return gauss_eval<double, false>(Pj.fwhm, c, (double)i, (double)j, a, b, e);
    }
    grid_corners_dw(P, c.y, c.x, c);
    return model_value<double, double>(P, P.data64, c, (double)i, (double)j);
}

// add_star! / subtract_star! (PSF.jl:420-447) over each star's box: one warp a
// star, lanes over the box pixels.  flags (nullable): stars with 0 are skipped.
__global__ void k_mp_addsub(int nL, const int4* __restrict__ boxes, const double* __restrict__ params,
                            const uint8_t* __restrict__ flags, double sign, DevPsf P, MPConst M, double* residual,
                            int ny) {
    const int lane = threadIdx.x & 31;
    const int s = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    if (s >= nL || (flags && !flags[s])) return;
    const int4 b = boxes[s];  // y1, x1, box rows, box columns
    const double* pr = params + (int64_t)s * M.np;
    for (int e = lane; e < b.z * b.w; e += 32) {
        const int i = b.x + e % b.z, j = b.y + e / b.z;
        const int64_t q = (i - 1) + (int64_t)(j - 1) * ny;
        residual[q] = residual[q] + sign * mp_model(P, M, pr, i, j);
    }
}

template <typename TI>
__global__ void k_mp_cutouts(int nL, const int4* __restrict__ boxes, const int64_t* __restrict__ offs,
                             const double* __restrict__ residual, const TI* __restrict__ iv, int ny,
                             double* __restrict__ pix, double* __restrict__ ivc) {
    const int lane = threadIdx.x & 31;
    const int s = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    if (s >= nL) return;
    const int4 b = boxes[s];
    const int64_t o = offs[s];
    for (int e = lane; e < b.z * b.w; e += 32) {
        const int i = b.x + e % b.z, j = b.y + e / b.z;
        const int64_t q = (i - 1) + (int64_t)(j - 1) * ny;
        pix[o + e] = residual[q];
        if (iv) ivc[o + e] = (double)iv[q];
    }
}

// _star_diagnostics! (psf_photometry_diagnostics.jl:154-231) over the fitted
// box: image is the original data, residual the star's fit residual (every
// model subtracted, its own included), star_model its best-fit render, kept in
// shared memory with its disk-correlated copy for spread_model (D.I null:
// spread_model off).  One block of kDiagThreads a star (grid-stride).  out:
// qfit, qfit_expected, qfit_z, crowding, spread_model, spread_model_err per
// star (NaN where undefined).
template <typename TI>
__global__ void __launch_bounds__(kDiagThreads, 3) k_mp_diag(int nL, const int4* __restrict__ boxes,
                                                         const double* __restrict__ params,
                                                         const uint8_t* __restrict__ flags,
                                                         const TI* __restrict__ img,
                                                         const double* __restrict__ residual,
                                                         const TI* __restrict__ iv, DevPsf P, MPConst M, int n_free,
                                                         int ny, SpreadDev D, int smode, int boxmax, double* __restrict__ out) {
    extern __shared__ double stamp[];  // model stamp, x-pass scratch, disk-correlated stamp
    __shared__ double red[12 * (kDiagThreads / 32)];
    const double NaN = __longlong_as_double(0x7ff8000000000000LL);
    const int mode = D.I ? smode : 0;
    double* Is = stamp + 7 * boxmax;  // mode 1: the six profiles
    if (mode == 1)
        for (int i = threadIdx.x; i < 6 * (2 * D.kh + 1); i += blockDim.x) Is[i] = D.I[i];
    for (int s = blockIdx.x; s < nL; s += gridDim.x) {
        __syncthreads();  // the previous star's stamps are no longer read
        double* o = out + (int64_t)s * 6;
        const double* pr = params + (int64_t)s * M.np;
        const double flux = pr[M.rf], bkg = pr[M.rb];
        if (flags[s] != 2 || !(flux > 0)) {  // 2: fitted in this batch
            if (threadIdx.x == 0) o[0] = o[1] = o[2] = o[3] = o[4] = o[5] = NaN;
            continue;
        }
        const int4 b = boxes[s];
        const int nb = b.z * b.w;
        const bool spread = mode != 0 && nb <= boxmax;
        double* G = stamp + 2 * boxmax;  // mode 2: the correlated stamp
        if (spread) {
            for (int e = threadIdx.x; e < nb; e += blockDim.x) stamp[e] = mp_model(P, M, pr, b.x + e % b.z, b.y + e / b.z);
            __syncthreads();
            if (mode == 1) {
                spread_xpass_all(D, Is, stamp, stamp + boxmax, boxmax, b.z, b.w);
                __syncthreads();
            } else {
                spread_stamp_block(D, stamp, stamp + boxmax, G, b.z, b.w);
            }
        }
        const double inv_flux = 1.0 / flux;
        // qv ncl ndi den ss ss2 Sp Sq Sp0 Sq0 SqG ngood
        double v[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int e = threadIdx.x; e < nb; e += blockDim.x) {
            const int i = b.x + e % b.z, j = b.y + e / b.z;
            const int64_t q = (i - 1) + (int64_t)(j - 1) * ny;
            const double wp = iv ? (double)iv[q] : 1.0;
            if (isfinite(wp) && wp > 0) {
                const double mv = spread ? stamp[e] : mp_model(P, M, pr, i, j);
                const double r = residual[q];
                v[0] += fabs(r);
                const double Pp = (mv - bkg) * inv_flux;
                const double wP = wp * Pp;
                const double p_i = r + mv - bkg;
                v[1] += wP * p_i;
                v[2] += wP * ((double)img[q] - bkg);
                v[3] += wP * Pp;
                if (spread) {
                    const double gm = mode == 1 ? spread_ypass(D, Is, stamp + boxmax, boxmax, b.z, e) : G[e];
                    const double g_i = (gm - bkg) * inv_flux;
                    v[6] += wP * p_i;
                    v[7] += wp * g_i * p_i;
                    v[8] += wP * Pp;
                    v[9] += wp * Pp * g_i;
                    v[10] += wp * g_i * g_i;
                }
            }
            if (iv) {
                const double vq = (double)iv[q];
                if (isfinite(vq) && vq > 0) {
                    const double si = 1.0 / sqrt(vq);
                    v[4] += si;
                    v[5] += si * si;
                    v[11] += 1.0;
                }
            }
        }
        block_sum_n<12>(v, red);
        if (threadIdx.x == 0) {
            const double qv = v[0], ncl = v[1], ndi = v[2], den = v[3], ss = v[4], ss2 = v[5];
            const double Sp = v[6], Sq = v[7], Sp0 = v[8], Sq0 = v[9], SqG = v[10];
            const int ngood = (int)v[11];
            const double c2p = 0.7978845608028654;  // sqrt(2 / pi)
            o[0] = qv * inv_flux;
            o[3] = (den > 0 && ncl > 0 && ndi > 0) ? 2.5 * log10(ndi / ncl) : NaN;
            o[1] = iv ? c2p * ss * inv_flux : NaN;
            o[2] = NaN;
            if (iv && ss2 > 0 && ngood > n_free) {
                const double dfac = sqrt(1.0 - (double)n_free / (double)ngood);
                o[2] = (qv - c2p * dfac * ss) / (sqrt((1.0 - 2.0 / 3.141592653589793) * ss2) * dfac);
            }
            o[4] = o[5] = NaN;
            if (spread && Sp > 0) {
                o[4] = Sq / Sp - Sq0 / Sp0;
                if (iv) o[5] = sqrt(fmax(0.0, Sp * Sp * SqG + Sq * Sq * Sp0 - 2 * Sq * Sp * Sq0)) / (Sp * Sp);
            }
        }
    }
}

template <typename TI>
__global__ void k_mp_init(int64_t npix, const TI* __restrict__ img, double* __restrict__ residual) {
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q < npix) residual[q] = (double)img[q];
}

// Bookkeeping of one batch after its fit_star launch (:373-401), one thread a
// star: on success the star's parameters, errors of the free parameters,
// convergence, chi^2 and iteration count are updated and its new model is
// queued for subtraction (flag 2); a fit that failed the input checks
// invalidates the star and, on passes 2+, queues its previous model again to
// undo the add-back (flag 1).  Positions index the batch; idx maps them to stars.
__global__ void k_mp_book(int nL, const int32_t* __restrict__ idx, int pass, int np, int nf, MPFree F,
                          const double* __restrict__ lm_params, const double* __restrict__ lm_cov,
                          const double* __restrict__ lm_chisq, const uint8_t* __restrict__ lm_conv,
                          const int32_t* __restrict__ lm_iters, const int32_t* __restrict__ lm_status,
                          const double* __restrict__ pin, double* __restrict__ prm, double* __restrict__ err,
                          uint8_t* __restrict__ conv, double* __restrict__ chisq, int32_t* __restrict__ niter,
                          uint8_t* __restrict__ valid, int* __restrict__ n_failed, double* __restrict__ psub,
                          uint8_t* __restrict__ flag) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nL) return;
    const int64_t s = idx[k];
    if (lm_status[k] != 0) {  // fit_star threw (:391-401)
        valid[s] = 0;
        atomicAdd(n_failed, 1);
        for (int q = 0; q < np; ++q) psub[(int64_t)k * np + q] = pin[(int64_t)k * np + q];
        flag[k] = pass > 1 ? 1 : 0;
        return;
    }
    for (int q = 0; q < np; ++q) {
        const double v = lm_params[(int64_t)k * np + q];
        prm[s * np + q] = v;
        psub[(int64_t)k * np + q] = v;
    }
    for (int a = 0; a < nf; ++a)
        err[s * np + F.idx[a]] = sqrt(fmax(0.0, lm_cov[(int64_t)k * nf * nf + a + a * nf]));
    conv[s] = lm_conv[k];
    chisq[s] = lm_chisq[k];
    niter[s] += lm_iters[k];
    flag[k] = 2;
}

inline unsigned warps_grid(int64_t n) { return (unsigned)std::max<int64_t>(1, (n * 32 + 255) / 256); }

}  // namespace

int fit_all_stars_dev(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* P, double fit_rad, int n_passes,
                      double spread_model_fwhm, const void* d_img, int32_t eltype, int64_t ny64, int64_t nx64,
                      const void* d_iv, int64_t n, const double* init, cpb_multipass_result* out) {
    if (!(n_passes > 0)) throw ArgError{"n_passes must be positive, got " + std::to_string(n_passes)};
    if (eltype != CPB_F32 && eltype != CPB_F64) throw ArgError{"unsupported image eltype"};
    if (ny64 <= 0 || nx64 <= 0 || ny64 * nx64 >= (1LL << 31)) throw ArgError{"image size out of range"};
    if (P->precision != CPB_PREC_FP64) throw ArgError{"only the FP64 precision form is built for fit_all_stars"};
    if (!out->params || !out->errors || !out->converged || !out->valid || !out->chisq || !out->n_iter)
        throw ArgError{"null output array"};
    const int ny = (int)ny64, nx = (int)nx64;
    const int64_t npix = ny64 * nx64;
    cudaStream_t st = ctx->stream;
    const DevPsf dp = psf->dev;
    MPConst M{};
    M.gauss = dp.kind == CPB_PSF_CIRCULAR_GAUSSIAN ? 1 : 0;
    M.np = M.gauss ? 5 : 4;
    M.ry = 0;
    M.rx = 1;
    M.rw = M.gauss ? 2 : -1;
    M.rf = M.gauss ? 3 : 2;
    M.rb = M.gauss ? 4 : 3;
    // free set in getproperties order (psf_fitting.jl:8-26)
    const int bits_g[5] = {CPB_FREE_Y, CPB_FREE_X, CPB_FREE_FWHM, CPB_FREE_FLUX, CPB_FREE_BKG};
    const int bits_i[4] = {CPB_FREE_Y, CPB_FREE_X, CPB_FREE_FLUX, CPB_FREE_BKG};
    std::vector<int> free_idx;
    for (int q = 0; q < M.np; ++q)
        if (P->free_mask & (M.gauss ? bits_g[q] : bits_i[q])) free_idx.push_back(q);
    if (free_idx.empty()) throw ArgError{"all model parameters are fixed; nothing to fit"};
    const int nf = (int)free_idx.size();
    const int np = M.np;
    const double NaN = std::numeric_limits<double>::quiet_NaN();

    out->n_passes = n_passes;
    out->n_failed = 0;
    out->n_levels = 0;
    out->n_fits = 0;
    out->device_seconds = 0;
    // per-star state (host): parameters, errors, flags (:282-323)
    std::vector<double> prm(init, init + n * np), err(n * np, NaN);
    for (int64_t s = 0; s < n; ++s)
        for (int q = 0; q < np; ++q)
            if (std::find(free_idx.begin(), free_idx.end(), q) == free_idx.end()) err[s * np + q] = 0.0;
    std::vector<uint8_t> valid(n, 1), conv(n, 0);
    std::vector<double> chisq(n, 0.0), diag(n * 6, NaN);
    std::vector<int32_t> niter(n, 0);
    if (n == 0) {
        if (out->residual) std::fill(out->residual, out->residual + npix, 0.0);
        return 0;
    }

    double* resid = (double*)scratch(ctx, "mp_residual", sizeof(double) * npix);
    check(cudaEventRecord(ctx->ev0, st), "event");
    if (eltype == CPB_F64)
        k_mp_init<double><<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(npix, (const double*)d_img, resid);
    else
        k_mp_init<float><<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(npix, (const float*)d_img, resid);
    check(cudaGetLastError(), "k_mp_init");

    // per-star state on the device (star order) and per-position buffers of a
    // pass (level order; a pass never holds more than n positions)
    const int Rmax = (int)std::ceil(std::max(fit_rad, 0.0)) + 1;
    const int64_t box_max = (int64_t)(2 * Rmax + 1) * (2 * Rmax + 1);
    double* d_prm = (double*)scratch(ctx, "mp_prm", sizeof(double) * n * np);
    double* d_err = (double*)scratch(ctx, "mp_err", sizeof(double) * n * np);
    double* d_chisq = (double*)scratch(ctx, "mp_chisq", sizeof(double) * n);
    int32_t* d_niter = (int32_t*)scratch(ctx, "mp_niter", sizeof(int32_t) * n);
    uint8_t* d_sflag = (uint8_t*)scratch(ctx, "mp_sflags", (size_t)n * 2);  // valid, converged
    uint8_t* d_valid = d_sflag;
    uint8_t* d_conv = d_sflag + n;
    int* d_nfail = (int*)scratch(ctx, "mp_nfail", sizeof(int));
    int32_t* d_idx = (int32_t*)scratch(ctx, "mp_idx", sizeof(int32_t) * n);
    int4* d_box = (int4*)scratch(ctx, "mp_box", sizeof(int4) * n);
    double* d_pin = (double*)scratch(ctx, "mp_pin", sizeof(double) * n * np);
    double* d_psub = (double*)scratch(ctx, "mp_psub", sizeof(double) * n * np);
    uint8_t* d_flag = (uint8_t*)scratch(ctx, "mp_flag", n);
    int64_t* d_off = (int64_t*)scratch(ctx, "mp_off", sizeof(int64_t) * n);
    int32_t* d_dims = (int32_t*)scratch(ctx, "mp_dims", sizeof(int32_t) * n * 4);  // ny, nx, y1, x1 planes
    double* d_lmd = (double*)scratch(ctx, "mp_lm_f64", sizeof(double) * n * (np + nf * nf + 4));
    uint8_t* d_lmu = (uint8_t*)scratch(ctx, "mp_lm_u8", (size_t)n * 4);
    int32_t* d_lmi = (int32_t*)scratch(ctx, "mp_lm_i32", sizeof(int32_t) * n * 2);
    double* d_diag = (double*)scratch(ctx, "mp_diag", sizeof(double) * n * 6);
    // cutout pixels of one batch: the largest batch of a pass sizes them (grown on demand)
    check(cudaMemcpyAsync(d_prm, prm.data(), sizeof(double) * n * np, cudaMemcpyHostToDevice, st), "h2d");
    check(cudaMemcpyAsync(d_err, err.data(), sizeof(double) * n * np, cudaMemcpyHostToDevice, st), "h2d");
    check(cudaMemsetAsync(d_chisq, 0, sizeof(double) * n, st), "memset");
    check(cudaMemsetAsync(d_niter, 0, sizeof(int32_t) * n, st), "memset");
    check(cudaMemsetAsync(d_conv, 0, (size_t)n, st), "memset");
    check(cudaMemsetAsync(d_nfail, 0, sizeof(int), st), "memset");
    MPFree F{};
    for (int a = 0; a < nf; ++a) F.idx[a] = free_idx[a];
    // spread_model reference disk (the first catalogue star fixes the PSF's effective width)
    SpreadHost sh;
    SpreadDev sd{};
    const int boxmax = (int)box_max;
    int smode = 0;
    if (spread_kernel(psf, psf->dev.fwhm, spread_model_fwhm, init[0], init[1], fit_rad, sh) &&
        (smode = spread_mode(boxmax, sh.kh)) != 0) {
        double* d_I = (double*)scratch(ctx, "mp_spread_I", sizeof(double) * sh.I.size());
        check(cudaMemcpyAsync(d_I, sh.I.data(), sizeof(double) * sh.I.size(), cudaMemcpyHostToDevice, st), "h2d");
        sd.I = d_I;
        sd.kh = sh.kh;
        for (int c = 0; c < 6; ++c) sd.alpha[c] = sh.alpha[c], sd.L[c] = sh.L[c];
    }
    const size_t diag_smem = spread_smem_bytes(smode, boxmax, sd.kh);
    if (diag_smem > 48 * 1024) {
        check(cudaFuncSetAttribute(k_mp_diag<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)diag_smem),
              "smem attr");
        check(cudaFuncSetAttribute(k_mp_diag<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)diag_smem),
              "smem attr");
    }

    // host plan of one pass (level order)
    std::vector<int32_t> hidx;
    std::vector<int4> hbox;
    std::vector<double> hpin;
    std::vector<int64_t> hoff;
    std::vector<int32_t> hdims;
    std::vector<int64_t> lev_start, lev_pix;
    std::vector<double> hdiag;
    const double FTfit = fit_rad;

    for (int pass = 1; pass <= n_passes; ++pass) {
        // brightest first, stable (sortperm(rev = true))
        std::vector<int64_t> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(),
                         [&](int64_t a, int64_t b) { return prm[a * np + M.rf] > prm[b * np + M.rf]; });
        // boxes at the pass start and the batch of every valid star
        std::vector<int4> box(n);
        std::vector<int> level(n, -1);
        int nlev = 0;
        {
            const int cell = 2 * Rmax + 2;
            const int gnx = nx / cell + 2;
            std::unordered_map<int64_t, std::vector<int64_t>> grid;
            for (int64_t s : order) {
                if (!valid[s]) continue;
                const double y = prm[s * np + M.ry], x = prm[s * np + M.rx];
                if (!(std::isfinite(y) && std::isfinite(x))) {
                    valid[s] = 0;
                    continue;
                }
                int ylo = (int)std::max(std::floor(y - FTfit), 1.0), yhi = (int)std::min(std::ceil(y + FTfit), (double)ny);
                int xlo = (int)std::max(std::floor(x - FTfit), 1.0), xhi = (int)std::min(std::ceil(x + FTfit), (double)nx);
                const int64_t by = std::max(yhi - ylo + 1, 0), bx = std::max(xhi - xlo + 1, 0);
                if (by * bx < 3) {  // :343-348
                    valid[s] = 0;
                    continue;
                }
                box[s] = make_int4(ylo, xlo, (int)by, (int)bx);
                int lv = 0;
                const int cy0 = (ylo - 1) / cell, cy1 = (yhi - 1) / cell, cx0 = (xlo - 1) / cell, cx1 = (xhi - 1) / cell;
                for (int cx = cx0; cx <= cx1; ++cx)
                    for (int cy = cy0; cy <= cy1; ++cy) {
                        auto it = grid.find((int64_t)cy * gnx + cx);
                        if (it == grid.end()) continue;
                        for (int64_t t : it->second) {
                            const int4& bt = box[t];
                            if (bt.x <= yhi && ylo <= bt.x + bt.z - 1 && bt.y <= xhi && xlo <= bt.y + bt.w - 1)
                                lv = std::max(lv, level[t] + 1);
                        }
                    }
                level[s] = lv;
                nlev = std::max(nlev, lv + 1);
                for (int cx = cx0; cx <= cx1; ++cx)
                    for (int cy = cy0; cy <= cy1; ++cy) grid[(int64_t)cy * gnx + cx].push_back(s);
            }
        }
        // positions in level order (brightness order inside a level), each
        // batch's cutouts packed from offset 0
        std::vector<int64_t> cnt(nlev + 1, 0);
        for (int64_t s : order)
            if (valid[s] && level[s] >= 0) cnt[level[s] + 1] += 1;
        lev_start.assign(nlev + 1, 0);
        for (int L = 0; L < nlev; ++L) lev_start[L + 1] = lev_start[L] + cnt[L + 1];
        const int64_t npos = lev_start[nlev];
        hidx.resize(npos);
        hbox.resize(npos);
        hpin.resize((size_t)npos * np);
        hoff.resize(npos);
        hdims.resize((size_t)npos * 4);
        lev_pix.assign(nlev, 0);
        {
            std::vector<int64_t> fill(lev_start.begin(), lev_start.end() - 1);
            for (int64_t s : order) {
                if (!(valid[s] && level[s] >= 0)) continue;
                const int L = level[s];
                const int64_t k = fill[L]++;
                hidx[k] = (int32_t)s;
                hbox[k] = box[s];
                std::memcpy(&hpin[(size_t)k * np], &prm[s * np], sizeof(double) * np);
                hoff[k] = lev_pix[L];
                lev_pix[L] += (int64_t)box[s].z * box[s].w;
                hdims[k] = box[s].z;
                hdims[npos + k] = box[s].w;
                hdims[2 * npos + k] = box[s].x;
                hdims[3 * npos + k] = box[s].y;
            }
        }
        out->n_levels += nlev;
        out->n_fits += npos;
        const int64_t pix_max = lev_pix.empty() ? 1 : std::max<int64_t>(1, *std::max_element(lev_pix.begin(), lev_pix.end()));
        double* d_cpix = (double*)scratch(ctx, "mp_cpix", sizeof(double) * pix_max);
        double* d_civ = d_iv ? (double*)scratch(ctx, "mp_civ", sizeof(double) * pix_max) : nullptr;
        if (npos > 0) {
            check(cudaMemcpyAsync(d_valid, valid.data(), (size_t)n, cudaMemcpyHostToDevice, st), "h2d");
            check(cudaMemcpyAsync(d_idx, hidx.data(), sizeof(int32_t) * npos, cudaMemcpyHostToDevice, st), "h2d");
            check(cudaMemcpyAsync(d_box, hbox.data(), sizeof(int4) * npos, cudaMemcpyHostToDevice, st), "h2d");
            check(cudaMemcpyAsync(d_pin, hpin.data(), sizeof(double) * npos * np, cudaMemcpyHostToDevice, st), "h2d");
            check(cudaMemcpyAsync(d_off, hoff.data(), sizeof(int64_t) * npos, cudaMemcpyHostToDevice, st), "h2d");
            check(cudaMemcpyAsync(d_dims, hdims.data(), sizeof(int32_t) * npos * 4, cudaMemcpyHostToDevice, st),
                  "h2d");
        }
        // fit_star results per position
        double* lm_par = d_lmd;
        double* lm_cov = d_lmd + (size_t)npos * np;
        double* lm_sc = d_lmd + (size_t)npos * (np + nf * nf);  // cost, cost_init, chisq, lambda planes
        for (int L = 0; L < nlev; ++L) {
            const int64_t p0 = lev_start[L];
            const int nL = (int)(lev_start[L + 1] - p0);
            if (nL == 0) continue;
            const int64_t tot = lev_pix[L];
            const int4* bx = d_box + p0;
            // passes 2+: the star's previous model goes back in (:360-365)
            if (pass > 1) {
                KernelScope ks_(ctx, "k_mp_addsub", (double)tot * 16);
                k_mp_addsub<<<warps_grid(nL), 256, 0, st>>>(nL, bx, d_pin + p0 * np, nullptr, 1.0, dp, M, resid, ny);
                check(cudaGetLastError(), "k_mp_addsub");
            }
            {
                KernelScope ks_(ctx, "k_mp_cutouts", (double)tot * (d_iv ? 32 : 16));
                if (eltype == CPB_F64)
                    k_mp_cutouts<double><<<warps_grid(nL), 256, 0, st>>>(nL, bx, d_off + p0, resid,
                                                                       (const double*)d_iv, ny, d_cpix, d_civ);
                else
                    k_mp_cutouts<float><<<warps_grid(nL), 256, 0, st>>>(nL, bx, d_off + p0, resid,
                                                                      (const float*)d_iv, ny, d_cpix, d_civ);
                check(cudaGetLastError(), "k_mp_cutouts");
            }
            // fit_star on every box of the batch (:367-371): the fit_star kernel
            cpb_lm_result r{};
            r.params = lm_par + p0 * np;
            r.cov = lm_cov + p0 * nf * nf;
            r.cost = lm_sc + p0;
            r.cost_init = lm_sc + npos + p0;
            r.chisq = lm_sc + 2 * npos + p0;
            r.lambda_final = lm_sc + 3 * npos + p0;
            r.converged = d_lmu + p0;
            r.x_converged = d_lmu + npos + p0;
            r.f_converged = d_lmu + 2 * npos + p0;
            r.g_converged = d_lmu + 3 * npos + p0;
            r.iterations = d_lmi + p0;
            r.status = d_lmi + npos + p0;
            lm_enqueue_device(ctx, psf, P, nL, d_off + p0, d_dims + p0, d_dims + npos + p0, d_dims + 2 * npos + p0,
                              d_dims + 3 * npos + p0, d_cpix, CPB_F64, d_civ, d_pin + p0 * np, tot, &r);
            // bookkeeping (:373-401) and what to subtract
            k_mp_book<<<(unsigned)((nL + 127) / 128), 128, 0, st>>>(
                nL, d_idx + p0, pass, np, nf, F, r.params, r.cov, r.chisq, r.converged, r.iterations, r.status,
                d_pin + p0 * np, d_prm, d_err, d_conv, d_chisq, d_niter, d_valid, d_nfail, d_psub + p0 * np,
                d_flag + p0);
            check(cudaGetLastError(), "k_mp_book");
            {
                KernelScope ks_(ctx, "k_mp_addsub", (double)tot * 16);
                k_mp_addsub<<<warps_grid(nL), 256, 0, st>>>(nL, bx, d_psub + p0 * np, d_flag + p0, -1.0, dp, M, resid,
                                                            ny);
                check(cudaGetLastError(), "k_mp_addsub");
            }
            if (pass == n_passes) {  // diagnostics of the fitted stars (:381-389)
                KernelScope ks_(ctx, "k_mp_diag", (double)tot * (d_iv ? 24 : 16));
                const unsigned g = (unsigned)std::min<int64_t>(nL, (int64_t)ctx->n_sm * 16);
                if (eltype == CPB_F64)
                    k_mp_diag<double><<<g, kDiagThreads, diag_smem, st>>>(
                        nL, bx, d_psub + p0 * np, d_flag + p0, (const double*)d_img, resid, (const double*)d_iv, dp,
                        M, nf, ny, sd, smode, boxmax, d_diag + p0 * 6);
                else
                    k_mp_diag<float><<<g, kDiagThreads, diag_smem, st>>>(
                        nL, bx, d_psub + p0 * np, d_flag + p0, (const float*)d_img, resid, (const float*)d_iv, dp,
                        M, nf, ny, sd, smode, boxmax, d_diag + p0 * 6);
                check(cudaGetLastError(), "k_mp_diag");
            }
        }
        // the pass's state back on the host: parameters and flags for the next
        // pass's plan; on the last pass also the diagnostics of every position
        check(cudaMemcpyAsync(prm.data(), d_prm, sizeof(double) * n * np, cudaMemcpyDeviceToHost, st), "d2h");
        std::vector<uint8_t> hflags((size_t)n * 2);
        check(cudaMemcpyAsync(hflags.data(), d_sflag, (size_t)n * 2, cudaMemcpyDeviceToHost, st), "d2h");
        if (pass == n_passes && npos > 0) {
            hdiag.resize((size_t)npos * 6);
            check(cudaMemcpyAsync(hdiag.data(), d_diag, sizeof(double) * npos * 6, cudaMemcpyDeviceToHost, st), "d2h");
        }
        check(cudaStreamSynchronize(st), "sync");
        if (npos > 0)
            for (int64_t s = 0; s < n; ++s) valid[s] = hflags[s];  // fit failures of this pass
        for (int64_t s = 0; s < n; ++s) conv[s] = hflags[n + s];
        if (pass == n_passes && npos > 0) {
            // diagnostics of the fitted positions (k_mp_diag wrote NaN for the others)
            for (int64_t k = 0; k < npos; ++k)
                for (int t = 0; t < 6; ++t) diag[(int64_t)hidx[k] * 6 + t] = hdiag[(size_t)k * 6 + t];
        }
        // between-pass validation (:404-412)
        for (int64_t s = 0; s < n; ++s) {
            const double y = prm[s * np + M.ry], x = prm[s * np + M.rx], f = prm[s * np + M.rf];
            valid[s] = valid[s] && conv[s] && std::isfinite(y) && std::isfinite(x) && std::isfinite(f) && f > 0;
        }
    }
    check(cudaEventRecord(ctx->ev1, st), "event");
    int nfail = 0;
    check(cudaMemcpyAsync(err.data(), d_err, sizeof(double) * n * np, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(chisq.data(), d_chisq, sizeof(double) * n, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(niter.data(), d_niter, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(&nfail, d_nfail, sizeof(int), cudaMemcpyDeviceToHost, st), "d2h");
    if (out->residual)
        check(cudaMemcpyAsync(out->residual, resid, sizeof(double) * npix, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaStreamSynchronize(st), "sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    out->device_seconds = ms * 1e-3;
    out->n_failed = nfail;
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
    return 0;
}

}  // namespace cpb
