// cpb_internal.cuh -- shared host/device definitions of the B200 PSF-fitting library.
//
// Device PSF arithmetic restates CrowdPhot.jl:
//   bicubic_interpolate / _cubic4        src/psf/empirical_models.jl:185-292
//   _gridded_corner_bicubic_pass!        src/psf/psf_fitting.jl:1233-1321
//   _grid_corners_dw                     src/psf/gridded_psf.jl:176-208
//   CircularGaussianPSF evaluate(_fg)    src/psf/parametric_models.jl:79-115
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <algorithm>
#include <exception>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/crowdphot_b200.h"

namespace cpb {

// ---------------------------------------------------------------------------
// device-side PSF description (passed by value to kernels)
// ---------------------------------------------------------------------------
struct DevNode {
    int64_t off;        // element offset of this node in the concatenated data
    int32_t ny, nx;
    double oy, ox;      // origin.y, origin.x
    double sx, sy;      // oversampling x, y
    double fill;
    // polyphase copy: sample (i, k) (0-based) lives at
    // poff + ((i % isy) + (k % isx) * isy) * PY * PX + (i / isy) + (k / isx) * PY,
    // so the samples one stencil tap needs at consecutive stamp rows are adjacent.
    int64_t poff;
    int32_t PY, PX;     // ceil(ny / isy), ceil(nx / isx)
    int32_t isy, isx;   // integer oversampling (the reference's oversampling is a pair of Ints)
    // edge-padded polyphase copy (fit_star): the node with one replicated sample
    // on every side, so that a clamped stencil (empirical_models.jl:270-285) reads
    // the same values as an interior one; padded sample (i + 1, k + 1) lives at
    // lpoff + (((i + 1) % isy) + ((k + 1) % isx) * isy) * LPY * LPX
    //       + (i + 1) / isy + ((k + 1) / isx) * LPY.
    int64_t lpoff;
    int32_t LPY, LPX;   // ceil((ny + 2) / isy), ceil((nx + 2) / isx)
};

constexpr int kMaxNodes = 64;

struct DevPsf {
    int32_t kind;       // CPB_PSF_*
    int32_t n_nodes;
    int32_t gny, gnx;   // node grid size
    double fwhm;        // CircularGaussianPSF FWHM (the fixed value of the fit)
    const double* data64;
    const float* data32;
    const double* pp64;       // polyphase copies of the node data (see DevNode)
    const float* pp32;
    const double* lpp64;      // edge-padded polyphase copies (see DevNode)
    const DevNode* nodes;     // n_nodes
    const double* ygrid;      // gny
    const double* xgrid;      // gnx
    const int32_t* index_grid;  // gny x gnx column-major, 0-based
    int64_t total_elems;      // sum of padded node sizes
};

// Per-star model coefficients for one parameter vector (theta or theta+delta).
struct StarCoef {
    double y, x, flux, bkg;
    double w[4], dwdy[4], dwdx[4];
    int32_t idx[4];           // node index, -1 = inactive corner
};

// ---------------------------------------------------------------------------
// device math
// ---------------------------------------------------------------------------
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// _grid_corners_dw (gridded_psf.jl:176-208).
__device__ inline void grid_corners_dw(const DevPsf& P, double Y, double X, StarCoef& c) {
    if (P.n_nodes == 1 || P.kind != CPB_PSF_GRIDDED_IMAGE) {
        c.idx[0] = 0;
        c.w[0] = 1.0;
        c.dwdy[0] = 0.0;
        c.dwdx[0] = 0.0;
        for (int k = 1; k < 4; ++k) {
            c.idx[k] = -1;
            c.w[k] = 0.0;
            c.dwdy[k] = 0.0;
            c.dwdx[k] = 0.0;
        }
        return;
    }
    int iy = 0, ix = 0;  // searchsortedlast (1-based count of elements <= value)
    for (int k = 0; k < P.gny; ++k) iy += (P.ygrid[k] <= Y) ? 1 : 0;
    for (int k = 0; k < P.gnx; ++k) ix += (P.xgrid[k] <= X) ? 1 : 0;
    iy = clampi(iy, 1, P.gny - 1);
    ix = clampi(ix, 1, P.gnx - 1);
    double y0 = P.ygrid[iy - 1], y1 = P.ygrid[iy], x0 = P.xgrid[ix - 1], x1 = P.xgrid[ix];
    double Yc = fmin(fmax(Y, y0), y1), Xc = fmin(fmax(X, x0), x1);
    double cy = (Y > y0 && Y < y1) ? 1.0 : 0.0;
    double cx = (X > x0 && X < x1) ? 1.0 : 0.0;
    double invnorm = 1.0 / ((x1 - x0) * (y1 - y0));
    double dy1 = y1 - Yc, dy0 = Yc - y0, dx1 = x1 - Xc, dx0 = Xc - x0;
    const int32_t* ig = P.index_grid;
    int g = P.gny;
    c.idx[0] = ig[(iy - 1) + (ix - 1) * g];
    c.w[0] = dx1 * dy1 * invnorm;
    c.dwdy[0] = -dx1 * cy * invnorm;
    c.dwdx[0] = -dy1 * cx * invnorm;
    c.idx[1] = ig[(iy - 1) + ix * g];
    c.w[1] = dx0 * dy1 * invnorm;
    c.dwdy[1] = -dx0 * cy * invnorm;
    c.dwdx[1] = dy1 * cx * invnorm;
    c.idx[2] = ig[iy + (ix - 1) * g];
    c.w[2] = dx1 * dy0 * invnorm;
    c.dwdy[2] = dx1 * cy * invnorm;
    c.dwdx[2] = -dy0 * cx * invnorm;
    c.idx[3] = ig[iy + ix * g];
    c.w[3] = dx0 * dy0 * invnorm;
    c.dwdy[3] = dx0 * cy * invnorm;
    c.dwdx[3] = dy0 * cx * invnorm;
    for (int k = 0; k < 4; ++k)
        if (c.w[k] == 0.0 && c.dwdy[k] == 0.0 && c.dwdx[k] == 0.0) c.idx[k] = -1;
}

// One node's bicubic value and grid derivatives at detector pixel (py, px)
// for a star centred at (Y, X) -- the per-pixel body of
// _gridded_corner_bicubic_pass!.  D = element type of the tabulated data,
// M = arithmetic type.  NEED_D = false skips the derivative arithmetic.
template <typename D, typename M, bool NEED_D>
__device__ __forceinline__ void corner_eval(const D* __restrict__ data, const DevNode& nd, M Y, M X, M py, M px, M& pv,
                                            M& pdv, M& pdu) {
    const M u = (M)nd.sx * (px - X) + (M)nd.ox;
    const M v = (M)nd.sy * (py - Y) + (M)nd.oy;
    const int nyd = nd.ny, nxd = nd.nx;
    const bool inb = isfinite(u) && isfinite(v) && u >= (M)1 && u <= (M)nxd && v >= (M)1 && v <= (M)nyd;
    const M uc = inb ? u : (M)1, vc = inb ? v : (M)1;
    const int lx = clampi((int)floor(uc), 1, nxd - 1);
    const int ly = clampi((int)floor(vc), 1, nyd - 1);
    const M du = uc - (M)lx, dv = vc - (M)ly;
    const int ix0 = clampi(lx - 1, 1, nxd) - 1, ix1 = lx - 1, ix2 = lx, ix3 = clampi(lx + 2, 1, nxd) - 1;
    const int iy0 = clampi(ly - 1, 1, nyd) - 1, iy1 = ly - 1, iy2 = ly, iy3 = clampi(ly + 2, 1, nyd) - 1;
    const D* c0 = data + (int64_t)ix0 * nyd;
    const D* c1 = data + (int64_t)ix1 * nyd;
    const D* c2 = data + (int64_t)ix2 * nyd;
    const D* c3 = data + (int64_t)ix3 * nyd;
    M row[4], drow[4];
    const int iys[4] = {iy0, iy1, iy2, iy3};
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const M a = (M)c0[iys[r]], b = (M)c1[iys[r]], c = (M)c2[iys[r]], e = (M)c3[iys[r]];
        const M k1 = (c - a) / 2;
        const M k4 = c - b - k1;
        const M k2 = 3 * k4 - (e - b) / 2 + k1;
        const M k3 = k4 - k2;
        row[r] = du * (du * (du * k3 + k2) + k1) + b;
        if (NEED_D) drow[r] = du * (3 * du * k3 + 2 * k2) + k1;
    }
    const M v1 = (row[2] - row[0]) / 2;
    const M v4 = row[2] - row[1] - v1;
    const M v2 = 3 * v4 - (row[3] - row[1]) / 2 + v1;
    const M v3 = v4 - v2;
    const M val = dv * (dv * (dv * v3 + v2) + v1) + row[1];
    pv = inb ? val : (M)nd.fill;
    if (NEED_D) {
        const M dpdv = dv * (3 * dv * v3 + 2 * v2) + v1;
        const M u1 = (drow[2] - drow[0]) / 2;
        const M u4 = drow[2] - drow[1] - u1;
        const M u2 = 3 * u4 - (drow[3] - drow[1]) / 2 + u1;
        const M u3 = u4 - u2;
        const M dpdu = dv * (dv * (dv * u3 + u2) + u1) + drow[1];
        pdv = inb ? dpdv : (M)0;
        pdu = inb ? dpdu : (M)0;
    }
}

template <typename D>
__device__ __forceinline__ const D* node_data(const DevPsf& P);
template <>
__device__ __forceinline__ const double* node_data<double>(const DevPsf& P) { return P.data64; }
template <>
__device__ __forceinline__ const float* node_data<float>(const DevPsf& P) { return P.data32; }

// Unit-flux profile s and ds/dY, ds/dX (gridded chain rule, psf_photometry_simultaneous.jl:500-512).
// `base` points at the (possibly shared-memory) concatenated node data.
template <typename D, typename M, bool NEED_D>
__device__ __forceinline__ void grid_profile(const DevPsf& P, const D* __restrict__ base, const StarCoef& c, M py,
                                             M px, M& s, M& dsdY, M& dsdX) {
    s = 0;
    dsdY = 0;
    dsdX = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (c.idx[k] < 0) continue;
        const DevNode nd = P.nodes[c.idx[k]];
        M pv, pdv = 0, pdu = 0;
        corner_eval<D, M, NEED_D>(base + nd.off, nd, (M)c.y, (M)c.x, py, px, pv, pdv, pdu);
        s += (M)c.w[k] * pv;
        if (NEED_D) {
            dsdY += (M)c.dwdy[k] * pv - (M)c.w[k] * (M)nd.sy * pdv;
            dsdX += (M)c.dwdx[k] * pv - (M)c.w[k] * (M)nd.sx * pdu;
        }
    }
}

// CircularGaussianPSF profile (parametric_models.jl:79-115): f and (df/dy, df/dx, df/dflux).
template <typename M, bool NEED_D>
__device__ __forceinline__ M gauss_eval(M fwhm, const StarCoef& c, M py, M px, M& gy, M& gx, M& gf) {
    const M gp = (M)(-2.772588722239781);  // -4 log(2)
    const M dx = px - (M)c.x, dy = py - (M)c.y;
    const M f2 = fwhm * fwhm;
    const M sq = (dx * dx + dy * dy) / f2;
    const M norm = -((M)3.141592653589793 * f2 / gp);
    const M amp = (M)c.flux / norm;
    const M g = exp(gp * sq);
    if (NEED_D) {
        const M Ag = amp * g;
        const M gf2 = gp / f2;
        gy = -2 * Ag * gf2 * dy;
        gx = -2 * Ag * gf2 * dx;
        gf = g / norm;
    }
    return amp * g + (M)c.bkg;
}

// Model value flux*s + bkg at one pixel for either PSF family.
template <typename D, typename M>
__device__ __forceinline__ M model_value(const DevPsf& P, const D* __restrict__ base, const StarCoef& c, M py, M px) {
    if (P.kind == CPB_PSF_CIRCULAR_GAUSSIAN) {
        M a, b, e;
        return gauss_eval<M, false>((M)P.fwhm, c, py, px, a, b, e);
    }
    M s, dY, dX;
    grid_profile<D, M, false>(P, base, c, py, px, s, dY, dX);
    return (M)c.flux * s + (M)c.bkg;
}

// Gradient (df/dy, df/dx, df/dflux) at one pixel.
template <typename D, typename M>
__device__ __forceinline__ void model_grad(const DevPsf& P, const D* __restrict__ base, const StarCoef& c, M py, M px,
                                           M g[3]) {
    if (P.kind == CPB_PSF_CIRCULAR_GAUSSIAN) {
        gauss_eval<M, true>((M)P.fwhm, c, py, px, g[0], g[1], g[2]);
        return;
    }
    M s, dY, dX;
    grid_profile<D, M, true>(P, base, c, py, px, s, dY, dX);
    g[0] = (M)c.flux * dY;
    g[1] = (M)c.flux * dX;
    g[2] = s;
}

// ---------------------------------------------------------------------------
// warp helpers
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// max that propagates NaN like Julia's max (fmax would drop it).
__device__ __forceinline__ double nan_max(double a, double b) { return (a != a || b != b) ? (a + b) : fmax(a, b); }
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nan_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// fit_all_stars (cpb_multipass.cu): per-star parameter rows.
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

// One dependency-driven fit_all_stars pass (k_mp_dag, cpb_lm.cu).
struct DagArgs {
    int npos, pass, ny, box_max;
    MPConst M;
    MPFree F;
    const int32_t* idx;         // position -> star
    const int4* box;            // per position: y1, x1, rows, columns
    const double* pin;          // per position: parameters at the pass start
    const int32_t* succ_start;  // per position (npos + 1): stars that wait for it
    const int32_t* succ_list;
    int32_t* indeg;             // per position: unfinished stars it waits for
    int32_t* plevel;            // per position: longest chain of stars before it (0 at the start)
    int32_t* queue;             // npos ready positions, -1 = not yet
    int32_t* counters;          // head, tail, error, deepest level
    double* resid;
    const void* iv;             // image inv_var (nullable), eltype of the image
    double *cpix, *civ;         // per team: box_max doubles each
    double *prm, *err;
    uint8_t *conv, *valid;
    double* chisq;
    int32_t* niter;
    int* n_failed;
    double* psub;               // per position: the subtracted model
    uint8_t* flag;              // per position: 2 fitted, 1 add-back undone, 0 none
    long long spin_limit;       // polls of the ready queue before a team gives up
    double* snap;               // last pass: residual box after the subtraction (nullable)
    const int64_t* snap_off;    // per position
};

// The spread_model reference disk on the device.  The band-limited disk is a
// sum of six separable Gaussian-mixture components, K = sum_c alpha_c I_c I_c',
// with I_c zero beyond |m| = L_c (the reference's overflow cutoff), so the
// zero-border correlation (correlate!(g, ms, K, :zero), correlation.jl:122-141)
// is run as one x pass and one y pass per component -- sum_c 2 (2 L_c + 1)
// multiply-adds a pixel instead of (2 kh + 1)^2.
struct SpreadDev {
    const double* I;  // 6 x (2 kh + 1), I_c(m) at c * (2 kh + 1) + m + kh
    double alpha[6];  // a_c / (sum of the unnormalised kernel)
    int L[6];         // support half-width of I_c (<= kh)
    int kh;
};

// G = K correlated with the bh x bw column-major stamp M (zero border), by the
// whole block (every thread calls it); T and G are block scratch of bh * bw
// doubles each.  Ends with a barrier: G is complete on return.
__device__ __forceinline__ void spread_stamp_block(const SpreadDev& D, const double* M, double* T, double* G, int bh,
                                                   int bw) {
    const int nb = bh * bw, n = 2 * D.kh + 1;
    for (int e = threadIdx.x; e < nb; e += blockDim.x) G[e] = 0.0;
    for (int c = 0; c < 6; ++c) {
        const int L = D.L[c];
        const double* I = D.I + c * n + D.kh;
        __syncthreads();
        for (int e = threadIdx.x; e < nb; e += blockDim.x) {  // x pass
            const int r = e % bh, col = e / bh;
            const int q0 = max(-L, -col), q1 = min(L, bw - 1 - col);
            double t = 0.0;
            for (int q = q0; q <= q1; ++q) t += I[q] * M[r + (col + q) * bh];
            T[e] = t;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < nb; e += blockDim.x) {  // y pass
            const int r = e % bh, col = e / bh;
            const int p0 = max(-L, -r), p1 = min(L, bh - 1 - r);
            double t = 0.0;
            for (int p = p0; p <= p1; ++p) t += I[p] * T[r + p + col * bh];
            G[e] += D.alpha[c] * t;
        }
    }
    __syncthreads();
}

// Block-wide sums of K values in a fixed order (warp sums, then the warps in
// index order); results valid in thread 0.  sh: K * (blockDim.x / 32) doubles.
template <int K>
__device__ __forceinline__ void block_sum_n(double (&v)[K], double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) sh[wid * K + k] = v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double t = 0.0;
            for (int w2 = 0; w2 < nw; ++w2) t += sh[w2 * K + k];
            v[k] = t;
        }
    }
}

// The x pass of all six components at once (each stamp value is loaded once
// for every component whose support reaches it): T[c * ld + e] = sum_q
// I_c(q) M[r, col + q] over the in-box columns, e = r + col * bh.  Is: the six
// profiles in shared memory, 6 x (2 kh + 1).  The y pass and the weighting are
// spread_ypass at each pixel.  Pixels t0, t0 + ts, ... (the block by default,
// a warp with t0 = lane, ts = 32).  No barrier inside.
__device__ __forceinline__ void spread_xpass_all(const SpreadDev& D, const double* Is, const double* M, double* T,
                                                 int ld, int bh, int bw, int t0 = -1, int ts = 0) {
    if (t0 < 0) {
        t0 = threadIdx.x;
        ts = blockDim.x;
    }
    const int n = 2 * D.kh + 1, nb = bh * bw;
    int Lmax = 0;
#pragma unroll
    for (int c = 0; c < 6; ++c) Lmax = max(Lmax, D.L[c]);
    for (int e = t0; e < nb; e += ts) {
        const int r = e % bh, col = e / bh;
        const int q0 = max(-Lmax, -col), q1 = min(Lmax, bw - 1 - col);
        double t[6] = {0, 0, 0, 0, 0, 0};
        for (int q = q0; q <= q1; ++q) {
            const double m = M[r + (col + q) * bh];
            const int aq = q < 0 ? -q : q;
#pragma unroll
            for (int c = 0; c < 6; ++c)
                if (aq <= D.L[c]) t[c] += Is[c * n + D.kh + q] * m;
        }
#pragma unroll
        for (int c = 0; c < 6; ++c) T[c * ld + e] = t[c];
    }
}

// The disk-correlated stamp value at pixel e = r + col * bh from the x-pass
// planes T (component c at T + c * ld): sum_c alpha_c sum_p I_c(p) T_c[r + p, col].
__device__ __forceinline__ double spread_ypass(const SpreadDev& D, const double* Is, const double* T, int ld, int bh,
                                               int e) {
    const int n = 2 * D.kh + 1, r = e % bh;
    double g = 0.0;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        const int L = D.L[c];
        const int p0 = max(-L, -r), p1 = min(L, bh - 1 - r);
        const double* I = Is + c * n + D.kh;
        const double* Tc = T + c * ld + e;
        double t = 0.0;
        for (int p = p0; p <= p1; ++p) t += I[p] * Tc[p];
        g += D.alpha[c] * t;
    }
    return g;
}

// Threads of a diagnostics block (one block a star) and its shared memory when
// spread_model is on.  Mode 1 (the usual): the model stamp, six x-pass planes
// and the profiles, (7 boxmax + 6 (2 kh + 1)) doubles; mode 2 (large boxes):
// the model stamp, one x-pass plane and the correlated stamp, one component at
// a time, 3 boxmax doubles.  Boxes beyond both within 200 KB (fit_rad above
// ~45 px) leave spread_model NaN (mode 0).
constexpr int kDiagThreads = 256;
inline size_t spread_smem_bytes(int mode, int boxmax, int kh) {
    return mode == 1 ? ((size_t)7 * boxmax + 6 * (2 * (size_t)kh + 1)) * sizeof(double)
                     : (mode == 2 ? (size_t)3 * boxmax * sizeof(double) : 0);
}
inline int spread_mode(int boxmax, int kh) {
    if (spread_smem_bytes(1, boxmax, kh) <= 200 * 1024) return 1;
    if (spread_smem_bytes(2, boxmax, kh) <= 200 * 1024) return 2;
    return 0;
}

// A spread_model disk built on the device, for fits whose disk width depends on
// a fitted position (the simultaneous fit sizes it from the first catalogue
// star's final parameters, psf_photometry_simultaneous.jl:1363-1365).  Table of
// spread_tab_len(kh) doubles: [0] the disk FWHM (spread_model is off unless it
// is finite and positive), [1..6] alpha_c, [7..12] L_c, then the six profiles
// I_c(m), m = -kh..kh, as in SpreadDev.  The quadrature rule (spread_rule in
// cpb_spread.cu, kSpreadRuleLen doubles): the 32 Gauss-Legendre nodes on
// [-1, 1], their weights, the six mixture amplitudes and the six variances.
constexpr int kSpreadHdr = 13;
constexpr int kSpreadGL = 32;
constexpr int kSpreadRuleLen = 2 * kSpreadGL + 12;
__host__ __device__ inline int spread_tab_len(int kh) { return kSpreadHdr + 6 * (2 * kh + 1); }
void spread_rule(double* out);  // host: fills kSpreadRuleLen doubles

__device__ inline bool spread_tab_on(const double* tab) { return isfinite(tab[0]) && tab[0] > 0; }

__device__ inline SpreadDev spread_dev(const double* tab, int kh) {
    SpreadDev D;
    D.I = tab + kSpreadHdr;
    D.kh = kh;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        D.alpha[c] = tab[1 + c];
        D.L[c] = (int)tab[7 + c];
    }
    return D;
}

// _spread_fwhm (psf_photometry_diagnostics.jl:113-125) by the whole block: the
// unit render centred at (Y, X) over PSF.extent(Int, m), sqrt(ea 2 ln2 / pi)
// with ea = (sum g)^2 / sum g^2.  P.fwhm is the PSF's own FWHM (Gaussian).
// red: 2 (blockDim.x / 32) + 1 doubles of shared memory.  Every thread gets
// the value; a non-finite position gives NaN.
__device__ inline double spread_fwhm_block(const DevPsf& P, double Y, double X, double* red) {
    if (!(isfinite(Y) && isfinite(X))) return __longlong_as_double(0x7ff8000000000000LL);
    StarCoef c;
    c.y = Y;
    c.x = X;
    c.flux = 1.0;
    c.bkg = 0.0;
    grid_corners_dw(P, Y, X, c);
    double e0 = 0, e1 = 0, e2 = 0, e3 = 0;
    if (P.kind == CPB_PSF_CIRCULAR_GAUSSIAN) {
        const double a = 5.0 * P.fwhm / 2;  // fwhm_factor 5, no rotation
        e0 = Y - a;
        e1 = Y + a;
        e2 = X - a;
        e3 = X + a;
    } else {
        bool first = true;
        for (int k = 0; k < 4; ++k) {
            if (c.idx[k] < 0 || c.w[k] == 0.0) continue;
            const DevNode nd = P.nodes[c.idx[k]];
            const double lo_y = Y - (nd.oy - 1.0) / nd.sy, hi_y = Y + ((double)nd.ny - nd.oy) / nd.sy;
            const double lo_x = X - (nd.ox - 1.0) / nd.sx, hi_x = X + ((double)nd.nx - nd.ox) / nd.sx;
            e0 = first ? lo_y : fmin(e0, lo_y);
            e1 = first ? hi_y : fmax(e1, hi_y);
            e2 = first ? lo_x : fmin(e2, lo_x);
            e3 = first ? hi_x : fmax(e3, hi_x);
            first = false;
        }
    }
    const int ylo = (int)floor(e0), yhi = (int)ceil(e1), xlo = (int)floor(e2), xhi = (int)ceil(e3);
    const int h = max(yhi - ylo + 1, 0), w = max(xhi - xlo + 1, 0);
    double v[2] = {0.0, 0.0};
    for (int e = threadIdx.x; e < h * w; e += blockDim.x) {
        const double g = model_value<double, double>(P, P.data64, c, (double)(ylo + e % h), (double)(xlo + e / h));
        v[0] += g;
        v[1] += g * g;
    }
    block_sum_n<2>(v, red);
    const int slot = 2 * (blockDim.x >> 5);
    if (threadIdx.x == 0) red[slot] = sqrt(v[0] * v[0] / v[1] * 2 * 0.6931471805599453 / 3.141592653589793);
    __syncthreads();
    const double f = red[slot];
    __syncthreads();
    return f;
}

// The disk table of one fit (layout above), by the whole block:
// _exp_disk_kernel_bandlimited(f; half = kh) (psf_photometry_diagnostics.jl:82-100)
// as six separable profiles I_c(m) = int_{-1/2}^{1/2} exp(-a_c k^2) cos(2 pi k m) dk,
// a_c = 2 pi^2 re^2 v_c, re = f / 16 * 1.67834699, zero where pi^2 m^2 / a_c > 690.
// The integral is composite 32-point Gauss-Legendre on max(4, 2 kh) equal panels
// of [-1/2, 1/2] (the host rule of cpb_exp_disk_kernel); the integrand is even,
// so the right half's panels are summed and doubled.  One panel at a time, the
// block tabulates the weighted exp(-a_c k^2) of the six components and
// cos(2 pi k m) of the kh + 1 orders at the panel's 32 nodes in `pan`
// ((7 + kh) * 32 doubles of shared memory), then one thread per (c, m) adds
// the panel's 32 products -- 7 + kh transcendentals a node instead of
// 12 (kh + 1).  f = param unless param is NaN (then _spread_fwhm at (Y, X));
// spread_tab_on(tab) tells whether spread_model is on.  Ends with a barrier.
__device__ inline void spread_disk_block(const DevPsf& P, double param, int kh, double Y, double X,
                                         const double* __restrict__ rule, double* tab, double* red, double* pan) {
    const double f = isnan(param) ? spread_fwhm_block(P, Y, X, red) : param;
    if (threadIdx.x == 0) tab[0] = f;
    if (!(isfinite(f) && f > 0)) {
        __syncthreads();
        return;
    }
    const double pi = 3.141592653589793;
    const int n = 2 * kh + 1, np = 6 * (kh + 1), rows = 7 + kh;
    const double re = f / 16 * 1.67834699;
    const int panels = max(4, 2 * kh);
    const double hw = 0.5 / panels;
    const double* gx = rule;
    const double* gw = rule + kSpreadGL;
    const double* amp = rule + 2 * kSpreadGL;
    const double* var = amp + 6;
    double* I0 = tab + kSpreadHdr;  // I_c(m) for m >= 0 accumulates at I0[c * n + kh + m]
    for (int t = threadIdx.x; t < np; t += blockDim.x) I0[(t / (kh + 1)) * n + kh + t % (kh + 1)] = 0.0;
    for (int pnl = panels / 2; pnl < panels; ++pnl) {
        const double mid = -0.5 + (2 * pnl + 1) * hw;
        __syncthreads();  // the previous panel's table is no longer read
        for (int t = threadIdx.x; t < rows * kSpreadGL; t += blockDim.x) {
            const int q = t % kSpreadGL, row = t / kSpreadGL;
            const double k = mid + hw * gx[q];
            pan[t] = row < 6 ? hw * gw[q] * exp(-(2 * pi * pi * re * re * var[row]) * k * k)
                             : cospi(2 * k * (double)(row - 6));
        }
        __syncthreads();
        for (int t = threadIdx.x; t < np; t += blockDim.x) {
            const int cc = t / (kh + 1), m = t % (kh + 1);
            const double a = 2 * pi * pi * re * re * var[cc];
            if (pi * pi * (double)m * m / a > 690) continue;
            const double* E = pan + cc * kSpreadGL;
            const double* Cm = pan + (6 + m) * kSpreadGL;
            double sp = 0.0;
#pragma unroll 8
            for (int q = 0; q < kSpreadGL; ++q) sp += E[q] * Cm[q];
            I0[cc * n + kh + m] += sp;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < np; t += blockDim.x) {
        const int cc = t / (kh + 1), m = t % (kh + 1);
        const double I = 2 * I0[cc * n + kh + m];
        I0[cc * n + kh + m] = I;
        I0[cc * n + kh - m] = I;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const double* Iv = I0 + threadIdx.x * n + kh;
        int L = 0;
        for (int m = kh; m > 0; --m)
            if (Iv[m] != 0.0) {
                L = m;
                break;
            }
        tab[7 + threadIdx.x] = (double)L;
    }
    if (threadIdx.x == 0) {
        double total = 0.0;
        for (int c = 0; c < 6; ++c) {
            double s = 0.0;
            for (int m = 0; m < n; ++m) s += I0[c * n + m];
            total += amp[c] * s * s;
        }
        for (int c = 0; c < 6; ++c) tab[1 + c] = amp[c] / total;
    }
    __syncthreads();
}

}  // namespace cpb

// ---------------------------------------------------------------------------
// host-side handles
// ---------------------------------------------------------------------------
struct cpb_psf {
    cpb::DevPsf dev;
    double* d_data64 = nullptr;
    float* d_data32 = nullptr;
    double* d_pp64 = nullptr;
    float* d_pp32 = nullptr;
    double* d_lpp64 = nullptr;
    cpb::DevNode* d_nodes = nullptr;
    double* d_ygrid = nullptr;
    double* d_xgrid = nullptr;
    int32_t* d_index_grid = nullptr;
    std::vector<cpb::DevNode> h_nodes;
    int64_t smem_bytes64 = 0;  // padded bytes of all nodes in FP64
    int64_t smem_bytes32 = 0;
    // host copies for the host-side curve of growth (model_rad = :auto)
    std::vector<double> h_data64;
    std::vector<double> h_ygrid, h_xgrid;
    std::vector<int32_t> h_index_grid;
    // unit-PSF annular surface brightness per (R_cap, fwhm), computed once
    std::mutex cog_mu;
    std::map<std::pair<int, double>, std::vector<double>> cog_sb;
};

struct cpb_ctx {
    int device = 0;
    int n_sm = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    std::string err;
    struct Buf {
        void* p = nullptr;
        size_t bytes = 0;
    };
    std::map<std::string, Buf> bufs;  // grow-only scratch, reused across calls (stream-ordered allocations)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t grow_ev = nullptr;    // orders the copy stream around a scratch buffer's reallocation
    // second stream for uploads that overlap kernels, with its hand-off events
    cudaStream_t copy_stream = nullptr;
    static constexpr int kCopyEvents = 16;
    cudaEvent_t copy_ev[kCopyEvents] = {};
    void* pinned = nullptr;  // small pinned staging for scalar readbacks
    // kernel instrumentation: launch counter (always on) and, when profiling is
    // enabled, CUDA-event timing of every launch on this context's stream
    int64_t launches = 0;
    bool profile = false;
    // bounded device waits: polls before a persistent kernel gives up (<= 0: default)
    int64_t wait_limit = 0;
    // one-shot host-side fault injection for tests (CPB_FAULT_*)
    int32_t fault = CPB_FAULT_NONE;
    struct KStat {
        int64_t launches = 0;
        double seconds = 0, bytes = 0;
    };
    std::map<std::string, KStat> kstats;
    struct Pending {
        std::string name;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    // When set (only inside cpb_fit_simultaneous_device_noalloc), scratch()
    // carves buffers from this caller-independent static region instead of
    // allocating; see cpb_noalloc.cu.
    struct Arena {
        char* base = nullptr;
        size_t cap = 0, used = 0;
        std::map<std::string, std::pair<size_t, size_t>> slots;  // name -> (offset, bytes)
    };
    Arena* arena = nullptr;
};

namespace cpb {

// Scratch arena: returns a device buffer of at least `bytes` under `name`.
void* scratch(cpb_ctx* ctx, const char* name, size_t bytes);
// Carves `bytes` for `name` from a fixed region (no allocation); throws when it is full.
void* arena_carve(cpb_ctx::Arena* a, const char* name, size_t bytes);

// Brackets one kernel launch: counts it and, when profiling, records CUDA
// events on the context stream with the launch's algorithmic bytes.
struct KernelScope {
    cpb_ctx* ctx;
    const char* name;
    double bytes;
    cudaEvent_t a = nullptr, b = nullptr;
    KernelScope(cpb_ctx* c, const char* n, double by);
    ~KernelScope();
};
// Resolves pending event pairs into ctx->kstats (after a stream sync).
void resolve_kernel_events(cpb_ctx* ctx);

// A named NVTX range over a host-side phase (set-up, fill, render, LSQR, trial,
// freeze, final pass, ...), visible in Nsight timelines; free when no tool is attached.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

struct CudaError {
    cudaError_t e;
    const char* what;
};

inline void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError{e, what};
}

struct ArgError {
    std::string msg;
};
struct OomError {
    std::string msg;
};
// A bounded device-side wait gave up (CPB_ERR_TIMEOUT).
struct WaitTimeout {
    std::string msg;
};

// Runs one C-ABI entry point's body under the context's lock, translating
// exceptions into CPB_* status codes and cpb_last_error() text.
template <typename F>
int guarded(cpb_ctx* ctx, F&& f) {
    if (!ctx) return CPB_ERR_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->err.clear();
    try {
        check(cudaSetDevice(ctx->device), "cudaSetDevice");
        return f();
    } catch (const ArgError& e) {
        ctx->err = e.msg;
        return CPB_ERR_ARGUMENT;
    } catch (const OomError& e) {
        ctx->err = e.msg;
        return CPB_ERR_OOM;
    } catch (const WaitTimeout& e) {
        ctx->err = e.msg;
        return CPB_ERR_TIMEOUT;
    } catch (const CudaError& e) {
        ctx->err = std::string(e.what) + ": " + cudaGetErrorString(e.e);
        return CPB_ERR_CUDA;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return CPB_ERR_INTERNAL;
    }
}


// Simultaneous fit driver (cpb_sim.cu).  Inputs are device pointers.
int fit_simultaneous_dev(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* P, const void* d_image,
                         int32_t eltype, int64_t ny, int64_t nx, const void* d_inv_var, const void* d_background,
                         int64_t n, const double* d_y0, const double* d_x0, const double* d_flux0,
                         cpb_sim_result* out);

// Upper bound of the scratch bytes one simultaneous fit carves from a fixed
// region (cpb_sim.cu), every catalogue star counted as active; with
// model_rad = :auto the model stamps are counted at the fit box and checked
// again inside the fit once the radii are known.
size_t sim_scratch_bound(const cpb_sim_params* P, int64_t ny, int64_t nx, int64_t n, bool dbg_pixels);

// model_rad = :auto (psf_photometry_simultaneous.jl:192-243), host side
// (cpb_radii.cu): per-star model radii from the unit PSF's curve of growth and
// the background noise of the weight sample.
void model_radii_auto(const cpb_psf* psf, double fwhm, double nsigma, int R_fit, int R_cap,
                      std::vector<double>& w_sample, const std::vector<double>& flux, std::vector<int32_t>& out);

// spread_model reference disk (cpb_spread.cu): the separable components of
// the band-limited exponential disk with support half = ceil(fit_rad); false
// when spread_model is off.
struct SpreadHost {
    int kh = 0;
    std::vector<double> I;  // 6 x (2 kh + 1)
    double alpha[6] = {0, 0, 0, 0, 0, 0};
    int L[6] = {0, 0, 0, 0, 0, 0};
};
bool spread_kernel(const cpb_psf* psf, double psf_fwhm, double param, double y1, double x1, double fit_rad,
                   SpreadHost& out);

// Batched simultaneous fits of small groups (cpb_groups.cu).  Device inputs and
// outputs; the h_*_opt arrays (nullable) are host copies of the group metadata.
int fit_groups_dev(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* P, int64_t G, const int64_t* d_off,
                   const int32_t* d_ny, const int32_t* d_nx, const void* d_pix, int32_t eltype, const void* d_iv,
                   const void* d_bkg, const int64_t* d_soff, const double* d_y0, const double* d_x0,
                   const double* d_f0, int64_t total_pixels, cpb_group_result* out, const int64_t* h_off_opt,
                   const int32_t* h_ny_opt, const int32_t* h_nx_opt, const int64_t* h_soff_opt);

// Bound batches over fixed device buffers (cpb_lm.cu, cpb_groups.cu): one
// launch each, no host synchronisation and no allocation, so that a CUDA graph
// can capture them; the *_signature strings key the launch-shape tuner.
struct LMBatch;
LMBatch* lm_batch_create(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* P, int64_t n_cut,
                         const int64_t* d_off, const int32_t* d_ny, const int32_t* d_nx, const int32_t* d_y1,
                         const int32_t* d_x1, const void* d_pix, int32_t eltype, const void* d_iv,
                         const double* d_init, int64_t total_pixels, const cpb_lm_result* out);
void lm_batch_enqueue(cpb_ctx* ctx, LMBatch* b, cudaStream_t st, int blocks_per_sm, int smem_node);
bool lm_batch_smem_possible(const LMBatch* b);
int64_t lm_batch_size(const LMBatch* b);
std::string lm_batch_signature(const LMBatch* b);
void lm_batch_destroy(LMBatch* b);

struct GroupBatch;
GroupBatch* group_batch_create(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* P, int64_t G,
                               const int64_t* d_off, const int32_t* d_ny, const int32_t* d_nx, const void* d_pix,
                               int32_t eltype, const void* d_iv, const void* d_bkg, const int64_t* d_soff,
                               const double* d_y0, const double* d_x0, const double* d_f0, int64_t total_pixels,
                               const cpb_group_result* out);
// Groups are launched in buckets of similar star count (one launch each).
int group_batch_buckets(const GroupBatch* b);
void group_batch_enqueue(cpb_ctx* ctx, GroupBatch* b, cudaStream_t st, int bucket, int threads);
void group_batch_set_threads(GroupBatch* b, int bucket, int threads);
int group_batch_threads(const GroupBatch* b, int bucket);
int group_batch_occupancy(GroupBatch* b, int bucket, int threads);
int64_t group_batch_size(const GroupBatch* b);
std::string group_batch_signature(const GroupBatch* b, int bucket);
void group_batch_destroy(GroupBatch* b);

// fit_all_stars (cpb_multipass.cu): device image / weights, host catalogue and outputs.
int fit_all_stars_dev(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* P, double fit_rad, int n_passes,
                      double spread_model_fwhm, const void* d_img, int32_t eltype, int64_t ny, int64_t nx,
                      const void* d_iv, int64_t n, const double* init, cpb_multipass_result* out);

// Batched LM driver (cpb_lm.cu).  Host inputs.
int fit_lm_batch(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* P, int64_t n_cutouts,
                 const int64_t* offsets, const int32_t* ny, const int32_t* nx, const int32_t* y_origin,
                 const int32_t* x_origin, const void* pixels, int32_t eltype, const void* inv_var,
                 const double* init, cpb_lm_result* out);
// fit_all_stars pass as one dependency-driven launch (cpb_lm.cu): whether the
// PSF / keywords allow it (single-node image PSFs and the Gaussian, no IRLS),
// the number of 128-thread teams the launch runs (its per-team scratch), and
// the launch itself (iv_eltype: element type of the image and inv_var).
bool mp_dag_supported(const cpb_psf* psf, const cpb_lm_params* P);
int mp_dag_teams(cpb_ctx* ctx);
void mp_dag_launch(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* P, int32_t iv_eltype, const DagArgs& A);

// The fit_star launch of fit_lm_batch_device on the context's stream, with no
// event, synchronisation or host read-back (callers chain further kernels).
// team_warps: warps a cutout (0: chosen by the batch size; 1 or 4);
// zeroed_queue (nullable): a work-queue counter already at zero.
void lm_enqueue_device(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* P, int64_t n_cut, const int64_t* d_off,
                       const int32_t* d_ny, const int32_t* d_nx, const int32_t* d_y1, const int32_t* d_x1,
                       const void* d_pix, int32_t eltype, const void* d_iv, const double* d_init, int64_t total_pixels,
                       const cpb_lm_result* out, int team_warps = 0,
                       unsigned long long* zeroed_queue = nullptr);
int fit_lm_batch_device(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* P, int64_t n_cut,
                        const int64_t* d_off, const int32_t* d_ny, const int32_t* d_nx, const int32_t* d_y1,
                        const int32_t* d_x1, const void* d_pix, int32_t eltype, const void* d_iv,
                        const double* d_init, int64_t total_pixels, cpb_lm_result* out);

}  // namespace cpb
