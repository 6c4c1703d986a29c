// cpb_sim.cu -- B200 simultaneous damped Gauss-Newton / LSQR PSF fit.
//
// Device restatement of CrowdPhot.fit_all_stars_simultaneous
// (src/photometry/psf_photometry_simultaneous.jl:953-1431).  Layout in HBM:
//   * per-pixel vectors (data, data_work, w, sqrt(w), union mask, residual,
//     LSQR u) are column-major npix arrays, as in the reference;
//   * stamp derivatives V are star-major: star j owns a contiguous block of
//     VS >= p*S2 values in the reference's (k fastest, then stamp pixel m)
//     order (StampDerivatives.values, :19-43), padded to 128 bytes;
//   * stamp pixel indices are not stored: they follow from the integer anchor
//     and the fit-box offset (the reference's `pixels` matrix is rebuilt only
//     for the bit-exact debug export);
//   * per-tile star lists (32 x 8 pixel tiles, stars in Morton order) turn the
//     reference's scatter-adds (apply_J!, _render_model!) into deterministic
//     pixel gathers with no atomics.
// Control flow per outer iteration follows :1186-1284; the LSQR inner solve
// runs entirely on the device with its stopping tests evaluated in-kernel.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>

#include "cpb_internal.cuh"
#include "cpb_linalg.cuh"
#include "cpb_reduce.cuh"

namespace cpb {
namespace {

constexpr int TY = 32;   // region rows (y, contiguous in memory)
constexpr int SW = 8;    // columns of one warp's strip
constexpr int NT = 128;  // threads of the region kernels (4 warps)
constexpr int TX = SW * (NT / 32);  // region columns
constexpr double kEps64 = 2.220446049250313e-16;

enum RenderMode { MODE_CUR = 0, MODE_CAND = 1, MODE_FREEZE = 2, MODE_FINAL = 3 };

// Device-resident scalars of one fit.
struct Scalars {
    double cost;       // current residual cost (over U)
    double cost_cand;  // candidate cost
    double gnorm;      // global gradient cosine
    double beta1;      // ||mrhs||
    // LSQR state (Krylov.jl lsqr recurrences)
    double alpha, beta, inv_alpha, inv_beta;
    double Anorm2, dNorm2, xNorm, xNorm2, c2, s2, z, xENorm2, res2, rhobar, phibar, ArNorm0;
    double err_vec[5];
    double wnorm2;
    double lambda, atol, btol;
    int iter, itmax, stopped, status;
    int n_new_frozen;
};

// ---------------------------------------------------------------------------
// setup kernels
// ---------------------------------------------------------------------------
template <typename TI>
__global__ void k_prepare(const TI* __restrict__ img, const TI* __restrict__ iv, const TI* __restrict__ bkg,
                          int64_t npix, double* data, double* data_work, double* w, double* sw,
                          unsigned* nonfinite) {
    int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= npix) return;
    double d = (double)img[q] - (bkg ? (double)bkg[q] : 0.0);
    double wv = 1.0;
    if (iv) {
        double v = (double)iv[q];
        wv = (isfinite(v) && v > 0) ? v : 0.0;
    }
    if (!isfinite(d)) {
        if (!iv) atomicAdd(nonfinite, 1u);
        d = 0.0;
        wv = 0.0;
    }
    data[q] = d;
    data_work[q] = d;
    w[q] = wv;
    sw[q] = sqrt(wv);
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

// _build_stamps! per catalogue star (:262-295): anchors (round half to even),
// usable-pixel test, active flag and Morton key (:163-174).
__global__ void k_anchor(int64_t n, const double* y0, const double* x0, const double* f0, int R, int ny, int nx,
                         const double* __restrict__ w, int32_t* ay, int32_t* ax, uint8_t* ok, uint64_t* key,
                         unsigned* neg) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool fin = isfinite(y0[i]) && isfinite(x0[i]);
    const int a_y = fin ? (int)__double2ll_rn(y0[i]) : 0;
    const int a_x = fin ? (int)__double2ll_rn(x0[i]) : 0;
    bool any = false;
    if (fin) {
        for (int dx = -R; dx <= R && !any; ++dx) {
            int gx = a_x + dx;
            if (gx < 1 || gx > nx) continue;
            for (int dy = -R; dy <= R; ++dy) {
                int gy = a_y + dy;
                if (gy < 1 || gy > ny) continue;
                if (w[(gy - 1) + (int64_t)(gx - 1) * ny] > 0) {
                    any = true;
                    break;
                }
            }
        }
    }
    const bool good = any && fin && isfinite(f0[i]);
    ay[i] = a_y;
    ax[i] = a_x;
    ok[i] = good;
    if (good && (a_y < 0 || a_x < 0)) atomicAdd(neg, 1u);
    key[i] = spread_bits((uint64_t)(uint32_t)a_y) | (spread_bits((uint64_t)(uint32_t)a_x) << 1);
}

__global__ void k_gather_active(int64_t n_act, const int32_t* act, const int32_t* ay_c, const int32_t* ax_c,
                                const double* y0, const double* x0, const double* f0, int p, int3 gc,
                                int32_t* ay, int32_t* ax, double* theta) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n_act) return;
    int i = act[j];
    ay[j] = ay_c[i];
    ax[j] = ax_c[i];
    int g[3] = {gc.x, gc.y, gc.z};
    for (int k = 0; k < p; ++k) theta[j * p + k] = g[k] == 1 ? y0[i] : (g[k] == 2 ? x0[i] : f0[i]);
}

// Union of usable stamp pixels (_touched_pixels, :329-335) and, on request,
// the reference's `pixels` matrix (1-based, 0 = unusable).
__global__ void k_union(int64_t n_act, const int32_t* ay, const int32_t* ax, int R, int ny, int nx,
                        const double* __restrict__ w, uint8_t* umask, int32_t* dbg_pixels) {
    int64_t j = blockIdx.x;
    const int S = 2 * R + 1, S2 = S * S;
    for (int m = threadIdx.x; m < S2; m += blockDim.x) {
        int gy = ay[j] + (m % S) - R, gx = ax[j] + (m / S) - R;
        int32_t fi = 0;
        if (gy >= 1 && gy <= ny && gx >= 1 && gx <= nx) {
            int64_t q = (gy - 1) + (int64_t)(gx - 1) * ny;
            if (w[q] > 0) {
                umask[q] = 1;
                fi = (int32_t)(q + 1);
            }
        }
        if (dbg_pixels) dbg_pixels[m + (int64_t)S2 * j] = fi;
    }
}

__global__ void k_count_u8(const uint8_t* m, int64_t n, unsigned long long* cnt) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    unsigned c = (i < n && m[i]) ? 1u : 0u;
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt, (unsigned long long)c);
}

// ---- per-tile star lists -------------------------------------------------
__device__ __forceinline__ bool star_tiles(int ay, int ax, int Rj, int ny, int nx, int& ty0, int& ty1, int& tx0,
                                           int& tx1) {
    int ylo = max(ay - Rj, 1), yhi = min(ay + Rj, ny), xlo = max(ax - Rj, 1), xhi = min(ax + Rj, nx);
    if (ylo > yhi || xlo > xhi) return false;
    ty0 = (ylo - 1) / TY;
    ty1 = (yhi - 1) / TY;
    tx0 = (xlo - 1) / TX;
    tx1 = (xhi - 1) / TX;
    return true;
}

__global__ void k_tile_count(int64_t n_act, const int32_t* ay, const int32_t* ax, const int32_t* Rs, int Rconst,
                             int ny, int nx, int32_t* cnt) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n_act) return;
    int Rj = Rs ? Rs[j] : Rconst, a, b, c, d;
    cnt[j] = star_tiles(ay[j], ax[j], Rj, ny, nx, a, b, c, d) ? (b - a + 1) * (d - c + 1) : 0;
}

__global__ void k_tile_emit(int64_t n_act, const int32_t* ay, const int32_t* ax, const int32_t* Rs, int Rconst,
                            int ny, int nx, int nty, const int32_t* offs, uint32_t* keys, int32_t* vals) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n_act) return;
    int Rj = Rs ? Rs[j] : Rconst, ty0, ty1, tx0, tx1;
    if (!star_tiles(ay[j], ax[j], Rj, ny, nx, ty0, ty1, tx0, tx1)) return;
    int o = offs[j];
    for (int tx = tx0; tx <= tx1; ++tx)
        for (int ty = ty0; ty <= ty1; ++ty) {
            keys[o] = (uint32_t)(ty + tx * nty);
            vals[o] = (int32_t)j;
            ++o;
        }
}

__global__ void k_tile_bounds(int64_t npairs, const uint32_t* keys, int32_t* start, int32_t* end) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= npairs) return;
    uint32_t k = keys[i];
    if (i == 0 || keys[i - 1] != k) start[k] = (int32_t)i;
    if (i == npairs - 1 || keys[i + 1] != k) end[k] = (int32_t)(i + 1);
}

// Sort keys of the regions by work: the number of (region, star) pairs.
__global__ void k_tile_work(int64_t ntiles, const int32_t* start, const int32_t* end, uint32_t* key, int32_t* idx) {
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    key[t] = (uint32_t)(end[t] - start[t]);
    idx[t] = (int32_t)t;
}

__global__ void k_tile_pack(int64_t npairs, const int32_t* sorted_j, const int32_t* ay, const int32_t* ax,
                            const int32_t* Rs, int Rconst, int4* packed) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= npairs) return;
    const int j = sorted_j[i];
    packed[i] = make_int4(j, ay[j], ax[j], Rs ? Rs[j] : Rconst);  // .w: the star's box radius
}

// ---------------------------------------------------------------------------
// per-iteration kernels
// ---------------------------------------------------------------------------
struct FitConst {
    int p;
    int gc[3];     // grad_col of free param k (1 = dy, 2 = dx, 3 = dflux)
    int ky, kx;    // index of y / x in the free list, -1 if fixed
    double fixed_y, fixed_x, fixed_flux, fixed_bkg;
    int R, S, S2, VS;
    int q32, r32;  // 32 / S and 32 % S: advancing a stamp index by one warp
    int ny, nx;
    int nty, ntx;
};

// model_from_vector for star j: theta (+ delta when cand).
__global__ void k_coef(int64_t n_act, FitConst fc, DevPsf P, const double* theta, const double* delta,
                       StarCoef* coef) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n_act) return;
    StarCoef c;
    c.y = fc.fixed_y;
    c.x = fc.fixed_x;
    c.flux = fc.fixed_flux;
    c.bkg = fc.fixed_bkg;
    for (int k = 0; k < fc.p; ++k) {
        double v = theta[j * fc.p + k];
        if (delta) v = v + delta[j * fc.p + k];
        if (fc.gc[k] == 1) c.y = v;
        else if (fc.gc[k] == 2) c.x = v;
        else c.flux = v;
    }
    grid_corners_dw(P, c.y, c.x, c);
    coef[j] = c;
}

// ---- separable cubic-convolution tables --------------------------------
// The cubic convolution of empirical_models.jl:185-196 (Keys, a = -1/2) is
// linear in the four samples: p(t) = sum_c w_c(t) f_c, p'(t) = sum_c d_c(t) f_c.
// Tabulating these weights once per stamp row and column turns each pixel's
// bicubic value and both derivatives into 16 sample loads and 44 FMAs.
// T is the arithmetic / storage type of the stamps (double for the plain
// form, float for the mixed-precision form); positions and weights are
// always derived in double and rounded once.
__device__ __forceinline__ void keys_weights(double t, double w[4], double d[4]) {
    const double t2 = t * t, t3 = t2 * t;
    w[0] = -0.5 * t + t2 - 0.5 * t3;
    w[1] = 1.0 - 2.5 * t2 + 1.5 * t3;
    w[2] = 0.5 * t + 2.0 * t2 - 1.5 * t3;
    w[3] = -0.5 * t2 + 0.5 * t3;
    d[0] = -0.5 + 2.0 * t - 1.5 * t2;
    d[1] = -5.0 * t + 4.5 * t2;
    d[2] = 0.5 + 4.0 * t - 4.5 * t2;
    d[3] = -t + 1.5 * t2;
}

// One axis of one node at one stamp row or column: clamped sample offsets
// (times the axis stride), weights, derivative weights, and the in-bounds
// half of bicubic_interpolate's `_inbound` test.
template <typename T>
struct AxisTab {
    T w[4], d[4];
    int off[4];
    int inb;
    int pad;
};

// Offsets address the node's polyphase copy (DevNode): an axis with integer
// oversampling s maps the 0-based sample index i to (i % s) * phase_stride +
// (i / s) * elem_stride, so the row and column parts add to the element offset.
template <typename T>
__device__ __forceinline__ void axis_tab(double coord, int n, int s, int phase_stride, int elem_stride,
                                         AxisTab<T>& t) {
    const bool inb = isfinite(coord) && coord >= 1.0 && coord <= (double)n;
    const double c = inb ? coord : 1.0;
    const int l = clampi((int)floor(c), 1, n - 1);
    const double f = c - (double)l;
    const int i0 = clampi(l - 1, 1, n) - 1, i1 = l - 1, i2 = l, i3 = clampi(l + 2, 1, n) - 1;
    t.off[0] = (i0 % s) * phase_stride + (i0 / s) * elem_stride;
    t.off[1] = (i1 % s) * phase_stride + (i1 / s) * elem_stride;
    t.off[2] = (i2 % s) * phase_stride + (i2 / s) * elem_stride;
    t.off[3] = (i3 % s) * phase_stride + (i3 / s) * elem_stride;
    double w[4], d[4];
    keys_weights(f, w, d);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        t.w[k] = (T)w[k];
        t.d[k] = (T)d[k];
    }
    t.inb = inb;
}
template <typename T>
__device__ __forceinline__ void axis_tab_x(const DevNode& nd, double u, AxisTab<T>& t) {
    axis_tab(u, nd.nx, nd.isx, nd.isy * nd.PY * nd.PX, nd.PY, t);
}
template <typename T>
__device__ __forceinline__ void axis_tab_y(const DevNode& nd, double v, AxisTab<T>& t) {
    axis_tab(v, nd.ny, nd.isy, nd.PY * nd.PX, 1, t);
}

template <typename T>
__device__ __forceinline__ const T* pp_data(const DevPsf& P);
template <>
__device__ __forceinline__ const double* pp_data<double>(const DevPsf& P) { return P.pp64; }
template <>
__device__ __forceinline__ const float* pp_data<float>(const DevPsf& P) { return P.pp32; }

// Bicubic value (and d/dv, d/du when GRAD) of one node from its tables.
template <bool GRAD, typename T>
__device__ __forceinline__ void tab_bicubic(const T* __restrict__ base, const AxisTab<T>& tx, const AxisTab<T>& ty,
                                            T fill, T& pv, T& pdv, T& pdu) {
    if (!(tx.inb && ty.inb)) {
        pv = fill;
        pdv = 0;
        pdu = 0;
        return;
    }
    T rv[4], rd[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const T* row = base + ty.off[r];
        const T a = __ldg(row + tx.off[0]), b = __ldg(row + tx.off[1]), c = __ldg(row + tx.off[2]),
                e = __ldg(row + tx.off[3]);
        rv[r] = tx.w[0] * a + tx.w[1] * b + tx.w[2] * c + tx.w[3] * e;
        if (GRAD) rd[r] = tx.d[0] * a + tx.d[1] * b + tx.d[2] * c + tx.d[3] * e;
    }
    pv = ty.w[0] * rv[0] + ty.w[1] * rv[1] + ty.w[2] * rv[2] + ty.w[3] * rv[3];
    if (GRAD) {
        pdv = ty.d[0] * rv[0] + ty.d[1] * rv[1] + ty.d[2] * rv[2] + ty.d[3] * rv[3];
        pdu = ty.w[0] * rd[0] + ty.w[1] * rd[1] + ty.w[2] * rd[2] + ty.w[3] * rd[3];
    }
}

// Star-parallel stamp evaluation, one block per star of `list` (grid-stride);
// the general path (any number of ePSF nodes).
// GRAD (with gram == nullptr): _fill_stamps! (:342-399, :437-543) -- raw =
//   sqrt(w) * gradient over the fit box, colnorm = max(||raw||, eps),
//   V = raw * (1 / colnorm); masked and off-image entries are exactly 0.
// GRAD with gram: the unscaled p x p Gram block sum(raw raw') of the error
//   estimate (:1305-1318), nothing else written.
// M != nullptr: the model value flux * s + bkg of every box pixel (the
//   per-star term of _render_model!, :545-577 / :605-673), box half-width Rb.
// Sums of squares and Gram entries accumulate in double for either T.
template <int NTF, int MAXE, bool GRAD, typename T>
__global__ void __launch_bounds__(NTF) k_eval(const int32_t* __restrict__ list, int64_t nlist, FitConst fc, DevPsf P,
                                              const StarCoef* __restrict__ coef, const int32_t* __restrict__ ay,
                                              const int32_t* __restrict__ ax, const double* __restrict__ w,
                                              const double* __restrict__ sw, T* __restrict__ V,
                                              double* __restrict__ colnorm, double* __restrict__ gram,
                                              T* __restrict__ M, int Rmax, int MS, const int32_t* __restrict__ Rs,
                                              const int64_t* __restrict__ moff) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    AxisTab<T>* tabs = (AxisTab<T>*)smem_raw;  // [corner][axis][Sb]
    __shared__ double sh[32];
    __shared__ double cn_sh[6];
    __shared__ StarCoef c;
    const bool gauss = P.kind == CPB_PSF_CIRCULAR_GAUSSIAN;
    const int p = fc.p;
    const int g0 = fc.gc[0] - 1, g1 = fc.gc[1] - 1, g2 = fc.gc[2] - 1;
    const T* data = pp_data<T>(P);
    for (int64_t li = blockIdx.x; li < nlist; li += gridDim.x) {
        const int j = list ? list[li] : (int)li;
        if (threadIdx.x == 0) c = coef[j];
        __syncthreads();
        const int Rb = Rs ? Rs[j] : Rmax;  // this star's box radius (<= Rmax, which sized the tables)
        const int Sb = 2 * Rb + 1, S2b = Sb * Sb;
        const int a_y = ay[j], a_x = ax[j];
        if (!gauss) {
            for (int e = threadIdx.x; e < 8 * Sb; e += NTF) {
                const int k = e / (2 * Sb), rem = e % (2 * Sb), axis = rem / Sb, idx = rem % Sb;
                if (c.idx[k] < 0) continue;
                const DevNode nd = P.nodes[c.idx[k]];
                if (axis == 0)
                    axis_tab_x(nd, nd.sx * ((double)(a_x - Rb + idx) - c.x) + nd.ox, tabs[(2 * k) * Sb + idx]);
                else
                    axis_tab_y(nd, nd.sy * ((double)(a_y - Rb + idx) - c.y) + nd.oy, tabs[(2 * k + 1) * Sb + idx]);
            }
            __syncthreads();
        }
        constexpr int RE = MAXE > 0 ? MAXE : 1;
        T raw[RE][3];
        double acc[6] = {0, 0, 0, 0, 0, 0};
        const int ne = MAXE > 0 ? MAXE : (S2b + NTF - 1) / NTF;  // MAXE 0: value-only, any box
#pragma unroll
        for (int e = 0; e < ne; ++e) {
            const int m = threadIdx.x + e * NTF;
            const int er = MAXE > 0 ? e : 0;
            raw[er][0] = raw[er][1] = raw[er][2] = 0;
            if (m >= S2b) continue;
            const int row = m % Sb, col = m / Sb;
            const int gy = a_y - Rb + row, gx = a_x - Rb + col;
            T s = 0, dY = 0, dX = 0, g[3];
            if (gauss) {
                const T val = gauss_eval<T, GRAD>((T)P.fwhm, c, (T)gy, (T)gx, g[0], g[1], g[2]);
                if (M) M[(moff ? moff[j] : (int64_t)j * MS) + m] = val;
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (c.idx[k] < 0) continue;
                    const DevNode nd = P.nodes[c.idx[k]];
                    T pv, pdv, pdu;
                    tab_bicubic<GRAD, T>(data + nd.poff, tabs[(2 * k) * Sb + col], tabs[(2 * k + 1) * Sb + row],
                                         (T)nd.fill, pv, pdv, pdu);
                    s += (T)c.w[k] * pv;
                    if (GRAD) {
                        dY += (T)c.dwdy[k] * pv - (T)c.w[k] * (T)nd.sy * pdv;
                        dX += (T)c.dwdx[k] * pv - (T)c.w[k] * (T)nd.sx * pdu;
                    }
                }
                if (M) M[(moff ? moff[j] : (int64_t)j * MS) + m] = (T)c.flux * s + (T)c.bkg;
                g[0] = (T)c.flux * dY;
                g[1] = (T)c.flux * dX;
                g[2] = s;
            }
            if (!GRAD) continue;
            if (gy < 1 || gy > fc.ny || gx < 1 || gx > fc.nx) continue;
            const int64_t q = (gy - 1) + (int64_t)(gx - 1) * fc.ny;
            if (!(w[q] > 0)) continue;
            const T sq = (T)sw[q];
            const T ga = g0 == 0 ? g[0] : (g0 == 1 ? g[1] : g[2]);
            const T gb = g1 == 0 ? g[0] : (g1 == 1 ? g[1] : g[2]);
            const T gc = g2 == 0 ? g[0] : (g2 == 1 ? g[1] : g[2]);
            raw[er][0] = sq * ga;
            raw[er][1] = p > 1 ? sq * gb : (T)0;
            raw[er][2] = p > 2 ? sq * gc : (T)0;
            const double r0 = raw[er][0], r1 = raw[er][1], r2 = raw[er][2];
            if (gram) {  // packed upper triangle (0,0) (0,1) (0,2) (1,1) (1,2) (2,2) for p = 3
                if (p == 1) {
                    acc[0] += r0 * r0;
                } else if (p == 2) {
                    acc[0] += r0 * r0;
                    acc[1] += r0 * r1;
                    acc[2] += r1 * r1;
                } else {
                    acc[0] += r0 * r0;
                    acc[1] += r0 * r1;
                    acc[2] += r0 * r2;
                    acc[3] += r1 * r1;
                    acc[4] += r1 * r2;
                    acc[5] += r2 * r2;
                }
            } else {
                acc[0] += r0 * r0;
                acc[1] += r1 * r1;
                acc[2] += r2 * r2;
            }
        }
        if (GRAD) {
            const int nacc = gram ? p * (p + 1) / 2 : p;
#pragma unroll
            for (int t = 0; t < 6; ++t) {
                if (t >= nacc) break;
                double tot = block_sum<NTF>(acc[t], sh);
                if (threadIdx.x == 0) {
                    if (gram) gram[(int64_t)j * 6 + t] = tot;
                    else cn_sh[t] = tot;
                }
            }
            __syncthreads();
            if (!gram) {
                T inv[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    double cn = sqrt(k < p ? cn_sh[k] : 1.0);
                    cn = cn < kEps64 ? kEps64 : cn;
                    inv[k] = (T)(1.0 / cn);
                    if (threadIdx.x == 0 && k < p) colnorm[(int64_t)j * p + k] = cn;
                }
                T* Vj = V + (int64_t)j * fc.VS;
#pragma unroll
                for (int e = 0; e < RE; ++e) {
                    const int m = threadIdx.x + e * NTF;
                    if (m >= S2b) continue;
                    Vj[m * p] = raw[e][0] * inv[0];
                    if (p > 1) Vj[m * p + 1] = raw[e][1] * inv[1];
                    if (p > 2) Vj[m * p + 2] = raw[e][2] * inv[2];
                }
            }
        }
        __syncthreads();
    }
}

// Warp-per-star stamp evaluation for single-node ePSFs and the Gaussian (the
// common case): no block barriers, each warp keeps its star's row / column
// tables in its own slice of shared memory, and GRAD runs two passes
// (colnorm, then the scaled stamp) instead of caching the raw values.
// Same outputs as k_eval.
template <bool GRAD, typename T>
__global__ void __launch_bounds__(256, 3) k_eval_warp(const int32_t* __restrict__ list, int64_t nlist, FitConst fc,
                                                      DevPsf P, const StarCoef* __restrict__ coef,
                                                      const int32_t* __restrict__ ay, const int32_t* __restrict__ ax,
                                                      const double* __restrict__ w, const double* __restrict__ sw,
                                                      T* __restrict__ V, double* __restrict__ colnorm,
                                                      double* __restrict__ gram, T* __restrict__ M, int Rmax, int MS,
                                                      const int32_t* __restrict__ Rs, const int64_t* __restrict__ moff) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    AxisTab<T>* tcol = (AxisTab<T>*)smem_raw + wid * 2 * (2 * Rmax + 1);
    const bool gauss = P.kind == CPB_PSF_CIRCULAR_GAUSSIAN;
    DevNode nd{};
    if (!gauss) nd = P.nodes[0];
    const T* base = gauss ? nullptr : pp_data<T>(P) + nd.poff;
    const T nfill = (T)nd.fill, nsy = (T)nd.sy, nsx = (T)nd.sx;
    const int p = fc.p;
    const int g0 = fc.gc[0] - 1, g1 = fc.gc[1] - 1, g2 = fc.gc[2] - 1;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (gridDim.x * (int64_t)blockDim.x) >> 5;
    for (int64_t li = warp; li < nlist; li += nwarps) {
        const int j = list ? list[li] : (int)li;
        const StarCoef& cg = coef[j];
        const double cy = cg.y, cx = cg.x;
        const T flux = (T)cg.flux, bkg = (T)cg.bkg;
        const T w0 = (T)cg.w[0], dwy = (T)cg.dwdy[0], dwx = (T)cg.dwdx[0];
        const int Rb = Rs ? Rs[j] : Rmax;  // this star's box radius
        const int Sb = 2 * Rb + 1, S2b = Sb * Sb;
        const int q32 = 32 / Sb, r32 = 32 % Sb;
        AxisTab<T>* trow = tcol + Sb;
        const int oy = ay[j] - Rb, ox = ax[j] - Rb;
        if (!gauss) {
            for (int idx = lane; idx < 2 * Sb; idx += 32) {
                if (idx < Sb) axis_tab_x(nd, nd.sx * ((double)(ox + idx) - cx) + nd.ox, tcol[idx]);
                else axis_tab_y(nd, nd.sy * ((double)(oy + idx - Sb) - cy) + nd.oy, trow[idx - Sb]);
            }
            __syncwarp();
        }
        StarCoef gc_;
        if (gauss) {
            gc_.y = cy;
            gc_.x = cx;
            gc_.flux = cg.flux;
            gc_.bkg = cg.bkg;
        }
        // value (and gradient) at stamp entry (row, col)
        auto eval_px = [&](int row, int col, T& val, T& ga, T& gb, T& gcc) {
            T g[3];
            if (gauss) {
                val = gauss_eval<T, GRAD>((T)P.fwhm, gc_, (T)(oy + row), (T)(ox + col), g[0], g[1], g[2]);
            } else {
                T pv, pdv = 0, pdu = 0;
                tab_bicubic<GRAD, T>(base, tcol[col], trow[row], nfill, pv, pdv, pdu);
                const T s = w0 * pv;
                val = flux * s + bkg;
                if (GRAD) {
                    g[0] = flux * (dwy * pv - w0 * nsy * pdv);
                    g[1] = flux * (dwx * pv - w0 * nsx * pdu);
                    g[2] = s;
                }
            }
            if (GRAD) {
                ga = g0 == 0 ? g[0] : (g0 == 1 ? g[1] : g[2]);
                gb = g1 == 0 ? g[0] : (g1 == 1 ? g[1] : g[2]);
                gcc = g2 == 0 ? g[0] : (g2 == 1 ? g[1] : g[2]);
            }
        };
        if (!GRAD) {
            int row = lane % Sb, col = lane / Sb;
            for (int m = lane; m < S2b; m += 32) {
                T val, a, b, c;
                eval_px(row, col, val, a, b, c);
                M[(moff ? moff[j] : (int64_t)j * MS) + m] = val;
                row += r32;
                col += q32;
                if (row >= Sb) {
                    row -= Sb;
                    col += 1;
                }
            }
        } else {
            // one evaluation a stamp entry: the weighted derivatives go to V
            // unscaled (and the model value to M) while the column norms
            // accumulate; a second sweep over the star's block, still in L2,
            // applies the inverse norms
            double acc[6] = {0, 0, 0, 0, 0, 0};
            T* Vj = gram ? nullptr : V + (int64_t)j * fc.VS;
            int row = lane % Sb, col = lane / Sb;
            for (int m = lane; m < S2b; m += 32) {
                const int gy = oy + row, gx = ox + col;
                const bool onimg = gy >= 1 && gy <= fc.ny && gx >= 1 && gx <= fc.nx;
                const int64_t q = onimg ? (gy - 1) + (int64_t)(gx - 1) * fc.ny : 0;
                const bool use = onimg && w[q] > 0;
                T r0 = 0, r1 = 0, r2 = 0;
                if (use || (M && !gram)) {
                    T val, a, b, c;
                    eval_px(row, col, val, a, b, c);
                    if (M && !gram) M[(moff ? moff[j] : (int64_t)j * MS) + m] = val;
                    if (use) {
                        const T sq = (T)sw[q];
                        r0 = sq * a;
                        r1 = sq * b;
                        r2 = sq * c;
                        const double d0 = r0, d1 = p > 1 ? (double)r1 : 0.0, d2 = p > 2 ? (double)r2 : 0.0;
                        if (gram) {
                            acc[0] += d0 * d0;
                            acc[1] += d0 * d1;
                            acc[2] += d0 * d2;
                            acc[3] += d1 * d1;
                            acc[4] += d1 * d2;
                            acc[5] += d2 * d2;
                        } else {
                            acc[0] += d0 * d0;
                            acc[1] += d1 * d1;
                            acc[2] += d2 * d2;
                        }
                    }
                }
                if (!gram) {
                    Vj[m * p] = r0;
                    if (p > 1) Vj[m * p + 1] = r1;
                    if (p > 2) Vj[m * p + 2] = r2;
                }
                row += r32;
                col += q32;
                if (row >= Sb) {
                    row -= Sb;
                    col += 1;
                }
            }
#pragma unroll
            for (int t = 0; t < 6; ++t) acc[t] = warp_sum(acc[t]);
            if (gram) {
                if (lane == 0) {
                    double* gj = gram + (int64_t)j * 6;
                    if (p == 1) gj[0] = acc[0];
                    else if (p == 2) {
                        gj[0] = acc[0];
                        gj[1] = acc[1];
                        gj[2] = acc[3];
                    } else {
                        for (int t = 0; t < 6; ++t) gj[t] = acc[t];
                    }
                }
            } else {
                T inv[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    double cn = sqrt(k < p ? acc[k] : 1.0);
                    cn = cn < kEps64 ? kEps64 : cn;
                    inv[k] = (T)(1.0 / cn);
                    if (lane == 0 && k < p) colnorm[(int64_t)j * p + k] = cn;
                }
                for (int m = lane; m < S2b; m += 32) {  // the entries this lane wrote above
                    Vj[m * p] *= inv[0];
                    if (p > 1) Vj[m * p + 1] *= inv[1];
                    if (p > 2) Vj[m * p + 2] *= inv[2];
                }
            }
        }
        __syncwarp();
    }
}

// Per-region pixel gather over the region's star list (stars in Morton
// order), the deterministic replacement of the reference's scatter-adds.
// A block owns a TY x TX pixel region; warp w owns the SW-column strip
// starting at column w*SW and accumulates it in shared memory.  For each star
// whose box meets its strip the warp streams the star's stamp entries for
// those (at most SW) columns -- a contiguous run of the star's block -- and
// adds them to the strip, one star after another (no atomics, fixed order).
//   KIND_JV: sum_k V[j, m, k] * v[j, k] / alpha  (apply_J!, :95-137)
//   KIND_M : sum M[j, m]                         (_render_model!)
// Epilogues (MODE): LSQR u update + beta (Krylov lsqr step 1); weighted
// residual + cost (_residual_cost!, :675-684); candidate cost (_cost!,
// :686-693); freeze subtraction (_freeze_star!, :739-754); final residual.
constexpr int KIND_JV = 0, KIND_M = 1;
constexpr int MODE_LSQR = 4;
// 32-entry slots a warp loads per round: 4 measured fastest on the 2048^2 fit
// (J.v 47.0 ms per fit; 3 slots 46.6 ms, 6 slots 58.5 ms and 8 slots 65.1 ms,
// their registers costing more resident warps than the extra loads in flight
// gain); J.v alone is held to 64 registers (8 blocks an SM: 45.7 ms), the
// model gathers keep the compiler's choice
constexpr int KSLOT = 4;

template <int KIND, int MODE, typename TS>
__global__ void __launch_bounds__(NT, KIND == KIND_JV ? 8 : 0) k_gather(FitConst fc, const int32_t* __restrict__ tstart,
                                               const int32_t* __restrict__ tend, const int4* __restrict__ tlist,
                                               const int32_t* __restrict__ tord,
                                               const uint8_t* __restrict__ incl, const TS* __restrict__ src,
                                               int Rbox, int64_t stride, const int64_t* __restrict__ soff,
                                               const double* __restrict__ vt,
                                               const double* u_src, double u_sign,
                                               double* out, const uint8_t* __restrict__ umask,
                                               const double* __restrict__ w, const double* __restrict__ sw,
                                               const double* __restrict__ data_ref, Scalars* sc, Reducer red,
                                               double* result) {
    __shared__ double s_acc[NT / 32][TY * SW];
    __shared__ int s_j[NT];
    __shared__ int s_ay[NT];
    __shared__ int s_ax[NT];
    __shared__ int s_rb[NT];
    __shared__ double s_v[3][NT];
    __shared__ int s_wcnt[NT / 32];
    __shared__ double sh[32];
    double inv_alpha = 1.0, alpha = 0.0, uscale = 1.0;
    if (KIND == KIND_JV) {
        if (sc->stopped) return;  // uniform across the grid
        inv_alpha = sc->inv_alpha;
        alpha = sc->alpha;
        uscale = u_sign * sc->inv_beta;
    }
    const int p = KIND == KIND_JV ? fc.p : 1;
    const int reg = tord[blockIdx.x];
    const int ry = reg % fc.nty, rx = reg / fc.nty;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int y0 = ry * TY + 1, xs0 = rx * TX + wid * SW + 1;
    const int yend = min(y0 + TY - 1, fc.ny), xend = min(xs0 + SW - 1, fc.nx);
    double* acc = s_acc[wid];
    for (int t = lane; t < TY * SW; t += 32) acc[t] = 0.0;
    const int s0 = tstart[reg], s1 = tend[reg];
    for (int c0 = s0; c0 < s1; c0 += NT) {
        const int li = c0 + threadIdx.x;
        int4 ent = make_int4(-1, 0, 0, 0);
        bool keep = false;
        if (li < s1) {
            ent = tlist[li];
            keep = incl ? incl[ent.x] != 0 : true;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_wcnt[wid] = __popc(bal);
        __syncthreads();
        int before = 0, total = 0;
#pragma unroll
        for (int q = 0; q < NT / 32; ++q) {
            total += s_wcnt[q];
            if (q < wid) before += s_wcnt[q];
        }
        if (keep) {
            const int pos = before + __popc(bal & ((1u << lane) - 1u));
            s_j[pos] = ent.x;
            s_ay[pos] = ent.y;
            s_ax[pos] = ent.z;
            s_rb[pos] = ent.w;
            if (KIND == KIND_JV)
                for (int k = 0; k < fc.p; ++k) s_v[k][pos] = vt[(int64_t)ent.x * fc.p + k] * inv_alpha;
        }
        __syncthreads();
        if (xs0 <= fc.nx) {
            // The warp walks its stars' entries in 32-entry slots (a slot holds
            // one star's entries, a star's last slot is padded) and takes four
            // slots a round -- up to four stars -- loading all of them before
            // adding any; slots are added in order, so every pixel still sums
            // its stars in list order, and one add instruction never holds two
            // stars (no lost updates between lanes).
            int e = 0, c = 0;  // current star and slot
            int tot = 0, nrows = 1, m0 = 0, a0 = 0, Sb = 1;
            float inv_nrows = 1.0f;
            const TS* base = src;
            auto seek = [&](int from) {  // the next star meeting the strip, from `from`
                c = 0;
                for (e = from; e < total; ++e) {
                    const int ax_ = s_ax[e], ay_ = s_ay[e];
                    // model renders: each star's own model radius; J v: the fit box
                    const int Rb = KIND == KIND_M ? s_rb[e] : Rbox;
                    Sb = 2 * Rb + 1;
                    const int c_lo = max(ax_ - Rb, xs0), c_hi = min(ax_ + Rb, xend);
                    const int r_lo = max(ay_ - Rb, y0), r_hi = min(ay_ + Rb, yend);
                    if (c_lo > c_hi || r_lo > r_hi) continue;  // warp-uniform
                    nrows = r_hi - r_lo + 1;
                    tot = nrows * (c_hi - c_lo + 1);
                    inv_nrows = 1.0f / (float)nrows;
                    m0 = (r_lo - ay_ + Rb) + (c_lo - ax_ + Rb) * Sb;
                    a0 = (r_lo - y0) + (c_lo - xs0) * TY;
                    base = src + (soff ? soff[s_j[e]] : (int64_t)s_j[e] * stride);
                    return;
                }
            };
            seek(0);
            while (e < total) {
                TS raw[KSLOT][3];
                int dst[KSLOT], eq[KSLOT];
#pragma unroll
                for (int q = 0; q < KSLOT; ++q) {
                    dst[q] = -1;
                    eq[q] = e;
                    raw[q][0] = raw[q][1] = raw[q][2] = (TS)0;
                    if (e < total) {
                        const int t = c * 32 + lane;
                        if (t < tot) {
                            const int cc = (int)(((float)t + 0.5f) * inv_nrows);
                            const int rr = t - cc * nrows;
                            const TS* ptr = base + (int64_t)(m0 + rr + cc * Sb) * p;
                            raw[q][0] = __ldg(ptr);
                            if (KIND == KIND_JV) {
                                if (p > 1) raw[q][1] = __ldg(ptr + 1);
                                if (p > 2) raw[q][2] = __ldg(ptr + 2);
                            }
                            dst[q] = a0 + rr + cc * TY;
                        }
                        if ((c + 1) * 32 < tot) ++c;
                        else seek(e + 1);
                    }
                }
#pragma unroll
                for (int q = 0; q < KSLOT; ++q) {
                    if (dst[q] >= 0) {
                        double v;
                        if (KIND == KIND_JV) {
                            v = (double)raw[q][0] * s_v[0][eq[q]];
                            if (p > 1) v += (double)raw[q][1] * s_v[1][eq[q]];
                            if (p > 2) v += (double)raw[q][2] * s_v[2][eq[q]];
                        } else {
                            v = (double)raw[q][0];
                        }
                        acc[dst[q]] += v;
                    }
                }
                __syncwarp();
            }
        }
        __syncthreads();
    }
    double part = 0.0;
    for (int t = lane; t < TY * SW; t += 32) {
        const int gy = y0 + (t % TY), gx = xs0 + t / TY;
        if (gy > fc.ny || gx > fc.nx) continue;
        const int64_t q = (gy - 1) + (int64_t)(gx - 1) * fc.ny;
        const double a = acc[t];
        if (MODE == MODE_LSQR) {
            const double un = a - alpha * (u_src[q] * uscale);
            out[q] = un;
            part += un * un;
        } else if (MODE == MODE_CUR) {
            double wr = 0.0;
            if (umask[q]) {
                wr = sw[q] * (a - data_ref[q]);
                part += wr * wr;
            }
            out[q] = wr;  // wt_resid (zero outside U)
        } else if (MODE == MODE_CAND) {
            if (umask[q]) {
                const double r = a - data_ref[q];
                part += w[q] * r * r;
            }
        } else if (MODE == MODE_FREEZE) {
            out[q] -= a;  // data_work
        } else {
            out[q] = data_ref[q] - a;  // residual against the original data
        }
    }
    if (MODE == MODE_LSQR) {
        double tot;
        if (grid_reduce<NT>(part, red, sh, &tot, reg) && threadIdx.x == 0) {
            const double beta = sqrt(tot);
            sc->beta = beta;
            if (beta != 0.0) {
                sc->inv_beta = 1.0 / beta;
                sc->Anorm2 = sc->Anorm2 + alpha * alpha + beta * beta;
                if (sc->lambda > 0) sc->Anorm2 += sc->lambda * sc->lambda;
            }
        }
    } else if (MODE == MODE_CUR || MODE == MODE_CAND) {
        grid_reduce<NT>(part, red, sh, result, reg);
    }
}

// J^T u for the stars of `list` (apply_JT!, :55-85): one warp per star,
// coalesced reads of the star's stamp block, gathers of u; stamp indices
// advance incrementally and four entries per lane are in flight at once.
// Writes z[j*p+k] = sum_m V[j,m,k] u[pix(m)] * uscale.  LSQR form: v_new =
// z - beta * v_old / alpha_old and alpha = ||v_new|| (Krylov lsqr step 2).
template <bool LSQR, typename TS>
__global__ void __launch_bounds__(256, 4) k_JT(const int32_t* __restrict__ list, int64_t nlist, FitConst fc,
                                            const int32_t* __restrict__ ay, const int32_t* __restrict__ ax,
                                            const TS* __restrict__ V, const double* __restrict__ u,
                                            double* __restrict__ z, Scalars* sc, Reducer red) {
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (gridDim.x * (int64_t)blockDim.x) >> 5;
    double uscale = 1.0, beta = 0.0, inv_alpha = 0.0;
    if (LSQR) {
        if (sc->stopped || sc->beta == 0.0) return;  // uniform across the grid
        uscale = sc->inv_beta;
        beta = sc->beta;
        inv_alpha = sc->inv_alpha;
    }
    const int p = fc.p, S = fc.S, S2 = fc.S2, R = fc.R;
    double part = 0.0;
    for (int64_t li = warp; li < nlist; li += nwarps) {
        const int j = list[li];
        const int a_y = ay[j] - R, a_x = ax[j] - R;
        const TS* Vj = V + (int64_t)j * fc.VS;
        double acc0 = 0, acc1 = 0, acc2 = 0;
        int r = lane % S, c = lane / S;
        for (int m0 = 0; m0 < S2; m0 += 128) {
            double uv[4], v0[4], v1[4], v2[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int m = m0 + lane + 32 * q;
                const int gy = a_y + r, gx = a_x + c;
                const bool ok = m < S2 && gy >= 1 && gy <= fc.ny && gx >= 1 && gx <= fc.nx;
                uv[q] = 0.0;
                v0[q] = v1[q] = v2[q] = 0.0;
                if (ok) {
                    uv[q] = __ldg(u + (gy - 1) + (int64_t)(gx - 1) * fc.ny);
                    const TS* vm = Vj + m * p;
                    v0[q] = (double)__ldg(vm);
                    if (p > 1) v1[q] = (double)__ldg(vm + 1);
                    if (p > 2) v2[q] = (double)__ldg(vm + 2);
                }
                r += fc.r32;
                c += fc.q32;
                if (r >= S) {
                    r -= S;
                    c += 1;
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double uq = LSQR ? uv[q] * uscale : uv[q];
                acc0 += v0[q] * uq;
                acc1 += v1[q] * uq;
                acc2 += v2[q] * uq;
            }
        }
        acc0 = warp_sum(acc0);
        acc1 = warp_sum(acc1);
        acc2 = warp_sum(acc2);
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (k >= p) break;
                double val = k == 0 ? acc0 : (k == 1 ? acc1 : acc2);
                if (LSQR) {
                    val = val - beta * (z[(int64_t)j * p + k] * inv_alpha);
                    part += val * val;
                }
                z[(int64_t)j * p + k] = val;
            }
        }
    }
    if (LSQR) {
        double tot;
        if (grid_reduce<256>(part, red, sh, &tot) && threadIdx.x == 0) {
            const double alpha = sqrt(tot);
            sc->alpha = alpha;
            sc->inv_alpha = alpha != 0.0 ? 1.0 / alpha : 0.0;
        }
    }
}


// LSQR init after b_scaled: v1 = A'u1 = -b_scaled / beta1 (the first
// adjoint product reuses the gradient pass), alpha1 = ||v1||, x = 0.
__global__ void k_lsqr_v0(int64_t n, const double* b_scaled, double* vt, double* x, Scalars* sc, Reducer red) {
    __shared__ double sh[32];
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const double inv_b1 = sc->inv_beta;
    double part = 0.0;
    if (i < n) {
        double v = -(b_scaled[i] * inv_b1);
        vt[i] = v;
        x[i] = 0.0;
        part = v * v;
    }
    double tot;
    if (grid_reduce<256>(part, red, sh, &tot) && threadIdx.x == 0) {
        double alpha = sqrt(tot);
        sc->alpha = alpha;
        sc->Anorm2 = tot;
        sc->inv_alpha = alpha != 0.0 ? 1.0 / alpha : 0.0;
        sc->ArNorm0 = alpha * sc->beta1;
        sc->rhobar = alpha;
        sc->phibar = sc->beta1;
        if (alpha == 0.0) {
            sc->stopped = 1;
            sc->status = 4;
        } else {
            double Anorm = alpha, rNorm = sc->beta1;
            double t = sc->ArNorm0 / (Anorm * rNorm);
            if (t <= 1.4901161193847656e-08 || 1.0 + t <= 1.0) {
                sc->stopped = 1;
                sc->status = 1;
            }
        }
    }
}

__global__ void k_lsqr_w0(int64_t n, const double* vt, double* wl, Scalars* sc, Reducer red) {
    __shared__ double sh[32];
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const double ia = sc->inv_alpha;
    double part = 0.0;
    if (i < n) {
        double v = vt[i] * ia;
        wl[i] = v;
        part = v * v;
    }
    double tot;
    if (grid_reduce<256>(part, red, sh, &tot) && threadIdx.x == 0) sc->wnorm2 = tot;
}

// QR continuation, x / w update and stopping tests (Krylov lsqr main loop
// after the Golub-Kahan step).  Every thread evaluates the same scalar
// recurrence from the state; the last block commits it.
__global__ void k_lsqr_update(int64_t n, const double* vt, double* x, double* wl, Scalars* sc, Reducer red) {
    __shared__ double sh[32];
    if (sc->stopped) return;
    const double alpha = sc->alpha, beta = sc->beta, lambda = sc->lambda;
    double c1, s1, rhobar1;
    sym_givens(sc->rhobar, lambda, c1, s1, rhobar1);
    double phibar = sc->phibar;
    const double psi = s1 * phibar;
    phibar = c1 * phibar;
    double c, s, rho;
    sym_givens(rhobar1, beta, c, s, rho);
    const double phi = c * phibar;
    phibar = s * phibar;
    const double theta = s * alpha;
    const double sigma = phi / rho, tr = -theta / rho;
    const double ia = sc->inv_alpha;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double part = 0.0;
    if (i < n) {
        double wi = wl[i];
        x[i] = x[i] + sigma * wi;
        double wn = vt[i] * ia + tr * wi;
        wl[i] = wn;
        part = wn * wn;
    }
    double tot;
    if (grid_reduce<256>(part, red, sh, &tot) && threadIdx.x == 0) {
        const double axtol = 1.4901161193847656e-08, etol = axtol, ctol = axtol;
        int iter = sc->iter + 1;
        double xENorm2 = sc->xENorm2 + phi * phi;
        sc->err_vec[iter % 5] = phi;
        double err_lbnd = 0;
        if (iter >= 5) {
            double e2 = 0;
            for (int k = 0; k < 5; ++k) e2 += sc->err_vec[k] * sc->err_vec[k];
            err_lbnd = sqrt(e2);
        }
        const double tau = s * phi;
        double dNorm2 = sc->dNorm2 + sc->wnorm2 / (rho * rho);
        double delta = sc->s2 * rho;
        double gambar = -sc->c2 * rho;
        double rhs = phi - delta * sc->z;
        double zbar = rhs / gambar;
        double xNorm = sqrt(sc->xNorm2 + zbar * zbar);
        double c2, s2, gamma;
        sym_givens(gambar, theta, c2, s2, gamma);
        double z = rhs / gamma;
        double xNorm2 = sc->xNorm2 + z * z;
        double Anorm = sqrt(sc->Anorm2);
        double Acond = Anorm * sqrt(dNorm2);
        double res1 = phibar * phibar;
        double res2 = sc->res2 + psi * psi;
        double rNorm = sqrt(res1 + res2);
        double ArNorm = alpha * fabs(tau);
        double test1 = rNorm / sc->beta1;
        double test2 = ArNorm / (Anorm * rNorm);
        double test3 = 1.0 / Acond;
        double t1 = test1 / (1.0 + Anorm * xNorm / sc->beta1);
        double rNormtol = sc->btol + axtol * Anorm * xNorm / sc->beta1;
        bool ill = (1.0 + test3 <= 1.0) || (test3 <= ctol);
        bool zr = (1.0 + t1 <= 1.0) || (test1 <= rNormtol);
        bool fwd = iter >= 5 && err_lbnd <= etol * sqrt(xENorm2);
        bool solved = (1.0 + test2 <= 1.0) || (test2 <= axtol) || (ArNorm <= sc->atol) || zr || fwd;
        bool tired = iter >= sc->itmax;
        sc->rhobar = -c * alpha;
        sc->phibar = phibar;
        sc->xENorm2 = xENorm2;
        sc->dNorm2 = dNorm2;
        sc->xNorm = xNorm;
        sc->xNorm2 = xNorm2;
        sc->c2 = c2;
        sc->s2 = s2;
        sc->z = z;
        sc->res2 = res2;
        sc->wnorm2 = tot;
        sc->iter = iter;
        if (solved || tired || ill) {
            sc->stopped = 1;
            sc->status = solved ? (zr ? 2 : 1) : (ill ? 3 : 0);
        }
    }
}

// delta = x / colnorm, position step cap (_cap_position_step!, :700-716),
// delta_scaled = colnorm * delta.
__global__ void k_step(int64_t n_act, FitConst fc, double max_step, const double* x, const double* cn, double* delta,
                       double* dsc) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n_act) return;
    const int p = fc.p;
    double d[3];
    for (int k = 0; k < p; ++k) d[k] = x[j * p + k] / cn[j * p + k];
    if (fc.ky >= 0 || fc.kx >= 0) {
        double dy = fc.ky < 0 ? 0.0 : d[fc.ky];
        double dx = fc.kx < 0 ? 0.0 : d[fc.kx];
        double len = sqrt(dy * dy + dx * dx);
        if (len > max_step) {
            double scl = max_step / len;
            if (fc.ky >= 0) d[fc.ky] *= scl;
            if (fc.kx >= 0) d[fc.kx] *= scl;
        }
    }
    for (int k = 0; k < p; ++k) {
        delta[j * p + k] = d[k];
        dsc[j * p + k] = cn[j * p + k] * d[k];
    }
}

// global gradient cosine (:1199-1213), max over all parameters
__global__ void k_gnorm(int64_t n, const double* cn, const double* b, double dof, Scalars* sc, Reducer red) {
    __shared__ double sh[32];
    const double C_r = sc->cost / dof;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double g = 0.0;
    if (i < n) {
        double bt = cn[i] * b[i];
        double Aii = cn[i] * cn[i];
        g = fabs(bt) / (sqrt(Aii * C_r) + kEps64);
    }
    double tot;
    if (grid_reduce<256, true>(g, red, sh, &tot) && threadIdx.x == 0) sc->gnorm = tot;
}

// Accepted step (:1245-1251) and per-star freeze tests (:1265-1283,
// _x_tol_local :810-823, _g_tol_local :789-801).
__global__ void k_accept_freeze(int64_t n_act, FitConst fc, double x_tol, double g_tol, double dof, int iter,
                                double* theta, const double* delta, const double* dsc, const double* cn, double* D,
                                const double* b, uint8_t* live, uint8_t* newf, int32_t* frozen_at, uint8_t* conv,
                                Scalars* sc) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n_act) return;
    const int p = fc.p;
    for (int k = 0; k < p; ++k) {
        int64_t i = j * p + k;
        theta[i] = theta[i] + delta[i];
        D[i] = fmax(D[i], cn[i]);
    }
    newf[j] = 0;
    if (!live[j]) return;
    const double C_r = sc->cost / dof;
    double num = 0, xn = 0, gn = 0;
    for (int k = 0; k < p; ++k) {
        int64_t i = j * p + k;
        double v = (D[i] / cn[i]) * dsc[i];
        num += v * v;
        double xv = D[i] * theta[i];
        xn += xv * xv;
        double bt = cn[i] * b[i];
        double Aii = cn[i] * cn[i];
        gn = nan_max(gn, fabs(bt) / (sqrt(Aii * C_r) + kEps64));
    }
    bool xt = sqrt(num) <= x_tol * (sqrt(xn) + x_tol);
    bool gt = gn <= g_tol;
    if (xt || gt) {
        live[j] = 0;
        newf[j] = 1;
        frozen_at[j] = iter;
        conv[j] = 1;
        atomicAdd(&sc->n_new_frozen, 1);
    }
}

__global__ void k_freeze_all(int64_t n_act, int iter, uint8_t* live, int32_t* frozen_at, uint8_t* conv) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n_act || !live[j]) return;
    live[j] = 0;
    frozen_at[j] = iter;
    conv[j] = 1;
}



__global__ void k_errors(int64_t n_act, int p, const double* gram, bool reweighted, double dof, const Scalars* sc,
                         double* err) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n_act) return;
    double A[9], inv[9];
    int t = 0;
    for (int k = 0; k < p; ++k)
        for (int l = k; l < p; ++l) {
            double v = gram[j * 6 + t++];
            A[k + l * p] = v;
            A[l + k * p] = v;
        }
    double tr = 0;
    for (int k = 0; k < p; ++k) tr += A[k + k * p];
    for (int k = 0; k < p; ++k) A[k + k * p] += 1.0e-12 * tr;
    if (!chol_inv_small(A, p, inv)) pinv_small(A, p, inv);
    double f = reweighted ? sc->cost / dof : 1.0;
    for (int k = 0; k < p; ++k) err[j * p + k] = sqrt(fmax(0.0, inv[k + k * p] * f));
}

// The spread_model disk of the simultaneous fit, one block.  Its width comes
// from the first catalogue star's parameters after the final bookkeeping
// (params[row_y, 1], params[row_x, 1], :1289-1299 and :1363-1364): the fitted
// position when that star is active (the block finds its slot in the
// Morton-ordered active list), its catalogue position when not, the fixed
// value of a fixed coordinate.  ky / kx: their rows in theta, -1 when fixed.
// Dynamic shared memory: the quadrature panel, (7 + kh) * 32 doubles.
__global__ void __launch_bounds__(256) k_spread_disk(DevPsf P, double param, int kh,
                                                     const double* __restrict__ theta,
                                                     const int32_t* __restrict__ act, int64_t n_act, int p, int ky,
                                                     int kx, double fixed_y, double fixed_x,
                                                     const double* __restrict__ y0, const double* __restrict__ x0,
                                                     const double* __restrict__ rule, double* tab) {
    extern __shared__ double pan[];
    __shared__ double red[2 * 8 + 1];
    __shared__ int64_t slot;
    if (threadIdx.x == 0) slot = -1;
    __syncthreads();
    for (int64_t j = threadIdx.x; j < n_act; j += blockDim.x)
        if (act[j] == 0) slot = j;  // catalogue indices are unique: one writer at most
    __syncthreads();
    const int64_t j0 = slot;
    const double Y = ky < 0 ? fixed_y : (j0 >= 0 ? theta[j0 * p + ky] : y0[0]);
    const double X = kx < 0 ? fixed_x : (j0 >= 0 ? theta[j0 * p + kx] : x0[0]);
    spread_disk_block(P, param, kh, Y, X, rule, tab, red, pan);
}

// chisq and the qfit / crowding / spread_model diagnostics per active star
// (:1358-1397, psf_photometry_diagnostics.jl:154-231); one block of
// kDiagThreads a star (grid-stride), the star's model stamp over its box and
// its disk-correlated copy kept in shared memory.  stab: the disk table
// (spread_disk_block; null or off: spread_model NaN), smode its layout.
template <typename TI>
__global__ void __launch_bounds__(kDiagThreads, 3) k_diag(int64_t n_act, FitConst fc, DevPsf P, double fit_rad,
                                                      const StarCoef* __restrict__ coef,
                                                      const double* __restrict__ resid, const TI* __restrict__ img,
                                                      const TI* __restrict__ bkgimg, const TI* __restrict__ iv,
                                                      const double* __restrict__ stab, int kh, int smode,
                                                      int boxmax,
                                                      double* out /* n_act x 7: chisq qfit qfit_exp qfit_z crowding
                                                                     spread spread_err */) {
    extern __shared__ double stamp[];  // model stamp, x-pass scratch, disk-correlated stamp
    __shared__ double red[14 * (kDiagThreads / 32)];
    __shared__ StarCoef c;
    const double NaN = __longlong_as_double(0x7ff8000000000000LL);
    const bool on = stab != nullptr && spread_tab_on(stab);
    const SpreadDev D = on ? spread_dev(stab, kh) : SpreadDev{};
    const int mode = on ? smode : 0;
    double* Is = stamp + 7 * boxmax;  // mode 1: the six profiles
    if (mode == 1)
        for (int i = threadIdx.x; i < 6 * (2 * D.kh + 1); i += blockDim.x) Is[i] = D.I[i];
    for (int64_t j = blockIdx.x; j < n_act; j += gridDim.x) {
        __syncthreads();  // the previous star's c and stamps are no longer read
        if (threadIdx.x == 0) c = coef[j];
        __syncthreads();
        double* o = out + j * 7;
        const bool validp = isfinite(c.y) && isfinite(c.x) && isfinite(c.flux) && c.flux > 0;
        if (!validp) {
            if (threadIdx.x == 0) {
                o[0] = 0.0;
                o[1] = o[2] = o[3] = o[4] = o[5] = o[6] = NaN;
            }
            continue;
        }
        const int ylo = max((int)floor(c.y - fit_rad), 1), yhi = min((int)ceil(c.y + fit_rad), fc.ny);
        const int xlo = max((int)floor(c.x - fit_rad), 1), xhi = min((int)ceil(c.x + fit_rad), fc.nx);
        const int h = max(yhi - ylo + 1, 0), wd = max(xhi - xlo + 1, 0);
        const int nb = h * wd;
        const double inv_flux = 1.0 / c.flux;
        const bool spread = mode != 0 && nb > 0 && nb <= boxmax;
        double* G = stamp + 2 * boxmax;  // mode 2: the correlated stamp
        if (spread) {
            for (int e = threadIdx.x; e < nb; e += blockDim.x)
                stamp[e] = model_value<double, double>(P, P.data64, c, (double)(ylo + e % h), (double)(xlo + e / h));
            __syncthreads();
            if (mode == 1) {
                spread_xpass_all(D, Is, stamp, stamp + boxmax, boxmax, h, wd);
                __syncthreads();
            } else {
                spread_stamp_block(D, stamp, stamp + boxmax, G, h, wd);
            }
        }
        // num qv ncl ndi den ss ss2 Sp Sq Sp0 Sq0 SqG ng ngi
        double v[14] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int e = threadIdx.x; e < nb; e += blockDim.x) {
            const int gy = ylo + e % h, gx = xlo + e / h;
            const int64_t q = (gy - 1) + (int64_t)(gx - 1) * fc.ny;
            const double r = resid[q];
            const double wp = iv ? (double)iv[q] : 1.0;
            if (isfinite(wp) && wp > 0) {
                v[0] += wp * (r * r);
                v[12] += 1.0;
                const double mv = spread ? stamp[e] : model_value<double, double>(P, P.data64, c, (double)gy, (double)gx);
                v[1] += fabs(r);
                const double Pp = (mv - c.bkg) * inv_flux;
                const double wP = wp * Pp;
                const double p_i = r + mv - c.bkg;
                v[2] += wP * p_i;
                const double im = (double)img[q] - (bkgimg ? (double)bkgimg[q] : 0.0);
                v[3] += wP * (im - c.bkg);
                v[4] += wP * Pp;
                if (spread) {
                    const double gm = mode == 1 ? spread_ypass(D, Is, stamp + boxmax, boxmax, h, e) : G[e];
                    const double g_i = (gm - c.bkg) * inv_flux;
                    v[7] += wP * p_i;
                    v[8] += wp * g_i * p_i;
                    v[9] += wP * Pp;
                    v[10] += wp * Pp * g_i;
                    v[11] += wp * g_i * g_i;
                }
                if (iv) {
                    const double si = 1.0 / sqrt(wp);
                    v[5] += si;
                    v[6] += si * si;
                    v[13] += 1.0;
                }
            }
        }
        block_sum_n<14>(v, red);
        if (threadIdx.x == 0) {
            const double num = v[0], qv = v[1], ncl = v[2], ndi = v[3], den = v[4], ss = v[5], ss2 = v[6];
            const double Sp = v[7], Sq = v[8], Sp0 = v[9], Sq0 = v[10], SqG = v[11];
            const int ng = (int)v[12], ngi = (int)v[13];
            o[0] = (ng - fc.p > 0) ? num / (double)(ng - fc.p) : 0.0;
            o[1] = qv * inv_flux;
            o[4] = (den > 0 && ncl > 0 && ndi > 0) ? 2.5 * log10(ndi / ncl) : NaN;
            o[5] = o[6] = NaN;
            if (spread && Sp > 0) {
                o[5] = Sq / Sp - Sq0 / Sp0;
                if (iv) o[6] = sqrt(fmax(0.0, Sp * Sp * SqG + Sq * Sq * Sp0 - 2 * Sq * Sp * Sq0)) / (Sp * Sp);
            }
            if (iv) {
                o[2] = sqrt(2.0 / 3.141592653589793) * ss * inv_flux;
                if (ss2 > 0 && ngi > fc.p) {
                    double dfac = sqrt(1.0 - (double)fc.p / (double)ngi);
                    o[3] = (qv - sqrt(2.0 / 3.141592653589793) * dfac * ss) /
                           (sqrt((1.0 - 2.0 / 3.141592653589793) * ss2) * dfac);
                } else {
                    o[3] = NaN;
                }
            } else {
                o[2] = o[3] = NaN;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
template <typename T>
T* S(cpb_ctx* ctx, const char* name, size_t count) {
    return (T*)scratch(ctx, name, std::max<size_t>(count, 1) * sizeof(T));
}

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

// k_eval with the register cache its box needs: 256 threads for boxes up to
// 2,048 pixels, 512 / 1,024 threads up to 4,096 / 8,192 (ceil(radius) <= 44);
// the value-only form (no cache) takes any box.  smem: the axis tables.
template <bool GRAD, typename T, typename... A>
void launch_k_eval(int64_t S2, unsigned grid, size_t smem, cudaStream_t st, A... args) {
    auto go = [&](auto kern, int threads) {
        if (smem > 48 * 1024)
            check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attr");
        kern<<<grid, threads, smem, st>>>(args...);
    };
    if (S2 <= 256)
        go(k_eval<256, 1, GRAD, T>, 256);
    else if (S2 <= 512)
        go(k_eval<256, 2, GRAD, T>, 256);
    else if (S2 <= 1024)
        go(k_eval<256, 4, GRAD, T>, 256);
    else if (S2 <= 2048)
        go(k_eval<256, 8, GRAD, T>, 256);
    else if (S2 <= 4096)
        go(k_eval<512, 8, GRAD, T>, 512);
    else if (S2 <= 8192)
        go(k_eval<1024, 8, GRAD, T>, 1024);
    else if constexpr (!GRAD)
        go(k_eval<256, 0, false, T>, 256);
    else
        throw ArgError{"fit_rad too large for the B200 stamp kernel of a gridded PSF (ceil(fit_rad) must be <= 44)"};
}

struct TileLists {
    int32_t *start = nullptr, *end = nullptr;
    int4* list = nullptr;     // (star, anchor y, anchor x, box radius) per (tile, star) pair
    int32_t* order = nullptr; // the regions by decreasing star count: block b of a gather takes order[b]
};

TileLists build_tiles(cpb_ctx* ctx, const char* tag, int64_t n_act, const int32_t* ay, const int32_t* ax,
                      const int32_t* Rs, int Rconst, int ny, int nx, int nty, int ntx) {
    cudaStream_t st = ctx->stream;
    std::string t(tag);
    int32_t* cnt = S<int32_t>(ctx, (t + "_cnt").c_str(), n_act + 1);
    int32_t* offs = S<int32_t>(ctx, (t + "_offs").c_str(), n_act + 1);
    k_tile_count<<<nblk(n_act), 256, 0, st>>>(n_act, ay, ax, Rs, Rconst, ny, nx, cnt);
    check(cudaGetLastError(), "k_tile_count");
    check(cudaMemsetAsync(cnt + n_act, 0, sizeof(int32_t), st), "memset");
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, offs, (int)(n_act + 1), st);
    void* dtmp = scratch(ctx, (t + "_scan_tmp").c_str(), tmp);
    cub::DeviceScan::ExclusiveSum(dtmp, tmp, cnt, offs, (int)(n_act + 1), st);
    int32_t npairs = 0;
    check(cudaMemcpyAsync(&npairs, offs + n_act, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "d2h npairs");
    check(cudaStreamSynchronize(st), "sync");
    uint32_t* k0 = S<uint32_t>(ctx, (t + "_k0").c_str(), npairs);
    uint32_t* k1 = S<uint32_t>(ctx, (t + "_k1").c_str(), npairs);
    int32_t* v0 = S<int32_t>(ctx, (t + "_v0").c_str(), npairs);
    TileLists tl;
    int32_t* sorted_j = S<int32_t>(ctx, (t + "_sorted").c_str(), npairs);
    tl.list = S<int4>(ctx, (t + "_list").c_str(), npairs);
    const int64_t ntiles = (int64_t)nty * ntx;
    tl.start = S<int32_t>(ctx, (t + "_start").c_str(), ntiles);
    tl.end = S<int32_t>(ctx, (t + "_end").c_str(), ntiles);
    tl.order = S<int32_t>(ctx, (t + "_order").c_str(), ntiles);
    check(cudaMemsetAsync(tl.start, 0, sizeof(int32_t) * ntiles, st), "memset");
    check(cudaMemsetAsync(tl.end, 0, sizeof(int32_t) * ntiles, st), "memset");
    if (npairs > 0) {
        k_tile_emit<<<nblk(n_act), 256, 0, st>>>(n_act, ay, ax, Rs, Rconst, ny, nx, nty, offs, k0, v0);
        check(cudaGetLastError(), "k_tile_emit");
        int end_bit = 1;
        while ((1LL << end_bit) < ntiles) ++end_bit;
        tmp = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tmp, k0, k1, v0, sorted_j, npairs, 0, end_bit, st);
        dtmp = scratch(ctx, (t + "_sort_tmp").c_str(), tmp);
        cub::DeviceRadixSort::SortPairs(dtmp, tmp, k0, k1, v0, sorted_j, npairs, 0, end_bit, st);
        k_tile_bounds<<<nblk(npairs), 256, 0, st>>>(npairs, k1, tl.start, tl.end);
        check(cudaGetLastError(), "k_tile_bounds");
        k_tile_pack<<<nblk(npairs), 256, 0, st>>>(npairs, sorted_j, ay, ax, Rs, Rconst, tl.list);
        check(cudaGetLastError(), "k_tile_pack");
    }
    // heaviest regions first, so that the last wave of a gather is its lightest
    // (the radix sort is stable: equal counts keep region order)
    uint32_t* wkey = S<uint32_t>(ctx, (t + "_wkey").c_str(), 2 * ntiles);
    int32_t* widx = S<int32_t>(ctx, (t + "_widx").c_str(), ntiles);
    k_tile_work<<<nblk(ntiles), 256, 0, st>>>(ntiles, tl.start, tl.end, wkey, widx);
    check(cudaGetLastError(), "k_tile_work");
    tmp = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, wkey, wkey + ntiles, widx, tl.order, (int)ntiles, 0, 32,
                                              st);
    dtmp = scratch(ctx, (t + "_wsort_tmp").c_str(), tmp);
    cub::DeviceRadixSort::SortPairsDescending(dtmp, tmp, wkey, wkey + ntiles, widx, tl.order, (int)ntiles, 0, 32, st);
    check(cudaGetLastError(), "region order");
    return tl;
}

}  // namespace

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
template <typename TS>
int fit_sim_impl(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* P, const void* d_image,
                         int32_t eltype, int64_t ny64, int64_t nx64, const void* d_inv_var, const void* d_background,
                         int64_t n_stars, const double* d_y0, const double* d_x0, const double* d_flux0,
                         cpb_sim_result* out) {
    cudaStream_t st = ctx->stream;
    const double NaN = std::numeric_limits<double>::quiet_NaN();
    // argument checks in the reference's order (:984-997)
    if (!(P->max_iter > 0)) throw ArgError{"max_iter must be positive"};
    if (!(P->inner_iterations > 0)) throw ArgError{"inner_iterations must be positive"};
    if (!(P->linear_tol > 0)) throw ArgError{"linear_tol must be positive"};
    if (!(P->max_trials > 0)) throw ArgError{"max_trials must be positive"};
    if (!P->model_rad_auto && !(P->model_rad > 0)) throw ArgError{"model_rad must be :auto or a positive real"};
    const double model_rad_max = P->model_rad_max < 0 ? 10 * P->fit_rad : P->model_rad_max;
    if (!(model_rad_max >= P->fit_rad)) throw ArgError{"model_rad_max must be >= fit_rad"};
    if (!(P->model_rad_nsigma > 0)) throw ArgError{"model_rad_nsigma must be positive"};
    if (P->solver != CPB_SOLVER_LSQR && P->solver != CPB_SOLVER_LSMR) throw ArgError{"solver must be :lsqr or :lsmr"};
    if (P->solver == CPB_SOLVER_LSMR) throw ArgError{"solver :lsmr is not supported by the B200 path; use :lsqr"};
    if (P->damping == CPB_DAMP_LEVENBERG)
        throw ArgError{
            "LevenbergDamping is not supported by fit_all_stars_simultaneous: it conflicts with the "
            "column-equilibrated x_tol scaling. Use MarquardtDamping."};
    if (!(P->fit_rad > 0)) throw ArgError{"fit_rad must be positive"};
    if (eltype != CPB_F32 && eltype != CPB_F64) throw ArgError{"unsupported image eltype"};
    if (ny64 <= 0 || nx64 <= 0 || ny64 * nx64 >= (1LL << 31)) throw ArgError{"image size out of range"};
    const int ny = (int)ny64, nx = (int)nx64;
    const int64_t npix = ny64 * nx64;
    const bool reweighted =
        P->covariance == CPB_COV_REWEIGHTED || (P->covariance == CPB_COV_AUTO && d_inv_var == nullptr);
    out->n_active = 0;
    out->n_union = 0;
    out->n_trials = 0;
    out->n_lsqr_iters = 0;
    out->model_px_evals = 0;
    out->lsqr_px_macs = 0;
    out->device_seconds = 0;
    auto nan_diag = [&](int64_t i) {
        if (out->qfit) out->qfit[i] = NaN;
        if (out->qfit_expected) out->qfit_expected[i] = NaN;
        if (out->qfit_z) out->qfit_z[i] = NaN;
        if (out->crowding) out->crowding[i] = NaN;
        if (out->spread_model) out->spread_model[i] = NaN;
        if (out->spread_model_err) out->spread_model_err[i] = NaN;
    };
    if (n_stars == 0) {
        out->n_passes = 0;
        out->n_failed = 0;
        if (out->residual) std::fill(out->residual, out->residual + npix, 0.0);
        return 0;
    }
    // free set (:1015-1051)
    FitConst fc{};
    fc.p = 0;
    if (P->free_mask & CPB_FREE_Y) fc.gc[fc.p++] = 1;
    if (P->free_mask & CPB_FREE_X) fc.gc[fc.p++] = 2;
    if (P->free_mask & CPB_FREE_FLUX) fc.gc[fc.p++] = 3;
    if (P->free_mask & ~(CPB_FREE_Y | CPB_FREE_X | CPB_FREE_FLUX))
        throw ArgError{
            "fit_all_stars_simultaneous fits only (y, x, flux) per star. Fix `bkg` (subtract the background first "
            "and pass `fixed = (; bkg = zero(eltype(image)))`), and fix all shape parameters."};
    if (fc.p == 0) throw ArgError{"all model parameters are fixed; nothing to fit"};
    const int p = fc.p;
    fc.ky = fc.kx = -1;
    for (int k = 0; k < p; ++k) {
        if (fc.gc[k] == 1) fc.ky = k;
        if (fc.gc[k] == 2) fc.kx = k;
    }
    for (int k = p; k < 3; ++k) fc.gc[k] = 3;
    fc.fixed_y = P->fixed_y;
    fc.fixed_x = P->fixed_x;
    fc.fixed_flux = P->fixed_flux;
    fc.fixed_bkg = P->fixed_bkg;
    fc.R = (int)std::ceil(P->fit_rad);
    fc.S = 2 * fc.R + 1;
    fc.S2 = fc.S * fc.S;
    fc.VS = ((p * fc.S2 + 15) / 16) * 16;
    fc.q32 = 32 / fc.S;
    fc.r32 = 32 % fc.S;
    fc.ny = ny;
    fc.nx = nx;
    fc.nty = (ny + TY - 1) / TY;
    fc.ntx = (nx + TX - 1) / TX;
    const int64_t ntiles = (int64_t)fc.nty * fc.ntx;
    DevPsf dp = psf->dev;
    dp.fwhm = P->fixed_fwhm;

    check(cudaEventRecord(ctx->ev0, st), "event");
    // device-resident scalars and reducers
    Scalars* sc = S<Scalars>(ctx, "scalars", 1);
    check(cudaMemsetAsync(sc, 0, sizeof(Scalars), st), "memset");
    const int64_t max_blocks = std::max<int64_t>(ntiles, nblk(std::max<int64_t>(n_stars * 3, npix)) + 1);
    Reducer red{S<double>(ctx, "red_partials", max_blocks), S<unsigned>(ctx, "red_counter", 1)};
    check(cudaMemsetAsync(red.counter, 0, sizeof(unsigned), st), "memset");
    Scalars* h_sc = (Scalars*)ctx->pinned;

    // ---- data and weights (:1056-1084)
    double* data = S<double>(ctx, "data", npix);
    double* data_work = S<double>(ctx, "data_work", npix);
    double* w = S<double>(ctx, "w", npix);
    double* sw = S<double>(ctx, "sw", npix);
    unsigned* flags = S<unsigned>(ctx, "flags", 4);
    check(cudaMemsetAsync(flags, 0, 4 * sizeof(unsigned), st), "memset");
    if (eltype == CPB_F64)
        k_prepare<double><<<nblk(npix), 256, 0, st>>>((const double*)d_image, (const double*)d_inv_var,
                                                      (const double*)d_background, npix, data, data_work, w, sw,
                                                      flags);
    else
        k_prepare<float><<<nblk(npix), 256, 0, st>>>((const float*)d_image, (const float*)d_inv_var,
                                                     (const float*)d_background, npix, data, data_work, w, sw, flags);
    check(cudaGetLastError(), "k_prepare");

    // ---- _build_stamps! (:245-323)
    int32_t* ay_c = S<int32_t>(ctx, "ay_c", n_stars);
    int32_t* ax_c = S<int32_t>(ctx, "ax_c", n_stars);
    uint8_t* ok = S<uint8_t>(ctx, "ok", n_stars);
    uint64_t* key = S<uint64_t>(ctx, "key", n_stars);
    k_anchor<<<nblk(n_stars), 256, 0, st>>>(n_stars, d_y0, d_x0, d_flux0, fc.R, ny, nx, w, ay_c, ax_c, ok, key,
                                            flags + 1);
    check(cudaGetLastError(), "k_anchor");
    // compact active stars in catalogue order, then stable radix sort by Morton key
    int32_t* iota = S<int32_t>(ctx, "iota", n_stars);
    int32_t* sel = S<int32_t>(ctx, "sel", n_stars);
    uint64_t* selkey = S<uint64_t>(ctx, "selkey", n_stars);
    uint64_t* selkey2 = S<uint64_t>(ctx, "selkey2", n_stars);
    int32_t* act = S<int32_t>(ctx, "act", n_stars);
    int* d_nsel = S<int>(ctx, "nsel", 1);
    {
        std::vector<int32_t> h_iota(n_stars);
        for (int64_t i = 0; i < n_stars; ++i) h_iota[i] = (int32_t)i;
        check(cudaMemcpyAsync(iota, h_iota.data(), sizeof(int32_t) * n_stars, cudaMemcpyHostToDevice, st), "h2d");
        size_t tmp = 0;
        cub::DeviceSelect::Flagged(nullptr, tmp, iota, ok, sel, d_nsel, (int)n_stars, st);
        void* dtmp = scratch(ctx, "sel_tmp", tmp);
        cub::DeviceSelect::Flagged(dtmp, tmp, iota, ok, sel, d_nsel, (int)n_stars, st);
        tmp = 0;
        cub::DeviceSelect::Flagged(nullptr, tmp, key, ok, selkey, d_nsel, (int)n_stars, st);
        dtmp = scratch(ctx, "sel_tmp2", tmp);
        cub::DeviceSelect::Flagged(dtmp, tmp, key, ok, selkey, d_nsel, (int)n_stars, st);
        check(cudaGetLastError(), "select");
    }
    int h_nsel = 0;
    unsigned h_flags[4];
    check(cudaMemcpyAsync(&h_nsel, d_nsel, sizeof(int), cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(h_flags, flags, sizeof(h_flags), cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaStreamSynchronize(st), "sync");
    if (!d_inv_var && h_flags[0] > 0)
        throw ArgError{
            "the image contains non-finite values but `inv_var` was not provided; pass `inv_var` to mask them or "
            "clean the image first"};
    const int64_t n_act = h_nsel;
    const int n_failed = (int)(n_stars - n_act);
    out->n_active = n_act;
    if (n_act == 0) {  // _empty_simultaneous_result (:1433-1445)
        std::vector<double> y(n_stars), x(n_stars), f(n_stars);
        check(cudaMemcpy(y.data(), d_y0, sizeof(double) * n_stars, cudaMemcpyDeviceToHost), "d2h");
        check(cudaMemcpy(x.data(), d_x0, sizeof(double) * n_stars, cudaMemcpyDeviceToHost), "d2h");
        check(cudaMemcpy(f.data(), d_flux0, sizeof(double) * n_stars, cudaMemcpyDeviceToHost), "d2h");
        for (int64_t i = 0; i < n_stars; ++i) {
            out->y[i] = y[i];
            out->x[i] = x[i];
            out->flux[i] = f[i];
            out->bkg[i] = 0.0;
            out->y_err[i] = (P->free_mask & CPB_FREE_Y) ? NaN : 0.0;
            out->x_err[i] = (P->free_mask & CPB_FREE_X) ? NaN : 0.0;
            out->flux_err[i] = (P->free_mask & CPB_FREE_FLUX) ? NaN : 0.0;
            out->bkg_err[i] = 0.0;
            out->converged[i] = 0;
            out->valid[i] = 0;
            if (out->chisq) out->chisq[i] = 0.0;
            nan_diag(i);
            out->n_iter[i] = 0;
        }
        out->n_passes = 0;
        out->n_failed = (int32_t)n_stars;
        if (out->residual) std::fill(out->residual, out->residual + npix, 0.0);
        return 0;
    }
    if (h_flags[1] > 0)
        throw ArgError{"InexactError: a star's integer anchor is negative (Morton key of a negative coordinate)"};
    {
        size_t tmp = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tmp, selkey, selkey2, sel, act, (int)n_act, 0, 64, st);
        void* dtmp = scratch(ctx, "sort_tmp", tmp);
        cub::DeviceRadixSort::SortPairs(dtmp, tmp, selkey, selkey2, sel, act, (int)n_act, 0, 64, st);
        check(cudaGetLastError(), "sort");
    }
    const int64_t n = (int64_t)p * n_act;
    int32_t* ay = S<int32_t>(ctx, "ay", n_act);
    int32_t* ax = S<int32_t>(ctx, "ax", n_act);
    double* theta = S<double>(ctx, "theta", n);
    k_gather_active<<<nblk(n_act), 256, 0, st>>>(n_act, act, ay_c, ax_c, d_y0, d_x0, d_flux0, p,
                                                 make_int3(fc.gc[0], fc.gc[1], fc.gc[2]), ay, ax, theta);
    check(cudaGetLastError(), "k_gather_active");

    // ---- union of stamp pixels (:329-335)
    uint8_t* umask = S<uint8_t>(ctx, "umask", npix);
    check(cudaMemsetAsync(umask, 0, npix, st), "memset");
    int32_t* dbg_pix = out->dbg_pixels ? S<int32_t>(ctx, "dbg_pix", (int64_t)fc.S2 * n_act) : nullptr;
    k_union<<<(unsigned)n_act, 256, 0, st>>>(n_act, ay, ax, fc.R, ny, nx, w, umask, dbg_pix);
    check(cudaGetLastError(), "k_union");
    unsigned long long* ucnt = S<unsigned long long>(ctx, "ucnt", 1);
    check(cudaMemsetAsync(ucnt, 0, sizeof(unsigned long long), st), "memset");
    k_count_u8<<<nblk(npix), 256, 0, st>>>(umask, npix, ucnt);
    unsigned long long h_ucnt = 0;
    check(cudaMemcpyAsync(&h_ucnt, ucnt, sizeof(h_ucnt), cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaStreamSynchronize(st), "sync");
    out->n_union = (int64_t)h_ucnt;

    // ---- model radii (:1111-1124)
    if (P->model_rad_auto && !d_inv_var)
        throw ArgError{
            "model_rad=:auto requires inv_var (it needs a noise scale); pass inv_var or an explicit scalar model_rad"};
    int model_R;                  // the largest model radius (sizes the model stamps)
    int32_t* d_modelR = nullptr;  // per active slot when model_rad = :auto
    std::vector<int32_t> h_modelR;
    double model_box_sum = 0;     // sum over active stars of (2 R_j + 1)^2
    if (P->model_rad_auto) {
        const int R_cap = (int)std::ceil(model_rad_max);
        // the noise sample w[1 : step : end] and the active stars' catalogue fluxes
        const int64_t step = std::max<int64_t>(1, npix / 65536);
        const int64_t nsamp = (npix + step - 1) / step;
        std::vector<double> wsamp(nsamp), f0(n_stars);
        std::vector<int32_t> h_act_order(n_act);
        check(cudaMemcpy2DAsync(wsamp.data(), sizeof(double), w, step * sizeof(double), sizeof(double), nsamp,
                                cudaMemcpyDeviceToHost, st), "d2h weight sample");
        check(cudaMemcpyAsync(f0.data(), d_flux0, sizeof(double) * n_stars, cudaMemcpyDeviceToHost, st), "d2h");
        check(cudaMemcpyAsync(h_act_order.data(), act, sizeof(int32_t) * n_act, cudaMemcpyDeviceToHost, st), "d2h");
        check(cudaStreamSynchronize(st), "sync");
        std::vector<double> fl(n_act);
        for (int64_t j = 0; j < n_act; ++j) fl[j] = f0[h_act_order[j]];
        model_radii_auto(psf, P->fixed_fwhm, P->model_rad_nsigma, fc.R, R_cap, wsamp, fl, h_modelR);
        model_R = *std::max_element(h_modelR.begin(), h_modelR.end());
        d_modelR = S<int32_t>(ctx, "model_R", n_act);
        check(cudaMemcpyAsync(d_modelR, h_modelR.data(), sizeof(int32_t) * n_act, cudaMemcpyHostToDevice, st),
              "h2d model radii");
        for (int32_t r : h_modelR) model_box_sum += (double)(2 * r + 1) * (2 * r + 1);
    } else {
        const int R_cap = (int)std::ceil(std::max(P->model_rad, P->fit_rad));
        model_R = std::min(std::max((int)std::ceil(P->model_rad), fc.R), R_cap);
        model_box_sum = (double)n_act * (2 * model_R + 1) * (2 * model_R + 1);
    }
    const double mean_box = model_box_sum / (double)n_act;  // per-star render work (instrumentation)
    const double dof = (double)std::max<int64_t>((int64_t)h_ucnt - n, 1);

    // ---- tile lists (fit box for J v; model box for renders)
    TileLists tfit = build_tiles(ctx, "tfit", n_act, ay, ax, nullptr, fc.R, ny, nx, fc.nty, fc.ntx);
    TileLists tmod = (model_R == fc.R && !d_modelR)
                         ? tfit
                         : build_tiles(ctx, "tmod", n_act, ay, ax, d_modelR, model_R, ny, nx, fc.nty, fc.ntx);

    // ---- working buffers (:1129-1166)
    TS* V = S<TS>(ctx, "V", (int64_t)fc.VS * n_act);
    double* cn = S<double>(ctx, "colnorm", n);
    double* D = S<double>(ctx, "D", n);
    double* bsc = S<double>(ctx, "b_scaled", n);
    double* delta = S<double>(ctx, "delta", n);
    double* dsc = S<double>(ctx, "delta_scaled", n);
    double* xl = S<double>(ctx, "lsqr_x", n);
    double* vt = S<double>(ctx, "lsqr_v", n);
    double* wl = S<double>(ctx, "lsqr_w", n);
    double* wt_resid = S<double>(ctx, "wt_resid", npix);
    double* u = S<double>(ctx, "lsqr_u", npix);
    StarCoef* coef = S<StarCoef>(ctx, "coef", n_act);
    StarCoef* coefc = S<StarCoef>(ctx, "coef_cand", n_act);
    uint8_t* live = S<uint8_t>(ctx, "live", n_act);
    uint8_t* newf = S<uint8_t>(ctx, "newf", n_act);
    uint8_t* conv = S<uint8_t>(ctx, "conv", n_act);
    int32_t* frozen_at = S<int32_t>(ctx, "frozen_at", n_act);
    int32_t* live_list = S<int32_t>(ctx, "live_list", n_act);
    int32_t* iota_act = S<int32_t>(ctx, "iota_act", n_act);
    int* d_nlive = S<int>(ctx, "nlive", 1);
    check(cudaMemsetAsync(live, 1, n_act, st), "memset");
    check(cudaMemsetAsync(conv, 0, n_act, st), "memset");
    check(cudaMemsetAsync(frozen_at, 0, sizeof(int32_t) * n_act, st), "memset");
    check(cudaMemsetAsync(cn, 0, sizeof(double) * n, st), "memset");
    check(cudaMemsetAsync(V, 0, sizeof(TS) * (int64_t)fc.VS * n_act, st), "memset");
    check(cudaMemcpyAsync(iota_act, iota, sizeof(int32_t) * n_act, cudaMemcpyDeviceToDevice, st), "d2d");
    int64_t n_live = n_act;
    check(cudaMemcpyAsync(live_list, iota, sizeof(int32_t) * n_act, cudaMemcpyDeviceToDevice, st), "d2d");
    size_t live_tmp_bytes = 0;
    cub::DeviceSelect::Flagged(nullptr, live_tmp_bytes, iota_act, live, live_list, d_nlive, (int)n_act, st);
    void* live_tmp = scratch(ctx, "live_tmp", live_tmp_bytes);

    const int fill_blocks = (int)std::min<int64_t>(n_act, (int64_t)ctx->n_sm * 16);
    // per-star model values of the render box: one block of MS per star, or with
    // per-star radii (:auto) each star's own (2 R_j + 1)^2 block at moff[j]
    const int Sm = 2 * model_R + 1;
    const int MS = ((Sm * Sm + 15) / 16) * 16;
    int64_t* d_moff = nullptr;
    int64_t mtotal = (int64_t)MS * n_act;
    if (d_modelR) {
        std::vector<int64_t> h_moff(n_act);
        mtotal = 0;
        for (int64_t j = 0; j < n_act; ++j) {
            h_moff[j] = mtotal;
            const int64_t sj = 2 * (int64_t)h_modelR[j] + 1;
            mtotal += (sj * sj + 15) / 16 * 16;
        }
        d_moff = S<int64_t>(ctx, "model_off", n_act);
        check(cudaMemcpyAsync(d_moff, h_moff.data(), sizeof(int64_t) * n_act, cudaMemcpyHostToDevice, st), "h2d");
    }
    TS* Mbuf = S<TS>(ctx, "model_stamps", mtotal);
    constexpr double bts = sizeof(TS);  // bytes per stored stamp / model value
    int32_t* evlist = S<int32_t>(ctx, "eval_list", n_act);
    const size_t tab_bytes = dp.kind == CPB_PSF_CIRCULAR_GAUSSIAN ? 0 : (size_t)(dp.n_nodes == 1 ? 2 : 8) * sizeof(AxisTab<TS>);
    bool m_fresh = false;  // Mbuf holds the current-theta model of the live stars (written by the fill)
    const bool warp_eval = dp.kind == CPB_PSF_CIRCULAR_GAUSSIAN || dp.n_nodes == 1;
    // model-value launches of the warp kernel: as many warps a block as their
    // row / column tables fit in shared memory (large :auto model boxes use fewer)
    int smem_optin = 0;
    check(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device), "attr");
    // warps per block of a k_eval_warp launch whose per-warp axis tables (2 Sx
    // entries) fit the opt-in shared memory
    auto warp_shape = [&](int Sx, size_t tab_size, unsigned& threads, size_t& smem) {
        int warps = 8;
        while (warps > 1 && (size_t)warps * 2 * Sx * tab_size > (size_t)smem_optin) warps /= 2;
        if ((size_t)warps * 2 * Sx * tab_size > (size_t)smem_optin)
            throw ArgError{"radius too large for the B200 stamp kernels"};
        threads = 32u * warps;
        smem = (size_t)warps * 2 * Sx * tab_size;
    };
    auto model_warp_shape = [&](size_t tab_size, unsigned& threads, size_t& smem) {
        warp_shape(Sm, tab_size, threads, smem);
    };
    auto eval_grid = [&](int64_t nlist) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>(nlist, (int64_t)ctx->n_sm * 16)); };
    auto launch_fill = [&](const int32_t* list, int64_t nlist, double* gram) {
        if (nlist <= 0) return;
        const bool writeM = !gram && model_R == fc.R && !d_modelR;
        KernelScope ks_(ctx, gram ? "k_eval_gram" : "k_eval_fill",
                        (double)nlist * ((gram ? 48.0 : (double)p * fc.S2 * bts + p * 8) + (writeM ? fc.S2 * bts : 0.0) +
                                         std::min<double>((double)fc.S2, (double)h_ucnt / std::max<int64_t>(n_act, 1)) * 16 +
                                         sizeof(StarCoef)));
        const size_t smem = tab_bytes * fc.S;
        TS* Mo = writeM ? Mbuf : nullptr;
        if (warp_eval) {
            unsigned thr;
            size_t sm_bytes;
            warp_shape(fc.S, sizeof(AxisTab<TS>), thr, sm_bytes);
            if (sm_bytes > 48 * 1024)
                check(cudaFuncSetAttribute(k_eval_warp<true, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)sm_bytes), "smem attr");
            const int wpb = (int)(thr / 32);
            const unsigned gbw = (unsigned)std::max<int64_t>(1, std::min<int64_t>((nlist + wpb - 1) / wpb, (int64_t)ctx->n_sm * 8));
            k_eval_warp<true, TS><<<gbw, thr, sm_bytes, st>>>(list, nlist, fc, dp, coef, ay, ax, w, sw, V, cn, gram, Mo, fc.R, MS, nullptr, nullptr);
        } else {
            launch_k_eval<true, TS>(fc.S2, eval_grid(nlist), smem, st, list, nlist, fc, dp, coef, ay, ax, w, sw, V, cn,
                                    gram, Mo, fc.R, MS, (const int32_t*)nullptr, (const int64_t*)nullptr);
        }
        check(cudaGetLastError(), "k_eval_fill");
        m_fresh = writeM;
    };
    (void)fill_blocks;
    // model values at `cf` for the stars of `list` into Mbuf (value-only stamp evaluation)
    auto launch_eval_model = [&](const int32_t* list, int64_t nlist, const StarCoef* cf) {
        if (nlist <= 0) return;
        KernelScope ks_(ctx, "k_eval_model", (double)nlist * ((double)Sm * Sm * bts + sizeof(StarCoef)));
        const size_t smem = tab_bytes * Sm;
        const unsigned gb = eval_grid(nlist);
        if (warp_eval) {
            unsigned thr;
            size_t sm_bytes;
            model_warp_shape(sizeof(AxisTab<TS>), thr, sm_bytes);
            if (sm_bytes > 48 * 1024)
                check(cudaFuncSetAttribute(k_eval_warp<false, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)sm_bytes), "smem attr");
            const int wpb = (int)(thr / 32);
            const unsigned gbw = (unsigned)std::max<int64_t>(1, std::min<int64_t>((nlist + wpb - 1) / wpb, (int64_t)ctx->n_sm * 8));
            k_eval_warp<false, TS><<<gbw, thr, sm_bytes, st>>>(list, nlist, fc, dp, cf, ay, ax, w, sw, V, cn, nullptr, Mbuf, model_R, MS, d_modelR, d_moff);
        } else {
            launch_k_eval<false, TS>((int64_t)Sm * Sm, gb, smem, st, list, nlist, fc, dp, cf, ay, ax, w, sw, V, cn,
                                     (double*)nullptr, Mbuf, model_R, MS, (const int32_t*)d_modelR,
                                     (const int64_t*)d_moff);
        }
        check(cudaGetLastError(), "k_eval_model");
    };
    auto launch_render = [&](int mode, const uint8_t* incl, const int32_t* list, int64_t nlist, const StarCoef* cf,
                             double* outp, const double* ref, double* result) {
        if (!(mode == MODE_CUR && m_fresh)) launch_eval_model(list, nlist, cf);
        m_fresh = false;
        const double px_bytes = mode == MODE_CUR ? 25.0 : (mode == MODE_CAND ? 17.0 : 16.0);
        KernelScope ks_(ctx, mode == MODE_CUR ? "k_gather_resid" : (mode == MODE_CAND ? "k_gather_cost" :
                                                   (mode == MODE_FREEZE ? "k_gather_freeze" : "k_gather_final")),
                        (double)npix * px_bytes + (double)nlist * Sm * Sm * bts);
        switch (mode) {
            case MODE_CUR:
                k_gather<KIND_M, MODE_CUR, TS><<<(unsigned)ntiles, NT, 0, st>>>(fc, tmod.start, tmod.end, tmod.list, tmod.order, incl, Mbuf, model_R, MS, d_moff, nullptr, nullptr, 0.0, outp, umask, w, sw, ref, sc, red, result);
                break;
            case MODE_CAND:
                k_gather<KIND_M, MODE_CAND, TS><<<(unsigned)ntiles, NT, 0, st>>>(fc, tmod.start, tmod.end, tmod.list, tmod.order, incl, Mbuf, model_R, MS, d_moff, nullptr, nullptr, 0.0, outp, umask, w, sw, ref, sc, red, result);
                break;
            case MODE_FREEZE:
                k_gather<KIND_M, MODE_FREEZE, TS><<<(unsigned)ntiles, NT, 0, st>>>(fc, tmod.start, tmod.end, tmod.list, tmod.order, incl, Mbuf, model_R, MS, d_moff, nullptr, nullptr, 0.0, outp, umask, w, sw, ref, sc, red, result);
                break;
            default:
                k_gather<KIND_M, MODE_FINAL, TS><<<(unsigned)ntiles, NT, 0, st>>>(fc, tmod.start, tmod.end, tmod.list, tmod.order, incl, Mbuf, model_R, MS, d_moff, nullptr, nullptr, 0.0, outp, umask, w, sw, ref, sc, red, result);
        }
        check(cudaGetLastError(), "k_gather");
    };
    auto update_live_list = [&]() {
        cub::DeviceSelect::Flagged(live_tmp, live_tmp_bytes, iota_act, live, live_list, d_nlive, (int)n_act, st);
        int h = 0;
        check(cudaMemcpyAsync(&h, d_nlive, sizeof(int), cudaMemcpyDeviceToHost, st), "d2h");
        check(cudaStreamSynchronize(st), "sync");
        n_live = h;
    };
    const unsigned jt_blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n_act + 7) / 8, (int64_t)ctx->n_sm * 8));
    auto read_scalars = [&]() {
        check(cudaMemcpyAsync(h_sc, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st), "d2h");
        check(cudaStreamSynchronize(st), "sync");
    };
    double evals = 0.0, macs = 0.0;

    // ---- initial fill and cost (:1171-1178)
    KernelScope(ctx, "k_coef", (double)n_act * (sizeof(StarCoef) + 3 * 8)), k_coef<<<nblk(n_act), 256, 0, st>>>(n_act, fc, dp, theta, nullptr, coef);
    launch_fill(live_list, n_live, nullptr);
    launch_render(MODE_CUR, live, live_list, n_live, coef, wt_resid, data_work, &sc->cost);
    check(cudaMemcpyAsync(D, cn, sizeof(double) * n, cudaMemcpyDeviceToDevice, st), "d2d");
    evals += (double)n_live * (fc.S2 + mean_box);
    bool fresh = true;  // V / wt_resid / cost are at the current theta and live set
    double lam = P->lambda_init;
    int n_run = 0;
    int64_t n_trials = 0, n_lsqr = 0;

    // ---- outer loop (:1186-1284)
    for (int iter = 1; iter <= P->max_iter; ++iter) {
        if (!fresh) {
            KernelScope(ctx, "k_coef", (double)n_act * (sizeof(StarCoef) + 3 * 8)), k_coef<<<nblk(n_act), 256, 0, st>>>(n_act, fc, dp, theta, nullptr, coef);
            launch_fill(live_list, n_live, nullptr);
            launch_render(MODE_CUR, live, live_list, n_live, coef, wt_resid, data_work, &sc->cost);
            evals += (double)n_live * (fc.S2 + mean_box);
        }
        fresh = false;
        // b_scaled = J' wt_resid (frozen stars stay 0)
        check(cudaMemsetAsync(bsc, 0, sizeof(double) * n, st), "memset");
        {
            KernelScope ks_(ctx, "k_JT", (double)n_live * ((double)p * fc.S2 * bts + 2.0 * p * 8) + std::min<double>((double)h_ucnt, (double)n_live * fc.S2) * 8);
            k_JT<false, TS><<<jt_blocks, 256, 0, st>>>(live_list, n_live, fc, ay, ax, V, wt_resid, bsc, sc, red);
        }
        check(cudaGetLastError(), "k_JT");
        macs += (double)n_live * fc.S2;
        {
            KernelScope ks_(ctx, "k_gnorm", (double)n * 8 * 2);
            k_gnorm<<<nblk(n), 256, 0, st>>>(n, cn, bsc, dof, sc, red);
        }
        check(cudaGetLastError(), "k_gnorm");
        read_scalars();
        const double cost = h_sc->cost;
        if (h_sc->gnorm <= P->g_tol) {
            k_freeze_all<<<nblk(n_act), 256, 0, st>>>(n_act, iter - 1, live, frozen_at, conv);
            n_run = iter - 1;
            break;
        }
        bool accepted = false, f_conv = false;
        for (int trial = 1; trial <= P->max_trials; ++trial) {
            ++n_trials;
            // LSQR init (Krylov lsqr: beta1 u1 = b, alpha1 v1 = A'u1)
            Scalars init{};
            init.cost = cost;
            init.beta1 = std::sqrt(cost);
            init.beta = init.beta1;
            init.inv_beta = init.beta1 != 0 ? 1.0 / init.beta1 : 0.0;
            init.lambda = std::sqrt(lam);
            init.atol = P->linear_tol;
            init.btol = P->linear_tol;
            init.itmax = P->inner_iterations;
            init.c2 = -1.0;
            init.stopped = init.beta1 == 0 ? 1 : 0;
            init.status = init.beta1 == 0 ? 4 : 0;
            *h_sc = init;
            check(cudaMemcpyAsync(sc, h_sc, sizeof(Scalars), cudaMemcpyHostToDevice, st), "h2d");
            if (init.beta1 == 0) {
                check(cudaMemsetAsync(xl, 0, sizeof(double) * n, st), "memset");
            } else {
                {
                    KernelScope ks_(ctx, "k_lsqr_v0", (double)n * 8 * 3);
                    k_lsqr_v0<<<nblk(n), 256, 0, st>>>(n, bsc, vt, xl, sc, red);
                }
                {
                    KernelScope ks_(ctx, "k_lsqr_w0", (double)n * 8 * 2);
                    k_lsqr_w0<<<nblk(n), 256, 0, st>>>(n, vt, wl, sc, red);
                }
                for (int it = 0; it < P->inner_iterations; ++it) {
                    {
                        KernelScope ks_(ctx, "k_gather_Jv", (double)n_live * ((double)p * fc.S2 * bts + p * 8) + 2.0 * npix * 8);
                        k_gather<KIND_JV, MODE_LSQR, TS><<<(unsigned)ntiles, NT, 0, st>>>(fc, tfit.start, tfit.end, tfit.list, tfit.order, live, V, fc.R, fc.VS, nullptr, vt, it == 0 ? wt_resid : u, it == 0 ? -1.0 : 1.0, u, umask, w, sw, nullptr, sc, red, nullptr);
                    }
                    {
                        KernelScope ks_(ctx, "k_JT_lsqr", (double)n_live * ((double)p * fc.S2 * bts + 2.0 * p * 8) + std::min<double>((double)h_ucnt, (double)n_live * fc.S2) * 8);
                        k_JT<true, TS><<<jt_blocks, 256, 0, st>>>(live_list, n_live, fc, ay, ax, V, u, vt, sc, red);
                    }
                    {
                        KernelScope ks_(ctx, "k_lsqr_update", (double)n * 8 * 5);
                        k_lsqr_update<<<nblk(n), 256, 0, st>>>(n, vt, xl, wl, sc, red);
                    }
                }
                check(cudaGetLastError(), "lsqr");
            }
            {
                KernelScope ks_(ctx, "k_step", (double)n * 8 * 4);
                k_step<<<nblk(n_act), 256, 0, st>>>(n_act, fc, P->max_step, xl, cn, delta, dsc);
            }
            KernelScope(ctx, "k_coef", (double)n_act * (sizeof(StarCoef) + 3 * 8)), k_coef<<<nblk(n_act), 256, 0, st>>>(n_act, fc, dp, theta, delta, coefc);
            launch_render(MODE_CAND, live, live_list, n_live, coefc, nullptr, data_work, &sc->cost_cand);
            evals += (double)n_live * mean_box;
            read_scalars();
            n_lsqr += h_sc->iter;
            macs += 2.0 * h_sc->iter * n_live * fc.S2;
            const double cost_cand = h_sc->cost_cand;
            const double dcost = cost - cost_cand;
            f_conv = (cost_cand < cost) && (dcost / cost <= P->f_tol);
            if (cost_cand < cost) {
                accepted = true;
                lam = std::max(lam / P->lambda_down, P->lambda_min);
                // cost := cost_cand is re-derived by the next residual pass
                Scalars s2 = *h_sc;
                s2.cost = cost_cand;
                s2.n_new_frozen = 0;
                *h_sc = s2;
                check(cudaMemcpyAsync(sc, h_sc, sizeof(Scalars), cudaMemcpyHostToDevice, st), "h2d");
                // C_r of the freeze test uses the cost at the start of this iteration
                Scalars* scf = S<Scalars>(ctx, "scalars_freeze", 1);
                Scalars s3 = s2;
                s3.cost = cost;
                check(cudaMemcpyAsync(scf, &s3, sizeof(Scalars), cudaMemcpyHostToDevice, st), "h2d");
                {
                    KernelScope ks_(ctx, "k_accept_freeze", (double)n * 8 * 7);
                    k_accept_freeze<<<nblk(n_act), 256, 0, st>>>(n_act, fc, P->x_tol, P->g_tol, dof, iter, theta, delta,
                                                            dsc, cn, D, bsc, live, newf, frozen_at, conv, scf);
                }
                check(cudaGetLastError(), "k_accept_freeze");
                int h_new = 0;
                check(cudaMemcpyAsync(&h_new, &scf->n_new_frozen, sizeof(int), cudaMemcpyDeviceToHost, st), "d2h");
                check(cudaStreamSynchronize(st), "sync");
                if (f_conv) {
                    // f_tol freezes everything without subtraction (:1259-1264); the
                    // per-star tests above are not part of that path, undo nothing:
                    // stars they froze are frozen at `iter` either way.
                    h_new = 0;
                }
                if (h_new > 0) {
                    KernelScope(ctx, "k_coef", (double)n_act * (sizeof(StarCoef) + 3 * 8)), k_coef<<<nblk(n_act), 256, 0, st>>>(n_act, fc, dp, theta, nullptr, coef);
                    {
                        size_t tb = 0;
                        cub::DeviceSelect::Flagged(nullptr, tb, iota_act, newf, evlist, d_nlive, (int)n_act, st);
                        void* tmpb = scratch(ctx, "newf_tmp", tb);
                        cub::DeviceSelect::Flagged(tmpb, tb, iota_act, newf, evlist, d_nlive, (int)n_act, st);
                    }
                    launch_render(MODE_FREEZE, newf, evlist, h_new, coef, data_work, nullptr, nullptr);
                    evals += (double)h_new * mean_box;
                    update_live_list();
                }
                break;
            } else {
                lam = std::min(lam * P->lambda_up, P->lambda_max);
            }
        }
        n_run = iter;
        if (f_conv) {
            k_freeze_all<<<nblk(n_act), 256, 0, st>>>(n_act, iter, live, frozen_at, conv);
            break;
        }
        if (accepted && n_live == 0) break;
    }

    // ---- errors at the final theta, every active star (:1302-1329)
    KernelScope(ctx, "k_coef", (double)n_act * (sizeof(StarCoef) + 3 * 8)), k_coef<<<nblk(n_act), 256, 0, st>>>(n_act, fc, dp, theta, nullptr, coef);
    double* gram = S<double>(ctx, "gram", (int64_t)n_act * 6);
    // the final pass (errors, residual, diagnostics) is FP64 for either precision form
    {
        KernelScope ks_(ctx, "k_eval_gram", (double)n_act * (48.0 + sizeof(StarCoef)));
        if (warp_eval) {
            unsigned thr;
            size_t sm_bytes;
            warp_shape(fc.S, sizeof(AxisTab<double>), thr, sm_bytes);
            if (sm_bytes > 48 * 1024)
                check(cudaFuncSetAttribute(k_eval_warp<true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)sm_bytes), "smem attr");
            const int wpb = (int)(thr / 32);
            const unsigned gbw = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n_act + wpb - 1) / wpb, (int64_t)ctx->n_sm * 8));
            k_eval_warp<true, double><<<gbw, thr, sm_bytes, st>>>(
                nullptr, n_act, fc, dp, coef, ay, ax, w, sw, nullptr, cn, gram, nullptr, fc.R, MS, nullptr, nullptr);
        } else {
            launch_k_eval<true, double>(fc.S2, eval_grid(n_act), (size_t)(dp.n_nodes == 1 ? 2 : 8) * sizeof(AxisTab<double>) * fc.S,
                                        st, (const int32_t*)nullptr, n_act, fc, dp, coef, ay, ax, w, sw, (double*)nullptr,
                                        cn, gram, (double*)nullptr, fc.R, MS, (const int32_t*)nullptr,
                                        (const int64_t*)nullptr);
        }
        check(cudaGetLastError(), "k_eval_gram");
    }
    double* err = S<double>(ctx, "err", n);
    read_scalars();  // final cost
    k_errors<<<nblk(n_act), 256, 0, st>>>(n_act, p, gram, reweighted, dof, sc, err);
    check(cudaGetLastError(), "k_errors");
    // ---- final render against the original data (:1344-1356) and diagnostics
    double* resid = S<double>(ctx, "resid", npix);
    {
        double* M64 = std::is_same<TS, double>::value ? (double*)Mbuf : S<double>(ctx, "model_stamps64", mtotal);
        {
            KernelScope ks_(ctx, "k_eval_model", (double)n_act * ((double)Sm * Sm * 8 + sizeof(StarCoef)));
            if (warp_eval) {
                unsigned thr;
                size_t sm_bytes;
                model_warp_shape(sizeof(AxisTab<double>), thr, sm_bytes);
                if (sm_bytes > 48 * 1024)
                    check(cudaFuncSetAttribute(k_eval_warp<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)sm_bytes), "smem attr");
                const int wpb = (int)(thr / 32);
                const unsigned gbw = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n_act + wpb - 1) / wpb, (int64_t)ctx->n_sm * 8));
                k_eval_warp<false, double><<<gbw, thr, sm_bytes, st>>>(
                    nullptr, n_act, fc, dp, coef, ay, ax, w, sw, nullptr, cn, nullptr, M64, model_R, MS, d_modelR, d_moff);
            } else {
                const size_t sm_ = (size_t)(dp.n_nodes == 1 ? 2 : 8) * sizeof(AxisTab<double>) * Sm;
                launch_k_eval<false, double>((int64_t)Sm * Sm, eval_grid(n_act), sm_, st, (const int32_t*)nullptr, n_act,
                                             fc, dp, coef, ay, ax, w, sw, (double*)nullptr, cn, (double*)nullptr, M64,
                                             model_R, MS, (const int32_t*)d_modelR, (const int64_t*)d_moff);
            }
            check(cudaGetLastError(), "k_eval_model");
        }
        KernelScope ks_(ctx, "k_gather_final", (double)npix * 16.0 + (double)n_act * Sm * Sm * 8);
        k_gather<KIND_M, MODE_FINAL, double><<<(unsigned)ntiles, NT, 0, st>>>(fc, tmod.start, tmod.end, tmod.list, tmod.order, nullptr, M64, model_R, MS, d_moff, nullptr, nullptr, 0.0, resid, umask, w, sw, data, sc, red, nullptr);
        check(cudaGetLastError(), "k_gather_final");
    }
    // spread_model reference disk, on the device: its width comes from the first
    // catalogue star's final parameters (k_spread_disk)
    const int kh = (int)std::ceil(P->fit_rad);
    const int boxmax = (2 * kh + 2) * (2 * kh + 2);
    const double sp_param = P->spread_model_fwhm;
    int smode = 0;
    double* d_stab = nullptr;
    if (n_stars > 0 && (std::isnan(sp_param) || (std::isfinite(sp_param) && sp_param > 0)) &&
        (smode = spread_mode(boxmax, kh)) != 0) {
        double h_rule[kSpreadRuleLen];
        spread_rule(h_rule);
        double* d_rule = S<double>(ctx, "spread_rule", kSpreadRuleLen);
        d_stab = S<double>(ctx, "spread_tab", spread_tab_len(kh));
        check(cudaMemcpyAsync(d_rule, h_rule, sizeof(h_rule), cudaMemcpyHostToDevice, st), "h2d");
        int ky = -1, kx = -1;
        for (int k = 0; k < p; ++k) {
            if (fc.gc[k] == 1) ky = k;
            if (fc.gc[k] == 2) kx = k;
        }
        DevPsf ps = dp;
        ps.fwhm = psf->dev.fwhm;  // _spread_fwhm renders the PSF object's own width
        KernelScope ks_(ctx, "k_spread_disk", 0.0);
        k_spread_disk<<<1, 256, sizeof(double) * (7 + kh) * kSpreadGL, st>>>(
            ps, sp_param, kh, theta, act, n_act, p, ky, kx, P->fixed_y, P->fixed_x, d_y0, d_x0, d_rule, d_stab);
        check(cudaGetLastError(), "k_spread_disk");
    }
    const size_t diag_smem = spread_smem_bytes(smode, boxmax, kh);
    const unsigned dgrid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(n_act, (int64_t)ctx->n_sm * 16));
    double* diag = S<double>(ctx, "diag", (int64_t)n_act * 7);
    {
        KernelScope ks_(ctx, "k_diag",
                        (double)n_act * boxmax * (8.0 + (d_inv_var ? 2.0 : 1.0) * (eltype == CPB_F64 ? 8 : 4)));
        if (eltype == CPB_F64) {
            if (diag_smem > 48 * 1024)
                check(cudaFuncSetAttribute(k_diag<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)diag_smem),
                      "smem attr");
            k_diag<double><<<dgrid, kDiagThreads, diag_smem, st>>>(n_act, fc, dp, P->fit_rad, coef, resid,
                                                               (const double*)d_image, (const double*)d_background,
                                                               (const double*)d_inv_var, d_stab, kh, smode, boxmax, diag);
        } else {
            if (diag_smem > 48 * 1024)
                check(cudaFuncSetAttribute(k_diag<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)diag_smem),
                      "smem attr");
            k_diag<float><<<dgrid, kDiagThreads, diag_smem, st>>>(n_act, fc, dp, P->fit_rad, coef, resid,
                                                              (const float*)d_image, (const float*)d_background,
                                                              (const float*)d_inv_var, d_stab, kh, smode, boxmax, diag);
        }
        check(cudaGetLastError(), "k_diag");
    }
    check(cudaEventRecord(ctx->ev1, st), "event");

    // ---- download and assemble (:1289-1300, :1331-1337, :1404-1430)
    std::vector<double> h_theta(n), h_err(n), h_diag(n_act * 7);
    std::vector<int32_t> h_act(n_act), h_frozen(n_act);
    std::vector<uint8_t> h_live(n_act), h_conv(n_act);
    std::vector<double> y0(n_stars), x0(n_stars), f0(n_stars);
    check(cudaMemcpyAsync(h_theta.data(), theta, sizeof(double) * n, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(h_err.data(), err, sizeof(double) * n, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(h_diag.data(), diag, sizeof(double) * n_act * 7, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(h_act.data(), act, sizeof(int32_t) * n_act, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(h_frozen.data(), frozen_at, sizeof(int32_t) * n_act, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(h_live.data(), live, n_act, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(h_conv.data(), conv, n_act, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(y0.data(), d_y0, sizeof(double) * n_stars, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(x0.data(), d_x0, sizeof(double) * n_stars, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(f0.data(), d_flux0, sizeof(double) * n_stars, cudaMemcpyDeviceToHost, st), "d2h");
    if (out->residual)
        check(cudaMemcpyAsync(out->residual, resid, sizeof(double) * npix, cudaMemcpyDeviceToHost, st), "d2h");
    if (out->dbg_pixels)
        check(cudaMemcpyAsync(out->dbg_pixels, dbg_pix, sizeof(int32_t) * fc.S2 * n_act, cudaMemcpyDeviceToHost, st),
              "d2h");
    check(cudaStreamSynchronize(st), "sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    out->device_seconds = ms * 1e-3;

    std::vector<double> oy(y0), ox(x0), of(f0);
    std::vector<double> ey(n_stars, NaN), ex(n_stars, NaN), ef(n_stars, NaN);
    std::vector<uint8_t> valid(n_stars, 0);
    for (int64_t j = 0; j < n_act; ++j) {
        int64_t i = h_act[j];
        valid[i] = 1;
        for (int k = 0; k < p; ++k) {
            double v = h_theta[j * p + k], e = h_err[j * p + k];
            if (fc.gc[k] == 1) {
                oy[i] = v;
                ey[i] = e;
            } else if (fc.gc[k] == 2) {
                ox[i] = v;
                ex[i] = e;
            } else {
                of[i] = v;
                ef[i] = e;
            }
        }
    }
    for (int64_t i = 0; i < n_stars; ++i) {
        if (!(P->free_mask & CPB_FREE_Y)) {
            oy[i] = P->fixed_y;
            ey[i] = 0.0;
        }
        if (!(P->free_mask & CPB_FREE_X)) {
            ox[i] = P->fixed_x;
            ex[i] = 0.0;
        }
        if (!(P->free_mask & CPB_FREE_FLUX)) {
            of[i] = P->fixed_flux;
            ef[i] = 0.0;
        }
        if (valid[i] && !(std::isfinite(oy[i]) && std::isfinite(ox[i]) && std::isfinite(of[i]) && of[i] > 0))
            valid[i] = 0;
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
        nan_diag(i);
    }
    for (int64_t j = 0; j < n_act; ++j) {
        int64_t i = h_act[j];
        out->converged[i] = h_conv[j];
        out->n_iter[i] = h_live[j] ? n_run : h_frozen[j];
        if (out->dbg_active) out->dbg_active[j] = h_act[j];
        if (out->dbg_model_R) out->dbg_model_R[j] = d_modelR ? h_modelR[j] : model_R;
        if (!valid[i]) continue;
        const double* dg = &h_diag[j * 7];
        if (out->spread_model) out->spread_model[i] = dg[5];
        if (out->spread_model_err) out->spread_model_err[i] = dg[6];
        if (out->chisq) out->chisq[i] = dg[0];
        if (out->qfit) out->qfit[i] = dg[1];
        if (out->qfit_expected) out->qfit_expected[i] = dg[2];
        if (out->qfit_z) out->qfit_z[i] = dg[3];
        if (out->crowding) out->crowding[i] = dg[4];
    }
    out->n_passes = n_run;
    out->n_failed = n_failed;
    out->n_trials = n_trials;
    out->n_lsqr_iters = n_lsqr;
    out->model_px_evals = evals;
    out->lsqr_px_macs = macs;
    return 0;
}

int fit_simultaneous_dev(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* P, const void* d_image,
                         int32_t eltype, int64_t ny, int64_t nx, const void* d_inv_var, const void* d_background,
                         int64_t n, const double* d_y0, const double* d_x0, const double* d_flux0,
                         cpb_sim_result* out) {
    if (P->precision == CPB_PREC_MIXED)
        return fit_sim_impl<float>(ctx, psf, P, d_image, eltype, ny, nx, d_inv_var, d_background, n, d_y0, d_x0,
                                   d_flux0, out);
    if (P->precision != CPB_PREC_FP64) throw ArgError{"precision must be CPB_PREC_FP64 or CPB_PREC_MIXED"};
    return fit_sim_impl<double>(ctx, psf, P, d_image, eltype, ny, nx, d_inv_var, d_background, n, d_y0, d_x0,
                                d_flux0, out);
}

}  // namespace cpb
