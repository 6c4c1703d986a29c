// cpb_sim.cu -- B200 simultaneous damped Gauss-Newton / LSQR PSF fit.
//
// Device restatement of CrowdPhot.fit_all_stars_simultaneous
// (src/photometry/psf_photometry_simultaneous.jl:953-1431).  Layout in HBM:
//   * per-pixel vectors (data, data_work, w, sqrt(w), union mask, residual,
//     LSQR u) are column-major npix arrays, as in the reference;
//   * stamp derivatives V (the unscaled weighted derivatives over each fit
//     box, StampDerivatives.values, :19-43, times colnorm) and the model
//     stamps are stored region-contiguously: the image is cut into 32 x 32
//     pixel regions, the part of a star's box inside one region is a dense
//     rectangle (p planes, one per free parameter, each column in 16-byte
//     granules aligned with image rows: gran_rows), and a region's rectangles
//     follow one another in its star-list order, so a region's stamps are one
//     contiguous run (RectMap);
//   * stamp pixel indices are not stored: they follow from the integer anchor
//     and the fit-box offset (the reference's `pixels` matrix is rebuilt only
//     for the bit-exact debug export);
//   * per-region star lists (stars in Morton order) turn the reference's
//     scatter-adds (apply_J!, _render_model!) into deterministic pixel
//     gathers with no atomics.
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

// Checked build (-DCPB_CHECKED): the stamp and pixel accesses of this file's
// kernels test their indexes against the buffers' lengths; a failed test skips
// the access and records its site (the first one) in g_check_err, which the
// host turns into an error return after the fit.  Normal builds test nothing.
#ifdef CPB_CHECKED
__device__ unsigned g_check_err;
#define CPB_CHECK(cond, site) ((cond) || (atomicCAS(&g_check_err, 0u, (unsigned)(site)), false))
#else
#define CPB_CHECK(cond, site) true
#endif

constexpr int TY = 32;   // region rows (y, contiguous in memory)
constexpr int TX = 32;   // region columns
constexpr int NT = 128;  // threads of the region kernels (4 warps)
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
    // LSMR state (solver = :lsmr; Fong & Saunders 2011 recurrences)
    double m_alphabar, m_rho, m_rhobar, m_cbar, m_sbar, m_zeta, m_zetabar;
    double m_betadd, m_betad, m_rhodold, m_tautildeold, m_thetatilde, m_d, m_maxrbar, m_minrbar;
    double lambda, atol, btol;
    int iter, itmax, stopped, status;
    int n_new_frozen;
};

// ---------------------------------------------------------------------------
// setup kernels
// ---------------------------------------------------------------------------
// data and weight sanitisation of one pixel (:1056-1084)
__device__ __forceinline__ void prepare_px(double d, bool have_iv, double v, double& dout, double& wout,
                                           unsigned& bad) {
    double wv = 1.0;
    if (have_iv) wv = (isfinite(v) && v > 0) ? v : 0.0;
    if (!isfinite(d)) {
        if (!have_iv) ++bad;
        d = 0.0;
        wv = 0.0;
    }
    dout = d;
    wout = wv;
}

// one 16-byte run of a user image (the caller checked its alignment)
__device__ __forceinline__ void ld_img16(const float* p, double (&o)[4]) {
    const float4 t = __ldg((const float4*)p);
    o[0] = t.x;
    o[1] = t.y;
    o[2] = t.z;
    o[3] = t.w;
}
__device__ __forceinline__ void ld_img16(const double* p, double (&o)[2]) {
    const double2 t = __ldg((const double2*)p);
    o[0] = t.x;
    o[1] = t.y;
}

// VEC: each thread takes one 16-byte run of every input (4 floats or 2 doubles)
// and writes its pixels' vectors with 16-byte stores; otherwise one pixel a thread.
template <typename TI, bool VEC>
__global__ void k_prepare(const TI* __restrict__ img, const TI* __restrict__ iv, const TI* __restrict__ bkg,
                          int64_t npix, double* data, double* data_work, double* w, double* sw,
                          unsigned* nonfinite) {
    constexpr int E = VEC ? 16 / (int)sizeof(TI) : 1;
    const int64_t q0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) * E;
    if (q0 >= npix) return;
    double d[E], v[E], b[E], dd[E], ww[E];
    unsigned bad = 0;
    if constexpr (VEC) {
        ld_img16(img + q0, d);
        if (iv) ld_img16(iv + q0, v);
        if (bkg) ld_img16(bkg + q0, b);
    } else {
        d[0] = (double)img[q0];
        if (iv) v[0] = (double)iv[q0];
        if (bkg) b[0] = (double)bkg[q0];
    }
#pragma unroll
    for (int e = 0; e < E; ++e) prepare_px(d[e] - (bkg ? b[e] : 0.0), iv != nullptr, iv ? v[e] : 0.0, dd[e], ww[e], bad);
#pragma unroll
    for (int e = 0; e < E; e += 2) {
        if constexpr (E == 1) {
            data[q0] = dd[0];
            data_work[q0] = dd[0];
            w[q0] = ww[0];
            sw[q0] = sqrt(ww[0]);
        } else {
            const double2 dv = make_double2(dd[e], dd[e + 1]), wv = make_double2(ww[e], ww[e + 1]);
            *(double2*)(data + q0 + e) = dv;
            *(double2*)(data_work + q0 + e) = dv;
            *(double2*)(w + q0 + e) = wv;
            *(double2*)(sw + q0 + e) = make_double2(sqrt(ww[e]), sqrt(ww[e + 1]));
        }
    }
    if (bad) atomicAdd(nonfinite, bad);
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

// A star's (region, star) pairs in emit order: regions column by column
// (tx0..tx1, then ty0..ty1 within), starting at offs[j]; vals carry the emit
// index through the sort so that every pair's star and every star's pairs can
// be found afterwards (emit_j, star_pairs).
__global__ void k_tile_emit(int64_t n_act, const int32_t* ay, const int32_t* ax, const int32_t* Rs, int Rconst,
                            int ny, int nx, int nty, const int32_t* offs, uint32_t* keys, int32_t* vals,
                            int32_t* emit_j) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n_act) return;
    int Rj = Rs ? Rs[j] : Rconst, ty0, ty1, tx0, tx1;
    if (!star_tiles(ay[j], ax[j], Rj, ny, nx, ty0, ty1, tx0, tx1)) return;
    int o = offs[j];
    for (int tx = tx0; tx <= tx1; ++tx)
        for (int ty = ty0; ty <= ty1; ++ty) {
            keys[o] = (uint32_t)(ty + tx * nty);
            vals[o] = o;
            emit_j[o] = (int32_t)j;
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

__global__ void k_tile_pack(int64_t npairs, const int32_t* sorted_o, const int32_t* emit_j, const int32_t* ay,
                            const int32_t* ax, const int32_t* Rs, int Rconst, int4* packed, int32_t* star_pairs) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= npairs) return;
    const int o = sorted_o[i];
    const int j = emit_j[o];
    packed[i] = make_int4(j, ay[j], ax[j], Rs ? Rs[j] : Rconst);  // .w: the star's box radius
    star_pairs[o] = (int32_t)i;
}


// ---------------------------------------------------------------------------
// per-iteration kernels
// ---------------------------------------------------------------------------
struct FitConst {
    int p;
    int gc[3];     // grad_col of free param k (1 = dy, 2 = dx, 3 = dflux)
    int ky, kx;    // index of y / x in the free list, -1 if fixed
    double fixed_y, fixed_x, fixed_flux, fixed_bkg;
    int R, S, S2;
    int q32, r32;  // 32 / S and 32 % S: advancing a stamp index by one warp
    int ny, nx;
    int nty, ntx;
};

// ---- stamp storage ("granule layout") ------------------------------------
// A star's box of Sb x Sb pixels is stored per plane (one plane per free
// parameter for the stamp derivatives, one for model values) as Sb columns of
// SR = gran_rows(Sb, GH) entries.  GH = 16 bytes / element size (4 floats or
// 2 doubles) is the granule height.  Box row r of column c lives at
// c * SR + o + r with o = top0 mod GH, top0 the box's first image row
// (0-based), so storage row 0 of every column sits on an image row that is a
// multiple of GH.  The pixel regions of the gathers start on rows that are
// multiples of 32, so every run of a column they need is made of whole
// 16-byte granules; entries outside the box stay zero.
template <typename T>
struct Gran {
    static constexpr int H = 16 / (int)sizeof(T);
};
__host__ __device__ __forceinline__ int gran_rows(int Sb, int gh) { return (Sb + 2 * gh - 2) / gh * gh; }
__device__ __forceinline__ int gran_base(int top0, int gh) { return top0 & ~(gh - 1); }  // floor to a multiple of gh

// one 16-byte granule; V / model stamps are streamed once per launch (evict first)
__device__ __forceinline__ void ld_gran(const float* p, float (&o)[4]) {
    const float4 t = __ldcs((const float4*)p);
    o[0] = t.x;
    o[1] = t.y;
    o[2] = t.z;
    o[3] = t.w;
}
__device__ __forceinline__ void ld_gran(const double* p, double (&o)[2]) {
    const double2 t = __ldcs((const double2*)p);
    o[0] = t.x;
    o[1] = t.y;
}
// one 16-byte run of a per-pixel vector (reused, read-only for the launch)
__device__ __forceinline__ void ld_px16(const float* p, float (&o)[4]) {
    const float4 t = __ldg((const float4*)p);
    o[0] = t.x;
    o[1] = t.y;
    o[2] = t.z;
    o[3] = t.w;
}
__device__ __forceinline__ void ld_px16(const double* p, double (&o)[2]) {
    const double2 t = __ldg((const double2*)p);
    o[0] = t.x;
    o[1] = t.y;
}

// ---- region-contiguous stamp storage ------------------------------------
// The stamps are stored per (region, star) pair in the order of the region
// lists: the pair's rectangle -- the star's granule-layout columns clipped to
// the region -- is dense (rectangle column c, storage row s at
// c * nrows + s, one plane after the other), and the rectangles of a region's
// stars follow one another, so a region's gather reads one contiguous run.
struct RectGeo {
    int c_lo, ncols;  // box columns held
    int s_lo, nrows;  // storage rows held (a multiple of GH)
};

// The part of the box of radius Rb anchored at (ay, ax) that region (ry, rx)
// holds, for granules of GH rows.
__host__ __device__ __forceinline__ RectGeo rect_geo(int ay, int ax, int Rb, int ry, int rx, int GH) {
    const int Sb = 2 * Rb + 1, left0 = ax - Rb - 1, top0 = ay - Rb - 1;
    const int b0 = top0 & ~(GH - 1), SRb = gran_rows(Sb, GH);
    const int C0 = rx * TX, R0 = ry * TY;
    RectGeo g;
    const int c0 = left0 > C0 ? left0 : C0, c1 = left0 + Sb - 1 < C0 + TX - 1 ? left0 + Sb - 1 : C0 + TX - 1;
    const int r_lo = b0 > R0 ? b0 : R0, r_hi = b0 + SRb < R0 + TY ? b0 + SRb : R0 + TY;
    g.c_lo = c0 - left0;
    g.ncols = c1 >= c0 ? c1 - c0 + 1 : 0;
    g.s_lo = r_lo - b0;
    g.nrows = r_hi > r_lo ? r_hi - r_lo : 0;
    return g;
}

// Where one list's stamps live: per star its pairs (soffs, star_pairs), per
// pair its rectangle's element offset (off), and the planes a rectangle holds.
struct RectMap {
    const int32_t* soffs;       // per star: its first emit index
    const int32_t* star_pairs;  // per emit index: the pair (list position)
    const int64_t* off;         // per pair: offset of the rectangle's plane 0
    const int64_t* srect;       // per star, when every box meets at most 2 x 2 regions: its
                                // rectangles' offsets in emit order (kStarRects a star), else null
    int64_t len;                // elements of the buffer (the checked build tests indexes against it)
    int planes;
};
constexpr int kStarRects = 4;

// srect of a list whose boxes meet at most 2 x 2 regions (box side <= TX + 1).
__global__ void k_star_rects(int64_t n_act, const int32_t* __restrict__ soffs, const int32_t* __restrict__ star_pairs,
                             const int64_t* __restrict__ off, int64_t* srect) {
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n_act * kStarRects) return;
    const int64_t j = t / kStarRects;
    const int l = (int)(t % kStarRects);
    const int o = soffs[j] + l;
    srect[t] = o < soffs[j + 1] ? off[star_pairs[o]] : -1;
}

// Element index of box entry (row, col) of star j in plane 0, or -1 when no
// region holds it (off the image); plane k is k * *pstride further on.
// ty0..tx1: the star's regions (star_tiles).
__device__ __forceinline__ int64_t rect_slot(const RectMap& m, int j, int ay, int ax, int Rb, int ty0, int ty1,
                                             int tx0, int tx1, int row, int col, int GH, int64_t* pstride) {
    const int y = ay - Rb - 1 + row, x = ax - Rb - 1 + col;
    if (y < 0 || x < 0) return -1;
    const int ry = y / TY, rx = x / TX;
    if (ry < ty0 || ry > ty1 || rx < tx0 || rx > tx1) return -1;
    const int i = m.star_pairs[m.soffs[j] + (rx - tx0) * (ty1 - ty0 + 1) + (ry - ty0)];
    const RectGeo g = rect_geo(ay, ax, Rb, ry, rx, GH);
    const int top0 = ay - Rb - 1, o = top0 - (top0 & ~(GH - 1));
    *pstride = (int64_t)g.ncols * g.nrows;
    return m.off[i] + (int64_t)(col - g.c_lo) * g.nrows + (o + row - g.s_lo);
}
__device__ __forceinline__ int64_t rect_index(const RectMap& m, int j, int ay, int ax, int Rb, int ty0, int ty1,
                                              int tx0, int tx1, int row, int col, int k, int GH) {
    int64_t ps = 0;
    const int64_t q = rect_slot(m, j, ay, ax, Rb, ty0, ty1, tx0, tx1, row, col, GH, &ps);
    return q < 0 ? q : q + k * ps;
}

// A star's rectangles as the stamp kernels store into them: geometry and the
// offsets in the stamp-derivative (V) and model (M) buffers.
struct StoreRect {
    int64_t offV, offM;
    int c_lo, s_lo, nrows, ps;  // ps = ncols * nrows: the plane stride of V
};
constexpr int kFillRects = 16;  // rectangles a stamp kernel tabulates per star (else rect_slot)

__device__ __forceinline__ int64_t star_rect_off(const RectMap& m, int j, int l) {
    return m.srect ? m.srect[(int64_t)j * kStarRects + l] : m.off[m.star_pairs[m.soffs[j] + l]];
}

// Threads t = first, first + step, ... < nrect tabulate rectangle t of star j
// (regions in emit order: column by column, nty_j regions a column).
__device__ __forceinline__ void store_rect_tab(StoreRect* tab, int first, int step, int nrect, int nty_j, int ty0,
                                               int tx0, int j, int a_y, int a_x, int Rb, int GH, const RectMap* vmap,
                                               const RectMap* mmap) {
    for (int l = first; l < nrect; l += step) {
        const RectGeo g = rect_geo(a_y, a_x, Rb, ty0 + l % nty_j, tx0 + l / nty_j, GH);
        StoreRect t;
        t.c_lo = g.c_lo;
        t.s_lo = g.s_lo;
        t.nrows = g.nrows;
        t.ps = g.ncols * g.nrows;
        t.offV = vmap ? star_rect_off(*vmap, j, l) : 0;
        t.offM = mmap ? star_rect_off(*mmap, j, l) : 0;
        tab[l] = t;
    }
}

// Index of box entry (row, col) inside its rectangle (plane 0), and the
// rectangle, or -1 when no region holds the entry.  o: storage row of box row 0.
__device__ __forceinline__ int tab_entry(int ty0, int ty1, int tx0, int tx1, int nty_j, int top0, int left0, int o,
                                         int row, int col, const StoreRect* tab, const StoreRect** rect) {
    const int y = top0 + row, x = left0 + col;
    if (y < 0 || x < 0) return -1;
    const int ry = y / TY, rx = x / TX;
    if (ry < ty0 || ry > ty1 || rx < tx0 || rx > tx1) return -1;
    const StoreRect& t = tab[(rx - tx0) * nty_j + (ry - ty0)];
    *rect = &t;
    return (col - t.c_lo) * t.nrows + (o + row - t.s_lo);
}

// The rectangles of a star whose box meets at most 2 x 2 regions, for the stamp
// kernels' storage-order walk: per rectangle (emit order) its offsets in the
// stamp-derivative (V) and model (M) buffers, first box column, first storage
// row, rows and entries (ncols * nrows, also V's plane stride).
struct StorePlan {
    int64_t offV[kStarRects], offM[kStarRects];
    int c_lo[kStarRects], s_lo[kStarRects], nrows[kStarRects], ps[kStarRects];
    float inv_nrows[kStarRects];
};

// Lanes 0 .. nrect - 1 of the warp fill their rectangle of the plan.
__device__ __forceinline__ void store_plan(StorePlan& sp, int lane, int nrect, int j, int a_y, int a_x, int Rb,
                                           int ty0, int ty1, int tx0, int GH, const RectMap* vmap,
                                           const RectMap* mmap) {
    const int nty_j = ty1 - ty0 + 1;
    if (lane < nrect) {
        const RectGeo g = rect_geo(a_y, a_x, Rb, ty0 + lane % nty_j, tx0 + lane / nty_j, GH);
        sp.offV[lane] = vmap ? star_rect_off(*vmap, j, lane) : 0;
        sp.offM[lane] = mmap ? star_rect_off(*mmap, j, lane) : 0;
        sp.c_lo[lane] = g.c_lo;
        sp.s_lo[lane] = g.s_lo;
        sp.nrows[lane] = g.nrows;
        sp.ps[lane] = g.ncols * g.nrows;
        sp.inv_nrows[lane] = 1.0f / (float)max(g.nrows, 1);
    }
}

// Elements of every pair's rectangle (all planes), for the offsets' prefix sum.
__global__ void k_rect_size(int64_t npairs, const int4* __restrict__ list, const uint32_t* __restrict__ region,
                            int nty, int GH, int planes, int64_t* size) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i > npairs) return;
    if (i == npairs) {
        size[i] = 0;
        return;
    }
    const int4 e = list[i];
    const int r = (int)region[i];
    const RectGeo g = rect_geo(e.y, e.z, e.w, r % nty, r / nty, GH);
    size[i] = (int64_t)planes * g.ncols * g.nrows;
}

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
//   sqrt(w) * gradient over the fit box, colnorm = max(||raw||, eps); V keeps
//   raw (the reference's values[:, m, a] = raw / colnorm; the J products
//   divide by colnorm per star); masked and off-image entries are exactly 0.
// GRAD with gram: the unscaled p x p Gram block sum(raw raw') of the error
//   estimate (:1305-1318), nothing else written.
// M != nullptr: the model value flux * s + bkg of every box pixel (the
//   per-star term of _render_model!, :545-577 / :605-673), box half-width Rb.
// Sums of squares and Gram entries accumulate in double for either T.
template <int NTF, int MAXE, bool GRAD, typename T>
__global__ void __launch_bounds__(NTF) k_eval(const int32_t* __restrict__ list, int64_t nlist, FitConst fc, DevPsf P,
                                              const StarCoef* __restrict__ coef, const int32_t* __restrict__ ay,
                                              const int32_t* __restrict__ ax, const double* __restrict__ w,
                                              const double* __restrict__ sw, T* __restrict__ V, RectMap vmap,
                                              double* __restrict__ colnorm, double* __restrict__ gram,
                                              T* __restrict__ M, RectMap mmap, int Rmax,
                                              const int32_t* __restrict__ Rs) {
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
        // the regions holding this star's box (stamp rectangles, rect_index)
        constexpr int GH = Gran<T>::H;
        int ty0 = 0, ty1 = -1, tx0 = 0, tx1 = -1;
        star_tiles(a_y, a_x, Rb, fc.ny, fc.nx, ty0, ty1, tx0, tx1);
        auto sidx = [&](const RectMap& m, int row, int col, int k) {
            return rect_index(m, j, a_y, a_x, Rb, ty0, ty1, tx0, tx1, row, col, k, GH);
        };
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
                if (M) {
                    const int64_t q = sidx(mmap, row, col, 0);
                    if (q >= 0 && CPB_CHECK(q < mmap.len, 0x11)) M[q] = val;
                }
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
                if (M) {
                    const int64_t q = sidx(mmap, row, col, 0);
                    if (q >= 0 && CPB_CHECK(q < mmap.len, 0x12)) M[q] = (T)c.flux * s + (T)c.bkg;
                }
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
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    double cn = sqrt(k < p ? cn_sh[k] : 1.0);
                    cn = cn < kEps64 ? kEps64 : cn;
                    if (threadIdx.x == 0 && k < p) colnorm[(int64_t)j * p + k] = cn;
                }
#pragma unroll
                for (int e = 0; e < RE; ++e) {
                    const int m = threadIdx.x + e * NTF;
                    if (m >= S2b) continue;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        if (k >= p) break;
                        const int64_t at = sidx(vmap, m % Sb, m / Sb, k);  // the fit box: Sb == fc.S
                        if (at >= 0 && CPB_CHECK(at < vmap.len, 0x13)) V[at] = raw[e][k];
                    }
                }
            }
        }
        __syncthreads();
    }
}

// Warp-per-star stamp evaluation for single-node ePSFs and the Gaussian (the
// common case): no block barriers, each warp keeps its star's row / column
// tables in its own slice of shared memory.  Same outputs as k_eval.
// PLAN: every box meets at most 2 x 2 regions and every map written has
// per-star rectangle offsets (srect), so only the storage-order walk is
// compiled (the general paths' registers would otherwise spill in it).
// GRAM: the Gram blocks (gram non-null) rather than the stamps.  Four blocks
// an SM for FP32 stamps, three for FP64 (four measured slower there: the FP64
// taps' registers spill).
template <bool GRAD, typename T, bool PLAN, bool GRAM>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 3) k_eval_warp(const int32_t* __restrict__ list, int64_t nlist, FitConst fc,
                                                      DevPsf P, const StarCoef* __restrict__ coef,
                                                      const int32_t* __restrict__ ay, const int32_t* __restrict__ ax,
                                                      const double* __restrict__ w, const double* __restrict__ sw,
                                                      T* __restrict__ V, RectMap vmap, double* __restrict__ colnorm,
                                                      double* __restrict__ gram, T* __restrict__ M, RectMap mmap,
                                                      int Rmax, const int32_t* __restrict__ Rs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if constexpr (!GRAM) gram = nullptr;  // the stamp instantiations carry no Gram code
    __shared__ StoreRect rtabs[256 / 32][kFillRects];
    __shared__ StorePlan plans[256 / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    StoreRect* rtab = rtabs[wid];
    StorePlan& plan = plans[wid];
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
        // the regions holding this star's box: its stamp rectangles, tabulated
        // when there are at most kFillRects (else rect_slot per entry)
        constexpr int GH = Gran<T>::H;
        int ty0 = 0, ty1 = -1, tx0 = 0, tx1 = -1;
        const int a_y = ay[j], a_x = ax[j];
        star_tiles(a_y, a_x, Rb, fc.ny, fc.nx, ty0, ty1, tx0, tx1);
        const int nty_j = ty1 - ty0 + 1, nrect = nty_j * (tx1 - tx0 + 1);
        const bool wantV = GRAD && !gram, wantM = M != nullptr && !gram;
        // a plan when every map has per-star rectangle offsets (boxes within 2 x 2 regions)
        const bool planned = PLAN || (nrect <= kStarRects && (!wantV || vmap.srect) && (!wantM || mmap.srect));
        const bool tabbed = !PLAN && !planned && nrect <= kFillRects;
        if (planned)
            store_plan(plan, lane, nrect, j, a_y, a_x, Rb, ty0, ty1, tx0, GH, wantV ? &vmap : nullptr,
                       wantM ? &mmap : nullptr);
        else if (tabbed)
            store_rect_tab(rtab, lane, 32, nrect, nty_j, ty0, tx0, j, a_y, a_x, Rb, GH, wantV ? &vmap : nullptr,
                           wantM ? &mmap : nullptr);
        __syncwarp();
        const int top0 = a_y - Rb - 1, left0 = a_x - Rb - 1, so = top0 - gran_base(top0, GH);
        // element index of entry (row, col) in plane 0 of V (isV) or M, and V's plane stride
        auto store_at = [&](int row, int col, bool isV, int64_t* ps) -> int64_t {
            if (tabbed) {
                const StoreRect* t = nullptr;
                const int e = tab_entry(ty0, ty1, tx0, tx1, nty_j, top0, left0, so, row, col, rtab, &t);
                if (e < 0) return -1;
                *ps = t->ps;
                return (isV ? t->offV : t->offM) + e;
            }
            return rect_slot(isV ? vmap : mmap, j, a_y, a_x, Rb, ty0, ty1, tx0, tx1, row, col, GH, ps);
        };
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
        if (planned) {
            // storage order: the star's rectangles one after another, each column
            // by column, so the stores of a warp are consecutive; pad rows skipped
            double acc[6] = {0, 0, 0, 0, 0, 0};
            int l = 0, t = lane;
            while (l < nrect && t >= plan.ps[l]) t -= plan.ps[l++];
            while (l < nrect) {
                const int cc = (int)(((float)t + 0.5f) * plan.inv_nrows[l]);
                const int row = plan.s_lo[l] + (t - cc * plan.nrows[l]) - so, col = plan.c_lo[l] + cc;
                if (row >= 0 && row < Sb) {
                    if (!GRAD) {
                        T val, a, b, c;
                        eval_px(row, col, val, a, b, c);
                        if (CPB_CHECK(plan.offM[l] + t < mmap.len, 0x21)) M[plan.offM[l] + t] = val;
                    } else {
                        const int gy = oy + row, gx = ox + col;
                        const bool onimg = gy >= 1 && gy <= fc.ny && gx >= 1 && gx <= fc.nx;
                        const int64_t q = onimg ? (gy - 1) + (int64_t)(gx - 1) * fc.ny : 0;
                        // the weights load beside the evaluation (no branch on them before it)
                        const double wq = onimg ? w[q] : 0.0, swq = onimg ? sw[q] : 0.0;
                        const bool use = onimg && wq > 0;
                        T r0 = 0, r1 = 0, r2 = 0;
                        if (onimg || wantM) {
                            T val, a, b, c;
                            eval_px(row, col, val, a, b, c);
                            if (wantM && CPB_CHECK(plan.offM[l] + t < mmap.len, 0x22)) M[plan.offM[l] + t] = val;
                            if (use) {
                                const T sq = (T)swq;
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
                        if (wantV && onimg && CPB_CHECK(plan.offV[l] + t + (int64_t)(p - 1) * plan.ps[l] < vmap.len, 0x23)) {
                            T* v = V + plan.offV[l] + t;
                            v[0] = r0;
                            if (p > 1) v[plan.ps[l]] = r1;
                            if (p > 2) v[2 * plan.ps[l]] = r2;
                        }
                    }
                }
                t += 32;
                while (l < nrect && t >= plan.ps[l]) t -= plan.ps[l++];
            }
            if (GRAD) {
#pragma unroll
                for (int k = 0; k < 6; ++k) acc[k] = warp_sum(acc[k]);
                if (gram) {
                    if (lane == 0) {
                        double* gj = gram + (int64_t)j * 6;
                        if (p == 1) gj[0] = acc[0];
                        else if (p == 2) {
                            gj[0] = acc[0];
                            gj[1] = acc[1];
                            gj[2] = acc[3];
                        } else {
                            for (int k = 0; k < 6; ++k) gj[k] = acc[k];
                        }
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        double cn = sqrt(k < p ? acc[k] : 1.0);
                        cn = cn < kEps64 ? kEps64 : cn;
                        if (lane == 0 && k < p) colnorm[(int64_t)j * p + k] = cn;
                    }
                }
            }
        } else if constexpr (PLAN) {
        } else if (!GRAD) {
            int row = lane % Sb, col = lane / Sb;
            for (int m = lane; m < S2b; m += 32) {
                T val, a, b, c;
                eval_px(row, col, val, a, b, c);
                int64_t ps;
                const int64_t q = store_at(row, col, false, &ps);
                if (q >= 0 && CPB_CHECK(q < mmap.len, 0x24)) M[q] = val;
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
                    if (M && !gram) {
                        int64_t ps;
                        const int64_t q = store_at(row, col, false, &ps);
                        if (q >= 0 && CPB_CHECK(q < mmap.len, 0x25)) M[q] = val;
                    }
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
                if (!gram && onimg) {  // the fit box; off-image entries are not stored
                    int64_t ps;
                    const int64_t q = store_at(row, col, true, &ps);
                    if (q >= 0 && CPB_CHECK(q + (p - 1) * ps < vmap.len, 0x26)) {
                        V[q] = r0;
                        if (p > 1) V[q + ps] = r1;
                        if (p > 2) V[q + 2 * ps] = r2;
                    }
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
                // the stamp keeps the unscaled derivatives; the J products divide by colnorm
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    double cn = sqrt(k < p ? acc[k] : 1.0);
                    cn = cn < kEps64 ? kEps64 : cn;
                    if (lane == 0 && k < p) colnorm[(int64_t)j * p + k] = cn;
                }
            }
        }
        __syncwarp();
    }
}

// Per-region pixel gather over the region's star list (stars in Morton
// order), the deterministic replacement of the reference's scatter-adds.
// A block owns a TY x TX pixel region; warp w takes the region's stars
// w, w + NW, w + 2 NW, ... in list order and adds them into its own copy of
// the region in shared memory.  A star's part of the region is a dense
// rectangle of stamp granules (GH rows of one stamp column, GH = 16 bytes /
// element) stored at the pair's offset (roff), the rectangles of a region's
// stars one after another: the region's stamps are one contiguous run, read
// in whole 16-byte granules.  The warp walks its stars' granules in
// 32-granule slots (one star a slot, a star's last slot padded) and loads
// KSLOT slots -- KSLOT * p granules a lane -- before adding any, slot by slot.
// Each pixel is the sum of the warps' copies in warp order: a fixed order
// (no atomics, bitwise reproducible).
//   KIND_JV: sum_k V[j, k, m] * v[j, k] / (alpha colnorm[j, k])  (apply_J!,
//            :95-137; V holds the unscaled weighted derivatives)
//   KIND_M : sum M[j, m]                                          (_render_model!)
// Epilogues (MODE): LSQR u update + beta (Krylov lsqr step 1); weighted
// residual + cost (_residual_cost!, :675-684); candidate cost (_cost!,
// :686-693); freeze subtraction (_freeze_star!, :739-754); final residual.
// TU: element type of the LSQR pixel vectors (u, weighted residual); all
// sums are FP64.
constexpr int KIND_JV = 0, KIND_M = 1;
constexpr int MODE_LSQR = 4;
// slots a warp loads per round before adding (J v: 12 granules a lane in flight;
// the one-plane model renders measured slower with 12 slots than with 4)
constexpr int KSLOT = 4;
// the warps' FP64 region copies (sums are FP64 for either stamp type: FP32
// sums of the mixed-precision form moved its fit measurably, FP32 storage did not)
constexpr size_t kGatherSmem = (size_t)(NT / 32) * TX * TY * sizeof(double);

template <int KIND, int MODE, typename TS, typename TU>
__global__ void __launch_bounds__(NT) k_gather(FitConst fc, const int32_t* __restrict__ tstart,
                                               const int32_t* __restrict__ tend, const int4* __restrict__ tlist,
                                               const int32_t* __restrict__ tord,
                                               const uint8_t* __restrict__ incl, const TS* __restrict__ src,
                                               int Rbox, const int64_t* __restrict__ roff, int64_t src_len,
                                               const double* __restrict__ vt, const double* __restrict__ cn,
                                               const TU* u_src, double u_sign,
                                               TU* outu, double* outd, const uint8_t* __restrict__ umask,
                                               const double* __restrict__ w, const double* __restrict__ sw,
                                               const double* __restrict__ data_ref, Scalars* sc, Reducer red,
                                               double* result) {
    constexpr int GH = Gran<TS>::H;      // rows of a granule
    constexpr int NGR = TY / GH;         // granule rows of the region
    constexpr int NW = NT / 32;
    constexpr int NPL = KIND == KIND_JV ? 3 : 1;
    extern __shared__ __align__(16) unsigned char g_smem[];
    // the warps' region copies, [NW][TX * TY] doubles each: granule g (= column *
    // NGR + granule row) keeps its rows 0-1 at 2 g and rows 2-3 (4-row granules)
    // at kHalf + 2 g, so a warp's 16-byte accesses to consecutive granules are
    // consecutive (no bank conflicts for either granule height)
    constexpr int kHalf = TX * TY / 2;
    double* parts = (double*)g_smem;
    __shared__ int64_t s_off[NT];
    __shared__ int s_ay[NT];
    __shared__ int s_ax[NT];
    __shared__ int s_rb[NT];
    __shared__ double s_v[3][NT];
    __shared__ int s_wcnt[NW];
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
    const int R0 = ry * TY, C0 = rx * TX;  // 0-based first row / column of the region
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int t = threadIdx.x * 2; t < NW * TX * TY; t += NT * 2) *(double2*)(parts + t) = make_double2(0.0, 0.0);
    __syncthreads();
    double* mine = parts + wid * TX * TY;
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
        for (int q = 0; q < NW; ++q) {
            total += s_wcnt[q];
            if (q < wid) before += s_wcnt[q];
        }
        if (keep) {
            const int pos = before + __popc(bal & ((1u << lane) - 1u));
            s_off[pos] = roff[li];  // the pair's stamp rectangle
            s_ay[pos] = ent.y;
            s_ax[pos] = ent.z;
            s_rb[pos] = ent.w;
            if (KIND == KIND_JV)
                for (int k = 0; k < fc.p; ++k)
                    s_v[k][pos] = vt[(int64_t)ent.x * fc.p + k] * inv_alpha / cn[(int64_t)ent.x * fc.p + k];
        }
        __syncthreads();
        // the current star's rectangle of granules inside the region
        int e = wid, c = 0;  // star (staged index) and slot
        int tot = 0, nga = 1, cl0 = 0, gl0 = 0;
        int64_t PSb = 0;
        float inv_nga = 1.0f;
        const TS* base = src;
        auto star_geometry = [&]() {
            if (e >= total) return;
            // model renders: each star's own model radius; J v: the fit box
            const int Rb = KIND == KIND_M ? s_rb[e] : Rbox;
            const int Sb = 2 * Rb + 1;
            const int left0 = s_ax[e] - Rb - 1, top0 = s_ay[e] - Rb - 1;
            const int b0 = gran_base(top0, GH);
            const int SRb = gran_rows(Sb, GH);
            cl0 = max(left0, C0) - C0;
            const int cl1 = min(left0 + Sb - 1, C0 + TX - 1) - C0;
            const int r_lo = max(b0, R0), r_hi = min(b0 + SRb, R0 + TY);  // multiples of GH
            gl0 = (r_lo - R0) / GH;
            nga = max((r_hi - r_lo) / GH, 0);
            tot = cl1 >= cl0 ? (cl1 - cl0 + 1) * nga : 0;
            inv_nga = 1.0f / (float)max(nga, 1);
            // the dense rectangle: granule t = cc * nga + gg at t * GH, planes tot * GH apart
            PSb = (int64_t)tot * GH;
            base = src + s_off[e];
        };
        star_geometry();
        while (e < total && tot == 0) {
            e += NW;
            star_geometry();
        }
        while (e < total) {
            TS raw[KSLOT][NPL][GH];
            int dst[KSLOT], eq[KSLOT];
#pragma unroll
            for (int q = 0; q < KSLOT; ++q) {
                dst[q] = -1;
                eq[q] = e;
                if (e < total) {
                    const int t = c * 32 + lane;
                    if (t < tot) {
                        const int cc = (int)(((float)t + 0.5f) * inv_nga);
                        const int gg = t - cc * nga;
                        const TS* g = base + (int64_t)t * GH;
                        if (CPB_CHECK(g - src + (p - 1) * PSb + GH <= src_len, 0x31) &&
                            CPB_CHECK((cl0 + cc) * NGR + (gl0 + gg) < TX * NGR, 0x32)) {
#pragma unroll
                            for (int k = 0; k < NPL; ++k)
                                if (k < p) ld_gran(g + k * PSb, raw[q][k]);
                            dst[q] = (cl0 + cc) * NGR + (gl0 + gg);  // granule index in the region
                        }
                    }
                    if ((c + 1) * 32 < tot) {
                        ++c;
                    } else {
                        c = 0;
                        do {
                            e += NW;
                            star_geometry();
                        } while (e < total && tot == 0);
                    }
                }
            }
            // slots in order; two slots of a round may meet at a pixel (different
            // lanes), so each slot's adds complete before the next slot's start
#pragma unroll
            for (int q = 0; q < KSLOT; ++q) {
                if (dst[q] >= 0) {
                    double v[GH];
#pragma unroll
                    for (int r = 0; r < GH; ++r) {
                        double t = (double)raw[q][0][r];
                        if (KIND == KIND_JV) {
                            t *= s_v[0][eq[q]];
                            if (p > 1) t += (double)raw[q][1][r] * s_v[1][eq[q]];
                            if (p > 2) t += (double)raw[q][2][r] * s_v[2][eq[q]];
                        }
                        v[r] = t;
                    }
#pragma unroll
                    for (int h = 0; h < GH; h += 2) {
                        double2* a = (double2*)(mine + (h >> 1) * kHalf + 2 * dst[q]);
                        double2 t = *a;
                        t.x += v[h];
                        t.y += v[h + 1];
                        *a = t;
                    }
                }
                __syncwarp();
            }
        }
        __syncthreads();
    }
    // sum the warps' copies in warp order, then the epilogue, GH pixels at a time
    double part = 0.0;
    for (int gi = threadIdx.x; gi < TX * NGR; gi += NT) {
        const int col = gi / NGR, gr = gi % NGR;
        const int gx = C0 + col;
        if (gx >= fc.nx) continue;
        double acc[GH];
#pragma unroll
        for (int r = 0; r < GH; ++r) acc[r] = parts[(r >> 1) * kHalf + 2 * gi + (r & 1)];
#pragma unroll
        for (int q = 1; q < NW; ++q)
#pragma unroll
            for (int r = 0; r < GH; ++r) acc[r] += parts[q * TX * TY + (r >> 1) * kHalf + 2 * gi + (r & 1)];
#pragma unroll
        for (int r = 0; r < GH; ++r) {
            const int gy = R0 + gr * GH + r;
            if (gy >= fc.ny) break;
            const int64_t q = gy + (int64_t)gx * fc.ny;
            const double av = acc[r];
            if (MODE == MODE_LSQR) {
                const TU un = (TU)(av - alpha * ((double)u_src[q] * uscale));
                outu[q] = un;
                part += (double)un * (double)un;
            } else if (MODE == MODE_CUR) {
                double wr = 0.0;
                if (umask[q]) {
                    wr = sw[q] * (av - data_ref[q]);
                    part += wr * wr;
                }
                outu[q] = (TU)wr;  // wt_resid (zero outside U)
            } else if (MODE == MODE_CAND) {
                if (umask[q]) {
                    const double rr = av - data_ref[q];
                    part += w[q] * rr * rr;
                }
            } else if (MODE == MODE_FREEZE) {
                outd[q] -= av;  // data_work
            } else {
                outd[q] = data_ref[q] - av;  // residual against the original data
            }
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

// J^T u for the stars of `list` (apply_JT!, :55-85): one warp per star.
// The star's stamp lives in the rectangles of the regions its box meets
// (tfit: soffs / star_pairs / off); the lanes walk the granules of those
// rectangles as one sequence (GH rows of one stamp column: the granule of each
// derivative plane and the matching GH pixels of u, all 16-byte loads), JU
// granules in flight per lane.  Writes z[j*p+k] = sum_m V[j,k,m] u[pix(m)] *
// uscale / colnorm[j,k] (V holds the unscaled weighted derivatives).  LSQR
// form: v_new = z - beta * v_old / alpha_old and alpha = ||v_new|| (Krylov
// lsqr step 2).  Sums are FP64 for either stamp type.
constexpr int kJTRects = 16;  // rectangles a warp tabulates at a time
// four blocks an SM (64 registers; three with 80 and five with 48 measured slower)
template <bool LSQR, typename TS, typename TU>
__global__ void __launch_bounds__(256, 4) k_JT(const int32_t* __restrict__ list, int64_t nlist, FitConst fc,
                                            const int32_t* __restrict__ ay, const int32_t* __restrict__ ax,
                                            const TS* __restrict__ V, RectMap vmap, const double* __restrict__ cn,
                                            const TU* __restrict__ u, double* __restrict__ z, Scalars* sc,
                                            Reducer red) {
    static_assert(sizeof(TS) == sizeof(TU), "u granules match stamp granules");
    constexpr int GH = Gran<TS>::H;
    constexpr int JU = 2;
    struct RectTab {
        int64_t off;
        int tot, nga, x0, y0;  // granules, granule rows, first image column and row (0-based)
        float inv_nga;
    };
    __shared__ RectTab tabs[256 / 32][kJTRects];
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    RectTab* tab = tabs[wid];
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (gridDim.x * (int64_t)blockDim.x) >> 5;
    double uscale = 1.0, beta = 0.0, inv_alpha = 0.0;
    if (LSQR) {
        if (sc->stopped || sc->beta == 0.0) return;  // uniform across the grid
        uscale = sc->inv_beta;
        beta = sc->beta;
        inv_alpha = sc->inv_alpha;
    }
    const int p = fc.p, R = fc.R;
    const int ny = fc.ny, nx = fc.nx;
    const bool uvec = (ny % GH) == 0;
    double part = 0.0;
    for (int64_t li = warp; li < nlist; li += nwarps) {
        const int j = list[li];
        const int a_y = ay[j], a_x = ax[j];
        int ty0 = 0, ty1 = -1, tx0 = 0, tx1 = -1;
        star_tiles(a_y, a_x, R, ny, nx, ty0, ty1, tx0, tx1);
        const int nty_j = ty1 - ty0 + 1, nrect = (tx1 - tx0 + 1) * nty_j;
        const int left0 = a_x - R - 1, b0 = gran_base(a_y - R - 1, GH);
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int r0 = 0; r0 < nrect; r0 += kJTRects) {
            const int nr = min(kJTRects, nrect - r0);
            __syncwarp();  // the previous star's / chunk's table is no longer read
            if (lane < nr) {
                const int l = r0 + lane;
                const int ry = ty0 + l % nty_j, rx = tx0 + l / nty_j;
                const RectGeo g = rect_geo(a_y, a_x, R, ry, rx, GH);
                RectTab t;
                t.off = star_rect_off(vmap, j, l);
                t.nga = g.nrows / GH;
                t.inv_nga = 1.0f / (float)max(t.nga, 1);
                t.tot = g.ncols * t.nga;
                t.x0 = left0 + g.c_lo;
                t.y0 = b0 + g.s_lo;
                tab[lane] = t;
            }
            __syncwarp();
            // this lane's granules: lane, lane + 32, ... of the chunk's rectangles in order
            int r = 0, t = lane;
            while (r < nr && t >= tab[r].tot) t -= tab[r++].tot;
            while (r < nr) {
                TS v[JU][3][GH];
                TU uu[JU][GH];
                bool ok[JU];
#pragma unroll
                for (int q = 0; q < JU; ++q) {
                    ok[q] = false;
                    if (r >= nr) continue;
                    const RectTab& T = tab[r];
                    const int cc = (int)(((float)t + 0.5f) * T.inv_nga);
                    const int gg = t - cc * T.nga;
                    const int gx = T.x0 + cc, gy = T.y0 + gg * GH;
                    ok[q] = gx < nx &&
                            CPB_CHECK(T.off + (int64_t)t * GH + (int64_t)(p - 1) * T.tot * GH + GH <= vmap.len, 0x41);
                    if (ok[q]) {
                        const TS* e = V + T.off + (int64_t)t * GH;
                        const int64_t ps = (int64_t)T.tot * GH;
                        ld_gran(e, v[q][0]);
                        if (p > 1) ld_gran(e + ps, v[q][1]);
                        if (p > 2) ld_gran(e + 2 * ps, v[q][2]);
                        const int64_t pq = gy + (int64_t)gx * ny;
                        if (uvec && gy + GH <= ny) {
                            ld_px16(u + pq, uu[q]);
                        } else {
#pragma unroll
                            for (int rr = 0; rr < GH; ++rr) uu[q][rr] = gy + rr < ny ? __ldg(u + pq + rr) : (TU)0;
                        }
                    }
                    t += 32;
                    while (r < nr && t >= tab[r].tot) t -= tab[r++].tot;
                }
#pragma unroll
                for (int q = 0; q < JU; ++q) {
                    if (!ok[q]) continue;
#pragma unroll
                    for (int rr = 0; rr < GH; ++rr) {
                        const double ur = (double)uu[q][rr];
                        a0 += (double)v[q][0][rr] * ur;
                        if (p > 1) a1 += (double)v[q][1][rr] * ur;
                        if (p > 2) a2 += (double)v[q][2][rr] * ur;
                    }
                }
            }
        }
        const double acc0 = warp_sum(a0) * uscale;
        const double acc1 = warp_sum(a1) * uscale;
        const double acc2 = warp_sum(a2) * uscale;
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (k >= p) break;
                double val = (k == 0 ? acc0 : (k == 1 ? acc1 : acc2)) / cn[(int64_t)j * p + k];
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
__global__ void k_lsqr_v0(int64_t n, const double* b_scaled, double* vt, double* x, Scalars* sc, Reducer red,
                          bool lsmr) {
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
        } else if (!lsmr) {  // lsqr's test before the first iteration (lsmr has none)
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

// LSMR start (solver = :lsmr) after k_lsqr_v0: h = v1, hbar = 0 and the
// recurrence state of Fong & Saunders' algorithm (zetabar = alpha1 beta1, ...).
__global__ void k_lsmr_init(int64_t n, const double* vt, double* h, double* hbar, Scalars* sc) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const double ia = sc->inv_alpha;
    if (i < n) {
        h[i] = vt[i] * ia;
        hbar[i] = 0.0;
    }
    if (i == 0) {
        sc->m_alphabar = sc->alpha;
        sc->m_rho = 1.0;
        sc->m_rhobar = 1.0;
        sc->m_cbar = 1.0;
        sc->m_sbar = 0.0;
        sc->m_zeta = 0.0;
        sc->m_zetabar = sc->alpha * sc->beta1;
        sc->m_betadd = sc->beta1;
        sc->m_betad = 0.0;
        sc->m_rhodold = 1.0;
        sc->m_tautildeold = 0.0;
        sc->m_thetatilde = 0.0;
        sc->m_d = 0.0;
        sc->m_maxrbar = 0.0;
        sc->m_minrbar = 1e100;
    }
}

// One LSMR iteration after the Golub-Kahan step (Krylov lsmr main loop): the
// rotations eliminating the damping and turning B into R and R' into Rbar,
// hbar / x / h updates with ||x||^2 reduced over the grid, then (last block)
// the ||r||, ||A|| and cond(A) estimates and the stopping tests.  Every
// thread evaluates the same rotations from the state; the last block commits.
__global__ void k_lsmr_update(int64_t n, const double* vt, double* x, double* h, double* hbar, Scalars* sc,
                              Reducer red) {
    __shared__ double sh[32];
    if (sc->stopped) return;
    const double alpha = sc->alpha, beta = sc->beta, lambda = sc->lambda;
    double chat, shat, alphahat;
    sym_givens(sc->m_alphabar, lambda, chat, shat, alphahat);
    const double rhoold = sc->m_rho;
    double c, s, rho;
    sym_givens(alphahat, beta, c, s, rho);
    const double thetanew = s * alpha;
    const double rhobarold = sc->m_rhobar, zetaold = sc->m_zeta;
    const double thetabar = sc->m_sbar * rho, rhotemp = sc->m_cbar * rho;
    double cbar, sbar, rhobar;
    sym_givens(sc->m_cbar * rho, thetanew, cbar, sbar, rhobar);
    const double zeta = cbar * sc->m_zetabar, zetabar = -sbar * sc->m_zetabar;
    const double kh = thetabar * rho / (rhoold * rhobarold), kx = zeta / (rho * rhobar), kv = thetanew / rho;
    const double ia = sc->inv_alpha;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double part = 0.0;
    if (i < n) {
        const double hb = h[i] - kh * hbar[i];
        hbar[i] = hb;
        const double xi = x[i] + kx * hb;
        x[i] = xi;
        h[i] = vt[i] * ia - kv * h[i];
        part = xi * xi;
    }
    double tot;
    if (grid_reduce<256>(part, red, sh, &tot) && threadIdx.x == 0) {
        const double axtol = 1.4901161193847656e-08, ctol = axtol;
        const int iter = sc->iter + 1;
        // ||r|| estimate
        const double betaacute = chat * sc->m_betadd, betacheck = -shat * sc->m_betadd;
        const double betahat = c * betaacute, betadd = -s * betaacute;
        const double thetatildeold = sc->m_thetatilde;
        double ctildeold, stildeold, rhotildeold;
        sym_givens(sc->m_rhodold, thetabar, ctildeold, stildeold, rhotildeold);
        const double thetatilde = stildeold * rhobar, rhodold = ctildeold * rhobar;
        const double betad = -stildeold * sc->m_betad + ctildeold * betahat;
        const double tautildeold = (zetaold - thetatildeold * sc->m_tautildeold) / rhotildeold;
        const double taud = (zeta - thetatilde * tautildeold) / rhodold;
        const double dsum = sc->m_d + betacheck * betacheck;
        const double rNorm = sqrt(dsum + (betad - taud) * (betad - taud) + betadd * betadd);
        // ||A||, cond(A)
        double Anorm2 = sc->Anorm2 + beta * beta;
        const double Anorm = sqrt(Anorm2);
        Anorm2 += alpha * alpha;
        const double maxrbar = fmax(sc->m_maxrbar, rhobarold);
        const double minrbar = iter > 1 ? fmin(sc->m_minrbar, rhobarold) : sc->m_minrbar;
        const double Acond = fmax(maxrbar, rhotemp) / fmin(minrbar, rhotemp);
        // stopping tests
        const double ArNorm = fabs(zetabar), xNorm = sqrt(tot);
        const double test1 = rNorm / sc->beta1;
        const double test2 = ArNorm / (Anorm * rNorm);
        const double test3 = 1.0 / Acond;
        const double t1 = test1 / (1.0 + Anorm * xNorm / sc->beta1);
        const double rNormtol = sc->btol + axtol * Anorm * xNorm / sc->beta1;
        const bool ill = (1.0 + test3 <= 1.0) || (test3 <= ctol);
        const bool zr = (1.0 + t1 <= 1.0) || (test1 <= rNormtol);
        const bool solved = (1.0 + test2 <= 1.0) || (test2 <= axtol) || (ArNorm <= sc->atol) || zr;
        const bool tired = iter >= sc->itmax;
        sc->m_alphabar = c * alpha;
        sc->m_rho = rho;
        sc->m_rhobar = rhobar;
        sc->m_cbar = cbar;
        sc->m_sbar = sbar;
        sc->m_zeta = zeta;
        sc->m_zetabar = zetabar;
        sc->m_betadd = betadd;
        sc->m_betad = betad;
        sc->m_rhodold = rhodold;
        sc->m_tautildeold = tautildeold;
        sc->m_thetatilde = thetatilde;
        sc->m_d = dsum;
        sc->m_maxrbar = maxrbar;
        sc->m_minrbar = minrbar;
        sc->Anorm2 = Anorm2;
        sc->xNorm = xNorm;
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
// k_eval_warp, the storage-order-walk-only instantiation when `plan` (every
// box within 2 x 2 regions, every map written with per-star offsets)
template <bool GRAD, typename TS, bool GRAM = false, typename... A>
void launch_eval_warp(bool plan, unsigned grid, unsigned thr, size_t smem, cudaStream_t st, A... args) {
    auto go = [&](auto kern) {
        if (smem > 48 * 1024)
            check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attr");
        kern<<<grid, thr, smem, st>>>(args...);
    };
    if (plan) go(k_eval_warp<GRAD, TS, true, GRAM>);
    else go(k_eval_warp<GRAD, TS, false, GRAM>);
}

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
    uint32_t* region = nullptr;   // per pair: its region (ty + tx * nty)
    int32_t* soffs = nullptr;     // per star: its first emit index (n_act + 1)
    int32_t* star_pairs = nullptr;  // per emit index: the pair's list position
    int64_t npairs = 0;
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
    int32_t* emit_j = S<int32_t>(ctx, (t + "_emit_j").c_str(), npairs);
    TileLists tl;
    tl.npairs = npairs;
    tl.region = k1;
    tl.soffs = offs;
    tl.star_pairs = S<int32_t>(ctx, (t + "_star_pairs").c_str(), npairs);
    int32_t* sorted_o = S<int32_t>(ctx, (t + "_sorted").c_str(), npairs);
    tl.list = S<int4>(ctx, (t + "_list").c_str(), npairs);
    const int64_t ntiles = (int64_t)nty * ntx;
    tl.start = S<int32_t>(ctx, (t + "_start").c_str(), ntiles);
    tl.end = S<int32_t>(ctx, (t + "_end").c_str(), ntiles);
    tl.order = S<int32_t>(ctx, (t + "_order").c_str(), ntiles);
    check(cudaMemsetAsync(tl.start, 0, sizeof(int32_t) * ntiles, st), "memset");
    check(cudaMemsetAsync(tl.end, 0, sizeof(int32_t) * ntiles, st), "memset");
    if (npairs > 0) {
        k_tile_emit<<<nblk(n_act), 256, 0, st>>>(n_act, ay, ax, Rs, Rconst, ny, nx, nty, offs, k0, v0, emit_j);
        check(cudaGetLastError(), "k_tile_emit");
        int end_bit = 1;
        while ((1LL << end_bit) < ntiles) ++end_bit;
        tmp = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tmp, k0, k1, v0, sorted_o, npairs, 0, end_bit, st);
        dtmp = scratch(ctx, (t + "_sort_tmp").c_str(), tmp);
        cub::DeviceRadixSort::SortPairs(dtmp, tmp, k0, k1, v0, sorted_o, npairs, 0, end_bit, st);
        k_tile_bounds<<<nblk(npairs), 256, 0, st>>>(npairs, k1, tl.start, tl.end);
        check(cudaGetLastError(), "k_tile_bounds");
        k_tile_pack<<<nblk(npairs), 256, 0, st>>>(npairs, sorted_o, emit_j, ay, ax, Rs, Rconst, tl.list,
                                                  tl.star_pairs);
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

// Element offsets of a list's rectangles for granules of GH rows and `planes`
// planes: a prefix sum of the rectangle sizes (npairs + 1 entries; the last is
// the total).  Returns the total.
int64_t rect_offsets(cpb_ctx* ctx, const char* tag, const TileLists& tl, int nty, int GH, int planes, int64_t* off) {
    cudaStream_t st = ctx->stream;
    const std::string t(tag);
    int64_t* size = S<int64_t>(ctx, (t + "_rsize").c_str(), tl.npairs + 1);
    k_rect_size<<<nblk(tl.npairs + 1), 256, 0, st>>>(tl.npairs, tl.list, tl.region, nty, GH, planes, size);
    check(cudaGetLastError(), "k_rect_size");
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, size, off, (int)(tl.npairs + 1), st);
    void* dtmp = scratch(ctx, (t + "_rscan_tmp").c_str(), tmp);
    cub::DeviceScan::ExclusiveSum(dtmp, tmp, size, off, (int)(tl.npairs + 1), st);
    int64_t total = 0;
    check(cudaMemcpyAsync(&total, off + tl.npairs, sizeof(int64_t), cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaStreamSynchronize(st), "sync");
    return total;
}

}  // namespace

// ---------------------------------------------------------------------------
// scratch bound of one fit (the no-allocation entry point's up-front check)
// ---------------------------------------------------------------------------
namespace {

// Bytes arena_carve reserves for one named buffer of `bytes`.
size_t carve_size(size_t bytes) { return (std::max<size_t>(bytes, 256) + 255) & ~size_t(255); }

// The tile lists of build_tiles for n stars of box radius Rb.
// Upper bound of the (region, star) pairs of n boxes of radius Rb.
int64_t pairs_bound(int64_t n, int Rb) {
    const int64_t Sb = 2 * (int64_t)Rb + 1;
    return std::max<int64_t>(n * ((Sb + TY - 1) / TY + 1) * ((Sb + TX - 1) / TX + 1), 1);
}

// One rect_map: the offsets, the rectangle sizes, the scan temporaries and the
// per-star offsets (srect).
size_t rect_map_bound(int64_t npairs, int64_t n) {
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, (int64_t*)nullptr, (int64_t*)nullptr, (int)(npairs + 1));
    return 2 * carve_size(8 * (npairs + 1)) + carve_size(tmp) + carve_size(8 * kStarRects * n);
}

size_t tiles_bound(int64_t n, int Rb, int64_t ntiles) {
    const int64_t npairs = pairs_bound(n, Rb);
    size_t b = 2 * carve_size(4 * (n + 1));
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, (int32_t*)nullptr, (int32_t*)nullptr, (int)(n + 1));
    b += carve_size(tmp);
    // keys (2), values, emit_j, star_pairs, sorted; the packed list
    b += 6 * carve_size(4 * npairs) + carve_size(16 * npairs);
    b += 3 * carve_size(4 * ntiles) + carve_size(8 * ntiles) + carve_size(4 * ntiles);
    int end_bit = 1;
    while ((1LL << end_bit) < ntiles) ++end_bit;
    tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, (uint32_t*)nullptr, (uint32_t*)nullptr, (int32_t*)nullptr,
                                    (int32_t*)nullptr, (int)npairs, 0, end_bit);
    b += carve_size(tmp);
    tmp = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                              (int32_t*)nullptr, (int32_t*)nullptr, (int)ntiles, 0, 32);
    b += carve_size(tmp);
    return b;
}

// One precision form (Form<TS, TU>): stamps and model stamps (a star's
// rectangles hold at most its column storage), their rectangle maps, pixel vectors.
template <typename TS, typename TU>
size_t form_bound(int64_t n, int p, int S, int64_t model_entries, int64_t npairs_fit, int64_t npairs_mod,
                  int64_t npix) {
    size_t b = carve_size((size_t)p * S * gran_rows(S, Gran<TS>::H) * n * sizeof(TS));
    b += carve_size((size_t)model_entries * sizeof(TS));
    b += rect_map_bound(npairs_fit, n) + rect_map_bound(npairs_mod, n);
    b += 2 * carve_size(npix * sizeof(TU));
    return b;
}

}  // namespace

size_t sim_scratch_bound(const cpb_sim_params* P, int64_t ny, int64_t nx, int64_t n, bool dbg_pixels) {
    const int p = std::max(1, __builtin_popcount((unsigned)(P->free_mask & (CPB_FREE_Y | CPB_FREE_X | CPB_FREE_FLUX))));
    const int R = (int)std::ceil(std::max(P->fit_rad, 0.0));
    const int S = 2 * R + 1;
    const int64_t S2 = (int64_t)S * S;
    // model boxes: the scalar radius as the driver clamps it; with :auto the
    // fit box (the driver checks the model buffers again once the radii are known)
    int Rm = R;
    if (!P->model_rad_auto) {
        const int R_cap = (int)std::ceil(std::max(P->model_rad, P->fit_rad));
        Rm = std::min(std::max((int)std::ceil(P->model_rad), R), R_cap);
    }
    const int Sm = 2 * Rm + 1;
    const int64_t npix = ny * nx;
    const int64_t ntiles = ((ny + TY - 1) / TY) * ((nx + TX - 1) / TX);
    const int64_t np = (int64_t)p * n;
    size_t b = 2 * carve_size(sizeof(Scalars));                                    // scalars, scalars_freeze
    b += carve_size(8 * std::max<int64_t>(ntiles, nblk(std::max<int64_t>(n * 3, npix)) + 1)) + carve_size(4);
    b += 4 * carve_size(8 * npix) + carve_size(16);                                // data, data_work, w, sw, flags
    b += 2 * carve_size(4 * n) + carve_size(n) + carve_size(8 * n);                // ay_c, ax_c, ok, key
    b += 2 * carve_size(4 * n) + 2 * carve_size(8 * n) + carve_size(4 * n) + carve_size(4);  // iota .. nsel
    size_t tmp = 0;
    cub::DeviceSelect::Flagged(nullptr, tmp, (int32_t*)nullptr, (uint8_t*)nullptr, (int32_t*)nullptr, (int*)nullptr,
                               (int)n);
    const size_t sel_tmp = tmp;
    tmp = 0;
    cub::DeviceSelect::Flagged(nullptr, tmp, (uint64_t*)nullptr, (uint8_t*)nullptr, (uint64_t*)nullptr,
                               (int*)nullptr, (int)n);
    b += carve_size(sel_tmp) + carve_size(tmp);
    tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, (uint64_t*)nullptr, (uint64_t*)nullptr, (int32_t*)nullptr,
                                    (int32_t*)nullptr, (int)n, 0, 64);
    b += carve_size(tmp);
    b += 2 * carve_size(4 * n) + carve_size(8 * np);                              // ay, ax, theta
    b += carve_size(npix) + carve_size(8);                                         // umask, ucnt
    if (dbg_pixels) b += carve_size(4 * S2 * n);
    if (P->model_rad_auto) b += carve_size(4 * n);
    b += tiles_bound(n, R, ntiles);
    if (Rm != R || P->model_rad_auto) b += tiles_bound(n, Rm, ntiles);
    b += (P->solver == CPB_SOLVER_LSMR ? 9 : 8) * carve_size(8 * np) +           // solver state (lsmr: hbar)
         2 * carve_size(sizeof(StarCoef) * n);
    b += 3 * carve_size(n) + 4 * carve_size(4 * n) + carve_size(4);
    b += 2 * carve_size(sel_tmp);                                                  // live_tmp, newf_tmp
    // with :auto the model lists are counted at the fit box here (checked again in the fit)
    const int64_t pf = pairs_bound(n, R), pm = pairs_bound(n, Rm);
    const int64_t me32 = (int64_t)Sm * gran_rows(Sm, Gran<float>::H) * n;
    const int64_t me64 = (int64_t)Sm * gran_rows(Sm, Gran<double>::H) * n;
    if (P->precision == CPB_PREC_MIXED) {
        b += form_bound<float, float>(n, p, S, me32, pf, pm, npix);
        if (P->refine_iters > 0) b += form_bound<double, double>(n, p, S, me64, pf, pm, npix);
    } else {
        b += form_bound<double, double>(n, p, S, me64, pf, pm, npix);
    }
    // final pass: gram, err, resid, FP64 model stamps and their map, spread tables, diagnostics
    b += carve_size(48 * n) + carve_size(8 * np) + carve_size(8 * npix);
    b += carve_size(me64 * 8) + rect_map_bound(pm, n);
    b += carve_size(8 * kSpreadRuleLen) + carve_size(8 * spread_tab_len(R)) + carve_size(56 * n);
    return b;
}

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
namespace {

// The buffers of one precision form of the outer loop: stamp derivatives and
// model stamps stored as TS in the granule layout of TS, the LSQR pixel
// vectors (weighted residual, u) as TU.
template <typename TS, typename TU>
struct Form {
    FitConst fc;              // the fit constants
    TS* V = nullptr;          // stamp derivatives: p planes per rectangle of the fit-box lists (vmap)
    TS* M = nullptr;          // model stamps: one plane per rectangle of the model-box lists (mmap)
    RectMap vmap{}, mmap{};
    TU* wt_resid = nullptr;
    TU* u = nullptr;
    bool m_fresh = false;     // M holds the current-theta model of the live stars (written by the fill)
};

class SimFit {
  public:
    SimFit(cpb_ctx* ctx_, const cpb_psf* psf_, const cpb_sim_params* P_, const void* d_image_, int32_t eltype_,
           int64_t ny_, int64_t nx_, const void* d_inv_var_, const void* d_background_, int64_t n_stars_,
           const double* d_y0_, const double* d_x0_, const double* d_flux0_, cpb_sim_result* out_)
        : ctx(ctx_), psf(psf_), P(P_), d_image(d_image_), eltype(eltype_), ny64(ny_), nx64(nx_),
          d_inv_var(d_inv_var_), d_background(d_background_), n_stars(n_stars_), d_y0(d_y0_), d_x0(d_x0_),
          d_flux0(d_flux0_), out(out_), st(ctx_->stream) {}

    int run();

  private:
    template <typename T>
    T* S_(const char* name, size_t count) {
        return (T*)scratch(ctx, name, std::max<size_t>(count, 1) * sizeof(T));
    }
    void nan_diag(int64_t i);
    bool setup();  // false: the fit ended early (no stars, nothing active)
    template <typename TS, typename TU>
    Form<TS, TU> make_form(const char* tag);
    RectMap rect_map(const char* tag, const TileLists& tl, int GH, int planes, int Rmax, int64_t& total);
    template <typename TS, typename TU>
    void launch_fill(Form<TS, TU>& F, const int32_t* list, int64_t nlist);
    template <typename TS>
    void launch_eval_model(const FitConst& f, TS* M, const RectMap& mmap, const int32_t* list, int64_t nlist,
                           const StarCoef* cf);
    template <typename TS, typename TU>
    void launch_render(Form<TS, TU>& F, int mode, const uint8_t* incl, const int32_t* list, int64_t nlist,
                       const StarCoef* cf, TU* outu, double* outd, const double* ref, double* result);
    void update_live_list();
    void read_scalars();
    template <typename TS, typename TU>
    void outer_loop(Form<TS, TU>& F, int it_first, int it_last, bool initial);
    void finish();
    void warp_shape(int Sx, size_t tab_size, unsigned& threads, size_t& smem) const;
    void arena_precheck();
    void launch_coef(const double* delta, StarCoef* dst);

    // arguments
    cpb_ctx* ctx;
    const cpb_psf* psf;
    const cpb_sim_params* P;
    const void* d_image;
    int32_t eltype;
    int64_t ny64, nx64;
    const void* d_inv_var;
    const void* d_background;
    int64_t n_stars;
    const double *d_y0, *d_x0, *d_flux0;
    cpb_sim_result* out;
    cudaStream_t st;
    // set-up
    int ny = 0, nx = 0;
    int64_t npix = 0, ntiles = 0;
    bool reweighted = false;
    FitConst fc{};
    int p = 0;
    DevPsf dp{};
    Scalars* sc = nullptr;
    Scalars* h_sc = nullptr;
    Reducer red{};
    double *data = nullptr, *data_work = nullptr, *w = nullptr, *sw = nullptr;
    int32_t* act = nullptr;
    int64_t n_act = 0, n = 0;
    int n_failed = 0;
    int32_t *ay = nullptr, *ax = nullptr;
    double* theta = nullptr;
    uint8_t* umask = nullptr;
    int32_t* dbg_pix = nullptr;
    unsigned long long h_ucnt = 0;
    int model_R = 0;
    int32_t* d_modelR = nullptr;
    std::vector<int32_t> h_modelR;
    double mean_box = 0, dof = 1;
    TileLists tfit, tmod;
    double *cn = nullptr, *D = nullptr, *bsc = nullptr, *delta = nullptr, *dsc = nullptr;
    double *xl = nullptr, *vt = nullptr, *wl = nullptr, *hbar = nullptr;
    StarCoef *coef = nullptr, *coefc = nullptr;
    uint8_t *live = nullptr, *newf = nullptr, *conv = nullptr;
    int32_t *frozen_at = nullptr, *live_list = nullptr, *iota_act = nullptr, *evlist = nullptr;
    int* d_nlive = nullptr;
    void* live_tmp = nullptr;
    size_t live_tmp_bytes = 0;
    int64_t n_live = 0;
    bool warp_eval = false;
    int smem_optin = 0;
    int Sm = 0;
    unsigned jt_blocks = 1;
    // loop state
    double evals = 0, macs = 0;
    double lam = 0;
    int n_run = 0;
    int64_t n_trials = 0, n_lsqr = 0;
};

void SimFit::nan_diag(int64_t i) {
    const double NaN = std::numeric_limits<double>::quiet_NaN();
    if (out->qfit) out->qfit[i] = NaN;
    if (out->qfit_expected) out->qfit_expected[i] = NaN;
    if (out->qfit_z) out->qfit_z[i] = NaN;
    if (out->crowding) out->crowding[i] = NaN;
    if (out->spread_model) out->spread_model[i] = NaN;
    if (out->spread_model_err) out->spread_model_err[i] = NaN;
}

void SimFit::warp_shape(int Sx, size_t tab_size, unsigned& threads, size_t& smem) const {
    // warps per block of a k_eval_warp launch whose per-warp axis tables (2 Sx
    // entries) fit the opt-in shared memory
    int warps = 8;
    while (warps > 1 && (size_t)warps * 2 * Sx * tab_size > (size_t)smem_optin) warps /= 2;
    if ((size_t)warps * 2 * Sx * tab_size > (size_t)smem_optin)
        throw ArgError{"radius too large for the B200 stamp kernels"};
    threads = 32u * warps;
    smem = (size_t)warps * 2 * Sx * tab_size;
}

void SimFit::launch_coef(const double* dlt, StarCoef* dst) {
    KernelScope ks_(ctx, "k_coef", (double)n_act * (sizeof(StarCoef) + 3 * 8));
    k_coef<<<nblk(n_act), 256, 0, st>>>(n_act, fc, dp, theta, dlt, dst);
    check(cudaGetLastError(), "k_coef");
}

void SimFit::read_scalars() {
    check(cudaMemcpyAsync(h_sc, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaStreamSynchronize(st), "sync");
}

void SimFit::update_live_list() {
    cub::DeviceSelect::Flagged(live_tmp, live_tmp_bytes, iota_act, live, live_list, d_nlive, (int)n_act, st);
    int h = 0;
    check(cudaMemcpyAsync(&h, d_nlive, sizeof(int), cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaStreamSynchronize(st), "sync");
    n_live = h;
}

// The rectangles of list tl with granules of GH rows and `planes` planes each:
// the pair map and the offsets (total: the elements of every rectangle).
RectMap SimFit::rect_map(const char* tag, const TileLists& tl, int GH, int planes, int Rmax, int64_t& total) {
    RectMap m;
    m.soffs = tl.soffs;
    m.star_pairs = tl.star_pairs;
    m.planes = planes;
    int64_t* off = S_<int64_t>(tag, tl.npairs + 1);
    total = rect_offsets(ctx, tag, tl, fc.nty, GH, planes, off);
    m.len = total;
    m.off = off;
    m.srect = nullptr;
    if (2 * Rmax + 1 <= TX + 1 && 2 * Rmax + 1 <= TY + 1) {  // every box meets at most 2 x 2 regions
        int64_t* sr = S_<int64_t>((std::string(tag) + "_srect").c_str(), n_act * kStarRects);
        k_star_rects<<<nblk(n_act * kStarRects), 256, 0, st>>>(n_act, tl.soffs, tl.star_pairs, off, sr);
        check(cudaGetLastError(), "k_star_rects");
        m.srect = sr;
    }
    return m;
}

template <typename TS, typename TU>
Form<TS, TU> SimFit::make_form(const char* tag) {
    Form<TS, TU> F;
    constexpr int GH = Gran<TS>::H;
    F.fc = fc;
    const std::string t(tag);
    int64_t nv = 0, nm = 0;
    F.vmap = rect_map(("V_off" + t).c_str(), tfit, GH, p, fc.R, nv);
    F.mmap = rect_map(("M_off" + t).c_str(), tmod, GH, 1, model_R, nm);
    F.V = S_<TS>(("V" + t).c_str(), nv);
    F.M = S_<TS>(("model_stamps" + t).c_str(), nm);
    // rectangle entries outside the boxes stay zero for the whole fit (the anchors are fixed)
    check(cudaMemsetAsync(F.V, 0, sizeof(TS) * std::max<int64_t>(nv, 1), st), "memset");
    check(cudaMemsetAsync(F.M, 0, sizeof(TS) * std::max<int64_t>(nm, 1), st), "memset");
    F.wt_resid = S_<TU>(("wt_resid" + t).c_str(), npix);
    F.u = S_<TU>(("lsqr_u" + t).c_str(), npix);
    return F;
}

// _fill_stamps! at coef for the stars of `list`: V (and, when the model box is
// the fit box, the model stamps) and colnorm
template <typename TS, typename TU>
void SimFit::launch_fill(Form<TS, TU>& F, const int32_t* list, int64_t nlist) {
    if (nlist <= 0) return;
    NvtxRange nv_("cpb:sim:fill");
    constexpr double bts = sizeof(TS);
    const bool writeM = model_R == fc.R && !d_modelR;
    KernelScope ks_(ctx, "k_eval_fill",
                    (double)nlist * ((double)p * fc.S2 * bts + p * 8 + (writeM ? fc.S2 * bts : 0.0) +
                                     std::min<double>((double)fc.S2, (double)h_ucnt / std::max<int64_t>(n_act, 1)) * 16 +
                                     sizeof(StarCoef)));
    TS* Mo = writeM ? F.M : nullptr;
    if (warp_eval) {
        unsigned thr;
        size_t sm_bytes;
        warp_shape(fc.S, sizeof(AxisTab<TS>), thr, sm_bytes);
        const int wpb = (int)(thr / 32);
        const unsigned gbw =
            (unsigned)std::max<int64_t>(1, std::min<int64_t>((nlist + wpb - 1) / wpb, (int64_t)ctx->n_sm * 8));
        const bool plan = F.vmap.srect && (!Mo || F.mmap.srect);
        launch_eval_warp<true, TS>(plan, gbw, thr, sm_bytes, st, list, nlist, F.fc, dp, coef, ay, ax, w, sw, F.V,
                                   F.vmap, cn, (double*)nullptr, Mo, F.mmap, fc.R, (const int32_t*)nullptr);
    } else {
        const size_t tab_bytes = (size_t)(dp.n_nodes == 1 ? 2 : 8) * sizeof(AxisTab<TS>);
        const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(nlist, (int64_t)ctx->n_sm * 16));
        launch_k_eval<true, TS>(fc.S2, grid, tab_bytes * fc.S, st, list, nlist, F.fc, dp, coef, ay, ax, w, sw, F.V,
                                F.vmap, cn, (double*)nullptr, Mo, F.mmap, fc.R, (const int32_t*)nullptr);
    }
    check(cudaGetLastError(), "k_eval_fill");
    F.m_fresh = writeM;
}

// model values at `cf` for the stars of `list` into M (value-only stamp evaluation)
template <typename TS>
void SimFit::launch_eval_model(const FitConst& f, TS* M, const RectMap& mmap, const int32_t* list, int64_t nlist,
                               const StarCoef* cf) {
    if (nlist <= 0) return;
    KernelScope ks_(ctx, "k_eval_model", (double)nlist * ((double)Sm * Sm * sizeof(TS) + sizeof(StarCoef)));
    if (warp_eval) {
        unsigned thr;
        size_t sm_bytes;
        warp_shape(Sm, sizeof(AxisTab<TS>), thr, sm_bytes);
        const int wpb = (int)(thr / 32);
        const unsigned gbw =
            (unsigned)std::max<int64_t>(1, std::min<int64_t>((nlist + wpb - 1) / wpb, (int64_t)ctx->n_sm * 8));
        launch_eval_warp<false, TS>(mmap.srect != nullptr, gbw, thr, sm_bytes, st, list, nlist, f, dp, cf, ay, ax,
                                    w, sw, (TS*)nullptr, RectMap{}, cn, (double*)nullptr, M, mmap, model_R,
                                    (const int32_t*)d_modelR);
    } else {
        const size_t tab_bytes = (size_t)(dp.n_nodes == 1 ? 2 : 8) * sizeof(AxisTab<TS>);
        const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(nlist, (int64_t)ctx->n_sm * 16));
        launch_k_eval<false, TS>((int64_t)Sm * Sm, grid, tab_bytes * Sm, st, list, nlist, f, dp, cf, ay, ax, w, sw,
                                 (TS*)nullptr, RectMap{}, cn, (double*)nullptr, M, mmap, model_R,
                                 (const int32_t*)d_modelR);
    }
    check(cudaGetLastError(), "k_eval_model");
}

template <typename TS, typename TU>
void SimFit::launch_render(Form<TS, TU>& F, int mode, const uint8_t* incl, const int32_t* list, int64_t nlist,
                           const StarCoef* cf, TU* outu, double* outd, const double* ref, double* result) {
    NvtxRange nv_(mode == MODE_CUR ? "cpb:sim:render_residual"
                                   : (mode == MODE_CAND ? "cpb:sim:render_trial" : "cpb:sim:render_freeze"));
    if (!(mode == MODE_CUR && F.m_fresh)) launch_eval_model<TS>(F.fc, F.M, F.mmap, list, nlist, cf);
    F.m_fresh = false;
    const double px_bytes =
        mode == MODE_CUR ? 17.0 + sizeof(TU) : (mode == MODE_CAND ? 17.0 : 16.0);
    KernelScope ks_(ctx,
                    mode == MODE_CUR ? "k_gather_resid"
                                     : (mode == MODE_CAND ? "k_gather_cost"
                                                          : (mode == MODE_FREEZE ? "k_gather_freeze" : "k_gather_final")),
                    (double)npix * px_bytes + (double)nlist * Sm * Sm * sizeof(TS));
    const unsigned g = (unsigned)ntiles;
    const auto& tl = tmod;
#define CPB_RENDER(MD)                                                                                               \
    k_gather<KIND_M, MD, TS, TU><<<g, NT, kGatherSmem, st>>>(F.fc, tl.start, tl.end, tl.list, tl.order, incl, F.M,   \
                                                             model_R, F.mmap.off, F.mmap.len, nullptr, nullptr,      \
                                                             nullptr, 0.0,                                            \
                                                             outu, outd, umask, w, sw, ref, sc, red, result)
    switch (mode) {
        case MODE_CUR: CPB_RENDER(MODE_CUR); break;
        case MODE_CAND: CPB_RENDER(MODE_CAND); break;
        case MODE_FREEZE: CPB_RENDER(MODE_FREEZE); break;
        default: CPB_RENDER(MODE_FINAL);
    }
#undef CPB_RENDER
    check(cudaGetLastError(), "k_gather");
}

bool SimFit::setup() {
    NvtxRange nv_("cpb:sim:setup");
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
    if (P->damping == CPB_DAMP_LEVENBERG)
        throw ArgError{
            "LevenbergDamping is not supported by fit_all_stars_simultaneous: it conflicts with the "
            "column-equilibrated x_tol scaling. Use MarquardtDamping."};
    if (!(P->fit_rad > 0)) throw ArgError{"fit_rad must be positive"};
    if (eltype != CPB_F32 && eltype != CPB_F64) throw ArgError{"unsupported image eltype"};
    if (ny64 <= 0 || nx64 <= 0 || ny64 * nx64 >= (1LL << 31)) throw ArgError{"image size out of range"};
    if (P->precision != CPB_PREC_FP64 && P->precision != CPB_PREC_MIXED)
        throw ArgError{"precision must be CPB_PREC_FP64 or CPB_PREC_MIXED"};
    if (P->refine_iters < 0) throw ArgError{"refine_iters must be >= 0"};
    ny = (int)ny64;
    nx = (int)nx64;
    npix = ny64 * nx64;
    reweighted = P->covariance == CPB_COV_REWEIGHTED || (P->covariance == CPB_COV_AUTO && d_inv_var == nullptr);
    out->n_active = 0;
    out->n_union = 0;
    out->n_trials = 0;
    out->n_lsqr_iters = 0;
    out->model_px_evals = 0;
    out->lsqr_px_macs = 0;
    out->device_seconds = 0;
    if (n_stars == 0) {
        out->n_passes = 0;
        out->n_failed = 0;
        if (out->residual) std::fill(out->residual, out->residual + npix, 0.0);
        return false;
    }
    // free set (:1015-1051)
    fc.p = 0;
    if (P->free_mask & CPB_FREE_Y) fc.gc[fc.p++] = 1;
    if (P->free_mask & CPB_FREE_X) fc.gc[fc.p++] = 2;
    if (P->free_mask & CPB_FREE_FLUX) fc.gc[fc.p++] = 3;
    if (P->free_mask & ~(CPB_FREE_Y | CPB_FREE_X | CPB_FREE_FLUX))
        throw ArgError{
            "fit_all_stars_simultaneous fits only (y, x, flux) per star. Fix `bkg` (subtract the background first "
            "and pass `fixed = (; bkg = zero(eltype(image)))`), and fix all shape parameters."};
    if (fc.p == 0) throw ArgError{"all model parameters are fixed; nothing to fit"};
    p = fc.p;
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
    fc.q32 = 32 / fc.S;
    fc.r32 = 32 % fc.S;
    fc.ny = ny;
    fc.nx = nx;
    fc.nty = (ny + TY - 1) / TY;
    fc.ntx = (nx + TX - 1) / TX;
    ntiles = (int64_t)fc.nty * fc.ntx;
    dp = psf->dev;
    dp.fwhm = P->fixed_fwhm;

    check(cudaEventRecord(ctx->ev0, st), "event");
    // device-resident scalars and reducers
    sc = S_<Scalars>("scalars", 1);
    check(cudaMemsetAsync(sc, 0, sizeof(Scalars), st), "memset");
    const int64_t max_blocks = std::max<int64_t>(ntiles, nblk(std::max<int64_t>(n_stars * 3, npix)) + 1);
    red = Reducer{S_<double>("red_partials", max_blocks), S_<unsigned>("red_counter", 1)};
    check(cudaMemsetAsync(red.counter, 0, sizeof(unsigned), st), "memset");
    h_sc = (Scalars*)ctx->pinned;

    // ---- data and weights (:1056-1084)
    data = S_<double>("data", npix);
    data_work = S_<double>("data_work", npix);
    w = S_<double>("w", npix);
    sw = S_<double>("sw", npix);
    unsigned* flags = S_<unsigned>("flags", 4);
    check(cudaMemsetAsync(flags, 0, 4 * sizeof(unsigned), st), "memset");
    {
        // 16-byte reads of the caller's images when every one of them allows it
        const int e16 = eltype == CPB_F64 ? 2 : 4;
        auto al16 = [](const void* q) { return q == nullptr || ((uintptr_t)q & 15) == 0; };
        const bool vec = npix % e16 == 0 && al16(d_image) && al16(d_inv_var) && al16(d_background);
        KernelScope ks_(ctx, "k_prepare", (double)npix * ((eltype == CPB_F64 ? 8.0 : 4.0) *
                                                          (1 + (d_inv_var ? 1 : 0) + (d_background ? 1 : 0)) +
                                                          32.0));
#define CPB_PREP(TI, V)                                                                                         \
    k_prepare<TI, V><<<nblk(V ? npix / e16 : npix), 256, 0, st>>>((const TI*)d_image, (const TI*)d_inv_var,     \
                                                                  (const TI*)d_background, npix, data,         \
                                                                  data_work, w, sw, flags)
        if (eltype == CPB_F64) {
            if (vec) CPB_PREP(double, true);
            else CPB_PREP(double, false);
        } else {
            if (vec) CPB_PREP(float, true);
            else CPB_PREP(float, false);
        }
#undef CPB_PREP
        check(cudaGetLastError(), "k_prepare");
    }

    // ---- _build_stamps! (:245-323)
    int32_t* ay_c = S_<int32_t>("ay_c", n_stars);
    int32_t* ax_c = S_<int32_t>("ax_c", n_stars);
    uint8_t* ok = S_<uint8_t>("ok", n_stars);
    uint64_t* key = S_<uint64_t>("key", n_stars);
    k_anchor<<<nblk(n_stars), 256, 0, st>>>(n_stars, d_y0, d_x0, d_flux0, fc.R, ny, nx, w, ay_c, ax_c, ok, key,
                                            flags + 1);
    check(cudaGetLastError(), "k_anchor");
    // compact active stars in catalogue order, then stable radix sort by Morton key
    int32_t* iota = S_<int32_t>("iota", n_stars);
    int32_t* sel = S_<int32_t>("sel", n_stars);
    uint64_t* selkey = S_<uint64_t>("selkey", n_stars);
    uint64_t* selkey2 = S_<uint64_t>("selkey2", n_stars);
    act = S_<int32_t>("act", n_stars);
    int* d_nsel = S_<int>("nsel", 1);
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
    n_act = h_nsel;
    n_failed = (int)(n_stars - n_act);
    out->n_active = n_act;
    if (n_act == 0) {  // _empty_simultaneous_result (:1433-1445)
        std::vector<double> y(n_stars), x(n_stars), f(n_stars);
        check(cudaMemcpyAsync(y.data(), d_y0, sizeof(double) * n_stars, cudaMemcpyDeviceToHost, st), "d2h");
        check(cudaMemcpyAsync(x.data(), d_x0, sizeof(double) * n_stars, cudaMemcpyDeviceToHost, st), "d2h");
        check(cudaMemcpyAsync(f.data(), d_flux0, sizeof(double) * n_stars, cudaMemcpyDeviceToHost, st), "d2h");
        check(cudaStreamSynchronize(st), "sync");
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
        return false;
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
    n = (int64_t)p * n_act;
    ay = S_<int32_t>("ay", n_act);
    ax = S_<int32_t>("ax", n_act);
    theta = S_<double>("theta", n);
    k_gather_active<<<nblk(n_act), 256, 0, st>>>(n_act, act, ay_c, ax_c, d_y0, d_x0, d_flux0, p,
                                                 make_int3(fc.gc[0], fc.gc[1], fc.gc[2]), ay, ax, theta);
    check(cudaGetLastError(), "k_gather_active");

    // ---- union of stamp pixels (:329-335)
    umask = S_<uint8_t>("umask", npix);
    check(cudaMemsetAsync(umask, 0, npix, st), "memset");
    dbg_pix = out->dbg_pixels ? S_<int32_t>("dbg_pix", (int64_t)fc.S2 * n_act) : nullptr;
    k_union<<<(unsigned)n_act, 256, 0, st>>>(n_act, ay, ax, fc.R, ny, nx, w, umask, dbg_pix);
    check(cudaGetLastError(), "k_union");
    unsigned long long* ucnt = S_<unsigned long long>("ucnt", 1);
    check(cudaMemsetAsync(ucnt, 0, sizeof(unsigned long long), st), "memset");
    k_count_u8<<<nblk(npix), 256, 0, st>>>(umask, npix, ucnt);
    check(cudaMemcpyAsync(&h_ucnt, ucnt, sizeof(h_ucnt), cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaStreamSynchronize(st), "sync");
    out->n_union = (int64_t)h_ucnt;

    // ---- model radii (:1111-1124)
    if (P->model_rad_auto && !d_inv_var)
        throw ArgError{
            "model_rad=:auto requires inv_var (it needs a noise scale); pass inv_var or an explicit scalar model_rad"};
    double model_box_sum = 0;  // sum over active stars of (2 R_j + 1)^2
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
        d_modelR = S_<int32_t>("model_R", n_act);
        check(cudaMemcpyAsync(d_modelR, h_modelR.data(), sizeof(int32_t) * n_act, cudaMemcpyHostToDevice, st),
              "h2d model radii");
        check(cudaStreamSynchronize(st), "sync");
        for (int32_t r : h_modelR) model_box_sum += (double)(2 * r + 1) * (2 * r + 1);
    } else {
        const int R_cap = (int)std::ceil(std::max(P->model_rad, P->fit_rad));
        model_R = std::min(std::max((int)std::ceil(P->model_rad), fc.R), R_cap);
        model_box_sum = (double)n_act * (2 * model_R + 1) * (2 * model_R + 1);
    }
    Sm = 2 * model_R + 1;
    mean_box = model_box_sum / (double)n_act;  // per-star render work (instrumentation)
    dof = (double)std::max<int64_t>((int64_t)h_ucnt - n, 1);

    // ---- tile lists (fit box for J v; model box for renders)
    tfit = build_tiles(ctx, "tfit", n_act, ay, ax, nullptr, fc.R, ny, nx, fc.nty, fc.ntx);
    tmod = (model_R == fc.R && !d_modelR)
               ? tfit
               : build_tiles(ctx, "tmod", n_act, ay, ax, d_modelR, model_R, ny, nx, fc.nty, fc.ntx);

    // ---- solver state (:1129-1166)
    cn = S_<double>("colnorm", n);
    D = S_<double>("D", n);
    bsc = S_<double>("b_scaled", n);
    delta = S_<double>("delta", n);
    dsc = S_<double>("delta_scaled", n);
    xl = S_<double>("lsqr_x", n);
    vt = S_<double>("lsqr_v", n);
    wl = S_<double>("lsqr_w", n);  // lsqr's w, or lsmr's h
    if (P->solver == CPB_SOLVER_LSMR) hbar = S_<double>("lsmr_hbar", n);
    coef = S_<StarCoef>("coef", n_act);
    coefc = S_<StarCoef>("coef_cand", n_act);
    live = S_<uint8_t>("live", n_act);
    newf = S_<uint8_t>("newf", n_act);
    conv = S_<uint8_t>("conv", n_act);
    frozen_at = S_<int32_t>("frozen_at", n_act);
    live_list = S_<int32_t>("live_list", n_act);
    iota_act = S_<int32_t>("iota_act", n_act);
    evlist = S_<int32_t>("eval_list", n_act);
    d_nlive = S_<int>("nlive", 1);
    check(cudaMemsetAsync(live, 1, n_act, st), "memset");
    check(cudaMemsetAsync(conv, 0, n_act, st), "memset");
    check(cudaMemsetAsync(frozen_at, 0, sizeof(int32_t) * n_act, st), "memset");
    check(cudaMemsetAsync(cn, 0, sizeof(double) * n, st), "memset");
    check(cudaMemcpyAsync(iota_act, iota, sizeof(int32_t) * n_act, cudaMemcpyDeviceToDevice, st), "d2d");
    n_live = n_act;
    check(cudaMemcpyAsync(live_list, iota, sizeof(int32_t) * n_act, cudaMemcpyDeviceToDevice, st), "d2d");
    live_tmp_bytes = 0;
    cub::DeviceSelect::Flagged(nullptr, live_tmp_bytes, iota_act, live, live_list, d_nlive, (int)n_act, st);
    live_tmp = scratch(ctx, "live_tmp", live_tmp_bytes);

    warp_eval = dp.kind == CPB_PSF_CIRCULAR_GAUSSIAN || dp.n_nodes == 1;
    check(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device), "attr");
    jt_blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n_act + 7) / 8, (int64_t)ctx->n_sm * 8));
    lam = P->lambda_init;
    if (ctx->arena) arena_precheck();
    return true;
}

// No-allocation entry point: with the active set and the model radii known,
// the buffers of the precision forms and of the final pass must fit what is
// left of the fixed region; refuse here, before the outer loop starts.
void SimFit::arena_precheck() {
    // stored model-stamp entries of every active star at granule height gh (a bound:
    // the rectangles hold at most the stars' column storage)
    auto model_entries = [&](int gh) {
        int64_t t = 0;
        if (d_modelR) {
            for (int32_t r : h_modelR) t += (int64_t)(2 * r + 1) * gran_rows(2 * r + 1, gh);
        } else {
            t = n_act * (int64_t)Sm * gran_rows(Sm, gh);
        }
        return t;
    };
    size_t need = 0;
    auto form = [&](size_t ts, int gh) {
        need += carve_size((size_t)p * fc.S * gran_rows(fc.S, gh) * n_act * ts) + carve_size(model_entries(gh) * ts) +
                rect_map_bound(tfit.npairs, n_act) + rect_map_bound(tmod.npairs, n_act) + 2 * carve_size(npix * ts);
    };
    if (P->precision == CPB_PREC_MIXED) {
        form(sizeof(float), Gran<float>::H);
        if (P->refine_iters > 0) form(sizeof(double), Gran<double>::H);
    } else {
        form(sizeof(double), Gran<double>::H);
    }
    need += carve_size(sizeof(Scalars)) + carve_size(live_tmp_bytes);  // scalars_freeze, newf_tmp
    need += carve_size(48 * n_act) + carve_size(8 * n) + carve_size(8 * npix);
    need += carve_size(model_entries(Gran<double>::H) * 8) + rect_map_bound(tmod.npairs, n_act);
    need += carve_size(8 * kSpreadRuleLen) + carve_size(8 * spread_tab_len(fc.R)) + carve_size(56 * n_act);
    const size_t used = (ctx->arena->used + 255) & ~size_t(255);
    if (used + need > ctx->arena->cap)
        throw ArgError{"field too large for the no-allocation entry point: needs about " +
                       std::to_string((used + need + (1 << 20) - 1) >> 20) + " MiB of scratch, the static region holds " +
                       std::to_string(ctx->arena->cap >> 20) + " MiB"};
}

// The outer Gauss-Newton loop (:1186-1284) over iterations it_first..it_last,
// with the stamps, model values and LSQR pixel vectors of form F.  `initial`:
// the first fill and cost of the fit (:1171-1178), which also start D.
template <typename TS, typename TU>
void SimFit::outer_loop(Form<TS, TU>& F, int it_first, int it_last, bool initial) {
    constexpr double bts = sizeof(TS), btu = sizeof(TU);
    const FitConst& f = F.fc;
    const bool lsmr = P->solver == CPB_SOLVER_LSMR;  // krylov_solve! with the :lsmr workspace
    bool fresh = false;  // V / wt_resid / cost are at the current theta and live set
    if (initial) {
        launch_coef(nullptr, coef);
        launch_fill(F, live_list, n_live);
        launch_render(F, MODE_CUR, live, live_list, n_live, coef, F.wt_resid, nullptr, data_work, &sc->cost);
        check(cudaMemcpyAsync(D, cn, sizeof(double) * n, cudaMemcpyDeviceToDevice, st), "d2d");
        evals += (double)n_live * (fc.S2 + mean_box);
        fresh = true;
    }
    for (int iter = it_first; iter <= it_last; ++iter) {
        if (!fresh) {
            launch_coef(nullptr, coef);
            launch_fill(F, live_list, n_live);
            launch_render(F, MODE_CUR, live, live_list, n_live, coef, F.wt_resid, nullptr, data_work, &sc->cost);
            evals += (double)n_live * (fc.S2 + mean_box);
        }
        fresh = false;
        // b_scaled = J' wt_resid (frozen stars stay 0)
        check(cudaMemsetAsync(bsc, 0, sizeof(double) * n, st), "memset");
        {
            KernelScope ks_(ctx, "k_JT",
                            (double)n_live * ((double)p * fc.S2 * bts + 2.0 * p * 8) +
                                std::min<double>((double)h_ucnt, (double)n_live * fc.S2) * btu);
            k_JT<false, TS, TU><<<jt_blocks, 256, 0, st>>>(live_list, n_live, f, ay, ax, F.V, F.vmap, cn, F.wt_resid,
                                                           bsc, sc, red);
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
            check(cudaGetLastError(), "k_freeze_all");
            n_run = iter - 1;
            return;
        }
        bool accepted = false, f_conv = false;
        for (int trial = 1; trial <= P->max_trials; ++trial) {
            NvtxRange nv_trial("cpb:sim:trial");
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
                NvtxRange nv_lsqr("cpb:sim:lsqr");
                {
                    KernelScope ks_(ctx, "k_lsqr_v0", (double)n * 8 * 3);
                    k_lsqr_v0<<<nblk(n), 256, 0, st>>>(n, bsc, vt, xl, sc, red, lsmr);
                }
                {
                    KernelScope ks_(ctx, lsmr ? "k_lsmr_init" : "k_lsqr_w0", (double)n * 8 * 2);
                    if (lsmr) k_lsmr_init<<<nblk(n), 256, 0, st>>>(n, vt, wl, hbar, sc);
                    else k_lsqr_w0<<<nblk(n), 256, 0, st>>>(n, vt, wl, sc, red);
                }
                for (int it = 0; it < P->inner_iterations; ++it) {
                    {
                        KernelScope ks_(ctx, "k_gather_Jv",
                                        (double)n_live * ((double)p * fc.S2 * bts + p * 8) + 2.0 * npix * btu);
                        k_gather<KIND_JV, MODE_LSQR, TS, TU>
                            <<<(unsigned)ntiles, NT, kGatherSmem, st>>>(
                            f, tfit.start, tfit.end, tfit.list, tfit.order, live, F.V, fc.R, F.vmap.off, F.vmap.len, vt, cn,
                            it == 0 ? F.wt_resid : F.u, it == 0 ? -1.0 : 1.0, F.u, nullptr, umask, w, sw, nullptr, sc,
                            red, nullptr);
                    }
                    {
                        KernelScope ks_(ctx, "k_JT_lsqr",
                                        (double)n_live * ((double)p * fc.S2 * bts + 2.0 * p * 8) +
                                            std::min<double>((double)h_ucnt, (double)n_live * fc.S2) * btu);
                        k_JT<true, TS, TU><<<jt_blocks, 256, 0, st>>>(live_list, n_live, f, ay, ax, F.V, F.vmap, cn,
                                                                      F.u, vt, sc, red);
                    }
                    {
                        KernelScope ks_(ctx, lsmr ? "k_lsmr_update" : "k_lsqr_update", (double)n * 8 * (lsmr ? 7 : 5));
                        if (lsmr) k_lsmr_update<<<nblk(n), 256, 0, st>>>(n, vt, xl, wl, hbar, sc, red);
                        else k_lsqr_update<<<nblk(n), 256, 0, st>>>(n, vt, xl, wl, sc, red);
                    }
                }
                check(cudaGetLastError(), "lsqr");
            }
            {
                KernelScope ks_(ctx, "k_step", (double)n * 8 * 4);
                k_step<<<nblk(n_act), 256, 0, st>>>(n_act, fc, P->max_step, xl, cn, delta, dsc);
            }
            launch_coef(delta, coefc);
            launch_render(F, MODE_CAND, live, live_list, n_live, coefc, (TU*)nullptr, nullptr, data_work,
                          &sc->cost_cand);
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
                Scalars* scf = S_<Scalars>("scalars_freeze", 1);
                Scalars s3 = s2;
                s3.cost = cost;
                check(cudaMemcpyAsync(scf, &s3, sizeof(Scalars), cudaMemcpyHostToDevice, st), "h2d");
                {
                    KernelScope ks_(ctx, "k_accept_freeze", (double)n * 8 * 7);
                    k_accept_freeze<<<nblk(n_act), 256, 0, st>>>(n_act, fc, P->x_tol, P->g_tol, dof, iter, theta,
                                                                delta, dsc, cn, D, bsc, live, newf, frozen_at, conv,
                                                                scf);
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
                    launch_coef(nullptr, coef);
                    {
                        size_t tb = 0;
                        cub::DeviceSelect::Flagged(nullptr, tb, iota_act, newf, evlist, d_nlive, (int)n_act, st);
                        void* tmpb = scratch(ctx, "newf_tmp", tb);
                        cub::DeviceSelect::Flagged(tmpb, tb, iota_act, newf, evlist, d_nlive, (int)n_act, st);
                    }
                    launch_render(F, MODE_FREEZE, newf, evlist, h_new, coef, (TU*)nullptr, data_work, nullptr,
                                  nullptr);
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
            check(cudaGetLastError(), "k_freeze_all");
            return;
        }
        if (accepted && n_live == 0) return;
    }
}

int SimFit::run() {
    if (!setup()) return 0;
    const bool mixed = P->precision == CPB_PREC_MIXED;
    if (mixed) {
        Form<float, float> F32 = make_form<float, float>("_f32");
        outer_loop(F32, 1, P->max_iter, true);
        if (P->refine_iters > 0) {
            // FP64 refinement: every active star live again on the original
            // data, from the mixed-precision parameters, with the same scaling D
            // and convergence tests (converged flags accumulate) and the damping
            // restarted at lambda_init: near its end the FP32-stamp loop rejects
            // steps on cost differences below what FP32 model values resolve, and
            // the damping those rejections piled up would hold the FP64 steps back
            Form<double, double> F64 = make_form<double, double>("_f64");
            lam = P->lambda_init;
            check(cudaMemcpyAsync(data_work, data, sizeof(double) * npix, cudaMemcpyDeviceToDevice, st), "d2d");
            check(cudaMemsetAsync(live, 1, n_act, st), "memset");
            check(cudaMemcpyAsync(live_list, iota_act, sizeof(int32_t) * n_act, cudaMemcpyDeviceToDevice, st), "d2d");
            n_live = n_act;
            NvtxRange nv_("cpb:sim:refine_fp64");
            outer_loop(F64, n_run + 1, n_run + P->refine_iters, false);
        }
    } else {
        Form<double, double> F64 = make_form<double, double>("_f64");
        outer_loop(F64, 1, P->max_iter, true);
    }
    finish();
    return 0;
}

// Errors (:1302-1329), the final render against the original data
// (:1344-1356), the diagnostics and the result assembly (:1289-1300,
// :1331-1337, :1404-1430); FP64 for either precision form.
void SimFit::finish() {
    NvtxRange nv_("cpb:sim:final");
    const double NaN = std::numeric_limits<double>::quiet_NaN();
    launch_coef(nullptr, coef);
    double* gram = S_<double>("gram", (int64_t)n_act * 6);
    const FitConst& f64 = fc;
    {
        KernelScope ks_(ctx, "k_eval_gram", (double)n_act * (48.0 + sizeof(StarCoef)));
        if (warp_eval) {
            unsigned thr;
            size_t sm_bytes;
            warp_shape(fc.S, sizeof(AxisTab<double>), thr, sm_bytes);
            const int wpb = (int)(thr / 32);
            const unsigned gbw =
                (unsigned)std::max<int64_t>(1, std::min<int64_t>((n_act + wpb - 1) / wpb, (int64_t)ctx->n_sm * 8));
            const bool plan = 2 * fc.R + 1 <= TX + 1 && 2 * fc.R + 1 <= TY + 1;  // the Gram needs no map
            launch_eval_warp<true, double, true>(plan, gbw, thr, sm_bytes, st, (const int32_t*)nullptr, (int64_t)n_act, f64,
                                           dp, coef, ay, ax, w, sw, (double*)nullptr, RectMap{}, cn, gram,
                                           (double*)nullptr, RectMap{}, fc.R, (const int32_t*)nullptr);
        } else {
            const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(n_act, (int64_t)ctx->n_sm * 16));
            launch_k_eval<true, double>(fc.S2, grid, (size_t)(dp.n_nodes == 1 ? 2 : 8) * sizeof(AxisTab<double>) * fc.S,
                                        st, (const int32_t*)nullptr, n_act, f64, dp, coef, ay, ax, w, sw,
                                        (double*)nullptr, RectMap{}, cn, gram, (double*)nullptr, RectMap{}, fc.R,
                                        (const int32_t*)nullptr);
        }
        check(cudaGetLastError(), "k_eval_gram");
    }
    double* err = S_<double>("err", n);
    read_scalars();  // final cost
    k_errors<<<nblk(n_act), 256, 0, st>>>(n_act, p, gram, reweighted, dof, sc, err);
    check(cudaGetLastError(), "k_errors");
    // ---- final render against the original data (:1344-1356)
    double* resid = S_<double>("resid", npix);
    {
        int64_t mtot64 = 0;
        const RectMap m64 = rect_map("M_off_final", tmod, Gran<double>::H, 1, model_R, mtot64);
        double* M64 = S_<double>("model_stamps_final", mtot64);
        check(cudaMemsetAsync(M64, 0, sizeof(double) * std::max<int64_t>(mtot64, 1), st), "memset");
        launch_eval_model<double>(f64, M64, m64, nullptr, n_act, coef);
        KernelScope ks_(ctx, "k_gather_final", (double)npix * 16.0 + (double)n_act * Sm * Sm * 8);
        k_gather<KIND_M, MODE_FINAL, double, double>
            <<<(unsigned)ntiles, NT, kGatherSmem, st>>>(
            f64, tmod.start, tmod.end, tmod.list, tmod.order, nullptr, M64, model_R, m64.off, m64.len, nullptr, nullptr,
            nullptr, 0.0, nullptr, resid, umask, w, sw, data, sc, red, nullptr);
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
        double* d_rule = S_<double>("spread_rule", kSpreadRuleLen);
        d_stab = S_<double>("spread_tab", spread_tab_len(kh));
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
        check(cudaStreamSynchronize(st), "sync");  // h_rule is a stack buffer
    }
    const size_t diag_smem = spread_smem_bytes(smode, boxmax, kh);
    const unsigned dgrid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(n_act, (int64_t)ctx->n_sm * 16));
    double* diag = S_<double>("diag", (int64_t)n_act * 7);
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
}

}  // namespace

int fit_simultaneous_dev(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* P, const void* d_image,
                         int32_t eltype, int64_t ny, int64_t nx, const void* d_inv_var, const void* d_background,
                         int64_t n, const double* d_y0, const double* d_x0, const double* d_flux0,
                         cpb_sim_result* out) {
    SimFit fit(ctx, psf, P, d_image, eltype, ny, nx, d_inv_var, d_background, n, d_y0, d_x0, d_flux0, out);
    const int rc = fit.run();
#ifdef CPB_CHECKED
    // the checked build: the first index check that failed in any kernel of the fit
    unsigned site = 0;
    check(cudaMemcpyFromSymbolAsync(&site, g_check_err, sizeof(site), 0, cudaMemcpyDeviceToHost, ctx->stream),
          "check flag");
    check(cudaStreamSynchronize(ctx->stream), "check flag");
    if (site) {
        const unsigned zero = 0;
        check(cudaMemcpyToSymbolAsync(g_check_err, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, ctx->stream),
              "check flag");
        check(cudaStreamSynchronize(ctx->stream), "check flag");
        char msg[96];
        snprintf(msg, sizeof msg, "index check 0x%x failed in the simultaneous fit (access skipped)", site);
        throw std::runtime_error(msg);
    }
#endif
    return rc;
}

}  // namespace cpb
