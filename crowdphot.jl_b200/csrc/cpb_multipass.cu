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

#include <cub/cub.cuh>

#include "cpb_internal.cuh"

namespace cpb {
namespace {

// Passes 2+: add_star! (PSF.jl:420-428) of the star's previous model over its
// box, then the fit_star cutout of the running residual (and of inv_var) at
// offs[s] -- one warp a star, lanes over the box pixels.
template <typename TI>
__global__ void k_mp_addcut(int nL, const int4* __restrict__ boxes, const double* __restrict__ params, int add,
                            DevPsf P, MPConst M, double* residual, const TI* __restrict__ iv, int ny,
                            const int64_t* __restrict__ offs, double* __restrict__ pix, double* __restrict__ ivc) {
    const int lane = threadIdx.x & 31;
    const int s = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    if (s >= nL) return;
    const int4 b = boxes[s];  // y1, x1, box rows, box columns
    const double* pr = params + (int64_t)s * M.np;
    const int64_t o = offs[s];
    for (int e = lane; e < b.z * b.w; e += 32) {
        const int i = b.x + e % b.z, j = b.y + e / b.z;
        const int64_t q = (i - 1) + (int64_t)(j - 1) * ny;
        double r = residual[q];
        if (add) {
            r = r + mp_model(P, M, pr, i, j);
            residual[q] = r;
        }
        pix[o + e] = r;
        if (iv) ivc[o + e] = (double)iv[q];
    }
}

// _star_diagnostics! (psf_photometry_diagnostics.jl:154-231) over the fitted
// box: image is the original data, residual the star's fit residual (every
// model subtracted, its own included), star_model its best-fit render, kept in
// shared memory with its disk-correlated copy for spread_model (D.I null:
// spread_model off).  One block of kDiagThreads a star (grid-stride).  out:
// qfit, qfit_expected, qfit_z, crowding, spread_model, spread_model_err per
// star (NaN where undefined).  snap (nullable): the star's residual box saved
// right after its subtraction (snap_off per position), used in place of the
// residual image when the diagnostics run after the whole pass.
template <typename TI>
__global__ void __launch_bounds__(kDiagThreads, 3) k_mp_diag(int nL, const int4* __restrict__ boxes,
                                                         const double* __restrict__ params,
                                                         const uint8_t* __restrict__ flags,
                                                         const TI* __restrict__ img,
                                                         const double* __restrict__ residual,
                                                         const double* __restrict__ snap,
                                                         const int64_t* __restrict__ snap_off,
                                                         const TI* __restrict__ iv, DevPsf P, MPConst M, int n_free,
                                                         int ny, SpreadDev D, int smode, int boxmax,
                                                         const int32_t* __restrict__ idx, double* __restrict__ out) {
    extern __shared__ double stamp[];  // model stamp, x-pass scratch, disk-correlated stamp
    __shared__ double red[12 * (kDiagThreads / 32)];
    const double NaN = __longlong_as_double(0x7ff8000000000000LL);
    const int mode = D.I ? smode : 0;
    double* Is = stamp + 7 * boxmax;  // mode 1: the six profiles
    if (mode == 1)
        for (int i = threadIdx.x; i < 6 * (2 * D.kh + 1); i += blockDim.x) Is[i] = D.I[i];
    for (int s = blockIdx.x; s < nL; s += gridDim.x) {
        __syncthreads();  // the previous star's stamps are no longer read
        double* o = out + (int64_t)idx[s] * 6;  // star order
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
                const double r = snap ? snap[snap_off[s] + e] : residual[q];
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

// Bookkeeping of one batch after its fit_star launch (:373-401) and the
// subtraction that follows, one warp a star: on success the star's parameters,
// errors of the free parameters, convergence, chi^2 and iteration count are
// updated and its new model is subtracted (flag 2); a fit that failed the input
// checks invalidates the star and, on passes 2+, subtracts its previous model
// again to undo the add-back (flag 1).  Positions index the batch; idx maps
// them to stars.  psub / flag keep the subtracted model for the diagnostics.
__global__ void k_mp_booksub(int nL, const int32_t* __restrict__ idx, int pass, int nf, MPFree F,
                             const double* __restrict__ lm_params, const double* __restrict__ lm_cov,
                             const double* __restrict__ lm_chisq, const uint8_t* __restrict__ lm_conv,
                             const int32_t* __restrict__ lm_iters, const int32_t* __restrict__ lm_status,
                             const double* __restrict__ pin, const int4* __restrict__ boxes, DevPsf P, MPConst M,
                             double* residual, int ny, double* __restrict__ prm, double* __restrict__ err,
                             uint8_t* __restrict__ conv, double* __restrict__ chisq, int32_t* __restrict__ niter,
                             uint8_t* __restrict__ valid, int* __restrict__ n_failed, double* __restrict__ psub,
                             uint8_t* __restrict__ flag) {
    const int lane = threadIdx.x & 31;
    const int k = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    if (k >= nL) return;
    const int np = M.np;
    const int64_t s = idx[k];
    const bool failed = lm_status[k] != 0;
    const double* src = failed ? pin + (int64_t)k * np : lm_params + (int64_t)k * np;
    double* ps = psub + (int64_t)k * np;
    if (lane == 0) {
        if (failed) {  // fit_star threw (:391-401)
            valid[s] = 0;
            atomicAdd(n_failed, 1);
            flag[k] = pass > 1 ? 1 : 0;
        } else {
            for (int q = 0; q < np; ++q) prm[s * np + q] = src[q];
            for (int a = 0; a < nf; ++a)
                err[s * np + F.idx[a]] = sqrt(fmax(0.0, lm_cov[(int64_t)k * nf * nf + a + a * nf]));
            conv[s] = lm_conv[k];
            chisq[s] = lm_chisq[k];
            niter[s] += lm_iters[k];
            flag[k] = 2;
        }
        for (int q = 0; q < np; ++q) ps[q] = src[q];
    }
    if (failed && pass == 1) return;
    // subtract_star! of the new (or, undoing the add-back, the previous) model
    double pr[5];
    for (int q = 0; q < np; ++q) pr[q] = src[q];
    const int4 b = boxes[k];
    for (int e = lane; e < b.z * b.w; e += 32) {
        const int i = b.x + e % b.z, j = b.y + e / b.z;
        const int64_t q = (i - 1) + (int64_t)(j - 1) * ny;
        residual[q] = residual[q] - mp_model(P, M, pr, i, j);
    }
}

// ---- the plan of a pass on the device ---------------------------------------
// Order-preserving 64-bit key of a double (NaN above +inf, as isless orders it).
__device__ __forceinline__ unsigned long long mp_dkey(double v) {
    if (v != v) return 0xffffffffffffffffull;
    const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
    return (bits >> 63) ? ~bits : (bits | 0x8000000000000000ull);
}

// Per star at the pass start: its +-fit_rad box clamped to the image (:343-348)
// or invalidation (non-finite position, fewer than 3 box pixels), its grid cell
// (cells at least one box wide, so overlapping boxes have their corners in
// neighbouring cells), and the brightness key (flux descending; invalid last).
__global__ void k_plan_box(int n, const double* __restrict__ prm, MPConst M, double fit_rad, int ny, int nx,
                           int cell, int gny, uint8_t* __restrict__ valid, int4* __restrict__ box,
                           int32_t* __restrict__ cellid, unsigned long long* __restrict__ fkey,
                           int32_t* __restrict__ iota, int32_t* __restrict__ cell_count) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    iota[s] = s;
    cellid[s] = -1;
    fkey[s] = 0xffffffffffffffffull;
    if (!valid[s]) return;
    const double y = prm[(int64_t)s * M.np + M.ry], x = prm[(int64_t)s * M.np + M.rx];
    if (!(isfinite(y) && isfinite(x))) {
        valid[s] = 0;
        return;
    }
    const int ylo = (int)fmax(floor(y - fit_rad), 1.0), yhi = (int)fmin(ceil(y + fit_rad), (double)ny);
    const int xlo = (int)fmax(floor(x - fit_rad), 1.0), xhi = (int)fmin(ceil(x + fit_rad), (double)nx);
    const int by = max(yhi - ylo + 1, 0), bx = max(xhi - xlo + 1, 0);
    if ((int64_t)by * bx < 3) {
        valid[s] = 0;
        return;
    }
    box[s] = make_int4(ylo, xlo, by, bx);
    const int c = ((xlo - 1) / cell) * gny + (ylo - 1) / cell;
    cellid[s] = c;
    atomicAdd(&cell_count[c], 1);
    // ascending key = descending flux; the sort is stable, so ties keep the star order
    fkey[s] = ~mp_dkey(prm[(int64_t)s * M.np + M.rf]);
}

__global__ void k_plan_rank(int n, const int32_t* __restrict__ order, int32_t* __restrict__ rank,
                            int32_t* __restrict__ level) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    rank[order[k]] = k;
    level[k] = 0;
}

__global__ void k_plan_cells(int n, const int32_t* __restrict__ cellid, const int32_t* __restrict__ cell_start,
                             int32_t* __restrict__ cell_fill, int32_t* __restrict__ cell_list) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || cellid[s] < 0) return;
    const int c = cellid[s];
    cell_list[cell_start[c] + atomicAdd(&cell_fill[c], 1)] = s;
}

// One relaxation sweep of level(s) = 1 + max level of the brighter stars whose
// boxes meet box(s) (0 if none).  Levels only grow towards the fixed point, so
// sweeps may run in place; a sweep that changes nothing ends the iteration.
__global__ void k_plan_relax(int n, const int4* __restrict__ box, const int32_t* __restrict__ cellid,
                             const int32_t* __restrict__ rank, const int32_t* __restrict__ cell_start,
                             const int32_t* __restrict__ cell_list, int gny, int gnx, int32_t* level,
                             int* __restrict__ changed) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || cellid[s] < 0) return;
    const int4 bs = box[s];
    const int ylo = bs.x, yhi = bs.x + bs.z - 1, xlo = bs.y, xhi = bs.y + bs.w - 1;
    const int rs = rank[s];
    const int cx = cellid[s] / gny, cy = cellid[s] % gny;
    int lv = 0;
    for (int gx = max(cx - 1, 0); gx <= min(cx + 1, gnx - 1); ++gx)
        for (int gy = max(cy - 1, 0); gy <= min(cy + 1, gny - 1); ++gy) {
            const int c = gx * gny + gy;
            for (int q = cell_start[c]; q < cell_start[c + 1]; ++q) {
                const int t = cell_list[q];
                if (rank[t] >= rs) continue;
                const int4 bt = box[t];
                if (bt.x <= yhi && ylo <= bt.x + bt.z - 1 && bt.y <= xhi && xlo <= bt.y + bt.w - 1)
                    lv = max(lv, ((volatile const int32_t*)level)[t] + 1);
            }
        }
    if (lv > level[s]) {
        atomicMax(&level[s], lv);
        *changed = 1;
    }
}

__global__ void k_plan_poskey(int n, const int32_t* __restrict__ cellid, const int32_t* __restrict__ level,
                              const int32_t* __restrict__ rank, unsigned long long* __restrict__ key) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    key[s] = cellid[s] < 0 ? 0xffffffffffffffffull
                           : ((unsigned long long)(unsigned)level[s] << 32) | (unsigned long long)(unsigned)rank[s];
}

// Per position (level order): box, initial parameters, fit_star dims planes,
// box size; level starts, and npos / nlev into meta.
__global__ void k_plan_pos(int n, const int32_t* __restrict__ idx, const unsigned long long* __restrict__ skey,
                           const int4* __restrict__ box_s, const double* __restrict__ prm, int np,
                           const int32_t* __restrict__ level, int4* __restrict__ box, double* __restrict__ pin,
                           int32_t* __restrict__ dims, int64_t* __restrict__ size, int32_t* __restrict__ lev_start,
                           int32_t* __restrict__ meta, int32_t* __restrict__ pos_of) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const bool ok = skey[k] != 0xffffffffffffffffull;
    const bool last = k == n - 1 || skey[k + 1] == 0xffffffffffffffffull;
    if (!ok) {
        size[k] = 0;
        if (k == 0) meta[0] = meta[1] = 0;
        return;
    }
    const int s = idx[k];
    pos_of[s] = k;
    const int4 b = box_s[s];
    box[k] = b;
    for (int q = 0; q < np; ++q) pin[(int64_t)k * np + q] = prm[(int64_t)s * np + q];
    dims[k] = b.z;
    dims[n + k] = b.w;
    dims[2 * n + k] = b.x;
    dims[3 * n + k] = b.y;
    size[k] = (int64_t)b.z * b.w;
    const int L = level[s];
    if (k == 0 || level[idx[k - 1]] != L) lev_start[L] = k;
    if (last) {
        meta[0] = k + 1;  // positions
        meta[1] = L + 1;  // levels
        lev_start[L + 1] = k + 1;
    }
}

// Cutout offsets from each level's first pixel, and each level's pixel count.
__global__ void k_plan_offsets(int npos, int nlev, const int32_t* __restrict__ idx,
                               const int32_t* __restrict__ level, const int64_t* __restrict__ scan,
                               const int32_t* __restrict__ lev_start, int64_t* __restrict__ off,
                               int64_t* __restrict__ lev_pix) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < npos) off[k] = scan[k] - scan[lev_start[level[idx[k]]]];
    if (k < nlev) lev_pix[k] = scan[lev_start[k + 1]] - scan[lev_start[k]];
}

// The dependency lists of a pass for k_mp_dag: per position, how many brighter
// overlapping stars it waits for (indeg) and how many dimmer ones wait for it
// (nsucc); then the waiting positions themselves (succ_list from succ_start).
template <bool FILL>
__global__ void k_dag_edges(int n, const int4* __restrict__ box, const int32_t* __restrict__ cellid,
                            const int32_t* __restrict__ rank, const int32_t* __restrict__ cell_start,
                            const int32_t* __restrict__ cell_list, int gny, int gnx, const int32_t* __restrict__ pos_of,
                            int32_t* __restrict__ indeg, int32_t* __restrict__ nsucc,
                            const int32_t* __restrict__ succ_start, int32_t* __restrict__ succ_list) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || cellid[s] < 0) return;
    const int4 bs = box[s];
    const int ylo = bs.x, yhi = bs.x + bs.z - 1, xlo = bs.y, xhi = bs.y + bs.w - 1;
    const int rs = rank[s];
    const int cx = cellid[s] / gny, cy = cellid[s] % gny;
    const int k = pos_of[s];
    int np_ = 0, ns = 0;
    for (int gx = max(cx - 1, 0); gx <= min(cx + 1, gnx - 1); ++gx)
        for (int gy = max(cy - 1, 0); gy <= min(cy + 1, gny - 1); ++gy) {
            const int c = gx * gny + gy;
            for (int q = cell_start[c]; q < cell_start[c + 1]; ++q) {
                const int t = cell_list[q];
                if (t == s) continue;
                const int4 bt = box[t];
                if (!(bt.x <= yhi && ylo <= bt.x + bt.z - 1 && bt.y <= xhi && xlo <= bt.y + bt.w - 1)) continue;
                if (rank[t] < rs) {
                    ++np_;
                } else {
                    if (FILL) succ_list[succ_start[k] + ns] = pos_of[t];
                    ++ns;
                }
            }
        }
    if (!FILL) {
        indeg[k] = np_;
        nsucc[k] = ns;
    }
}

// Positions of a dependency-driven pass in brightness order (order: stars by
// rank, the invalid ones last): box, initial parameters and box size per
// position, the star -> position map, and the number of positions into meta.
__global__ void k_dag_pos(int n, const int32_t* __restrict__ order, const unsigned long long* __restrict__ skey,
                          const int4* __restrict__ box_s, const double* __restrict__ prm, int np,
                          int4* __restrict__ box, double* __restrict__ pin, int64_t* __restrict__ size,
                          int32_t* __restrict__ pos_of, int32_t* __restrict__ meta) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const bool ok = skey[k] != 0xffffffffffffffffull;
    if (!ok) {
        size[k] = 0;
        if (k == 0) meta[0] = 0;
        return;
    }
    if (k == n - 1 || skey[k + 1] == 0xffffffffffffffffull) meta[0] = k + 1;
    const int s = order[k];
    pos_of[s] = k;
    const int4 b = box_s[s];
    box[k] = b;
    for (int q = 0; q < np; ++q) pin[(int64_t)k * np + q] = prm[(int64_t)s * np + q];
    size[k] = (int64_t)b.z * b.w;
}

// The ready queue of a pass: every position that waits for nobody.
__global__ void k_dag_queue(int npos, const int32_t* __restrict__ indeg, int32_t* __restrict__ queue,
                            int32_t* __restrict__ counters) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npos || indeg[k] != 0) return;
    queue[atomicAdd(&counters[1], 1)] = k;
}

// Between-pass validation (:404-412).
__global__ void k_mp_validate(int n, const double* __restrict__ prm, MPConst M, const uint8_t* __restrict__ conv,
                              uint8_t* __restrict__ valid) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double y = prm[(int64_t)s * M.np + M.ry], x = prm[(int64_t)s * M.np + M.rx];
    const double f = prm[(int64_t)s * M.np + M.rf];
    valid[s] = valid[s] && conv[s] && isfinite(y) && isfinite(x) && isfinite(f) && f > 0;
}

template <typename T>
__global__ void k_mp_fill(int64_t n, T v, T* __restrict__ a) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

inline unsigned warps_grid(int64_t n) { return (unsigned)std::max<int64_t>(1, (n * 32 + 255) / 256); }

// Counts a launch that has no KernelScope (the context's launch counter).
inline void counted(cpb_ctx* ctx) { ctx->launches += 1; }

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
    counted(ctx);
    if (eltype == CPB_F64)
        k_mp_init<double><<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(npix, (const double*)d_img, resid);
    else
        k_mp_init<float><<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(npix, (const float*)d_img, resid);
    check(cudaGetLastError(), "k_mp_init");

    // per-star state on the device (star order) and per-position buffers of a
    // pass (level order; a pass never holds more than n positions)
    const int Rmax = (int)std::ceil(std::max(fit_rad, 0.0)) + 1;
    const int64_t box_max = (int64_t)(2 * Rmax + 1) * (2 * Rmax + 1);
    const int cell = 2 * Rmax + 2;  // >= every box side
    const int gny = (ny - 1) / cell + 1, gnx = (nx - 1) / cell + 1;
    const int ncell = gny * gnx;
    auto I32 = [&](const char* name, size_t cnt) { return (int32_t*)scratch(ctx, name, sizeof(int32_t) * std::max<size_t>(cnt, 1)); };
    auto U64 = [&](const char* name, size_t cnt) {
        return (unsigned long long*)scratch(ctx, name, sizeof(unsigned long long) * std::max<size_t>(cnt, 1));
    };
    double* d_prm = (double*)scratch(ctx, "mp_prm", sizeof(double) * n * np);
    double* d_err = (double*)scratch(ctx, "mp_err", sizeof(double) * n * np);
    double* d_chisq = (double*)scratch(ctx, "mp_chisq", sizeof(double) * n);
    int32_t* d_niter = I32("mp_niter", n);
    uint8_t* d_sflag = (uint8_t*)scratch(ctx, "mp_sflags", (size_t)n * 2);  // valid, converged
    uint8_t* d_valid = d_sflag;
    uint8_t* d_conv = d_sflag + n;
    int32_t* d_misc = I32("mp_misc", 4);  // failures, changed, positions, levels
    int* d_nfail = d_misc;
    int* d_changed = d_misc + 1;
    int32_t* d_meta = d_misc + 2;
    double* d_diagS = (double*)scratch(ctx, "mp_diag", sizeof(double) * n * 6);
    // plan
    int4* d_boxs = (int4*)scratch(ctx, "mp_box_star", sizeof(int4) * n);
    int32_t* d_cellid = I32("mp_cellid", n);
    unsigned long long* d_fkey = U64("mp_fkey", n);
    unsigned long long* d_fkey2 = U64("mp_fkey2", n);
    int32_t* d_iota = I32("mp_iota", n);
    int32_t* d_order = I32("mp_order", n);
    int32_t* d_rank = I32("mp_rank", n);
    int32_t* d_level = I32("mp_level", n);
    int32_t* d_ccount = I32("mp_cell_count", ncell + 1);
    int32_t* d_cstart = I32("mp_cell_start", ncell + 1);
    int32_t* d_cfill = I32("mp_cell_fill", ncell);
    int32_t* d_clist = I32("mp_cell_list", n);
    unsigned long long* d_pkey = U64("mp_pkey", n);
    unsigned long long* d_pkey2 = U64("mp_pkey2", n);
    int32_t* d_idx = I32("mp_idx", n);
    int64_t* d_size = (int64_t*)scratch(ctx, "mp_size", sizeof(int64_t) * (n + 1));
    int64_t* d_scan = (int64_t*)scratch(ctx, "mp_scan", sizeof(int64_t) * (n + 1));
    int32_t* d_lstart = I32("mp_lev_start", n + 1);
    int64_t* d_lpix = (int64_t*)scratch(ctx, "mp_lev_pix", sizeof(int64_t) * n);
    unsigned long long* d_queues = U64("mp_queues", n);
    int32_t* d_posof = I32("mp_pos_of", n);
    // dependency-driven passes (k_mp_dag): edges, ready queue, per-team cutouts
    const bool dag = mp_dag_supported(psf, P);
    int32_t *d_indeg = nullptr, *d_nsucc = nullptr, *d_sstart = nullptr, *d_queue = nullptr, *d_dagc = nullptr;
    double *d_tpix = nullptr, *d_tiv = nullptr;
    if (dag) {
        d_indeg = I32("mp_indeg", n);
        d_nsucc = I32("mp_nsucc", n + 1);
        d_sstart = I32("mp_succ_start", n + 1);
        d_queue = I32("mp_queue", n);
        d_dagc = I32("mp_dag_counters", 4);
        const int teams = mp_dag_teams(ctx);
        d_tpix = (double*)scratch(ctx, "mp_team_pix", sizeof(double) * teams * box_max);
        if (d_iv) d_tiv = (double*)scratch(ctx, "mp_team_iv", sizeof(double) * teams * box_max);
    }
    // per position
    int4* d_box = (int4*)scratch(ctx, "mp_box", sizeof(int4) * n);
    double* d_pin = (double*)scratch(ctx, "mp_pin", sizeof(double) * n * np);
    double* d_psub = (double*)scratch(ctx, "mp_psub", sizeof(double) * n * np);
    uint8_t* d_flag = (uint8_t*)scratch(ctx, "mp_flag", n);
    int64_t* d_off = (int64_t*)scratch(ctx, "mp_off", sizeof(int64_t) * n);
    int32_t* d_dims = I32("mp_dims", (size_t)n * 4);  // ny, nx, y1, x1 planes
    double* d_lmd = (double*)scratch(ctx, "mp_lm_f64", sizeof(double) * n * (np + nf * nf + 4));
    uint8_t* d_lmu = (uint8_t*)scratch(ctx, "mp_lm_u8", (size_t)n * 4);
    int32_t* d_lmi = I32("mp_lm_i32", (size_t)n * 2);
    // CUB temporary storage (the largest of the sorts and scans)
    size_t tmp_bytes = 0, t = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t, d_fkey, d_fkey2, d_iota, d_order, (int)n, 0, 64, st);
    tmp_bytes = std::max(tmp_bytes, t);
    cub::DeviceScan::ExclusiveSum(nullptr, t, d_ccount, d_cstart, ncell + 1, st);
    tmp_bytes = std::max(tmp_bytes, t);
    cub::DeviceScan::ExclusiveSum(nullptr, t, d_size, d_scan, (int)n + 1, st);
    tmp_bytes = std::max(tmp_bytes, t);
    cub::DeviceScan::ExclusiveSum(nullptr, t, d_ccount, d_cstart, (int)n + 1, st);
    tmp_bytes = std::max(tmp_bytes, t);
    void* d_tmp = scratch(ctx, "mp_cub_tmp", std::max<size_t>(tmp_bytes, 16));

    check(cudaMemcpyAsync(d_prm, prm.data(), sizeof(double) * n * np, cudaMemcpyHostToDevice, st), "h2d");
    check(cudaMemcpyAsync(d_err, err.data(), sizeof(double) * n * np, cudaMemcpyHostToDevice, st), "h2d");
    check(cudaMemsetAsync(d_chisq, 0, sizeof(double) * n, st), "memset");
    check(cudaMemsetAsync(d_niter, 0, sizeof(int32_t) * n, st), "memset");
    check(cudaMemsetAsync(d_valid, 1, (size_t)n, st), "memset");
    check(cudaMemsetAsync(d_conv, 0, (size_t)n, st), "memset");
    check(cudaMemsetAsync(d_misc, 0, sizeof(int32_t) * 4, st), "memset");
    counted(ctx);
    k_mp_fill<double><<<(unsigned)((n * 6 + 255) / 256), 256, 0, st>>>(n * 6, NaN, d_diagS);
    check(cudaGetLastError(), "k_mp_fill");
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
    const unsigned gs = (unsigned)((n + 255) / 256);
    std::vector<int32_t> lev_start;
    std::vector<int64_t> lev_pix;

    for (int pass = 1; pass <= n_passes; ++pass) {
        NvtxRange nv_("cpb:fit_all_stars:pass");
        // ---- plan (:326-348): brightness order, boxes, and the batch (level)
        // of every valid star, all on the device
        check(cudaMemsetAsync(d_ccount, 0, sizeof(int32_t) * (ncell + 1), st), "memset");
        check(cudaMemsetAsync(d_cfill, 0, sizeof(int32_t) * ncell, st), "memset");
        counted(ctx);
        k_plan_box<<<gs, 256, 0, st>>>((int)n, d_prm, M, fit_rad, ny, nx, cell, gny, d_valid, d_boxs, d_cellid, d_fkey,
                                       d_iota, d_ccount);
        check(cudaGetLastError(), "k_plan_box");
        t = tmp_bytes;
        check(cub::DeviceRadixSort::SortPairs(d_tmp, t, d_fkey, d_fkey2, d_iota, d_order, (int)n, 0, 64, st), "sort");
        counted(ctx);
        k_plan_rank<<<gs, 256, 0, st>>>((int)n, d_order, d_rank, d_level);
        t = tmp_bytes;
        check(cub::DeviceScan::ExclusiveSum(d_tmp, t, d_ccount, d_cstart, ncell + 1, st), "scan");
        counted(ctx);
        k_plan_cells<<<gs, 256, 0, st>>>((int)n, d_cellid, d_cstart, d_cfill, d_clist);
        check(cudaGetLastError(), "k_plan_cells");
        if (dag) {
            // positions in brightness order, the dependency lists, the ready
            // queue, and one launch for the whole pass
            counted(ctx);
            k_dag_pos<<<gs, 256, 0, st>>>((int)n, d_order, d_fkey2, d_boxs, d_prm, np, d_box, d_pin, d_size, d_posof,
                                          d_meta);
            check(cudaGetLastError(), "k_dag_pos");
            check(cudaMemsetAsync(d_size + n, 0, sizeof(int64_t), st), "memset");
            t = tmp_bytes;
            check(cub::DeviceScan::ExclusiveSum(d_tmp, t, d_size, d_scan, (int)n + 1, st), "scan");
            counted(ctx);
            k_dag_edges<false><<<gs, 256, 0, st>>>((int)n, d_boxs, d_cellid, d_rank, d_cstart, d_clist, gny, gnx, d_posof,
                                                   d_indeg, d_nsucc, nullptr, nullptr);
            check(cudaGetLastError(), "k_dag_edges");
            int32_t meta[2] = {0, 0};
            check(cudaMemcpyAsync(meta, d_meta, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "d2h");
            check(cudaStreamSynchronize(st), "sync");
            const int npos = meta[0];
            out->n_fits += npos;
            if (npos > 0) {
                check(cudaMemsetAsync(d_nsucc + npos, 0, sizeof(int32_t), st), "memset");
                t = tmp_bytes;
                check(cub::DeviceScan::ExclusiveSum(d_tmp, t, d_nsucc, d_sstart, npos + 1, st), "scan");
                int32_t nedge = 0;
                int64_t tot_all = 0;
                check(cudaMemcpyAsync(&nedge, d_sstart + npos, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "d2h");
                check(cudaMemcpyAsync(&tot_all, d_scan + npos, sizeof(int64_t), cudaMemcpyDeviceToHost, st), "d2h");
                check(cudaStreamSynchronize(st), "sync");
                int32_t* d_slist = I32("mp_succ_list", (size_t)nedge);
                counted(ctx);
                k_dag_edges<true><<<gs, 256, 0, st>>>((int)n, d_boxs, d_cellid, d_rank, d_cstart, d_clist, gny, gnx,
                                                      d_posof, nullptr, nullptr, d_sstart, d_slist);
                check(cudaGetLastError(), "k_dag_edges");
                counted(ctx);
                k_mp_fill<int32_t><<<(unsigned)((npos + 255) / 256), 256, 0, st>>>(npos, -1, d_queue);
                check(cudaMemsetAsync(d_level, 0, sizeof(int32_t) * npos, st), "memset");
                check(cudaMemsetAsync(d_dagc, 0, sizeof(int32_t) * 4, st), "memset");
                if (ctx->fault == CPB_FAULT_HOLD_READY_STAR && pass == 1) {
                    // test hook: the brightest star (position 0, which waits for nobody) is
                    // kept out of the ready queue, so the stars behind it never become ready
                    const int32_t held = 1;
                    check(cudaMemcpyAsync(d_indeg, &held, sizeof(int32_t), cudaMemcpyHostToDevice, st), "h2d");
                    check(cudaStreamSynchronize(st), "sync");
                    ctx->fault = CPB_FAULT_NONE;
                }
                counted(ctx);
                k_dag_queue<<<(unsigned)((npos + 255) / 256), 256, 0, st>>>(npos, d_indeg, d_queue, d_dagc);
                check(cudaGetLastError(), "k_dag_queue");
                double* d_snap = pass == n_passes
                                     ? (double*)scratch(ctx, "mp_snap", sizeof(double) * std::max<int64_t>(tot_all, 1))
                                     : nullptr;
                DagArgs A{};
                A.npos = npos;
                A.pass = pass;
                A.ny = ny;
                A.box_max = boxmax;
                A.M = M;
                A.F = F;
                A.idx = d_order;
                A.box = d_box;
                A.pin = d_pin;
                A.succ_start = d_sstart;
                A.succ_list = d_slist;
                A.indeg = d_indeg;
                A.plevel = d_level;
                A.queue = d_queue;
                A.counters = d_dagc;
                A.resid = resid;
                A.iv = d_iv;
                A.cpix = d_tpix;
                A.civ = d_tiv;
                A.prm = d_prm;
                A.err = d_err;
                A.conv = d_conv;
                A.valid = d_valid;
                A.chisq = d_chisq;
                A.niter = d_niter;
                A.n_failed = d_nfail;
                A.psub = d_psub;
                A.flag = d_flag;
                A.snap = d_snap;
                A.snap_off = d_scan;
                mp_dag_launch(ctx, psf, P, eltype, A);
                if (pass == n_passes) {  // diagnostics of the fitted stars (:381-389), from the snapshots
                    KernelScope ks_(ctx, "k_mp_diag", (double)tot_all * (d_iv ? 24 : 16));
                    const unsigned g = (unsigned)std::min<int64_t>(npos, (int64_t)ctx->n_sm * 16);
                    if (eltype == CPB_F64)
                        k_mp_diag<double><<<g, kDiagThreads, diag_smem, st>>>(
                            npos, d_box, d_psub, d_flag, (const double*)d_img, resid, d_snap, d_scan,
                            (const double*)d_iv, dp, M, nf, ny, sd, smode, boxmax, d_order, d_diagS);
                    else
                        k_mp_diag<float><<<g, kDiagThreads, diag_smem, st>>>(
                            npos, d_box, d_psub, d_flag, (const float*)d_img, resid, d_snap, d_scan,
                            (const float*)d_iv, dp, M, nf, ny, sd, smode, boxmax, d_order, d_diagS);
                    check(cudaGetLastError(), "k_mp_diag");
                }
                int32_t dc[4] = {0, 0, 0, 0};
                check(cudaMemcpyAsync(dc, d_dagc, sizeof(dc), cudaMemcpyDeviceToHost, st), "d2h");
                check(cudaStreamSynchronize(st), "sync");
                if (dc[2]) throw WaitTimeout{"fit_all_stars: a pass stalled waiting for ready stars"};
                out->n_levels += dc[3] + 1;  // the longest chain of dependent fits
            }
            counted(ctx);
            k_mp_validate<<<gs, 256, 0, st>>>((int)n, d_prm, M, d_conv, d_valid);
            check(cudaGetLastError(), "k_mp_validate");
            continue;
        }
        for (int64_t sweep = 0;; sweep += 2) {
            if (sweep > n + 2) throw CudaError{cudaErrorUnknown, "fit_all_stars: the batch plan did not converge"};
            int changed = 0;
            check(cudaMemsetAsync(d_changed, 0, sizeof(int), st), "memset");
            for (int k = 0; k < 2; ++k) {
                counted(ctx);
                k_plan_relax<<<gs, 256, 0, st>>>((int)n, d_boxs, d_cellid, d_rank, d_cstart, d_clist, gny, gnx,
                                                 d_level, d_changed);
            }
            check(cudaGetLastError(), "k_plan_relax");
            check(cudaMemcpyAsync(&changed, d_changed, sizeof(int), cudaMemcpyDeviceToHost, st), "d2h");
            check(cudaStreamSynchronize(st), "sync");
            if (!changed) break;
        }
        counted(ctx);
        k_plan_poskey<<<gs, 256, 0, st>>>((int)n, d_cellid, d_level, d_rank, d_pkey);
        t = tmp_bytes;
        check(cub::DeviceRadixSort::SortPairs(d_tmp, t, d_pkey, d_pkey2, d_iota, d_idx, (int)n, 0, 64, st), "sort");
        counted(ctx);
        k_plan_pos<<<gs, 256, 0, st>>>((int)n, d_idx, d_pkey2, d_boxs, d_prm, np, d_level, d_box, d_pin, d_dims, d_size,
                                       d_lstart, d_meta, d_posof);
        check(cudaGetLastError(), "k_plan_pos");
        check(cudaMemsetAsync(d_size + n, 0, sizeof(int64_t), st), "memset");
        t = tmp_bytes;
        check(cub::DeviceScan::ExclusiveSum(d_tmp, t, d_size, d_scan, (int)n + 1, st), "scan");
        int32_t meta[2] = {0, 0};
        check(cudaMemcpyAsync(meta, d_meta, sizeof(meta), cudaMemcpyDeviceToHost, st), "d2h");
        check(cudaStreamSynchronize(st), "sync");
        const int npos = meta[0], nlev = meta[1];
        out->n_levels += nlev;
        out->n_fits += npos;
        lev_start.assign(nlev + 1, 0);
        lev_pix.assign(std::max(nlev, 1), 0);
        if (npos > 0) {
            counted(ctx);
            k_plan_offsets<<<(unsigned)((std::max(npos, nlev) + 255) / 256), 256, 0, st>>>(npos, nlev, d_idx, d_level,
                                                                                        d_scan, d_lstart, d_off, d_lpix);
            check(cudaGetLastError(), "k_plan_offsets");
            check(cudaMemcpyAsync(lev_start.data(), d_lstart, sizeof(int32_t) * (nlev + 1), cudaMemcpyDeviceToHost, st),
                  "d2h");
            check(cudaMemcpyAsync(lev_pix.data(), d_lpix, sizeof(int64_t) * nlev, cudaMemcpyDeviceToHost, st), "d2h");
            check(cudaMemsetAsync(d_queues, 0, sizeof(unsigned long long) * nlev, st), "memset");
            check(cudaStreamSynchronize(st), "sync");
        }
        const int64_t pix_max = std::max<int64_t>(1, *std::max_element(lev_pix.begin(), lev_pix.end()));
        double* d_cpix = (double*)scratch(ctx, "mp_cpix", sizeof(double) * pix_max);
        double* d_civ = d_iv ? (double*)scratch(ctx, "mp_civ", sizeof(double) * pix_max) : nullptr;
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
            {  // passes 2+: the star's previous model goes back in (:360-365); the cutouts
                KernelScope ks_(ctx, "k_mp_addcut", (double)tot * (pass > 1 ? 32 : 16) + (d_iv ? tot * 16.0 : 0.0));
                if (eltype == CPB_F64)
                    k_mp_addcut<double><<<warps_grid(nL), 256, 0, st>>>(nL, bx, d_pin + p0 * np, pass > 1, dp, M, resid,
                                                                      (const double*)d_iv, ny, d_off + p0, d_cpix,
                                                                      d_civ);
                else
                    k_mp_addcut<float><<<warps_grid(nL), 256, 0, st>>>(nL, bx, d_pin + p0 * np, pass > 1, dp, M, resid,
                                                                     (const float*)d_iv, ny, d_off + p0, d_cpix,
                                                                     d_civ);
                check(cudaGetLastError(), "k_mp_addcut");
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
            lm_enqueue_device(ctx, psf, P, nL, d_off + p0, d_dims + p0, d_dims + n + p0, d_dims + 2 * n + p0,
                              d_dims + 3 * n + p0, d_cpix, CPB_F64, d_civ, d_pin + p0 * np, tot, &r, 4, d_queues + L);
            {  // bookkeeping (:373-401) and the subtraction
                KernelScope ks_(ctx, "k_mp_booksub", (double)tot * 16);
                k_mp_booksub<<<warps_grid(nL), 256, 0, st>>>(
                    nL, d_idx + p0, pass, nf, F, r.params, r.cov, r.chisq, r.converged, r.iterations, r.status,
                    d_pin + p0 * np, bx, dp, M, resid, ny, d_prm, d_err, d_conv, d_chisq, d_niter, d_valid, d_nfail,
                    d_psub + p0 * np, d_flag + p0);
                check(cudaGetLastError(), "k_mp_booksub");
            }
            if (pass == n_passes) {  // diagnostics of the fitted stars (:381-389)
                KernelScope ks_(ctx, "k_mp_diag", (double)tot * (d_iv ? 24 : 16));
                const unsigned g = (unsigned)std::min<int64_t>(nL, (int64_t)ctx->n_sm * 16);
                if (eltype == CPB_F64)
                    k_mp_diag<double><<<g, kDiagThreads, diag_smem, st>>>(
                        nL, bx, d_psub + p0 * np, d_flag + p0, (const double*)d_img, resid, nullptr, nullptr,
                        (const double*)d_iv, dp, M, nf, ny, sd, smode, boxmax, d_idx + p0, d_diagS);
                else
                    k_mp_diag<float><<<g, kDiagThreads, diag_smem, st>>>(
                        nL, bx, d_psub + p0 * np, d_flag + p0, (const float*)d_img, resid, nullptr, nullptr,
                        (const float*)d_iv, dp, M, nf, ny, sd, smode, boxmax, d_idx + p0, d_diagS);
                check(cudaGetLastError(), "k_mp_diag");
            }
        }
        // between-pass validation (:404-412)
        counted(ctx);
        k_mp_validate<<<gs, 256, 0, st>>>((int)n, d_prm, M, d_conv, d_valid);
        check(cudaGetLastError(), "k_mp_validate");
    }
    check(cudaEventRecord(ctx->ev1, st), "event");
    check(cudaMemcpyAsync(prm.data(), d_prm, sizeof(double) * n * np, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(valid.data(), d_valid, (size_t)n, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(conv.data(), d_conv, (size_t)n, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(diag.data(), d_diagS, sizeof(double) * n * 6, cudaMemcpyDeviceToHost, st), "d2h");
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
