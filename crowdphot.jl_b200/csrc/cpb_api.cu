// cpb_api.cu -- the extern "C" boundary (include/crowdphot_b200.h).
//
// Context and PSF handles, argument validation that mirrors the reference's
// constructors, host<->device staging, and error translation: C++ exceptions
// never cross the ABI; every entry point returns a CPB_* status and leaves a
// message for cpb_last_error().
#include <algorithm>
#include <cmath>
#include <cstring>
#include <set>
#include <string>
#include <vector>

#include "cpb_internal.cuh"

namespace cpb {

// A named grow-only scratch buffer of at least `bytes`.  Growth frees and
// allocates in stream order on the context's stream (cudaFreeAsync /
// cudaMallocAsync from the device's memory pool): no device-wide
// synchronisation, so contexts sharing the GPU -- the server's slots -- keep
// running while one of them grows.  The copy stream's work is ordered before
// the free and after the new allocation.
void* scratch(cpb_ctx* ctx, const char* name, size_t bytes) {
    if (ctx->arena) return arena_carve(ctx->arena, name, bytes);
    auto& b = ctx->bufs[name];
    if (b.bytes >= bytes && b.p) return b.p;
    if (b.p) {
        check(cudaEventRecord(ctx->grow_ev, ctx->copy_stream), "grow order");
        check(cudaStreamWaitEvent(ctx->stream, ctx->grow_ev, 0), "grow order");
        check(cudaFreeAsync(b.p, ctx->stream), "cudaFreeAsync");
        b.p = nullptr;
        b.bytes = 0;
    }
    size_t want = std::max<size_t>(bytes, 256);
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, want, ctx->stream);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        throw OomError{std::string("device memory exhausted allocating ") + name};
    }
    check(e, "cudaMallocAsync");
    check(cudaEventRecord(ctx->grow_ev, ctx->stream), "grow order");
    check(cudaStreamWaitEvent(ctx->copy_stream, ctx->grow_ev, 0), "grow order");
    b.p = p;
    b.bytes = want;
    return p;
}

static cudaEvent_t pool_event(cpb_ctx* ctx) {
    if (!ctx->event_pool.empty()) {
        cudaEvent_t e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    check(cudaEventCreate(&e), "cudaEventCreate");
    return e;
}

KernelScope::KernelScope(cpb_ctx* c, const char* n, double by) : ctx(c), name(n), bytes(by) {
    ctx->launches += 1;
    if (ctx->profile) {
        a = pool_event(ctx);
        b = pool_event(ctx);
        cudaEventRecord(a, ctx->stream);
    }
}

KernelScope::~KernelScope() {
    if (a) {
        cudaEventRecord(b, ctx->stream);
        ctx->pending.push_back({name, a, b, bytes});
    }
}

void resolve_kernel_events(cpb_ctx* ctx) {
    if (ctx->pending.empty()) return;
    cudaStreamSynchronize(ctx->stream);
    for (auto& p : ctx->pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.a, p.b);
        auto& k = ctx->kstats[p.name];
        k.launches += 1;
        k.seconds += ms * 1e-3;
        k.bytes += p.bytes;
        ctx->event_pool.push_back(p.a);
        ctx->event_pool.push_back(p.b);
    }
    ctx->pending.clear();
}

}  // namespace cpb

using namespace cpb;

extern "C" {

const char* cpb_version(void) { return "crowdphot_b200 0.1 (sm_100a)"; }

int cpb_ctx_create(int device, cpb_ctx** out) {
    if (!out) return CPB_ERR_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return CPB_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return CPB_ERR_ARGUMENT;
    auto* ctx = new cpb_ctx();
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->grow_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost(&ctx->pinned, 4096) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return CPB_ERR_CUDA;
    }
    for (int k = 0; k < cpb_ctx::kCopyEvents; ++k)
        if (cudaEventCreateWithFlags(&ctx->copy_ev[k], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return CPB_ERR_CUDA;
        }
    cudaDeviceGetAttribute(&ctx->n_sm, cudaDevAttrMultiProcessorCount, device);
    *out = ctx;
    return CPB_OK;
}

int cpb_ctx_destroy(cpb_ctx* ctx) {
    if (!ctx) return CPB_OK;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        cudaSetDevice(ctx->device);
        if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
        for (auto& kv : ctx->bufs)
            if (kv.second.p) cudaFreeAsync(kv.second.p, ctx->stream);
        ctx->bufs.clear();
        cudaStreamSynchronize(ctx->stream);
        if (ctx->pinned) cudaFreeHost(ctx->pinned);
        for (auto e : ctx->event_pool) cudaEventDestroy(e);
        for (auto& p : ctx->pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        if (ctx->ev0) cudaEventDestroy(ctx->ev0);
        if (ctx->ev1) cudaEventDestroy(ctx->ev1);
        if (ctx->grow_ev) cudaEventDestroy(ctx->grow_ev);
        if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
        for (auto e : ctx->copy_ev)
            if (e) cudaEventDestroy(e);
        if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
    return CPB_OK;
}

const char* cpb_last_error(const cpb_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int cpb_ctx_set_profiling(cpb_ctx* ctx, int enable) {
    return guarded(ctx, [&]() -> int {
        resolve_kernel_events(ctx);
        ctx->profile = enable != 0;
        return CPB_OK;
    });
}

int cpb_ctx_set_wait_limit(cpb_ctx* ctx, int64_t polls) {
    return guarded(ctx, [&]() -> int {
        ctx->wait_limit = polls;
        return CPB_OK;
    });
}

int cpb_ctx_inject_fault(cpb_ctx* ctx, int32_t fault) {
    return guarded(ctx, [&]() -> int {
        if (fault != CPB_FAULT_NONE && fault != CPB_FAULT_HOLD_READY_STAR) throw ArgError{"unknown fault kind"};
        ctx->fault = fault;
        return CPB_OK;
    });
}

int cpb_ctx_kernel_stats(cpb_ctx* ctx, cpb_kernel_stat* out, int max_out, int* n_out, int64_t* launches, int reset) {
    return guarded(ctx, [&]() -> int {
        resolve_kernel_events(ctx);
        int k = 0;
        for (auto& kv : ctx->kstats) {
            if (out && k < max_out) {
                std::memset(&out[k], 0, sizeof(cpb_kernel_stat));
                std::strncpy(out[k].name, kv.first.c_str(), sizeof(out[k].name) - 1);
                out[k].launches = kv.second.launches;
                out[k].seconds = kv.second.seconds;
                out[k].bytes = kv.second.bytes;
            }
            ++k;
        }
        if (n_out) *n_out = k;
        if (launches) *launches = ctx->launches;
        if (reset) {
            ctx->kstats.clear();
            ctx->launches = 0;
        }
        return CPB_OK;
    });
}

int cpb_psf_upload(cpb_ctx* ctx, const cpb_psf_desc* d, cpb_psf** out) {
    return guarded(ctx, [&]() -> int {
        if (!d || !out) throw ArgError{"null argument"};
        *out = nullptr;
        auto* ps = new cpb_psf();
        DevPsf& dp = ps->dev;
        std::memset(&dp, 0, sizeof(dp));
        dp.kind = d->kind;
        dp.fwhm = d->fwhm;
        try {
            if (d->kind == CPB_PSF_CIRCULAR_GAUSSIAN) {
                if (!(std::isfinite(d->fwhm))) throw ArgError{"CircularGaussianPSF fwhm must be finite"};
                dp.n_nodes = 0;
                *out = ps;
                return CPB_OK;
            }
            if (d->kind != CPB_PSF_GRIDDED_IMAGE && d->kind != CPB_PSF_IMAGE) throw ArgError{"unsupported PSF kind"};
            const int nn = d->n_nodes;
            if (nn < 1) throw ArgError{"`psfs` must be non-empty"};
            if (d->kind == CPB_PSF_IMAGE && nn != 1) throw ArgError{"ImagePSF takes exactly one node"};
            if (nn > kMaxNodes) throw ArgError{"too many PSF nodes"};
            if (d->eltype != CPB_F32 && d->eltype != CPB_F64) throw ArgError{"unsupported PSF eltype"};
            // ImagePSF checks (empirical_models.jl:101-140)
            std::vector<double> h64;
            std::vector<DevNode> nodes(nn);
            int64_t off = 0;
            for (int k = 0; k < nn; ++k) {
                DevNode& nd = nodes[k];
                const int64_t nyd = d->node_ny[k], nxd = d->node_nx[k];
                if (nyd < 4 || nxd < 4) throw ArgError{"each axis of `data` must have at least 4 samples"};
                nd.ny = (int32_t)nyd;
                nd.nx = (int32_t)nxd;
                nd.off = off;
                nd.sx = (double)d->node_os[2 * k];
                nd.sy = (double)d->node_os[2 * k + 1];
                if (!(nd.sx > 0 && nd.sy > 0)) throw ArgError{"`oversampling` values must be positive"};
                nd.oy = d->node_origin[2 * k];
                nd.ox = d->node_origin[2 * k + 1];
                if (!std::isfinite(nd.oy) || !std::isfinite(nd.ox)) throw ArgError{"`origin` must be finite"};
                nd.fill = d->node_fill_value ? d->node_fill_value[k] : 0.0;
                const int64_t ne = nyd * nxd;
                const int64_t padded = (ne + 3) / 4 * 4;  // 32-byte (FP64) / 16-byte (FP32) node alignment
                h64.resize(off + padded, 0.0);
                for (int64_t q = 0; q < ne; ++q) {
                    double v = d->eltype == CPB_F64 ? ((const double*)d->node_data[k])[q]
                                                    : (double)((const float*)d->node_data[k])[q];
                    if (!std::isfinite(v)) throw ArgError{"all elements of `data` must be finite"};
                    h64[off + q] = v;
                }
                off += padded;
            }
            // node grid (gridded_psf.jl:106-134)
            std::vector<double> yg, xg;
            std::vector<int32_t> ig;
            if (nn == 1 || d->kind == CPB_PSF_IMAGE) {
                yg = {d->grid_y ? d->grid_y[0] : 0.0};
                xg = {d->grid_x ? d->grid_x[0] : 0.0};
                ig = {0};
            } else {
                for (int k = 0; k < nn; ++k)
                    if (!std::isfinite(d->grid_y[k]) || !std::isfinite(d->grid_x[k]))
                        throw ArgError{"`grid_y` and `grid_x` must be finite"};
                std::set<double> ys(d->grid_y, d->grid_y + nn), xs(d->grid_x, d->grid_x + nn);
                yg.assign(ys.begin(), ys.end());
                xg.assign(xs.begin(), xs.end());
                if (yg.size() < 2 || xg.size() < 2)
                    throw ArgError{
                        "`grid_y` and `grid_x` must each contain at least 2 unique values unless a single PSF is "
                        "supplied"};
                if ((size_t)nn != yg.size() * xg.size())
                    throw ArgError{"`grid_y`/`grid_x` positions do not form a complete rectangular grid"};
                ig.assign(yg.size() * xg.size(), -1);
                for (int k = 0; k < nn; ++k) {
                    size_t iy = std::lower_bound(yg.begin(), yg.end(), d->grid_y[k]) - yg.begin();
                    size_t ix = std::lower_bound(xg.begin(), xg.end(), d->grid_x[k]) - xg.begin();
                    int32_t& slot = ig[iy + ix * yg.size()];
                    if (slot != -1) throw ArgError{"duplicate node position"};
                    slot = k;
                }
            }
            std::vector<float> h32(h64.size());
            for (size_t q = 0; q < h64.size(); ++q) h32[q] = (float)h64[q];
            // polyphase copies (DevNode): samples regrouped by oversampling phase
            std::vector<double> pp;
            for (int k = 0; k < nn; ++k) {
                DevNode& nd = nodes[k];
                nd.isy = (int32_t)d->node_os[2 * k + 1];
                nd.isx = (int32_t)d->node_os[2 * k];
                nd.PY = (nd.ny + nd.isy - 1) / nd.isy;
                nd.PX = (nd.nx + nd.isx - 1) / nd.isx;
                nd.poff = (int64_t)pp.size();
                const int64_t plane = (int64_t)nd.PY * nd.PX;
                pp.resize(pp.size() + (size_t)(plane * nd.isy * nd.isx + 3) / 4 * 4, 0.0);
                for (int64_t kk = 0; kk < nd.nx; ++kk)
                    for (int64_t ii = 0; ii < nd.ny; ++ii)
                        pp[nd.poff + ((ii % nd.isy) + (kk % nd.isx) * nd.isy) * plane + ii / nd.isy + (kk / nd.isx) * nd.PY] =
                            h64[nd.off + ii + kk * nd.ny];
            }
            std::vector<double> lpp;
            for (int k = 0; k < nn; ++k) {
                DevNode& nd = nodes[k];
                nd.LPY = (nd.ny + 2 + nd.isy - 1) / nd.isy;
                nd.LPX = (nd.nx + 2 + nd.isx - 1) / nd.isx;
                nd.lpoff = (int64_t)lpp.size();
                const int64_t plane = (int64_t)nd.LPY * nd.LPX;
                lpp.resize(lpp.size() + (size_t)(plane * nd.isy * nd.isx + 3) / 4 * 4, 0.0);
                for (int64_t kk = 0; kk < nd.nx + 2; ++kk)
                    for (int64_t ii = 0; ii < nd.ny + 2; ++ii) {
                        const int64_t si = std::min<int64_t>(std::max<int64_t>(ii - 1, 0), nd.ny - 1);
                        const int64_t sk = std::min<int64_t>(std::max<int64_t>(kk - 1, 0), nd.nx - 1);
                        lpp[nd.lpoff + ((ii % nd.isy) + (kk % nd.isx) * nd.isy) * plane + ii / nd.isy +
                            (kk / nd.isx) * nd.LPY] = h64[nd.off + si + sk * nd.ny];
                    }
            }
            check(cudaMalloc(&ps->d_lpp64, sizeof(double) * std::max<size_t>(lpp.size(), 1)), "cudaMalloc");
            check(cudaMemcpy(ps->d_lpp64, lpp.data(), sizeof(double) * lpp.size(), cudaMemcpyHostToDevice), "h2d");
            std::vector<float> pp32(pp.size());
            for (size_t q = 0; q < pp.size(); ++q) pp32[q] = (float)pp[q];
            check(cudaMalloc(&ps->d_pp64, sizeof(double) * std::max<size_t>(pp.size(), 1)), "cudaMalloc");
            check(cudaMalloc(&ps->d_pp32, sizeof(float) * std::max<size_t>(pp.size(), 1)), "cudaMalloc");
            check(cudaMemcpy(ps->d_pp64, pp.data(), sizeof(double) * pp.size(), cudaMemcpyHostToDevice), "h2d");
            check(cudaMemcpy(ps->d_pp32, pp32.data(), sizeof(float) * pp32.size(), cudaMemcpyHostToDevice), "h2d");
            check(cudaMalloc(&ps->d_data64, sizeof(double) * h64.size()), "cudaMalloc");
            check(cudaMalloc(&ps->d_data32, sizeof(float) * h32.size()), "cudaMalloc");
            check(cudaMalloc(&ps->d_nodes, sizeof(DevNode) * nn), "cudaMalloc");
            check(cudaMalloc(&ps->d_ygrid, sizeof(double) * yg.size()), "cudaMalloc");
            check(cudaMalloc(&ps->d_xgrid, sizeof(double) * xg.size()), "cudaMalloc");
            check(cudaMalloc(&ps->d_index_grid, sizeof(int32_t) * ig.size()), "cudaMalloc");
            check(cudaMemcpy(ps->d_data64, h64.data(), sizeof(double) * h64.size(), cudaMemcpyHostToDevice), "h2d");
            check(cudaMemcpy(ps->d_data32, h32.data(), sizeof(float) * h32.size(), cudaMemcpyHostToDevice), "h2d");
            check(cudaMemcpy(ps->d_nodes, nodes.data(), sizeof(DevNode) * nn, cudaMemcpyHostToDevice), "h2d");
            check(cudaMemcpy(ps->d_ygrid, yg.data(), sizeof(double) * yg.size(), cudaMemcpyHostToDevice), "h2d");
            check(cudaMemcpy(ps->d_xgrid, xg.data(), sizeof(double) * xg.size(), cudaMemcpyHostToDevice), "h2d");
            check(cudaMemcpy(ps->d_index_grid, ig.data(), sizeof(int32_t) * ig.size(), cudaMemcpyHostToDevice), "h2d");
            dp.n_nodes = nn;
            dp.gny = (int32_t)yg.size();
            dp.gnx = (int32_t)xg.size();
            dp.data64 = ps->d_data64;
            dp.data32 = ps->d_data32;
            dp.pp64 = ps->d_pp64;
            dp.pp32 = ps->d_pp32;
            dp.lpp64 = ps->d_lpp64;
            dp.nodes = ps->d_nodes;
            dp.ygrid = ps->d_ygrid;
            dp.xgrid = ps->d_xgrid;
            dp.index_grid = ps->d_index_grid;
            dp.total_elems = (int64_t)h64.size();
            ps->h_nodes = nodes;
            ps->h_data64 = h64;
            ps->h_ygrid = yg;
            ps->h_xgrid = xg;
            ps->h_index_grid = ig;
            ps->smem_bytes64 = (int64_t)h64.size() * 8;
            ps->smem_bytes32 = (int64_t)h64.size() * 4;
        } catch (...) {
            cudaFree(ps->d_data64);
            cudaFree(ps->d_data32);
            cudaFree(ps->d_pp64);
            cudaFree(ps->d_pp32);
            cudaFree(ps->d_lpp64);
            cudaFree(ps->d_nodes);
            cudaFree(ps->d_ygrid);
            cudaFree(ps->d_xgrid);
            cudaFree(ps->d_index_grid);
            delete ps;
            throw;
        }
        *out = ps;
        return CPB_OK;
    });
}

int cpb_psf_free(cpb_ctx* ctx, cpb_psf* ps) {
    if (!ps) return CPB_OK;
    return guarded(ctx, [&]() -> int {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ps->d_data64);
        cudaFree(ps->d_data32);
        cudaFree(ps->d_pp64);
        cudaFree(ps->d_pp32);
        cudaFree(ps->d_lpp64);
        cudaFree(ps->d_nodes);
        cudaFree(ps->d_ygrid);
        cudaFree(ps->d_xgrid);
        cudaFree(ps->d_index_grid);
        delete ps;
        return CPB_OK;
    });
}

int cpb_fit_simultaneous_device(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* params, const void* d_image,
                                int32_t eltype, int64_t ny, int64_t nx, const void* d_inv_var,
                                const void* d_background, int64_t n, const double* d_y0, const double* d_x0,
                                const double* d_flux0, cpb_sim_result* out) {
    return guarded(ctx, [&]() -> int {
        if (!psf || !params || !out || (n > 0 && (!d_y0 || !d_x0 || !d_flux0)) || !d_image)
            throw ArgError{"null argument"};
        return fit_simultaneous_dev(ctx, psf, params, d_image, eltype, ny, nx, d_inv_var, d_background, n, d_y0, d_x0,
                                    d_flux0, out);
    });
}

int cpb_fit_simultaneous(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* params, const void* image,
                         int32_t eltype, int64_t ny, int64_t nx, const void* inv_var, const void* background,
                         int64_t n, const double* y0, const double* x0, const double* flux0, cpb_sim_result* out) {
    return guarded(ctx, [&]() -> int {
        if (!psf || !params || !out || !image || (n > 0 && (!y0 || !x0 || !flux0))) throw ArgError{"null argument"};
        if (eltype != CPB_F32 && eltype != CPB_F64) throw ArgError{"unsupported image eltype"};
        if (ny <= 0 || nx <= 0) throw ArgError{"image must be non-empty"};
        const size_t esz = eltype == CPB_F64 ? 8 : 4;
        const size_t bytes = esz * (size_t)ny * (size_t)nx;
        cudaStream_t st = ctx->stream;
        void* d_img = scratch(ctx, "in_image", bytes);
        void* d_iv = inv_var ? scratch(ctx, "in_inv_var", bytes) : nullptr;
        void* d_bk = background ? scratch(ctx, "in_background", bytes) : nullptr;
        double* d_y = (double*)scratch(ctx, "in_y", sizeof(double) * std::max<int64_t>(n, 1));
        double* d_x = (double*)scratch(ctx, "in_x", sizeof(double) * std::max<int64_t>(n, 1));
        double* d_f = (double*)scratch(ctx, "in_flux", sizeof(double) * std::max<int64_t>(n, 1));
        check(cudaMemcpyAsync(d_img, image, bytes, cudaMemcpyHostToDevice, st), "h2d image");
        if (d_iv) check(cudaMemcpyAsync(d_iv, inv_var, bytes, cudaMemcpyHostToDevice, st), "h2d inv_var");
        if (d_bk) check(cudaMemcpyAsync(d_bk, background, bytes, cudaMemcpyHostToDevice, st), "h2d background");
        if (n > 0) {
            check(cudaMemcpyAsync(d_y, y0, sizeof(double) * n, cudaMemcpyHostToDevice, st), "h2d y");
            check(cudaMemcpyAsync(d_x, x0, sizeof(double) * n, cudaMemcpyHostToDevice, st), "h2d x");
            check(cudaMemcpyAsync(d_f, flux0, sizeof(double) * n, cudaMemcpyHostToDevice, st), "h2d flux");
        }
        return fit_simultaneous_dev(ctx, psf, params, d_img, eltype, ny, nx, d_iv, d_bk, n, d_y, d_x, d_f, out);
    });
}

int cpb_fit_simultaneous_batch_device(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* params,
                                      int64_t n_groups, const int64_t* d_pix_offsets, const int32_t* d_ny,
                                      const int32_t* d_nx, const void* d_pixels, int32_t eltype,
                                      const void* d_inv_var, const void* d_background,
                                      const int64_t* d_star_offsets, const double* d_y0, const double* d_x0,
                                      const double* d_flux0, int64_t total_pixels, cpb_group_result* out) {
    return guarded(ctx, [&]() -> int {
        if (!psf || !params || !out || (n_groups > 0 && (!d_pix_offsets || !d_ny || !d_nx || !d_pixels ||
                                                         !d_star_offsets || !d_y0 || !d_x0 || !d_flux0)))
            throw ArgError{"null argument"};
        return fit_groups_dev(ctx, psf, params, n_groups, d_pix_offsets, d_ny, d_nx, d_pixels, eltype, d_inv_var,
                              d_background, d_star_offsets, d_y0, d_x0, d_flux0, total_pixels, out, nullptr,
                              nullptr, nullptr, nullptr);
    });
}

int cpb_fit_simultaneous_batch(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* params, int64_t n_groups,
                               const int64_t* pix_offsets, const int32_t* ny, const int32_t* nx, const void* pixels,
                               int32_t eltype, const void* inv_var, const void* background,
                               const int64_t* star_offsets, const double* y0, const double* x0, const double* flux0,
                               cpb_group_result* out) {
    return guarded(ctx, [&]() -> int {
        if (!psf || !params || !out || n_groups < 0 || (n_groups > 0 && (!pix_offsets || !ny || !nx || !pixels ||
                                                                          !star_offsets || !y0 || !x0 || !flux0)))
            throw ArgError{"null argument"};
        if (eltype != CPB_F32 && eltype != CPB_F64) throw ArgError{"unsupported image eltype"};
        if (!out->y || !out->x || !out->flux || !out->y_err || !out->x_err || !out->flux_err || !out->converged ||
            !out->valid || !out->n_iter || !out->n_passes || !out->n_failed || !out->status)
            throw ArgError{"null output array"};
        const int64_t G = n_groups;
        if (G == 0) {
            out->n_kernel_groups = out->n_routed_groups = 0;
            out->device_seconds = 0;
            return CPB_OK;
        }
        int64_t npx = 0;
        for (int64_t g = 0; g < G; ++g) {
            if (ny[g] <= 0 || nx[g] <= 0) throw ArgError{"group image size out of range"};
            if (pix_offsets[g] < 0) throw ArgError{"pixel offsets must be non-negative"};
            npx = std::max<int64_t>(npx, pix_offsets[g] + (int64_t)ny[g] * nx[g]);
        }
        if (star_offsets[0] != 0) throw ArgError{"star_offsets[0] must be 0"};
        for (int64_t g = 0; g < G; ++g)
            if (star_offsets[g + 1] < star_offsets[g]) throw ArgError{"star_offsets must be non-decreasing"};
        const int64_t ns = star_offsets[G];
        const size_t esz = eltype == CPB_F64 ? 8 : 4;
        cudaStream_t st = ctx->stream;
        auto up = [&](const char* name, const void* src, size_t bytes) -> void* {
            void* d = scratch(ctx, name, std::max<size_t>(bytes, 8));
            if (src && bytes) check(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, st), "h2d batch input");
            return d;
        };
        const void* d_pix = up("gb_pix", pixels, esz * npx);
        const void* d_iv = inv_var ? up("gb_iv", inv_var, esz * npx) : nullptr;
        const void* d_bk = background ? up("gb_bkg", background, esz * npx) : nullptr;
        const int64_t* d_off = (const int64_t*)up("gb_off", pix_offsets, 8 * G);
        const int32_t* d_ny = (const int32_t*)up("gb_ny", ny, 4 * G);
        const int32_t* d_nx = (const int32_t*)up("gb_nx", nx, 4 * G);
        const int64_t* d_so = (const int64_t*)up("gb_soff", star_offsets, 8 * (G + 1));
        const double* d_y = (const double*)up("gb_y0", y0, 8 * ns);
        const double* d_x = (const double*)up("gb_x0", x0, 8 * ns);
        const double* d_f = (const double*)up("gb_f0", flux0, 8 * ns);
        // device outputs
        cpb_group_result d = *out;
        auto dout = [&](const char* name, void* host, size_t bytes) -> void* {
            return host ? scratch(ctx, name, std::max<size_t>(bytes, 8)) : nullptr;
        };
        d.y = (double*)dout("gb_o_y", out->y, 8 * ns);
        d.x = (double*)dout("gb_o_x", out->x, 8 * ns);
        d.flux = (double*)dout("gb_o_f", out->flux, 8 * ns);
        d.y_err = (double*)dout("gb_o_ey", out->y_err, 8 * ns);
        d.x_err = (double*)dout("gb_o_ex", out->x_err, 8 * ns);
        d.flux_err = (double*)dout("gb_o_ef", out->flux_err, 8 * ns);
        d.converged = (uint8_t*)dout("gb_o_cv", out->converged, ns);
        d.valid = (uint8_t*)dout("gb_o_va", out->valid, ns);
        d.n_iter = (int32_t*)dout("gb_o_it", out->n_iter, 4 * ns);
        d.chisq = (double*)dout("gb_o_chi", out->chisq, 8 * ns);
        d.qfit = (double*)dout("gb_o_q1", out->qfit, 8 * ns);
        d.qfit_expected = (double*)dout("gb_o_q2", out->qfit_expected, 8 * ns);
        d.qfit_z = (double*)dout("gb_o_q3", out->qfit_z, 8 * ns);
        d.crowding = (double*)dout("gb_o_cr", out->crowding, 8 * ns);
        d.spread_model = (double*)dout("gb_o_sm", out->spread_model, 8 * ns);
        d.spread_model_err = (double*)dout("gb_o_sme", out->spread_model_err, 8 * ns);
        d.residual = (double*)dout("gb_o_res", out->residual, 8 * npx);
        d.n_passes = (int32_t*)dout("gb_o_np", out->n_passes, 4 * G);
        d.n_failed = (int32_t*)dout("gb_o_nf", out->n_failed, 4 * G);
        d.status = (int32_t*)dout("gb_o_st", out->status, 4 * G);
        d.error_kind = (int32_t*)dout("gb_o_ek", out->error_kind, 4 * G);
        d.n_active = (int32_t*)dout("gb_o_na", out->n_active, 4 * G);
        d.n_union = (int32_t*)dout("gb_o_nu", out->n_union, 4 * G);
        d.n_trials = (int32_t*)dout("gb_o_nt", out->n_trials, 4 * G);
        d.n_lsqr_iters = (int32_t*)dout("gb_o_nl", out->n_lsqr_iters, 4 * G);
        fit_groups_dev(ctx, psf, params, G, d_off, d_ny, d_nx, d_pix, eltype, d_iv, d_bk, d_so, d_y, d_x, d_f, npx, &d,
                       pix_offsets, ny, nx, star_offsets);
        auto down = [&](void* host, const void* dev, size_t bytes) {
            if (host && bytes) check(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, st), "d2h batch output");
        };
        down(out->y, d.y, 8 * ns);
        down(out->x, d.x, 8 * ns);
        down(out->flux, d.flux, 8 * ns);
        down(out->y_err, d.y_err, 8 * ns);
        down(out->x_err, d.x_err, 8 * ns);
        down(out->flux_err, d.flux_err, 8 * ns);
        down(out->converged, d.converged, ns);
        down(out->valid, d.valid, ns);
        down(out->n_iter, d.n_iter, 4 * ns);
        down(out->chisq, d.chisq, 8 * ns);
        down(out->qfit, d.qfit, 8 * ns);
        down(out->qfit_expected, d.qfit_expected, 8 * ns);
        down(out->qfit_z, d.qfit_z, 8 * ns);
        down(out->crowding, d.crowding, 8 * ns);
        down(out->spread_model, d.spread_model, 8 * ns);
        down(out->spread_model_err, d.spread_model_err, 8 * ns);
        down(out->residual, d.residual, 8 * npx);
        down(out->n_passes, d.n_passes, 4 * G);
        down(out->n_failed, d.n_failed, 4 * G);
        down(out->status, d.status, 4 * G);
        down(out->error_kind, d.error_kind, 4 * G);
        down(out->n_active, d.n_active, 4 * G);
        down(out->n_union, d.n_union, 4 * G);
        down(out->n_trials, d.n_trials, 4 * G);
        down(out->n_lsqr_iters, d.n_lsqr_iters, 4 * G);
        check(cudaStreamSynchronize(st), "sync");
        out->n_kernel_groups = d.n_kernel_groups;
        out->n_routed_groups = d.n_routed_groups;
        out->device_seconds = d.device_seconds;
        return CPB_OK;
    });
}

int cpb_fit_all_stars(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* params, double fit_rad,
                      int32_t n_passes, double spread_model_fwhm, const void* image, int32_t eltype, int64_t ny,
                      int64_t nx, const void* inv_var, int64_t n, const double* init, cpb_multipass_result* out) {
    return guarded(ctx, [&]() -> int {
        if (!psf || !params || !out || !image || (n > 0 && !init)) throw ArgError{"null argument"};
        if (eltype != CPB_F32 && eltype != CPB_F64) throw ArgError{"unsupported image eltype"};
        if (ny <= 0 || nx <= 0) throw ArgError{"image must be non-empty"};
        const size_t bytes = (eltype == CPB_F64 ? 8 : 4) * (size_t)ny * (size_t)nx;
        void* d_img = scratch(ctx, "mp_in_image", bytes);
        void* d_iv = inv_var ? scratch(ctx, "mp_in_inv_var", bytes) : nullptr;
        check(cudaMemcpyAsync(d_img, image, bytes, cudaMemcpyHostToDevice, ctx->stream), "h2d image");
        if (d_iv) check(cudaMemcpyAsync(d_iv, inv_var, bytes, cudaMemcpyHostToDevice, ctx->stream), "h2d inv_var");
        return fit_all_stars_dev(ctx, psf, params, fit_rad, n_passes, spread_model_fwhm, d_img, eltype, ny, nx, d_iv,
                                 n, init, out);
    });
}

int cpb_fit_lm_batch(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* params, int64_t n_cutouts,
                     const int64_t* offsets, const int32_t* ny, const int32_t* nx, const int32_t* y_origin,
                     const int32_t* x_origin, const void* pixels, int32_t eltype, const void* inv_var,
                     const double* init, cpb_lm_result* out) {
    return guarded(ctx, [&]() -> int {
        if (!psf || !params || !out || (n_cutouts > 0 && (!offsets || !ny || !nx || !y_origin || !x_origin ||
                                                          !pixels || !init || !out->params || !out->iterations ||
                                                          !out->status)))
            throw ArgError{"null argument"};
        return fit_lm_batch(ctx, psf, params, n_cutouts, offsets, ny, nx, y_origin, x_origin, pixels, eltype, inv_var,
                            init, out);
    });
}

int cpb_fit_lm_batch_device(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* params, int64_t n_cutouts,
                            const int64_t* d_offsets, const int32_t* d_ny, const int32_t* d_nx,
                            const int32_t* d_y_origin, const int32_t* d_x_origin, const void* d_pixels,
                            int32_t eltype, const void* d_inv_var, const double* d_init, int64_t total_pixels,
                            cpb_lm_result* out) {
    return guarded(ctx, [&]() -> int {
        if (!psf || !params || !out || (n_cutouts > 0 && (!d_offsets || !d_ny || !d_nx || !d_y_origin ||
                                                          !d_x_origin || !d_pixels || !d_init || !out->status)))
            throw ArgError{"null argument"};
        return fit_lm_batch_device(ctx, psf, params, n_cutouts, d_offsets, d_ny, d_nx, d_y_origin, d_x_origin,
                                   d_pixels, eltype, d_inv_var, d_init, total_pixels, out);
    });
}

}  // extern "C"
