// cpb_noalloc.cu -- the simultaneous fit without any device allocation.
//
// Some callers cannot call cudaMalloc while they fit: Julia hosts whose device
// memory belongs to CUDA.jl's pool allocator (or a PyTorch process whose
// memory belongs to its caching allocator), where a direct cudaMalloc behind
// the pool's back can fail once the pool holds most of the GPU or fragment
// what it holds, and latency-critical loops that cannot take the implicit
// device synchronisation of cudaMalloc / cudaFree.  For them
// cpb_fit_simultaneous_device_noalloc runs the same fit as
// cpb_fit_simultaneous_device, but every scratch buffer (stamps, residuals,
// LSQR vectors, tile lists, sort temporaries, reduction partials) is carved
// from one file-scope device array of kNoAllocScratchBytes that the library
// holds on every GPU that loads it, for the life of the process.
//
// Set-up: the array's device address is looked up once per device with
// cudaGetSymbolAddress (in host code the symbol is only a host-side stand-in,
// never a device address).  The first call of the entry point on a device
// does that look-up, so it should come before any stream capture.  The
// address is kept for the life of the process: after a cudaDeviceReset of that
// device the module is loaded again and the kept address is stale, so do not
// call this entry point after resetting a device it has used.
//
// Sizes: a field is refused with CPB_ERR_ARGUMENT ("too large for the
// no-allocation entry point") when its scratch bound (sim_scratch_bound, every
// catalogue star counted as active) exceeds the array; with model_rad = :auto
// the model stamps are checked again once the per-star radii are known, before
// the outer loop starts.
//
// Sharing: every call uses the same array and finds the previous call's
// contents there; the fit clears everything that must start at zero.  Calls
// whose GPU work overlaps (two host threads, two contexts on one device)
// race on the array: serialise them.
#include <cstring>
#include <mutex>
#include <string>

#include "cpb_internal.cuh"

namespace cpb {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;  // 64 MiB per device

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_setup_mu;
void* g_scratch_addr[256] = {nullptr};

// Device address of g_noalloc_scratch on `device` (which must be current).
void* noalloc_base(int device) {
    if (device < 0 || device >= 256) throw ArgError{"device ordinal out of range"};
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            throw CudaError{e == cudaSuccess ? cudaErrorInvalidSymbol : e,
                            "cudaGetSymbolAddress(no-allocation scratch)"};
        }
        g_scratch_addr[device] = p;
    }
    return g_scratch_addr[device];
}

}  // namespace

void* arena_carve(cpb_ctx::Arena* a, const char* name, size_t bytes) {
    auto it = a->slots.find(name);
    if (it != a->slots.end() && it->second.second >= bytes) return a->base + it->second.first;
    const size_t off = (a->used + 255) & ~size_t(255);
    const size_t want = std::max<size_t>(bytes, 256);
    if (off + want > a->cap)
        throw ArgError{std::string("the fit needs more scratch than the no-allocation entry point's ") +
                       std::to_string(a->cap >> 20) + " MiB static region (buffer '" + name +
                       "'); use cpb_fit_simultaneous_device for this field"};
    a->used = off + want;
    a->slots[name] = {off, want};
    return a->base + off;
}

}  // namespace cpb

using namespace cpb;

extern "C" int cpb_fit_simultaneous_device_noalloc(cpb_ctx* ctx, const cpb_psf* psf, const cpb_sim_params* params,
                                                   const void* d_image, int32_t eltype, int64_t ny, int64_t nx,
                                                   const void* d_inv_var, const void* d_background, int64_t n,
                                                   const double* d_y0, const double* d_x0, const double* d_flux0,
                                                   cpb_sim_result* out) {
    if (!ctx) return CPB_ERR_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->err.clear();
    cpb_ctx::Arena arena;
    try {
        check(cudaSetDevice(ctx->device), "cudaSetDevice");
        if (!psf || !params || !out || !d_image || (n > 0 && (!d_y0 || !d_x0 || !d_flux0)))
            throw ArgError{"null argument"};
        if (ny <= 0 || nx <= 0) throw ArgError{"image must be non-empty"};
        const size_t need = sim_scratch_bound(params, ny, nx, n, out->dbg_pixels != nullptr);
        if (need > kNoAllocScratchBytes)
            throw ArgError{"field too large for the no-allocation entry point: needs about " +
                           std::to_string((need + (1 << 20) - 1) >> 20) + " MiB of scratch, the static region holds " +
                           std::to_string(kNoAllocScratchBytes >> 20) + " MiB"};
        arena.base = (char*)noalloc_base(ctx->device);
        arena.cap = kNoAllocScratchBytes;
        ctx->arena = &arena;
        int rc = fit_simultaneous_dev(ctx, psf, params, d_image, eltype, ny, nx, d_inv_var, d_background, n, d_y0,
                                      d_x0, d_flux0, out);
        ctx->arena = nullptr;
        return rc;
    } catch (const ArgError& e) {
        ctx->arena = nullptr;
        ctx->err = e.msg;
        return CPB_ERR_ARGUMENT;
    } catch (const OomError& e) {
        ctx->arena = nullptr;
        ctx->err = e.msg;
        return CPB_ERR_OOM;
    } catch (const CudaError& e) {
        ctx->arena = nullptr;
        ctx->err = std::string(e.what) + ": " + cudaGetErrorString(e.e);
        return CPB_ERR_CUDA;
    } catch (const std::exception& e) {
        ctx->arena = nullptr;
        ctx->err = e.what();
        return CPB_ERR_INTERNAL;
    }
}
