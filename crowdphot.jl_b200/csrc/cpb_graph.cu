// cpb_graph.cu -- one captured CUDA graph for a mixed batch of fit_star cutouts
// and star groups, and the launch-shape tuner that picks its kernels' shapes.
//
// The graph forks the context stream onto a side stream: the fit_star branch
// (work-queue reset + persistent k_lm_t) and the group branch (work-queue
// reset + persistent k_groups) run concurrently and join before the graph
// ends.  A replay is one cudaGraphLaunch; nothing is read back in between.
//
// Tuner: candidates are timed with CUDA events on the bound batch itself, one
// launch at a time, after one untimed run of the default shape; the fastest
// shape is kept -- for the fit_star kernel, blocks per SM and the node in
// shared memory or not; for each bucket of similar-size groups, the block size.  Choices are cached in a text file, one line per
// (device, kernel signature): "<device>|<signature>\t<a> <b> <ms>".
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "cpb_internal.cuh"

struct cpb_batch_graph {
    cpb::LMBatch* lm = nullptr;
    cpb::GroupBatch* grp = nullptr;
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, t0 = nullptr, t1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;
    cpb_tune_info info{};
};

namespace cpb {
namespace {

std::string device_name(int dev) {
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) {
        cudaGetLastError();
        return "cuda";
    }
    return p.name;
}

std::map<std::string, std::string> read_cache(const std::string& path) {
    std::map<std::string, std::string> m;
    if (path.empty()) return m;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        const size_t t = line.find('\t');
        if (t != std::string::npos) m[line.substr(0, t)] = line.substr(t + 1);
    }
    return m;
}

// Rewrites the cache with `key` set (write to a temporary file, then rename).
void write_cache(const std::string& path, const std::string& key, const std::string& value) {
    if (path.empty()) return;
    auto m = read_cache(path);
    m[key] = value;
    const std::string tmp = path + ".tmp";
    {
        std::ofstream f(tmp, std::ios::trunc);
        if (!f) return;  // an unwritable cache only costs a re-tune next time
        for (auto& kv : m) f << kv.first << '\t' << kv.second << '\n';
    }
    std::rename(tmp.c_str(), path.c_str());
}

template <typename F>
double time_ms(cpb_ctx* ctx, F&& launch) {
    cudaStream_t st = ctx->stream;
    check(cudaEventRecord(ctx->ev0, st), "event");
    launch();
    check(cudaEventRecord(ctx->ev1, st), "event");
    check(cudaStreamSynchronize(st), "sync");
    float ms = 0;
    check(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1), "elapsed");
    return ms;
}

}  // namespace
}  // namespace cpb

using namespace cpb;

extern "C" {

int cpb_batch_graph_create(cpb_ctx* ctx, const cpb_psf* psf, const cpb_lm_params* lm_params, int64_t n_cutouts,
                           const int64_t* d_offsets, const int32_t* d_ny, const int32_t* d_nx,
                           const int32_t* d_y_origin, const int32_t* d_x_origin, const void* d_pixels,
                           int32_t lm_eltype, const void* d_inv_var, const double* d_init, int64_t lm_total_pixels,
                           const cpb_lm_result* d_lm_out, const cpb_sim_params* sim_params, int64_t n_groups,
                           const int64_t* d_pix_offsets, const int32_t* d_gny, const int32_t* d_gnx,
                           const void* d_gpixels, int32_t g_eltype, const void* d_ginv_var,
                           const void* d_gbackground, const int64_t* d_star_offsets, const double* d_y0,
                           const double* d_x0, const double* d_flux0, int64_t g_total_pixels,
                           const cpb_group_result* d_g_out, int32_t autotune, const char* cache_path,
                           cpb_batch_graph** out, cpb_tune_info* info) {
    return guarded(ctx, [&]() -> int {
        if (!psf || !out) throw ArgError{"null argument"};
        *out = nullptr;
        if (n_cutouts < 0 || n_groups < 0) throw ArgError{"batch sizes must be >= 0"};
        if (n_cutouts > 0 && !lm_params) throw ArgError{"null lm_params"};
        if (n_groups > 0 && !sim_params) throw ArgError{"null sim_params"};
        if (autotune < 0 || autotune > 2) throw ArgError{"autotune must be 0, 1 or 2"};
        auto* g = new cpb_batch_graph();
        const bool prof = ctx->profile;
        try {
            if (n_cutouts > 0)
                g->lm = lm_batch_create(ctx, psf, lm_params, n_cutouts, d_offsets, d_ny, d_nx, d_y_origin, d_x_origin,
                                        d_pixels, lm_eltype, d_inv_var, d_init, lm_total_pixels, d_lm_out);
            if (n_groups > 0)
                g->grp = group_batch_create(ctx, psf, sim_params, n_groups, d_pix_offsets, d_gny, d_gnx, d_gpixels,
                                            g_eltype, d_ginv_var, d_gbackground, d_star_offsets, d_y0, d_x0, d_flux0,
                                            g_total_pixels, d_g_out);
            // ---- launch shapes
            cpb_tune_info& ti = g->info;
            ti.lm_blocks_per_sm = 2;
            ti.lm_node_in_smem = g->lm && lm_batch_smem_possible(g->lm) ? 1 : 0;
            ti.grp_threads = 0;
            ti.grp_blocks_per_sm = 0;
            ti.from_cache = 0;
            ti.n_timed = 0;
            if (autotune) {
                std::string path = cache_path ? cache_path : "";
                if (path.empty() && std::getenv("CPB_TUNE_CACHE")) path = std::getenv("CPB_TUNE_CACHE");
                const auto cache = autotune == 1 ? read_cache(path) : std::map<std::string, std::string>();
                const std::string dev = device_name(ctx->device);
                ctx->profile = false;
                int cached = 0, halves = 0;
                if (g->lm) {
                    ++halves;
                    const std::string key = dev + "|" + lm_batch_signature(g->lm);
                    auto it = cache.find(key);
                    int a = 0, b = 0;
                    double ms = 0;
                    if (it != cache.end() && std::sscanf(it->second.c_str(), "%d %d %lf", &a, &b, &ms) == 3 &&
                        (a == 1 || a == 2) && (b == 0 || (b == 1 && lm_batch_smem_possible(g->lm)))) {
                        ti.lm_blocks_per_sm = a;
                        ti.lm_node_in_smem = b;
                        ti.lm_ms = ms;
                        ++cached;
                    } else {
                        lm_batch_enqueue(ctx, g->lm, ctx->stream, ti.lm_blocks_per_sm, ti.lm_node_in_smem);  // warm
                        double best = 1e300;
                        for (int bps : {2, 1})
                            for (int sm : {1, 0}) {
                                if (sm && !lm_batch_smem_possible(g->lm)) continue;
                                const double t =
                                    time_ms(ctx, [&] { lm_batch_enqueue(ctx, g->lm, ctx->stream, bps, sm); });
                                ++ti.n_timed;
                                if (t < best) {
                                    best = t;
                                    ti.lm_blocks_per_sm = bps;
                                    ti.lm_node_in_smem = sm;
                                }
                            }
                        ti.lm_ms = best;
                        char v[64];
                        std::snprintf(v, sizeof(v), "%d %d %.4f", ti.lm_blocks_per_sm, ti.lm_node_in_smem, best);
                        write_cache(path, key, v);
                    }
                }
                if (g->grp) {
                    // one block size per bucket of similar group sizes
                    const int nb = group_batch_buckets(g->grp);
                    double total_ms = 0;
                    for (int k = 0; k < nb; ++k) {
                        ++halves;
                        const std::string key = dev + "|" + group_batch_signature(g->grp, k);
                        auto it = cache.find(key);
                        int a = 0, b = 0;
                        double ms = 0;
                        if (it != cache.end() && std::sscanf(it->second.c_str(), "%d %d %lf", &a, &b, &ms) >= 2 &&
                            (a == 64 || a == 128 || a == 256)) {
                            group_batch_set_threads(g->grp, k, a);
                            total_ms += ms;
                            ++cached;
                            continue;
                        }
                        group_batch_enqueue(ctx, g->grp, ctx->stream, k, 0);  // warm
                        double best = 1e300;
                        int best_nt = group_batch_threads(g->grp, k);
                        for (int nt : {64, 128, 256}) {
                            const double t = time_ms(ctx, [&] { group_batch_enqueue(ctx, g->grp, ctx->stream, k, nt); });
                            ++ti.n_timed;
                            if (t < best) {
                                best = t;
                                best_nt = nt;
                            }
                        }
                        group_batch_set_threads(g->grp, k, best_nt);
                        total_ms += best;
                        char v[64];
                        std::snprintf(v, sizeof(v), "%d %d %.4f", best_nt,
                                      group_batch_occupancy(g->grp, k, best_nt), best);
                        write_cache(path, key, v);
                    }
                    ti.grp_ms = total_ms;
                }
                ti.from_cache = (halves > 0 && cached == halves) ? 1 : 0;
                ctx->profile = prof;
            }
            // ---- capture: fork, the two branches, join
            check(cudaStreamCreateWithFlags(&g->side, cudaStreamNonBlocking), "stream");
            check(cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming), "event");
            check(cudaEventCreateWithFlags(&g->join, cudaEventDisableTiming), "event");
            check(cudaEventCreate(&g->t0), "event");
            check(cudaEventCreate(&g->t1), "event");
            // attribute calls happen here, outside the capture
            if (g->lm) lm_batch_enqueue(ctx, g->lm, ctx->stream, ti.lm_blocks_per_sm, ti.lm_node_in_smem);
            if (g->grp) {
                group_batch_enqueue(ctx, g->grp, ctx->stream, -1, 0);
                const int nb = group_batch_buckets(g->grp);
                if (nb > 0) {  // buckets are ordered by group size: report the largest groups' launch
                    ti.grp_threads = group_batch_threads(g->grp, nb - 1);
                    ti.grp_blocks_per_sm = group_batch_occupancy(g->grp, nb - 1, ti.grp_threads);
                }
            }
            check(cudaStreamSynchronize(ctx->stream), "sync");
            ctx->profile = false;
            const int64_t l0 = ctx->launches;
            check(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed), "begin capture");
            try {
                check(cudaEventRecord(g->fork, ctx->stream), "fork");
                check(cudaStreamWaitEvent(g->side, g->fork, 0), "fork wait");
                if (g->lm) lm_batch_enqueue(ctx, g->lm, ctx->stream, ti.lm_blocks_per_sm, ti.lm_node_in_smem);
                if (g->grp) group_batch_enqueue(ctx, g->grp, g->side, -1, 0);
                check(cudaEventRecord(g->join, g->side), "join");
                check(cudaStreamWaitEvent(ctx->stream, g->join, 0), "join wait");
            } catch (...) {
                cudaGraph_t dead = nullptr;
                cudaStreamEndCapture(ctx->stream, &dead);
                if (dead) cudaGraphDestroy(dead);
                cudaGetLastError();
                throw;
            }
            check(cudaStreamEndCapture(ctx->stream, &g->graph), "end capture");
            g->kernels = (int)(ctx->launches - l0);
            ctx->launches = l0;  // counted per replay instead
            ctx->profile = prof;
            check(cudaGraphInstantiate(&g->exec, g->graph, 0), "graph instantiate");
        } catch (...) {
            ctx->profile = prof;
            if (g->exec) cudaGraphExecDestroy(g->exec);
            if (g->graph) cudaGraphDestroy(g->graph);
            for (cudaEvent_t e : {g->fork, g->join, g->t0, g->t1})
                if (e) cudaEventDestroy(e);
            if (g->side) cudaStreamDestroy(g->side);
            lm_batch_destroy(g->lm);
            group_batch_destroy(g->grp);
            delete g;
            throw;
        }
        if (info) *info = g->info;
        *out = g;
        return CPB_OK;
    });
}

int cpb_batch_graph_launch(cpb_ctx* ctx, cpb_batch_graph* g, double* device_seconds) {
    return guarded(ctx, [&]() -> int {
        if (!g) throw ArgError{"null graph"};
        cudaStream_t st = ctx->stream;
        check(cudaEventRecord(g->t0, st), "event");
        check(cudaGraphLaunch(g->exec, st), "graph launch");
        check(cudaEventRecord(g->t1, st), "event");
        check(cudaStreamSynchronize(st), "sync");
        ctx->launches += g->kernels;
        if (device_seconds) {
            float ms = 0;
            check(cudaEventElapsedTime(&ms, g->t0, g->t1), "elapsed");
            *device_seconds = ms * 1e-3;
        }
        return CPB_OK;
    });
}

int cpb_batch_graph_destroy(cpb_ctx* ctx, cpb_batch_graph* g) {
    if (!g) return CPB_OK;
    return guarded(ctx, [&]() -> int {
        cudaStreamSynchronize(ctx->stream);
        if (g->exec) cudaGraphExecDestroy(g->exec);
        if (g->graph) cudaGraphDestroy(g->graph);
        for (cudaEvent_t e : {g->fork, g->join, g->t0, g->t1})
            if (e) cudaEventDestroy(e);
        if (g->side) cudaStreamDestroy(g->side);
        lm_batch_destroy(g->lm);
        group_batch_destroy(g->grp);
        delete g;
        return CPB_OK;
    });
}

}  // extern "C"
