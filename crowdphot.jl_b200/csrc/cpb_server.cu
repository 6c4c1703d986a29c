// cpb_server.cu -- continuous batching of fit_all_stars_simultaneous requests.
//
// One worker thread per slot; each slot owns a full context (stream, copy
// stream, events, grow-only device scratch), so requests running in different
// slots never share device state and their kernels overlap on the GPU.  PSFs
// are uploaded once and read by every slot.  Admission happens under one
// mutex: an idle worker takes the first queued request (arrival order) whose
// device-memory estimate fits the budget next to what the other slots hold;
// when only memory cached by idle slots stands in the way, that cache is
// released first.  Host code only: every fit goes through cpb_fit_simultaneous.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cpb_internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t id = 0;
    int32_t psf_id = 0;
    cpb_sim_params params{};
    const void* image = nullptr;
    int32_t eltype = CPB_F64;
    int64_t ny = 0, nx = 0;
    const void* inv_var = nullptr;
    const void* background = nullptr;
    int64_t n = 0;
    const double *y0 = nullptr, *x0 = nullptr, *f0 = nullptr;
    cpb_sim_result* out = nullptr;
    int64_t est = 0;
    int32_t state = CPB_REQ_QUEUED;
    int32_t status = 0;
    int32_t slot = -1;
    double device_seconds = 0;
    std::string error;
    Clock::time_point t_submit, t_start, t_end;
};

struct Slot {
    cpb_ctx* ctx = nullptr;
    std::thread worker;
    std::shared_ptr<Request> running;
};

// Device bytes one request's fit holds at its peak (fit_sim_impl's scratch,
// cpb_sim.cu): per-pixel vectors, stamp derivatives and model stamps of every
// star, per-star solver state and the region lists, plus the staged inputs.
int64_t estimate_bytes(const cpb_sim_params& P, int32_t eltype, int64_t ny, int64_t nx, int64_t n) {
    const int64_t npix = ny * nx;
    const int64_t esz = eltype == CPB_F64 ? 8 : 4;
    int p = 0;
    for (int b : {CPB_FREE_Y, CPB_FREE_X, CPB_FREE_FLUX}) p += (P.free_mask & b) ? 1 : 0;
    p = std::max(p, 1);
    const int R = (int)std::ceil(std::max(P.fit_rad, 0.0));
    const int S2 = (2 * R + 1) * (2 * R + 1);
    const int mR = std::max((int)std::ceil(std::max(P.model_rad, 0.0)), R);
    const int MS = ((2 * mR + 1) * (2 * mR + 1) + 15) / 16 * 16;
    const int VS = (p * S2 + 15) / 16 * 16;
    const int64_t bst = P.precision == CPB_PREC_MIXED ? 4 : 8;
    const int64_t per_px = 57 + 3 * esz;
    const int64_t per_star = VS * bst + MS * bst + (P.precision == CPB_PREC_MIXED ? MS * 8 : 0) + 1100;
    const int64_t bytes = npix * per_px + n * per_star + (64LL << 20);
    return bytes + bytes / 5;  // 20% margin for allocator rounding and CUB temporaries
}

int64_t held_bytes(cpb_ctx* ctx) {
    int64_t s = 0;
    for (auto& kv : ctx->bufs) s += (int64_t)kv.second.bytes;
    return s;
}

void release_scratch(cpb_ctx* ctx) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->copy_stream);
    for (auto& kv : ctx->bufs)
        if (kv.second.p) cudaFreeAsync(kv.second.p, ctx->stream);
    ctx->bufs.clear();
    cudaStreamSynchronize(ctx->stream);
}

}  // namespace

struct cpb_server {
    cpb_server_config cfg{};
    std::mutex mu;
    std::condition_variable work_cv;  // workers wait for admissible requests
    std::condition_variable done_cv;  // waiters wait for completions
    std::deque<std::shared_ptr<Request>> queue;
    std::map<int64_t, std::shared_ptr<Request>> all;
    std::vector<Slot> slots;
    std::vector<cpb_psf*> psfs;
    std::vector<int64_t> held;  // per slot: device bytes its context caches (updated by its worker)
    int64_t budget = 0;
    int64_t next_id = 1;
    Clock::time_point t0 = Clock::now();
    bool stop = false;
    std::string err;

    // Called with mu held by the worker of slot s: the first queued request that
    // fits, or null.  May release idle slots' caches to make room.
    std::shared_ptr<Request> admit(int s) {
        for (auto it = queue.begin(); it != queue.end(); ++it) {
            auto& r = *it;
            int64_t others = 0, idle_held = 0;
            for (size_t t = 0; t < slots.size(); ++t) {
                if ((int)t == s) continue;
                if (slots[t].running) others += std::max(slots[t].running->est, held[t]);
                else {
                    others += held[t];
                    idle_held += held[t];
                }
            }
            const int64_t need = std::max(r->est, held[s]);
            if (others + need <= budget) {
                auto req = r;
                queue.erase(it);
                return req;
            }
            if (others - idle_held + need <= budget) {
                // only idle caches are in the way: drop them (their owners are waiting on work_cv)
                for (size_t t = 0; t < slots.size(); ++t)
                    if ((int)t != s && !slots[t].running && held[t] > 0) {
                        release_scratch(slots[t].ctx);
                        held[t] = 0;
                    }
                auto req = r;
                queue.erase(it);
                return req;
            }
        }
        return nullptr;
    }

    void worker_loop(int s) {
        cpb_ctx* ctx = slots[s].ctx;
        for (;;) {
            std::shared_ptr<Request> r;
            {
                std::unique_lock<std::mutex> lk(mu);
                for (;;) {
                    if (stop) return;
                    r = admit(s);
                    if (r) break;
                    work_cv.wait(lk);
                }
                r->state = CPB_REQ_RUNNING;
                r->slot = s;
                r->t_start = Clock::now();
                slots[s].running = r;
                // the slot's cache grows to the request's size
                held[s] = std::max(held[s], r->est);
            }
            const int rc = cpb_fit_simultaneous(ctx, psfs[r->psf_id], &r->params, r->image, r->eltype, r->ny, r->nx,
                                                r->inv_var, r->background, r->n, r->y0, r->x0, r->f0, r->out);
            const std::string e = rc == CPB_OK ? std::string() : std::string(cpb_last_error(ctx));
            const int64_t h = held_bytes(ctx);
            {
                std::lock_guard<std::mutex> lk(mu);
                r->status = rc;
                r->error = e;
                r->device_seconds = rc == CPB_OK ? r->out->device_seconds : 0.0;
                r->t_end = Clock::now();
                r->state = rc == CPB_OK ? CPB_REQ_DONE : CPB_REQ_FAILED;
                slots[s].running.reset();
                held[s] = h;
            }
            done_cv.notify_all();
            work_cv.notify_all();  // memory and a slot came free
        }
    }

    void fill_info(const Request& r, cpb_request_info* info) {
        if (!info) return;
        std::memset(info, 0, sizeof(*info));
        info->state = r.state;
        info->status = r.status;
        info->slot = r.slot;
        info->est_bytes = r.est;
        auto secs = [](Clock::time_point a, Clock::time_point b) {
            return std::chrono::duration<double>(b - a).count();
        };
        const Clock::time_point now = Clock::now();
        if (r.state == CPB_REQ_QUEUED) {
            info->queued_seconds = secs(r.t_submit, now);
        } else if (r.state == CPB_REQ_RUNNING) {
            info->queued_seconds = secs(r.t_submit, r.t_start);
            info->run_seconds = secs(r.t_start, now);
        } else if (r.state == CPB_REQ_DONE || r.state == CPB_REQ_FAILED) {
            info->queued_seconds = secs(r.t_submit, r.t_start);
            info->run_seconds = secs(r.t_start, r.t_end);
            info->latency_seconds = secs(r.t_submit, r.t_end);
        } else {
            info->queued_seconds = secs(r.t_submit, r.t_end);
        }
        info->device_seconds = r.device_seconds;
        if (r.state >= CPB_REQ_RUNNING && r.state != CPB_REQ_CANCELLED) info->start_time = secs(t0, r.t_start);
        if (r.state == CPB_REQ_DONE || r.state == CPB_REQ_FAILED) info->end_time = secs(t0, r.t_end);
        std::strncpy(info->error, r.error.c_str(), sizeof(info->error) - 1);
    }
};

extern "C" {

int cpb_server_create(const cpb_server_config* config, cpb_server** out) {
    if (!config || !out) return CPB_ERR_ARGUMENT;
    *out = nullptr;
    auto* sv = new cpb_server();
    sv->cfg = *config;
    const int k = config->max_inflight > 0 ? config->max_inflight : 4;
    const int64_t reserve = config->hbm_reserve_bytes < 0 ? (2LL << 30) : config->hbm_reserve_bytes;
    sv->slots.resize(k);
    sv->held.assign(k, 0);
    for (int s = 0; s < k; ++s) {
        const int rc = cpb_ctx_create(config->device, &sv->slots[s].ctx);
        if (rc != CPB_OK) {
            for (int t = 0; t < s; ++t) cpb_ctx_destroy(sv->slots[t].ctx);
            delete sv;
            return rc;
        }
    }
    size_t free_b = 0, total_b = 0;
    cudaSetDevice(config->device);
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        for (auto& sl : sv->slots) cpb_ctx_destroy(sl.ctx);
        delete sv;
        return CPB_ERR_CUDA;
    }
    sv->budget = std::max<int64_t>((int64_t)free_b - reserve, 0);
    for (int s = 0; s < k; ++s) sv->slots[s].worker = std::thread([sv, s] { sv->worker_loop(s); });
    *out = sv;
    return CPB_OK;
}

int cpb_server_add_psf(cpb_server* sv, const cpb_psf_desc* desc, int32_t* psf_id) {
    if (!sv || !desc || !psf_id) return CPB_ERR_ARGUMENT;
    cpb_psf* p = nullptr;
    const int rc = cpb_psf_upload(sv->slots[0].ctx, desc, &p);
    std::lock_guard<std::mutex> lk(sv->mu);
    if (rc != CPB_OK) {
        sv->err = cpb_last_error(sv->slots[0].ctx);
        return rc;
    }
    sv->psfs.push_back(p);
    *psf_id = (int32_t)sv->psfs.size() - 1;
    sv->err.clear();
    return CPB_OK;
}

int cpb_server_submit(cpb_server* sv, int32_t psf_id, const cpb_sim_params* params, const void* image,
                      int32_t eltype, int64_t ny, int64_t nx, const void* inv_var, const void* background, int64_t n,
                      const double* y0, const double* x0, const double* flux0, cpb_sim_result* out,
                      int64_t* request_id) {
    if (!sv || !request_id) return CPB_ERR_ARGUMENT;
    std::unique_lock<std::mutex> lk(sv->mu);
    sv->err.clear();
    if (psf_id < 0 || psf_id >= (int32_t)sv->psfs.size()) {
        sv->err = "unknown psf_id";
        return CPB_ERR_ARGUMENT;
    }
    if (!params || !image || !out || ny <= 0 || nx <= 0 || n < 0 || (n > 0 && (!y0 || !x0 || !flux0))) {
        sv->err = "null argument or empty image";
        return CPB_ERR_ARGUMENT;
    }
    if (sv->stop) {
        sv->err = "server is shutting down";
        return CPB_ERR_ARGUMENT;
    }
    auto r = std::make_shared<Request>();
    r->id = sv->next_id++;
    r->psf_id = psf_id;
    r->params = *params;
    r->image = image;
    r->eltype = eltype;
    r->ny = ny;
    r->nx = nx;
    r->inv_var = inv_var;
    r->background = background;
    r->n = n;
    r->y0 = y0;
    r->x0 = x0;
    r->f0 = flux0;
    r->out = out;
    r->est = estimate_bytes(*params, eltype, ny, nx, n);
    r->t_submit = Clock::now();
    sv->all[r->id] = r;
    *request_id = r->id;
    if (r->est > sv->budget) {
        r->state = CPB_REQ_FAILED;
        r->status = CPB_ERR_OOM;
        r->error = "admission refused: the request needs an estimated " + std::to_string(r->est) +
                   " bytes of device memory; the server's budget is " + std::to_string(sv->budget);
        r->t_start = r->t_end = r->t_submit;
        lk.unlock();
        sv->done_cv.notify_all();
        return CPB_OK;
    }
    sv->queue.push_back(r);
    lk.unlock();
    sv->work_cv.notify_all();
    return CPB_OK;
}

int cpb_server_poll(cpb_server* sv, int64_t id, cpb_request_info* info) {
    if (!sv) return CPB_ERR_ARGUMENT;
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->all.find(id);
    if (it == sv->all.end()) {
        sv->err = "unknown request id";
        return CPB_ERR_ARGUMENT;
    }
    sv->fill_info(*it->second, info);
    return CPB_OK;
}

int cpb_server_wait(cpb_server* sv, int64_t id, double timeout_seconds, cpb_request_info* info) {
    if (!sv) return CPB_ERR_ARGUMENT;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->all.find(id);
    if (it == sv->all.end()) {
        sv->err = "unknown request id";
        return CPB_ERR_ARGUMENT;
    }
    std::shared_ptr<Request> r = it->second;
    auto finished = [&] { return r->state >= CPB_REQ_DONE; };
    if (timeout_seconds < 0) {
        sv->done_cv.wait(lk, finished);
    } else if (!sv->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_seconds), finished)) {
        sv->fill_info(*r, info);
        return CPB_ERR_TIMEOUT;
    }
    sv->fill_info(*r, info);
    return CPB_OK;
}

int cpb_server_cancel(cpb_server* sv, int64_t id) {
    if (!sv) return CPB_ERR_ARGUMENT;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = std::find_if(sv->queue.begin(), sv->queue.end(), [&](const std::shared_ptr<Request>& r) {
        return r->id == id;
    });
    if (it == sv->queue.end()) {
        sv->err = "request is not queued";
        return CPB_ERR_ARGUMENT;
    }
    (*it)->state = CPB_REQ_CANCELLED;
    (*it)->t_end = Clock::now();
    sv->queue.erase(it);
    lk.unlock();
    sv->done_cv.notify_all();
    return CPB_OK;
}

int cpb_server_destroy(cpb_server* sv) {
    if (!sv) return CPB_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
        for (auto& r : sv->queue) {
            r->state = CPB_REQ_CANCELLED;
            r->t_end = Clock::now();
        }
        sv->queue.clear();
    }
    sv->work_cv.notify_all();
    sv->done_cv.notify_all();
    for (auto& s : sv->slots)
        if (s.worker.joinable()) s.worker.join();
    for (cpb_psf* p : sv->psfs) cpb_psf_free(sv->slots[0].ctx, p);
    for (auto& s : sv->slots) cpb_ctx_destroy(s.ctx);
    delete sv;
    return CPB_OK;
}

const char* cpb_server_last_error(const cpb_server* sv) { return sv ? sv->err.c_str() : "null server"; }

}  // extern "C"
