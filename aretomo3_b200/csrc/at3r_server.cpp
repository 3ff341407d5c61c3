// Serving loop: tilt series are submitted as they are collected and
// reconstructed concurrently on one GPU.
//
// A request (geometry + host frames + host volume frames, as for
// at3r_run_host) waits in a FIFO queue until the device bytes it will hold
// (at3r_plan_estimate_bytes) fit the server's HBM budget next to the requests
// already running, and a worker is free.  Each of max_inflight workers owns a
// CUDA stream; it builds the request's plan with workspace taken
// stream-ordered from the device's memory pool (so finishing a request does
// not synchronise the device), runs it with the slab-streaming host path
// (volume slabs go back to the host as they finish, so a request holds only
// its slab buffers), releases the plan and admits the next request.  Kernels
// of concurrent requests overlap on the device.  Per-request latency runs from
// submission to the moment the volume is in host memory.
#include "at3r_internal.h"

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t id = 0;
    at3r_geom g{};
    std::vector<float> tilts;
    std::vector<const float*> frames;
    std::vector<float*> vols;
    size_t bytes = 0;
    Clock::time_point t_submit, t_start, t_done;
    at3r_status status = AT3R_OK;
    std::string err;
    bool done = false;
    bool waited = false;   // a caller is in at3r_server_wait for it (one waiter per request)
};

}  // namespace

struct at3r_server {
    int device = 0;
    size_t budget = 0;
    int max_inflight = 4;
    std::mutex mu;
    std::condition_variable cv;   // queue changes and completions
    std::deque<Request*> pending;
    std::map<int64_t, Request*> reqs;
    int64_t next_id = 1;
    size_t in_use = 0;
    int running = 0;
    bool stop = false;
    std::vector<std::thread> workers;
};

namespace {

void worker_main(at3r_server* s)
{
    cudaSetDevice(s->device);
    cudaStream_t st = nullptr;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (;;) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait(lk, [s] {
                return (s->stop && s->pending.empty()) ||
                       (!s->pending.empty() && s->in_use + s->pending.front()->bytes <= s->budget);
            });
            if (s->pending.empty()) break;
            r = s->pending.front();
            s->pending.pop_front();
            s->in_use += r->bytes;
            s->running++;
            r->t_start = Clock::now();
        }
        at3r_plan* plan = nullptr;
        at3r_status rc = plan_create_impl(&r->g, st, &plan);
        if (rc == AT3R_OK) rc = at3r_run_host(plan, r->frames.data(), r->vols.data(), st);
        std::string err = rc == AT3R_OK ? std::string() : std::string(at3r_last_error());
        if (plan) at3r_plan_destroy(plan);
        cudaStreamSynchronize(st);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->in_use -= r->bytes;
            s->running--;
            r->status = rc;
            r->err = err;
            r->t_done = Clock::now();
            r->done = true;
        }
        s->cv.notify_all();
    }
    cudaStreamDestroy(st);
}

}  // namespace

extern "C" {

at3r_status at3r_server_create(const at3r_server_opts* o, at3r_server** out)
{
    if (!out) return AT3R_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int dev = 0, ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        at3r_set_last_error("no CUDA device");
        return AT3R_ERR_NO_DEVICE;
    }
    cudaGetDevice(&dev);
    at3r_server* s = new at3r_server();
    s->device = dev;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    s->budget = (o && o->hbm_budget_bytes) ? o->hbm_budget_bytes : free_b / 10 * 9;
    s->max_inflight = (o && o->max_inflight > 0) ? o->max_inflight : 4;
    // keep freed workspace in the pool for the next request
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    for (int i = 0; i < s->max_inflight; i++) s->workers.emplace_back(worker_main, s);
    *out = s;
    return AT3R_OK;
}

at3r_status at3r_server_submit(at3r_server* s, const at3r_geom* g, const float* const* frames,
                               float* const* vol_frames, int64_t* id)
{
    if (!s || !g || !frames || !vol_frames || !g->tilts_deg || g->n_tilts < 1 || g->ny < 1) {
        at3r_set_last_error("null argument or empty series");
        return AT3R_ERR_INVALID_ARGUMENT;
    }
    Request* r = new Request();
    r->g = *g;
    r->tilts.assign(g->tilts_deg, g->tilts_deg + g->n_tilts);
    r->g.tilts_deg = r->tilts.data();
    r->frames.assign(frames, frames + g->n_tilts);
    r->vols.assign(vol_frames, vol_frames + g->ny);
    r->bytes = at3r_plan_estimate_bytes(g);
    if (r->bytes > s->budget) {
        delete r;
        at3r_set_last_error("the series needs more device memory than the server's budget");
        return AT3R_ERR_TOO_LARGE;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        r->t_submit = Clock::now();
        s->reqs[r->id] = r;
        s->pending.push_back(r);
        if (id) *id = r->id;
    }
    s->cv.notify_all();
    return AT3R_OK;
}

at3r_status at3r_server_wait(at3r_server* s, int64_t id, double* latency_s, double* queued_s)
{
    if (!s) return AT3R_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) {
        at3r_set_last_error("unknown request id");
        return AT3R_ERR_INVALID_ARGUMENT;
    }
    Request* r = it->second;
    if (r->waited) {
        at3r_set_last_error("another thread is already waiting for this request");
        return AT3R_ERR_INVALID_ARGUMENT;
    }
    r->waited = true;
    s->cv.wait(lk, [r] { return r->done; });
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    if (queued_s) *queued_s = std::chrono::duration<double>(r->t_start - r->t_submit).count();
    const at3r_status rc = r->status;
    if (rc != AT3R_OK) at3r_set_last_error(r->err.c_str());
    s->reqs.erase(it);
    delete r;
    return rc;
}

size_t at3r_server_in_use_bytes(at3r_server* s)
{
    if (!s) return 0;
    std::lock_guard<std::mutex> lk(s->mu);
    return s->in_use;
}

void at3r_server_destroy(at3r_server* s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto& kv : s->reqs) delete kv.second;
    delete s;
}

}  // extern "C"
