// Serving loop: tilt series are submitted as they are collected and
// reconstructed concurrently on one GPU, with continuous batching at y-slab
// granularity.
//
// A request (geometry + host frames + host volume frames, as for
// at3r_run_host) is admitted as soon as the device bytes it holds —
// its plan's workspace, its projections kept on the device for the whole
// request, two volume slabs (at3r_estimate_resident_bytes) — fit the HBM
// budget beside the admitted requests and fewer than max_inflight are
// active.  Admission scans the whole queue, so a request that does not fit
// yet does not hold back smaller ones behind it; a request passed over
// kMaxOvertakes times stops the scan until it fits, so none starves.
//
// One engine thread drives every active request on streams of its own: at
// admission it builds the plan (workspace stream-ordered from the device's
// memory pool, so no request synchronises the device), allocates and
// uploads the projections once; then it keeps up to two slabs of each
// active request queued — reconstruct the slab from the resident
// projections, copy its volume rows out to the host frames — and retires
// finished slabs as their events complete.  Slabs of different requests
// interleave on the device, a short request finishes while a long one is
// still running, and each finished slab leaves the device at once.  Slabs go
// to a stream whose priority follows the request's age among the active
// ones (the oldest the greatest), so the device serves the oldest request
// first and the younger ones take the SMs it leaves idle.  Every slab is computed by the request's own plan on its
// own buffers, so a result does not depend on what else is running.
// Pageable host frames are copied through pinned bounce buffers; pinned
// frames move directly.  Per-request latency runs from submission to the
// moment the whole volume is in host memory.
#include "at3r_internal.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

constexpr int kMaxOvertakes = 8;   // admissions that may pass a waiting request

struct Slab {
    int y0 = 0, n = 0, buf = 0;
    cudaEvent_t done = nullptr;   // rows computed and copied out (to the bounce buffer when pageable)
};

struct Request {
    int64_t id = 0;
    at3r_geom g{};
    std::vector<float> tilts;
    std::vector<const float*> frames;
    std::vector<float*> vols;
    size_t bytes = 0;
    int slab = 1;
    Clock::time_point t_submit, t_start, t_done;
    at3r_status status = AT3R_OK;
    std::string err;
    bool done = false;
    bool waited = false;   // a caller is in at3r_server_wait for it (one waiter per request)
    int overtaken = 0;
    // engine state
    cudaStream_t st = nullptr;               // set-up, upload and release
    cudaStream_t pst[8] = {};                // slab work, one stream per priority level used
    cudaStream_t last = nullptr;             // the stream of the last slab issued
    cudaEvent_t up = nullptr;                // upload done
    at3r_plan* plan = nullptr;
    float* d_proj = nullptr;
    float* d_vol[2] = {nullptr, nullptr};
    char* h_bounce[2] = {nullptr, nullptr};   // pinned, pageable output only
    bool out_pinned = false;
    int next_y = 0, rows_done = 0;
    std::deque<Slab> inflight;
    std::vector<cudaEvent_t> events;
};

}  // namespace

struct at3r_server {
    int device = 0;
    int prio_greatest = 0, prio_levels = 1;   // stream priorities: rank 0 (the oldest request) the greatest
    size_t budget = 0;
    int max_inflight = 4;
    std::mutex mu;
    std::condition_variable cv;   // queue changes and completions
    std::list<Request*> pending;
    std::map<int64_t, Request*> reqs;
    int64_t next_id = 1;
    size_t in_use = 0;
    int running = 0;
    bool stop = false;
    std::thread engine;
};

namespace {

bool is_pinned(const void* ptr)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

std::string cuda_msg(const char* what, cudaError_t e) { return std::string(what) + ": " + cudaGetErrorString(e); }

// Sets up an admitted request: stream, plan, resident projections, slab
// buffers; queues the upload.  Returns false (status and message set) on error.
bool start_request(Request* r)
{
    cudaError_t e = cudaStreamCreateWithFlags(&r->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        r->status = AT3R_ERR_CUDA;
        r->err = cuda_msg("stream", e);
        return false;
    }
    r->g.slab_slices = r->slab;
    at3r_status rc = plan_create_impl(&r->g, r->st, &r->plan);
    if (rc != AT3R_OK) {
        r->status = rc;
        r->err = at3r_last_error();
        return false;
    }
    const size_t T = r->g.n_tilts, ny = r->g.ny, nx = r->g.nx, Nx = nx & ~1, Nz = r->g.vol_z;
    const size_t frame = ny * nx, vslab = (size_t)r->slab * Nx * Nz;
    e = cudaMallocAsync(reinterpret_cast<void**>(&r->d_proj), sizeof(float) * T * frame, r->st);
    for (int b = 0; b < 2 && e == cudaSuccess; b++)
        e = cudaMallocAsync(reinterpret_cast<void**>(&r->d_vol[b]), sizeof(float) * vslab, r->st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        r->status = e == cudaErrorMemoryAllocation ? AT3R_ERR_OUT_OF_MEMORY : AT3R_ERR_CUDA;
        r->err = cuda_msg("request buffers", e);
        return false;
    }
    // the projections stay on the device for the whole request: one copy per frame
    for (size_t t = 0; t < T && e == cudaSuccess; t++)
        e = cudaMemcpyAsync(r->d_proj + t * frame, r->frames[t], sizeof(float) * frame, cudaMemcpyHostToDevice, r->st);
    r->out_pinned = is_pinned(r->vols[0]);
    if (!r->out_pinned && e == cudaSuccess)
        for (int b = 0; b < 2 && e == cudaSuccess; b++)
            e = cudaHostAlloc(reinterpret_cast<void**>(&r->h_bounce[b]), sizeof(float) * vslab, cudaHostAllocPortable);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->up, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(r->up, r->st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        r->status = AT3R_ERR_CUDA;
        r->err = cuda_msg("request upload", e);
        return false;
    }
    return true;
}

// Releases a request's device resources (stream-ordered) and its stream.
void end_request(Request* r)
{
    if (r->st) cudaStreamSynchronize(r->st);
    r->inflight.clear();
    if (r->plan) at3r_plan_destroy(r->plan);
    r->plan = nullptr;
    for (cudaStream_t& q : r->pst)
        if (q) { cudaStreamSynchronize(q); cudaStreamDestroy(q); q = nullptr; }
    r->last = nullptr;
    if (r->up) { cudaEventDestroy(r->up); r->up = nullptr; }
    if (r->st) {
        if (r->d_proj) cudaFreeAsync(r->d_proj, r->st);
        for (float* v : r->d_vol)
            if (v) cudaFreeAsync(v, r->st);
        cudaStreamSynchronize(r->st);
        cudaStreamDestroy(r->st);
    }
    r->d_proj = nullptr;
    r->d_vol[0] = r->d_vol[1] = nullptr;
    r->st = nullptr;
    for (char*& h : r->h_bounce)
        if (h) { cudaFreeHost(h); h = nullptr; }
    for (cudaEvent_t ev : r->events) cudaEventDestroy(ev);
    r->events.clear();
    cudaGetLastError();
}

// Queues the next slab of r: reconstruct, then copy the rows out, on the
// request's stream of priority level `level` (0 = the greatest).  A slab on
// another stream than the previous one waits for the previous slab (or the
// upload) first, so a request's slabs stay in order.
bool issue_slab(Request* r, int level, int prio)
{
    cudaStream_t& sq = r->pst[level];
    if (!sq && cudaStreamCreateWithPriority(&sq, cudaStreamNonBlocking, prio) != cudaSuccess) {
        cudaGetLastError();
        r->status = AT3R_ERR_CUDA;
        r->err = "stream creation failed";
        return false;
    }
    if (sq != r->last) {
        const cudaEvent_t prev = r->last ? r->inflight.empty() ? nullptr : r->inflight.back().done : r->up;
        if (prev && cudaStreamWaitEvent(sq, prev, 0) != cudaSuccess) {
            cudaGetLastError();
            r->status = AT3R_ERR_CUDA;
            r->err = "stream ordering failed";
            return false;
        }
        r->last = sq;
    }
    const cudaStream_t st = sq;
    const int y0 = r->next_y, n = std::min(r->slab, r->g.ny - y0);
    const int buf = (int)((y0 / r->slab) & 1);
    Slab s{y0, n, buf, nullptr};
    if (r->events.size() < 2) {
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            r->status = AT3R_ERR_CUDA;
            r->err = "event creation failed";
            return false;
        }
        r->events.push_back(ev);
    }
    s.done = r->events[buf];
    at3r_status rc = at3r_plan_run_slab(r->plan, r->d_proj, y0, n, r->d_vol[buf], st);
    if (rc != AT3R_OK) {
        r->status = rc;
        r->err = at3r_last_error();
        return false;
    }
    const size_t slice = (size_t)(r->g.nx & ~1) * r->g.vol_z;
    cudaError_t e = cudaSuccess;
    if (r->out_pinned) {
        // frames that sit back to back in host memory go out as one copy
        int j = 0;
        while (j < n && e == cudaSuccess) {
            int k = j + 1;
            while (k < n && r->vols[y0 + k] == r->vols[y0 + k - 1] + slice) k++;
            e = cudaMemcpyAsync(r->vols[y0 + j], r->d_vol[buf] + (size_t)j * slice, sizeof(float) * slice * (k - j),
                                cudaMemcpyDeviceToHost, st);
            j = k;
        }
    } else {
        e = cudaMemcpyAsync(r->h_bounce[buf], r->d_vol[buf], sizeof(float) * slice * n, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaEventRecord(s.done, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        r->status = AT3R_ERR_CUDA;
        r->err = cuda_msg("slab copy-out", e);
        return false;
    }
    r->inflight.push_back(s);
    r->next_y += n;
    return true;
}

// Retires r's finished slabs (in order); returns how many.
int retire_slabs(Request* r)
{
    int k = 0;
    const size_t slice = (size_t)(r->g.nx & ~1) * r->g.vol_z;
    while (!r->inflight.empty()) {
        Slab& s = r->inflight.front();
        const cudaError_t q = cudaEventQuery(s.done);
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) {
            cudaGetLastError();
            r->status = AT3R_ERR_CUDA;
            r->err = cuda_msg("slab", q);
            r->inflight.clear();
            return k;
        }
        if (!r->out_pinned) {
            std::vector<at3r::Piece> pc;
            for (int j = 0; j < s.n; j++)
                pc.push_back({reinterpret_cast<char*>(r->vols[s.y0 + j]),
                              r->h_bounce[s.buf] + sizeof(float) * slice * j, sizeof(float) * slice});
            at3r::parallel_copy(pc);
        }
        r->rows_done += s.n;
        r->inflight.pop_front();
        k++;
    }
    return k;
}

void finish(at3r_server* s, Request* r)
{
    end_request(r);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->in_use -= r->bytes;
        s->running--;
        r->t_done = Clock::now();
        r->done = true;
    }
    s->cv.notify_all();
}

void engine_main(at3r_server* s)
{
    cudaSetDevice(s->device);
    std::vector<Request*> active;
    for (;;) {
        // admission: any queued request that fits, in submission order; a
        // request passed over too often stops the scan until it fits
        std::vector<Request*> admit;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (active.empty()) {
                s->cv.wait(lk, [s] { return s->stop || !s->pending.empty(); });
                if (s->pending.empty() && s->stop) break;
            }
            for (auto it = s->pending.begin(); it != s->pending.end();) {
                Request* r = *it;
                if (s->running + (int)admit.size() >= s->max_inflight) break;
                if (s->in_use + r->bytes <= s->budget) {
                    s->in_use += r->bytes;
                    r->t_start = Clock::now();
                    admit.push_back(r);
                    it = s->pending.erase(it);
                    continue;
                }
                if (++r->overtaken > kMaxOvertakes) break;
                ++it;
            }
            s->running += (int)admit.size();
        }
        for (Request* r : admit) {
            if (start_request(r))
                active.push_back(r);
            else
                finish(s, r);
        }
        // progress: retire finished slabs, keep two slabs of every request queued
        bool moved = !admit.empty();
        for (size_t i = 0; i < active.size();) {
            Request* r = active[i];
            moved |= retire_slabs(r) > 0;
            // the older the request, the higher its streams' priority, so the
            // device finishes the oldest first and the younger ones fill in
            const int level = std::min((int)i, s->prio_levels - 1);
            while (r->status == AT3R_OK && r->inflight.size() < 2 && r->next_y < r->g.ny) {
                if (!issue_slab(r, level, s->prio_greatest + level)) break;
                moved = true;
            }
            if (r->status != AT3R_OK || (r->rows_done == r->g.ny && r->inflight.empty())) {
                finish(s, r);
                active.erase(active.begin() + (long)i);
                moved = true;
                continue;
            }
            i++;
        }
        if (!moved && !active.empty()) {
            // nothing finished: wait for the oldest queued slab of any request
            // (every request still has work queued on the device meanwhile)
            Request* oldest = nullptr;
            for (Request* r : active)
                if (!r->inflight.empty()) { oldest = r; break; }
            if (oldest) {
                cudaEventSynchronize(oldest->inflight.front().done);
                cudaGetLastError();
            } else {
                std::this_thread::sleep_for(std::chrono::microseconds(50));
            }
        }
    }
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
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess) {
        s->prio_greatest = greatest;
        s->prio_levels = std::max(1, std::min(8, least - greatest + 1));
    }
    // keep freed workspace in the pool for the next request
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    s->engine = std::thread(engine_main, s);
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
    for (int t = 0; t < g->n_tilts; t++)
        if (!frames[t]) {
            at3r_set_last_error("null tilt frame");
            return AT3R_ERR_INVALID_ARGUMENT;
        }
    for (int y = 0; y < g->ny; y++)
        if (!vol_frames[y]) {
            at3r_set_last_error("null volume frame");
            return AT3R_ERR_INVALID_ARGUMENT;
        }
    Request* r = new Request();
    r->g = *g;
    r->tilts.assign(g->tilts_deg, g->tilts_deg + g->n_tilts);
    r->g.tilts_deg = r->tilts.data();
    r->frames.assign(frames, frames + g->n_tilts);
    r->vols.assign(vol_frames, vol_frames + g->ny);
    r->bytes = at3r_estimate_resident_bytes(g, &r->slab);
    if (r->bytes == 0) {
        delete r;
        at3r_set_last_error("invalid series size");
        return AT3R_ERR_INVALID_ARGUMENT;
    }
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
    if (s->engine.joinable()) s->engine.join();
    for (auto& kv : s->reqs) delete kv.second;
    delete s;
}

}  // extern "C"
