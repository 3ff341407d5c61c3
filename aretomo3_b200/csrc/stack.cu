// C-ABI implementation of the input stage (at3r_stack_*: the aligned, binned
// tilt series of AreTomo/Correct/CCorrTomoStack.cpp and CBinStack::DoFFT) and
// of the thickness measurement (at3r_thickness_*: AreTomo/Recon/
// CCalcVolThick.cpp).  Kernels: stack_kernels.cuh.
#include "at3r.h"
#include "at3r_internal.h"
#include "fft_host.h"
#include "stack_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

using namespace at3r;

struct at3r_stack {
    at3r_stack_geom g{};
    int device = 0;
    int nx = 0, ny = 0, T = 0;
    int ax = 0, ay = 0, W = 0;     // aligned frame; W = width the reference's kernels cover
    int bx = 0, by = 0, KXo = 0;   // binned frame; kept row bins
    bool same = false;             // binned size == aligned size: no Fourier crop
    int P = 0;                     // local-alignment patches
    int by_rows = 0;               // k_corr visits tiles along aligned y (axis nearer 90 than 0 degrees)
    int chunk = 1;                 // tilts per device pass
    int c2r = AT3R_C2R_HERMITIAN;
    float norm = 1.f;
    float2* d_shift = nullptr;     // [T]
    float2* d_cs = nullptr;        // [T] cos / sin of the rotation
    float* d_local = nullptr;      // [T][5][P]
    int* d_rand = nullptr;         // [W * ay] random table of the fill
    int* d_flags = nullptr;        // [chunk] frames whose fill needs the mean
    float* d_aln = nullptr;        // [chunk][ay][ax]
    uint8_t* d_empty = nullptr;    // [chunk][W * ay]
    float2* d_Y = nullptr;         // [chunk][ay][KXo]
    float2* d_Wc = nullptr;        // [chunk][by][KXo]
    // host path: two buffers of hc tilts each, raw in and binned out, on
    // their own copy streams (double-buffered against the compute stream)
    int hc = 0;
    float* d_raw2[2] = {nullptr, nullptr};
    float* d_out2[2] = {nullptr, nullptr};
    cudaStream_t s_in = nullptr, s_out = nullptr;
    cudaEvent_t ev_in[2] = {}, ev_comp[2] = {}, ev_outdone[2] = {}, ev_slot[4] = {};
    HostFft frow, fcin, fcout, fbx;
    int b_row = 1, b_c2r = 1, cb = 1, col_pitch = 0, rs_col = 0;
    size_t smem_row = 0, smem_col = 0, smem_c2r = 0;
};

namespace {

at3r_status st_err(at3r_status s, const std::string& msg)
{
    at3r_set_last_error(msg.c_str());
    return s;
}

#define ST_CUDA(call)                                                                                      \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) {                                                                           \
            cudaGetLastError();                                                                            \
            return st_err(e_ == cudaErrorMemoryAllocation ? AT3R_ERR_OUT_OF_MEMORY : AT3R_ERR_CUDA,        \
                          std::string(#call) + ": " + cudaGetErrorString(e_));                             \
        }                                                                                                  \
    } while (0)

// CCorrectUtil::CalcAlignedSize (AreTomo/Correct/CCorrectUtil.cpp:11-21):
// x and y swap when the tilt axis is closer to x than to y.
void aligned_size(int nx, int ny, float axis_deg, int* a)
{
    a[0] = nx;
    a[1] = ny;
    const double rot = std::fabs(std::sin(axis_deg * 3.14 / 180.0));
    if (rot <= 0.707) return;
    a[0] = ny;
    a[1] = nx;
}

// GFourierResize2D::GetBinnedImgSize (MaUtil/GFourierResize2D.cu:75-88).
void binned_size(const int* a, float bin, int* b)
{
    b[0] = a[0];
    b[1] = a[1];
    if (bin == 1.0f) return;
    b[0] = (int)(a[0] / bin) / 2 * 2;
    b[1] = (int)(a[1] / bin) / 2 * 2;
}

at3r_status set_smem_attr(const void* fn, size_t bytes)
{
    int dev = 0, optin = 0;
    ST_CUDA(cudaGetDevice(&dev));
    ST_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa{};
    ST_CUDA(cudaFuncGetAttributes(&fa, fn));
    const size_t kMax = (size_t)optin - fa.sharedSizeBytes;
    if (bytes > kMax)
        return st_err(AT3R_ERR_TOO_LARGE, "shared-memory need " + std::to_string(bytes) + " exceeds " +
                                              std::to_string(kMax) + " bytes (frame too large for the binning FFT)");
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, bool> done;
    std::lock_guard<std::mutex> lk(mu);
    if (!done[{fn, dev}]) {
        ST_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMax));
        done[{fn, dev}] = true;
    }
    return AT3R_OK;
}

template <typename T>
at3r_status salloc(T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) return AT3R_OK;
    ST_CUDA(cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T)));
    return AT3R_OK;
}

at3r_status make_fft_tables(int n, HostFft& h)
{
    std::vector<float2> tables;
    plan_fft(n, h, tables);
    ST_CUDA(cudaMalloc(reinterpret_cast<void**>(&h.d_tables), h.bytes));
    ST_CUDA(cudaMemcpy(h.d_tables, tables.data(), h.bytes, cudaMemcpyHostToDevice));
    bind_fft(h);
    return AT3R_OK;
}

int row_batch(int work)
{
    int b = 1;
    while (b < 8 && (size_t)work * b * 2 <= 4096) b *= 2;
    while (b > 1 && 2 * sizeof(float2) * (size_t)fft_pitch(work) * b > (96u << 10)) b /= 2;
    return b;
}

// One pass over n tilts (first tilt t0) already on the device: align (+ fill)
// into d_aln, then bin into out.
at3r_status run_chunk(at3r_stack* s, const float* raw, int t0, int n, float* out, cudaStream_t st)
{
    const float* src = raw;
    if (s->g.correct) {
        const int fill = s->g.rand_fill ? 1 : 0;
        const dim3 grid = s->by_rows ? dim3((s->ay + 31) / 32, (s->ax + 31) / 32, n)
                                     : dim3((s->ax + 31) / 32, (s->ay + 31) / 32, n);
        k_corr<<<grid, 256, 0, st>>>(raw, s->nx, s->ny, s->ax, s->ay, s->W, s->d_shift + t0, s->d_cs + t0,
                                     s->d_local ? s->d_local + (size_t)t0 * 5 * s->P : nullptr, s->P, fill,
                                     s->by_rows, s->d_aln, s->d_empty);
        ST_CUDA(cudaGetLastError());
        if (fill) {
            ST_CUDA(cudaMemsetAsync(s->d_flags, 0, sizeof(int) * n, st));
            const int npx = s->W * s->ay;
            k_fill<<<dim3((npx + 1023) / 1024, n), 256, 0, st>>>(s->d_aln, s->d_empty, s->d_rand, s->W, s->ax, s->ay,
                                                               s->d_flags);
            k_fill_mean<<<n, 512, 0, st>>>(s->d_aln, s->d_empty, s->W, s->ax, s->ay, s->d_flags);
            ST_CUDA(cudaGetLastError());
        }
        src = s->d_aln;
    }
    if (s->same) {
        ST_CUDA(cudaMemcpyAsync(out, src, sizeof(float) * (size_t)n * s->ax * s->ay, cudaMemcpyDeviceToDevice, st));
        return AT3R_OK;
    }
    dispatch_rs(s->frow.rs, [&](auto R) {
        k_bin_r2c<decltype(R)::value><<<dim3(((s->ay + 1) / 2 + s->b_row - 1) / s->b_row, n), 512, s->smem_row, st>>>(
            src, s->ax, s->ay, s->KXo, s->frow.plan, s->b_row, s->d_Y);
    });
    dispatch_rs(s->rs_col, [&](auto R) {
        k_bin_cols<decltype(R)::value><<<dim3((s->KXo + s->cb - 1) / s->cb, n), 512, s->smem_col, st>>>(
            s->d_Y, s->KXo, s->ay, s->by, s->cb, s->col_pitch, s->fcin.plan, s->fcout.plan, s->norm, s->d_Wc);
    });
    dispatch_rs(s->fbx.rs, [&](auto R) {
        k_bin_c2r<decltype(R)::value><<<dim3(((s->by + 1) / 2 + s->b_c2r - 1) / s->b_c2r, n), 512, s->smem_c2r, st>>>(
            s->d_Wc, s->bx, s->by, s->fbx.plan, s->b_c2r, s->c2r == AT3R_C2R_PACKED, out);
    });
    ST_CUDA(cudaGetLastError());
    return AT3R_OK;
}

at3r_status check_device(const at3r_stack* s)
{
    int dev = -1;
    ST_CUDA(cudaGetDevice(&dev));
    if (dev != s->device) return st_err(AT3R_ERR_INVALID_ARGUMENT, "stack was created on another device");
    return AT3R_OK;
}

// Host-path buffers and streams, made on first use: chunks of about 256 MB
// of raw frames (at least one tilt, at most a device pass).
at3r_status ensure_host_path(at3r_stack* s)
{
    if (s->hc) return AT3R_OK;
    const size_t fin = (size_t)s->nx * s->ny * sizeof(float);
    const int hc = (int)std::max<size_t>(1, std::min<size_t>((size_t)s->chunk, (256ull << 20) / fin));
    at3r_status rc;
    for (int b = 0; b < 2; b++)
        if ((rc = salloc(&s->d_raw2[b], (size_t)hc * s->nx * s->ny)) ||
            (rc = salloc(&s->d_out2[b], (size_t)hc * s->bx * s->by)))
            return rc;
    ST_CUDA(cudaStreamCreateWithFlags(&s->s_in, cudaStreamNonBlocking));
    ST_CUDA(cudaStreamCreateWithFlags(&s->s_out, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&s->ev_in[0], &s->ev_in[1], &s->ev_comp[0], &s->ev_comp[1], &s->ev_outdone[0],
                           &s->ev_outdone[1], &s->ev_slot[0], &s->ev_slot[1], &s->ev_slot[2], &s->ev_slot[3]})
        ST_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    s->hc = hc;
    return AT3R_OK;
}

// Copies between pageable host frames and the device through the four
// pinned slots of a staging set: slots 0 and 1 carry frames in (a parallel
// host memcpy into a slot, then its copy to the device on s_in), slots 2 and 3
// carry binned frames out (a copy from the device on s_out; the host memcpy
// out of the slot runs when the slot is next needed, or at the end), so host
// copies overlap the GPU's copies and passes.
struct Stager {
    at3r_stack* s;
    char* set;
    int in_slot = 0, out_slot = 0;
    std::vector<Piece> pending[2];   // host copies still owed by out slots 0 / 1

    char* slot(int i) const { return set + (size_t)i * kStageBytes; }

    at3r_status direct(const std::vector<Piece>& pcs, cudaMemcpyKind kind, cudaStream_t strm)
    {
        for (const Piece& pc : merge_pieces(pcs)) ST_CUDA(cudaMemcpyAsync(pc.dst, pc.src, pc.bytes, kind, strm));
        return AT3R_OK;
    }

    at3r_status in(const std::vector<Piece>& pcs)
    {
        std::vector<Piece> group;
        size_t used = 0;
        auto flush = [&]() -> at3r_status {
            if (group.empty()) return AT3R_OK;
            ST_CUDA(cudaEventSynchronize(s->ev_slot[in_slot]));
            char* sl = slot(in_slot);
            std::vector<Piece> host, dev;
            size_t o = 0;
            for (const Piece& pc : group) {
                host.push_back({sl + o, pc.src, pc.bytes});
                dev.push_back({pc.dst, sl + o, pc.bytes});
                o += pc.bytes;
            }
            parallel_copy(host);
            for (const Piece& pc : merge_pieces(dev))
                ST_CUDA(cudaMemcpyAsync(pc.dst, pc.src, pc.bytes, cudaMemcpyHostToDevice, s->s_in));
            ST_CUDA(cudaEventRecord(s->ev_slot[in_slot], s->s_in));
            in_slot ^= 1;
            group.clear();
            used = 0;
            return AT3R_OK;
        };
        at3r_status rc;
        for (const Piece& pc : split_pieces(pcs)) {
            if (used + pc.bytes > kStageBytes && (rc = flush())) return rc;
            group.push_back(pc);
            used += pc.bytes;
        }
        return flush();
    }

    at3r_status drain(int k)
    {
        if (pending[k].empty()) return AT3R_OK;
        ST_CUDA(cudaEventSynchronize(s->ev_slot[2 + k]));
        parallel_copy(pending[k]);
        pending[k].clear();
        return AT3R_OK;
    }

    at3r_status out(const std::vector<Piece>& pcs)
    {
        std::vector<Piece> group;
        size_t used = 0;
        at3r_status rc;
        auto flush = [&]() -> at3r_status {
            if (group.empty()) return AT3R_OK;
            if ((rc = drain(out_slot))) return rc;
            char* sl = slot(2 + out_slot);
            std::vector<Piece> dev;
            size_t o = 0;
            for (const Piece& pc : group) {
                dev.push_back({sl + o, pc.src, pc.bytes});
                pending[out_slot].push_back({pc.dst, sl + o, pc.bytes});
                o += pc.bytes;
            }
            for (const Piece& pc : merge_pieces(dev))
                ST_CUDA(cudaMemcpyAsync(pc.dst, pc.src, pc.bytes, cudaMemcpyDeviceToHost, s->s_out));
            ST_CUDA(cudaEventRecord(s->ev_slot[2 + out_slot], s->s_out));
            out_slot ^= 1;
            group.clear();
            used = 0;
            return AT3R_OK;
        };
        for (const Piece& pc : split_pieces(pcs)) {
            if (used + pc.bytes > kStageBytes && (rc = flush())) return rc;
            group.push_back(pc);
            used += pc.bytes;
        }
        return flush();
    }

    at3r_status drain_all()
    {
        at3r_status rc;
        // the older slot first, so the frames land in order
        if ((rc = drain(out_slot)) || (rc = drain(out_slot ^ 1))) return rc;
        return AT3R_OK;
    }
};

// CCalcVolThick::mSmooth (CCalcVolThick.cpp:114-132): 11-sample box filter,
// indices clamped at the ends, sums in double.
void smooth_profile(std::vector<float>& cc)
{
    const int n = (int)cc.size(), win = 11;
    std::vector<float> buf(n);
    for (int i = 0; i < n; i++) {
        const int start = i - win / 2;
        double sum = 0.0;
        for (int j = 0; j < win; j++) {
            int k = j + start;
            if (k < 0) k = 0;
            else if (k >= n) k = n - 1;
            sum += cc[k];
        }
        buf[i] = (float)sum / win;
    }
    cc = buf;
}

// CCalcVolThick::mDetectEdges (CCalcVolThick.cpp:209-284): the lower edge is
// the first sample of [n/10, n/2) at or above the mean of the central 80 %,
// moved halfway towards the lowest sample below it; the upper edge likewise
// from the top.  Edges scale by the binning (int *= float).  The reference
// leaves an edge at its previous value when no sample reaches the mean; here
// it starts at the search bound.  mSearchMin / mSearchMax are computed there
// but not used, so they are not repeated.
void detect_edges(const std::vector<float>& cc, float bin, at3r_thickness* r)
{
    const int n = (int)cc.size(), half = n / 2;
    const int bot = (int)(n * 0.1), top = n - bot;
    float mean = 0.f;
    for (int i = bot; i < top; i++) mean += cc[i];
    mean = mean / (top - bot);
    int e0 = bot, e1 = top;
    for (int i = bot; i < half; i++) {
        if (cc[i] < mean) continue;
        e0 = i;
        break;
    }
    float minv = mean;
    int imin = e0;
    for (int i = bot; i < e0; i++) {
        if (cc[i] >= minv) continue;
        minv = cc[i];
        imin = i;
    }
    e0 = (e0 + imin) / 2;
    for (int i = top; i > half; i--) {
        if (cc[i] < mean) continue;
        e1 = i;
        break;
    }
    minv = mean;
    imin = e1;
    for (int i = top; i > e1; i--) {
        if (cc[i] >= minv) continue;
        minv = cc[i];
        imin = i;
    }
    e1 = (e1 + imin) / 2;
    e0 = (int)(e0 * bin);
    e1 = (int)(e1 * bin);
    r->edges[0] = e0;
    r->edges[1] = e1;
    r->thickness = e1 - e0;
    r->offset_z = (e0 + e1) / 2 - (int)(half * bin);
}


// The host path: tilt chunks of s->hc frames double-buffered over the copy
// streams and the compute stream.  Binned frames go to binned_frames (host)
// or, with binned_dev, stay on the device at binned_dev[T][by][bx].
at3r_status stack_pipeline(at3r_stack* s, const float* const* frames, float* const* binned_frames, float* binned_dev,
                           void* stream)
{
    at3r_status rc;
    const size_t fin = (size_t)s->nx * s->ny * sizeof(float), fout = (size_t)s->bx * s->by * sizeof(float);
    if ((rc = ensure_host_path(s))) return rc;
    bool pin_in = true, pin_out = true;
    for (int t = 0; t < s->T && (pin_in || pin_out); t++) {
        pin_in = pin_in && host_pinned(frames[t]);
        pin_out = pin_out && (binned_dev || host_pinned(binned_frames[t]));
    }
    char* stage = nullptr;
    if (!(pin_in && pin_out) && !(stage = stage_acquire()))
        return st_err(AT3R_ERR_OUT_OF_MEMORY, "pinned staging allocation failed");
    cudaStream_t st = (cudaStream_t)stream;
    Stager sg{s, stage};
    auto body = [&]() -> at3r_status {
        const int hc = s->hc;
        for (int k = 0, t0 = 0; t0 < s->T; k++, t0 += hc) {
            const int n = std::min(hc, s->T - t0), b = k & 1;
            // raw frames in, once the pass two chunks back has read this buffer
            if (k >= 2) ST_CUDA(cudaStreamWaitEvent(s->s_in, s->ev_comp[b], 0));
            std::vector<Piece> in;
            for (int j = 0; j < n; j++)
                in.push_back({reinterpret_cast<char*>(s->d_raw2[b]) + j * fin,
                              reinterpret_cast<const char*>(frames[t0 + j]), fin});
            if ((rc = pin_in ? sg.direct(in, cudaMemcpyHostToDevice, s->s_in) : sg.in(in))) return rc;
            ST_CUDA(cudaEventRecord(s->ev_in[b], s->s_in));
            // the pass, once its frames are in and this output buffer went out
            ST_CUDA(cudaStreamWaitEvent(st, s->ev_in[b], 0));
            if (k >= 2) ST_CUDA(cudaStreamWaitEvent(st, s->ev_outdone[b], 0));
            float* dst = binned_dev ? binned_dev + (size_t)t0 * s->bx * s->by : s->d_out2[b];
            if ((rc = run_chunk(s, s->d_raw2[b], t0, n, dst, st))) return rc;
            ST_CUDA(cudaEventRecord(s->ev_comp[b], st));
            if (binned_dev) continue;
            // binned frames out
            ST_CUDA(cudaStreamWaitEvent(s->s_out, s->ev_comp[b], 0));
            std::vector<Piece> out;
            for (int j = 0; j < n; j++)
                out.push_back({reinterpret_cast<char*>(binned_frames[t0 + j]),
                               reinterpret_cast<const char*>(s->d_out2[b]) + j * fout, fout});
            if ((rc = pin_out ? sg.direct(out, cudaMemcpyDeviceToHost, s->s_out) : sg.out(out))) return rc;
            ST_CUDA(cudaEventRecord(s->ev_outdone[b], s->s_out));
        }
        if ((rc = sg.drain_all())) return rc;
        ST_CUDA(cudaStreamSynchronize(s->s_out));
        ST_CUDA(cudaStreamSynchronize(st));
        return AT3R_OK;
    };
    rc = body();
    if (rc) {
        cudaStreamSynchronize(s->s_in);
        cudaStreamSynchronize(s->s_out);
        cudaStreamSynchronize(st);
        cudaGetLastError();
    }
    stage_release(stage);
    return rc;
}

// CCalcVolThick::DoIt on a device-resident (raw) or host (frames) series.
at3r_status thickness_impl(const at3r_stack_geom* g, const float* tilts_deg, float pix_size, const float* raw,
                           const float* const* frames, float* profile, float* profile_smoothed, int profile_cap,
                           at3r_thickness* res, void* stream)
{
    if (!g || !tilts_deg || !(raw || frames) || !res) return st_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    if (!(pix_size > 0.f)) return st_err(AT3R_ERR_INVALID_ARGUMENT, "pixel size must be > 0");
    std::memset(res, 0, sizeof(*res));
    cudaStream_t st = (cudaStream_t)stream;
    // CCalcVolThick::DoIt: binning max(20 A / pixel, 20), Fourier crop with
    // random fill, rotation by the tilt axis, no local patches
    at3r_stack_geom h = *g;
    h.correct = 1;
    h.rand_fill = 1;
    h.num_patches = 0;
    h.local_params = nullptr;
    h.bin = std::fmax(20.0f / pix_size, 20.0f);
    res->binning = h.bin;
    at3r_stack* s = nullptr;
    at3r_status rc = at3r_stack_create(&h, &s);
    if (rc) return rc;
    const int bx = s->bx, by = s->by, T = s->T;
    res->binned_xy[0] = bx;
    res->binned_xy[1] = by;
    const int vol_z = (int)(bx * 0.8) / 2 * 2;
    res->vol_z = vol_z;
    const int n = vol_z - 1;
    if (n < 10 || bx < 4) {
        at3r_stack_destroy(s);
        return st_err(AT3R_ERR_INVALID_ARGUMENT, "series too small for the thickness measurement after binning by " +
                                                     std::to_string(h.bin));
    }
    float* binned = nullptr;
    float* vol = nullptr;
    float* d_prof = nullptr;
    at3r_plan* plan = nullptr;
    auto cleanup = [&](at3r_status r) {
        if (plan) at3r_plan_destroy(plan);
        cudaStreamSynchronize(st);
        for (void* p : {(void*)binned, (void*)vol, (void*)d_prof})
            if (p) cudaFree(p);
        at3r_stack_destroy(s);
        return r;
    };
    if ((rc = salloc(&binned, (size_t)T * bx * by))) return cleanup(rc);
    if ((rc = raw ? at3r_stack_run_device(s, raw, binned, stream)
                  : stack_pipeline(s, frames, nullptr, binned, stream)))
        return cleanup(rc);
    // low-resolution WBP (CDoWbpRecon::DoIt) of the binned series
    at3r_geom wg;
    at3r_geom_init(&wg, AT3R_WBP);
    wg.nx = bx;
    wg.ny = by;
    wg.n_tilts = T;
    wg.tilts_deg = tilts_deg;
    wg.vol_z = vol_z;
    if ((rc = at3r_plan_create(&wg, &plan))) return cleanup(rc);
    const int Nx = bx & ~1;
    if ((rc = salloc(&vol, (size_t)by * vol_z * Nx))) return cleanup(rc);
    if ((rc = at3r_run_device(plan, binned, vol, stream))) return cleanup(rc);
    // plane statistics of FlipVol(true) (CCalcVolThick.cpp:85-103, 172-197,
    // 199-206): tile 40 % of x and y (even), centred in x; its rows start at
    // row 0 because mMeasureStd indexes row j, not start + j
    const int tx = (int)(Nx * 0.4f) / 2 * 2, ty = (int)(by * 0.4f) / 2 * 2;
    const int x0 = (Nx - tx) / 2;
    if ((rc = salloc(&d_prof, (size_t)n))) return cleanup(rc);
    k_plane_std<<<n, 256, 0, st>>>(vol, Nx, vol_z, x0, 0, tx, ty, d_prof);
    std::vector<float> cc(n);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(cc.data(), d_prof, sizeof(float) * n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return cleanup(st_err(AT3R_ERR_CUDA, "plane statistics failed"));
    }
    if (profile) std::memcpy(profile, cc.data(), sizeof(float) * std::min(n, std::max(profile_cap, 0)));
    smooth_profile(cc);
    if (profile_smoothed) std::memcpy(profile_smoothed, cc.data(), sizeof(float) * std::min(n, std::max(profile_cap, 0)));
    detect_edges(cc, h.bin, res);
    res->n_profile = n;
    return cleanup(AT3R_OK);
}

}  // namespace

extern "C" {

void at3r_stack_geom_init(at3r_stack_geom* g)
{
    if (!g) return;
    std::memset(g, 0, sizeof(*g));
    g->correct = 1;
    g->rand_fill = 1;
    g->bin = 1.0f;
}

void at3r_stack_destroy(at3r_stack* s)
{
    if (!s) return;
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != s->device) cudaSetDevice(s->device);
    cudaDeviceSynchronize();
    for (void* p : {(void*)s->d_shift, (void*)s->d_cs, (void*)s->d_local, (void*)s->d_rand, (void*)s->d_flags,
                    (void*)s->d_aln, (void*)s->d_empty, (void*)s->d_Y, (void*)s->d_Wc, (void*)s->d_raw2[0],
                    (void*)s->d_raw2[1], (void*)s->d_out2[0], (void*)s->d_out2[1], (void*)s->frow.d_tables,
                    (void*)s->fcin.d_tables, (void*)s->fcout.d_tables, (void*)s->fbx.d_tables})
        if (p) cudaFree(p);
    for (cudaEvent_t* e : {&s->ev_in[0], &s->ev_in[1], &s->ev_comp[0], &s->ev_comp[1], &s->ev_outdone[0],
                           &s->ev_outdone[1], &s->ev_slot[0], &s->ev_slot[1], &s->ev_slot[2], &s->ev_slot[3]})
        if (*e) cudaEventDestroy(*e);
    if (s->s_in) cudaStreamDestroy(s->s_in);
    if (s->s_out) cudaStreamDestroy(s->s_out);
    cudaGetLastError();
    if (cur >= 0 && cur != s->device) cudaSetDevice(cur);
    delete s;
}

at3r_status at3r_stack_create(const at3r_stack_geom* g, at3r_stack** out)
{
    if (!g || !out) return st_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (g->nx < 2 || g->ny < 2 || g->n_tilts < 1)
        return st_err(AT3R_ERR_INVALID_ARGUMENT, "sizes must satisfy nx >= 2, ny >= 2, n_tilts >= 1");
    if (!(g->bin >= 1.0f)) return st_err(AT3R_ERR_INVALID_ARGUMENT, "bin must be >= 1");
    if (g->num_patches < 0 || (g->num_patches > 0 && !g->local_params))
        return st_err(AT3R_ERR_INVALID_ARGUMENT, "num_patches > 0 needs local_params");
    if ((long long)g->nx * g->ny >= (1LL << 31))
        return st_err(AT3R_ERR_TOO_LARGE, "frames must hold fewer than 2^31 pixels");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return st_err(AT3R_ERR_NO_DEVICE, "no CUDA device");
    }
    at3r_stack* s = new at3r_stack();
    auto fail = [&](at3r_status rc) {
        at3r_stack_destroy(s);
        return rc;
    };
    s->g = *g;
    s->g.shifts = s->g.tilt_axes_deg = s->g.local_params = nullptr;
    cudaGetDevice(&s->device);
    s->nx = g->nx;
    s->ny = g->ny;
    s->T = g->n_tilts;
    int a[2] = {g->nx, g->ny}, b[2];
    if (g->correct) aligned_size(g->nx, g->ny, g->size_axis_deg, a);
    s->ax = a[0];
    s->ay = a[1];
    // the width GCorrPatchShift / GFillEmpty2D cover: (padX / 2 - 1) * 2, padX = (ax / 2 + 1) * 2
    s->W = ((s->ax / 2 + 1) * 2 / 2 - 1) * 2;
    binned_size(a, g->bin, b);
    s->bx = b[0];
    s->by = b[1];
    if (s->bx < 2 || s->by < 2) return fail(st_err(AT3R_ERR_INVALID_ARGUMENT, "binned frame smaller than 2 x 2"));
    s->same = (s->bx == s->ax && s->by == s->ay);
    s->KXo = s->bx / 2 + 1;
    s->P = g->correct ? g->num_patches : 0;
    s->norm = (float)(1.0 / s->ax / s->ay);
    at3r_status rc;

    // per-tilt alignment: shifts, rotation (GCorrPatchShift::DoIt's degree-to-radian factor), patches
    const size_t T = s->T;
    if (g->correct) {
        std::vector<float2> sh(T, make_float2(0.f, 0.f));
        if (g->shifts)
            for (size_t t = 0; t < T; t++) sh[t] = make_float2(g->shifts[2 * t], g->shifts[2 * t + 1]);
        const float d2r = 3.141592654f / 180.0f;
        std::vector<float> rad(T, 0.f);
        if (g->tilt_axes_deg)
            for (size_t t = 0; t < T; t++) rad[t] = g->tilt_axes_deg[t] * d2r;
        double sum_c = 0.0, sum_s = 0.0;
        for (size_t t = 0; t < T; t++) {
            sum_c += std::fabs(std::cos((double)rad[t]));
            sum_s += std::fabs(std::sin((double)rad[t]));
        }
        s->by_rows = sum_s > sum_c ? 1 : 0;
        float* d_rad = nullptr;
        if ((rc = salloc(&s->d_shift, T)) || (rc = salloc(&s->d_cs, T)) || (rc = salloc(&d_rad, T)))
            return fail(rc);
        // set-up kernels on a private stream, so that other work on the device is not waited for
        cudaStream_t ss = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&ss, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_shift, sh.data(), sizeof(float2) * T, cudaMemcpyHostToDevice, ss);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_rad, rad.data(), sizeof(float) * T, cudaMemcpyHostToDevice, ss);
        if (e == cudaSuccess) {
            k_axis_cs<<<(s->T + 127) / 128, 128, 0, ss>>>(d_rad, s->T, s->d_cs);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && g->rand_fill) {
            // one table per set-up, as GFillEmpty2D::SetSize draws it (GFillEmpty2D.cu:100-116)
            const int npx = s->W * s->ay;
            if ((rc = salloc(&s->d_rand, (size_t)npx))) {
                cudaStreamSynchronize(ss);
                cudaStreamDestroy(ss);
                cudaFree(d_rad);
                return fail(rc);
            }
            k_rand_table<<<(npx + 255) / 256, 256, 0, ss>>>(s->d_rand, npx, g->seed);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(ss);
        if (ss) cudaStreamDestroy(ss);
        cudaFree(d_rad);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(st_err(AT3R_ERR_CUDA, std::string("alignment tables: ") + cudaGetErrorString(e)));
        }
        if (s->P > 0) {
            if ((rc = salloc(&s->d_local, T * 5 * s->P))) return fail(rc);
            if (cudaMemcpy(s->d_local, g->local_params, sizeof(float) * T * 5 * s->P, cudaMemcpyHostToDevice) !=
                cudaSuccess)
                return fail(st_err(AT3R_ERR_CUDA, "local alignment upload failed"));
        }
    }

    // FFT plans of the binning (row length ax, column lengths ay -> by, C2R length bx)
    if (!s->same) {
        bool measured = false;
        s->c2r = probe_cufft_c2r(s->by, s->bx, &measured);
        if (!measured)
            return fail(st_err(AT3R_ERR_UNSUPPORTED, "cannot ask cuFFT which C2R convention it uses for the "
                                                     "binned size (libcufft not loadable)"));
        if ((rc = make_fft_tables(s->ax, s->frow)) || (rc = make_fft_tables(s->ay, s->fcin)) ||
            (rc = make_fft_tables(s->by, s->fcout)) || (rc = make_fft_tables(s->bx, s->fbx)))
            return fail(rc);
        s->b_row = row_batch(s->frow.plan.work);
        s->b_c2r = row_batch(s->fbx.plan.work);
        s->smem_row = 2 * sizeof(float2) * fft_pitch(s->frow.plan.work) * s->b_row;
        s->smem_c2r = 2 * sizeof(float2) * fft_pitch(s->fbx.plan.work) * s->b_c2r;
        s->col_pitch = (fft_pitch(std::max(s->fcin.plan.work, s->fcout.plan.work)) + 1) / 2 * 2 + 1;
        s->cb = std::max(1, std::min(32, 4096 / s->ay));
        while (s->cb > 1 && 2 * sizeof(float2) * s->cb * s->col_pitch > 227 * 1024) s->cb /= 2;
        s->smem_col = 2 * sizeof(float2) * s->cb * s->col_pitch;
        s->rs_col = std::max(s->fcin.rs, s->fcout.rs);
        std::vector<std::pair<const void*, size_t>> fns;
        dispatch_rs(s->frow.rs, [&](auto R) { fns.push_back({(const void*)k_bin_r2c<decltype(R)::value>, s->smem_row}); });
        dispatch_rs(s->rs_col, [&](auto R) { fns.push_back({(const void*)k_bin_cols<decltype(R)::value>, s->smem_col}); });
        dispatch_rs(s->fbx.rs, [&](auto R) { fns.push_back({(const void*)k_bin_c2r<decltype(R)::value>, s->smem_c2r}); });
        for (auto& f : fns)
            if ((rc = set_smem_attr(f.first, f.second))) return fail(rc);
    }

    // tilts per pass: the per-tilt workspace of a pass stays within 8 GB
    size_t per_tilt = 0;
    if (g->correct) per_tilt += sizeof(float) * (size_t)s->ax * s->ay + (g->rand_fill ? (size_t)s->W * s->ay : 0);
    if (!s->same) per_tilt += sizeof(float2) * (size_t)s->KXo * (s->ay + s->by);
    s->chunk = (int)std::max<size_t>(1, std::min<size_t>(T, (size_t)(8ull << 30) / std::max<size_t>(per_tilt, 1)));
    const size_t C = s->chunk;
    if (g->correct) {
        if ((rc = salloc(&s->d_aln, C * s->ax * s->ay))) return fail(rc);
        if (g->rand_fill && ((rc = salloc(&s->d_empty, C * s->W * s->ay)) || (rc = salloc(&s->d_flags, C))))
            return fail(rc);
    }
    if (!s->same) {
        if ((rc = salloc(&s->d_Y, C * s->ay * s->KXo)) || (rc = salloc(&s->d_Wc, C * s->by * s->KXo)))
            return fail(rc);
    }
    *out = s;
    return AT3R_OK;
}

at3r_status at3r_stack_sizes(const at3r_stack* s, int* aligned_xy, int* binned_xy)
{
    if (!s) return st_err(AT3R_ERR_INVALID_ARGUMENT, "null stack");
    if (aligned_xy) {
        aligned_xy[0] = s->ax;
        aligned_xy[1] = s->ay;
    }
    if (binned_xy) {
        binned_xy[0] = s->bx;
        binned_xy[1] = s->by;
    }
    return AT3R_OK;
}

int at3r_stack_c2r(const at3r_stack* s) { return s ? s->c2r : 0; }

at3r_status at3r_stack_fill_table(const at3r_stack* s, int* table, size_t n)
{
    if (!s || !table) return st_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    if (!s->d_rand) return st_err(AT3R_ERR_INVALID_ARGUMENT, "the stack has no random fill");
    const size_t need = (size_t)s->W * s->ay;
    if (n < need) return st_err(AT3R_ERR_INVALID_ARGUMENT, "table capacity below " + std::to_string(need));
    at3r_status rc;
    if ((rc = check_device(s))) return rc;
    ST_CUDA(cudaMemcpy(table, s->d_rand, sizeof(int) * need, cudaMemcpyDeviceToHost));
    return AT3R_OK;
}

at3r_status at3r_stack_run_device(at3r_stack* s, const float* raw, float* binned, void* stream)
{
    if (!s || !raw || !binned) return st_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    at3r_status rc;
    if ((rc = check_device(s))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    for (int t0 = 0; t0 < s->T; t0 += s->chunk) {
        const int n = std::min(s->chunk, s->T - t0);
        if ((rc = run_chunk(s, raw + (size_t)t0 * s->nx * s->ny, t0, n, binned + (size_t)t0 * s->bx * s->by, st)))
            return rc;
    }
    return AT3R_OK;
}

at3r_status at3r_stack_run_host(at3r_stack* s, const float* const* frames, float* const* binned_frames, void* stream)
{
    if (!s || !frames || !binned_frames) return st_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    at3r_status rc;
    if ((rc = check_device(s))) return rc;
    for (int t = 0; t < s->T; t++)
        if (!frames[t] || !binned_frames[t]) return st_err(AT3R_ERR_INVALID_ARGUMENT, "null frame pointer");
    return stack_pipeline(s, frames, binned_frames, nullptr, stream);
}

at3r_status at3r_thickness_device(const at3r_stack_geom* g, const float* tilts_deg, float pix_size, const float* raw,
                                  float* profile, float* profile_smoothed, int profile_cap, at3r_thickness* res,
                                  void* stream)
{
    if (!raw) return st_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    return thickness_impl(g, tilts_deg, pix_size, raw, nullptr, profile, profile_smoothed, profile_cap, res, stream);
}

at3r_status at3r_thickness_host(const at3r_stack_geom* g, const float* tilts_deg, float pix_size,
                                const float* const* frames, float* profile, float* profile_smoothed, int profile_cap,
                                at3r_thickness* res, void* stream)
{
    if (!g || !frames) return st_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    if (g->nx < 2 || g->ny < 2 || g->n_tilts < 1) return st_err(AT3R_ERR_INVALID_ARGUMENT, "invalid sizes");
    for (int t = 0; t < g->n_tilts; t++)
        if (!frames[t]) return st_err(AT3R_ERR_INVALID_ARGUMENT, "null frame pointer");
    return thickness_impl(g, tilts_deg, pix_size, nullptr, frames, profile, profile_smoothed, profile_cap, res, stream);
}

}  // extern "C"
