// C-ABI implementation: plans, workspace, the y-slab loop and the host-buffer
// path.  Declarations and data layouts: include/at3r.h.
#include "at3r.h"
#include "at3r_internal.h"
#include "fft_host.h"
#include "recon_kernels.cuh"

#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <ctime>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

using namespace at3r;

namespace {

thread_local std::string g_last_error;

at3r_status set_err(at3r_status s, const std::string& msg)
{
    g_last_error = msg;
    return s;
}

#define AT3R_CUDA(call)                                                                        \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return set_err(e_ == cudaErrorMemoryAllocation ? AT3R_ERR_OUT_OF_MEMORY : AT3R_ERR_CUDA, \
                           std::string(#call) + ": " + cudaGetErrorString(e_));                \
    } while (0)

at3r_status dalloc_bytes(at3r_plan* p, void** ptr, size_t bytes);   // defined with the plan

at3r_status make_fft(at3r_plan* pl, int n, HostFft& h)
{
    std::vector<float2> all;
    plan_fft(n, h, all);
    at3r_status ra = dalloc_bytes(pl, reinterpret_cast<void**>(&h.d_tables), h.bytes);
    if (ra != AT3R_OK) return ra;
    AT3R_CUDA(cudaMemcpy(h.d_tables, all.data(), h.bytes, cudaMemcpyHostToDevice));
    bind_fft(h);
    return AT3R_OK;
}

int round_up(int a, int b) { return (a + b - 1) / b * b; }

enum KernelKind { KK_GATHER, KK_RWEIGHT, KK_BP_SART, KK_BP_WBP, KK_FP_DIFF, KK_FILL, KK_ROW_R2C, KK_ZCROP, KK_XC2R,
                  KK_UNGROUP, KK_COUNT };
const char* kKernelNames[KK_COUNT] = {"gather_weight", "rweight", "bp_sart", "bp_wbp_2x", "fp_diff",
                                      "fill_empty", "row_r2c", "zcrop", "x_c2r", "ungroup"};
struct KStat {
    int64_t launches;
    double bytes, units, ms;
};

}  // namespace

struct at3r_plan {
    at3r_geom g{};
    std::vector<float> tilts;
    int nx = 0, ny = 0, T = 0, N = 0, Nx = 0, Nz = 0, KX = 0;
    int slab = 1;
    int slab_cap = 1;   // slices the workspace holds; the autotuner picks slab <= slab_cap
    cudaStream_t alloc_stream = nullptr;   // set: workspace from the memory pool, ordered on this stream
    int device = 0;
    int c2r = AT3R_C2R_HERMITIAN;
    float relax = 1.f;
    std::vector<int> sub_start, sub_size;
    float2* d_cs = nullptr;
    // staged sinograms: element size by storage type; row scales for 16-bit storage
    size_t esz = sizeof(float);
    float* d_scale = nullptr;
    // SART
    void* d_raw = nullptr;
    void* d_diff = nullptr;
    void* d_shadow = nullptr;   // 16-bit storage: the volume shadow the forward projector reads
    float4* d_w = nullptr;      // SART working volume, slice groups [ceil(S/4)][Nz][Nx] x 4 slices
    int* d_flags = nullptr;
    int* d_seen = nullptr;                 // run summary: every slice's flag bits ORed in
    unsigned long long fill_seed = 0;      // seed of the empty-voxel fill's random table
    double* d_rf = nullptr;
    std::vector<double> h_rf;
    // WBP
    float* d_h = nullptr;
    void* d_filt = nullptr;
    float* d_g2 = nullptr;    // also holds the cropped spectrum w
    float2* d_y = nullptr;
    // WBP: a second workspace and stream, so that alternate slabs overlap
    // (one slab's kernel tails fill with the next slab's kernels)
    struct WbpLane {
        void* filt = nullptr;
        float* scale = nullptr;
        int* flags = nullptr;
        float* g2 = nullptr;
        float2* y = nullptr;
    } lane2;
    cudaStream_t s_lane2 = nullptr;
    cudaEvent_t ev_lane[2] = {};
    HostFft fN, f2x, f2z, fz, fx;
    int zcrop_cb = 4, zcrop_pitch = 0;
    int b_rweight = 1, b_row = 1, b_xc2r = 1;   // sequences per CTA of the row FFT kernels
    int rs_zcrop = 0;                           // radix set of the z-crop kernel (both its lengths)
    size_t smem_rweight = 0, smem_row = 0, smem_zcrop = 0, smem_xc2r = 0;
    int bp_ww_sart = 0, bp_ww_wbp = 0;
    int bp_bulk = 0;   // FP32 back-projection staging by bulk asynchronous copies (AT3R_BP_BULK_STAGING)
    // host path
    float* d_proj_slab[2] = {nullptr, nullptr};
    float* d_vol_slab[2] = {nullptr, nullptr};
    float* d_xyz_slab[2] = {nullptr, nullptr};   // XY-frame copy of a slab (output stage)
    // pinned staging rings for pageable caller frames (input, output), borrowed
    // from the process-wide staging pool for one run
    char* h_stage_in[2] = {nullptr, nullptr};
    char* h_stage_out[2] = {nullptr, nullptr};
    cudaEvent_t ev_stage[4] = {};               // [0,1]: input ring slot free; [2,3]: output ring slot filled
    bool pooled = false;                        // workspace from the library memory pool
    cudaStream_t s_copy_in = nullptr, s_copy_out = nullptr;
    cudaEvent_t ev[8] = {};
    size_t ws_bytes = 0;
    int64_t launches = 0;
    // per-kernel accounting of the last run; device times only with timing on
    bool timing = false;
    std::vector<cudaEvent_t> evpool;
    size_t evused = 0;
    std::vector<std::pair<int, size_t>> pending;  // (kind, index of the start event)
    KStat stats[KK_COUNT] = {};
    std::vector<int> ray_len;                     // forward-projection samples per ray, per tilt
};

namespace {

// Workspace allocation: cudaMalloc, or — for plans made by the serving loop —
// stream-ordered from the device's memory pool on the plan's allocation
// stream, so that freeing it does not synchronise the device.
// The library's device memory pool (one per device): plan workspaces come
// from it and go back to it, so creating and destroying plans does not map
// and unmap device memory each time (a cudaFree of a 1k SART plan's 7.5 GB
// took 0.6 s).  at3r_release_cached_memory hands the pool's free memory back.
struct DevicePool {
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
};
std::mutex g_pool_mu;
std::map<int, DevicePool> g_pools;

DevicePool* device_pool(int dev)
{
    std::lock_guard<std::mutex> lk(g_pool_mu);
    DevicePool& dp = g_pools[dev];
    if (!dp.pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        if (cudaMemPoolCreate(&dp.pool, &props) != cudaSuccess) {
            cudaGetLastError();
            dp.pool = nullptr;
            return nullptr;
        }
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(dp.pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (cudaStreamCreateWithFlags(&dp.stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            cudaMemPoolDestroy(dp.pool);
            dp.pool = nullptr;
            return nullptr;
        }
    }
    return &dp;
}

at3r_status dalloc_bytes(at3r_plan* p, void** ptr, size_t bytes)
{
    cudaError_t e;
    if (p->alloc_stream) {
        e = cudaMallocAsync(ptr, bytes, p->alloc_stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(p->alloc_stream);
    } else if (DevicePool* dp = p->pooled ? device_pool(p->device) : nullptr) {
        e = cudaMallocFromPoolAsync(ptr, bytes, dp->pool, dp->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(dp->stream);
    } else {
        e = cudaMalloc(ptr, bytes);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_err(AT3R_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    p->ws_bytes += bytes;
    return AT3R_OK;
}

template <typename T>
at3r_status dalloc(at3r_plan* p, T** ptr, size_t count)
{
    return dalloc_bytes(p, reinterpret_cast<void**>(ptr), count * sizeof(T));
}

void dfree(at3r_plan* p, void* ptr)
{
    if (!ptr) return;
    if (p->alloc_stream) cudaFreeAsync(ptr, p->alloc_stream);
    else if (DevicePool* dp = p->pooled ? device_pool(p->device) : nullptr) cudaFreeAsync(ptr, dp->stream);
    else cudaFree(ptr);
}

int bp_window(int tx, int tz, double scale, const std::vector<float>& cs, int T)
{
    double span = 0;
    for (int t = 0; t < T; t++)
        span = std::max(span, (std::fabs(cs[2 * t]) * (tx - 1) + std::fabs(cs[2 * t + 1]) * (tz - 1)) * scale);
    return (int)std::ceil(span) + 6;
}

// tilts are staged in chunks, so the window buffer does not grow with the tilt count
// dynamic shared memory of a back-projection launch (bulk: the bulk-copy
// staging's raw rows and mbarrier on top)
size_t bp_smem(int bulk) { return bp_smem_bytes(bulk); }

// Back-projection window staging by bulk asynchronous copies (FP32 storage,
// N a multiple of 4): off unless AT3R_BP_BULK_STAGING=1 at plan creation; an
// alternative to the load path, kept for comparison.
bool bp_bulk_from_env()
{
    const char* e = std::getenv("AT3R_BP_BULK_STAGING");
    return e && e[0] == '1';
}

// Threads of a row / column FFT launch: 1024 when two CTAs' shared memory
// would not fit one SM (so one CTA holds 32 warps) and the radix set allows.
int fft_threads(int rs, size_t smem)
{
    const bool one_cta = 2 * (smem + 1024) > (228u << 10);
    return rs < 2 && one_cta ? 1024 : 512;
}

// Every plan raises a kernel's dynamic shared-memory limit to the device
// maximum (once per kernel and device), so plans of different sizes can
// coexist; the amount a launch uses is still its own.
at3r_status set_smem(const void* fn, size_t bytes)
{
    int dev = 0, optin = 0;
    AT3R_CUDA(cudaGetDevice(&dev));
    AT3R_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa{};
    AT3R_CUDA(cudaFuncGetAttributes(&fa, fn));
    const size_t kMax = (size_t)optin - fa.sharedSizeBytes;   // dynamic part the kernel may ask for
    if (bytes > kMax)
        return set_err(AT3R_ERR_TOO_LARGE, "shared-memory need " + std::to_string(bytes) + " exceeds " +
                                               std::to_string(kMax) + " bytes");
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, bool> done;
    std::lock_guard<std::mutex> lk(mu);
    if (!done[{fn, dev}]) {
        AT3R_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMax));
        done[{fn, dev}] = true;
    }
    return AT3R_OK;
}

// Launch bookkeeping: tbegin/tend bracket every kernel launch.  With timing
// enabled each launch is bracketed by two events on its own stream; the
// algorithmic bytes (compulsory DRAM reads + writes) and work units of every
// launch are tallied always.
at3r_status tbegin(at3r_plan* p, cudaStream_t st)
{
    if (!p->timing) return AT3R_OK;
    if (p->evused + 2 > p->evpool.size()) {
        for (int i = 0; i < 256; i++) {
            cudaEvent_t e;
            AT3R_CUDA(cudaEventCreate(&e));
            p->evpool.push_back(e);
        }
    }
    AT3R_CUDA(cudaEventRecord(p->evpool[p->evused], st));
    return AT3R_OK;
}

at3r_status tend(at3r_plan* p, cudaStream_t st, int kind, double bytes, double units)
{
    p->launches++;
    KStat& k = p->stats[kind];
    k.launches++;
    k.bytes += bytes;
    k.units += units;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(AT3R_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    if (p->timing) {
        AT3R_CUDA(cudaEventRecord(p->evpool[p->evused + 1], st));
        p->pending.push_back({kind, p->evused});
        p->evused += 2;
    }
    return AT3R_OK;
}

#define TB(p, st)                                  \
    do {                                           \
        at3r_status r_ = tbegin((p), (st));        \
        if (r_ != AT3R_OK) return r_;              \
    } while (0)
#define TE(p, st, kind, bytes, units)                                  \
    do {                                                               \
        at3r_status r_ = tend((p), (st), (kind), (double)(bytes), (double)(units)); \
        if (r_ != AT3R_OK) return r_;                                  \
    } while (0)

// One slab of slices [y0, y0 + S): proj points at tilt 0 row 0 of a
// [T][rows][nx] block whose row `proj_y0` is slice y0; vol points at the
// slab's first output slice.
template <typename ST, typename VT>
at3r_status run_slab_t(at3r_plan* p, const float* proj, size_t tilt_stride, int proj_y0, int S, float* vol,
                       cudaStream_t st, int lane)
{
    // WBP slabs on the second lane use its workspace
    int* const flags = lane ? p->lane2.flags : p->d_flags;
    float* const scale = lane ? p->lane2.scale : p->d_scale;
    void* const filt_ws = lane ? p->lane2.filt : p->d_filt;
    float* const g2 = lane ? p->lane2.g2 : p->d_g2;
    float2* const yws = lane ? p->lane2.y : p->d_y;
    ST* raw = static_cast<ST*>(p->d_raw);
    ST* dif = static_cast<ST*>(p->d_diff);
    ST* filt = static_cast<ST*>(filt_ws);
    const double es = (double)sizeof(ST), vs = std::is_same<VT, float>::value ? 4.0 : 2.0;
    const int T = p->T, N = p->N, Nx = p->Nx, Nz = p->Nz, KX = p->KX;
    const double f4 = 4.0, vox = (double)S * Nx * Nz;
    const int SG = (S + SB - 1) / SB;   // slice groups: each thread carries SB slices
    AT3R_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * S, st));
    if (p->g.method == AT3R_SART) {
        TB(p, st);
        k_gather_weight<ST><<<dim3(T, S), 256, 0, st>>>(proj, tilt_stride, p->nx, proj_y0, p->d_cs, T, N, Nz, raw,
                                                        p->d_scale, p->d_flags);
        TE(p, st, KK_GATHER, (f4 + es) * S * T * N, (double)S * T * N);
        // the working volume in slice groups: one 16-byte (or 8-byte shadow)
        // load gives a tap of four slices; unpacked into vol at the end
        AT3R_CUDA(cudaMemsetAsync(p->d_w, 0, sizeof(float4) * (size_t)SG * Nx * Nz, st));
        // the 16-bit shadow: eight slices per voxel
        const int SG8 = (S + 7) / 8;
        if (p->d_shadow) AT3R_CUDA(cudaMemsetAsync(p->d_shadow, 0, sizeof(uint4) * (size_t)SG8 * Nx * Nz, st));
        BpArgs a{};
        a.T = T; a.N = N; a.cs = p->d_cs; a.GX = Nx; a.GZ = Nz; a.S = S;
        a.out = reinterpret_cast<float*>(p->d_w); a.out_slice = (size_t)Nx * Nz; a.ww = p->bp_ww_sart;
        a.flags = p->d_flags; a.seen = p->d_seen; a.bulk = p->bp_bulk;
        a.scale = p->d_scale; a.shadow = p->d_shadow;
        const dim3 bgrid = bp_paired<VT>()
                               ? dim3(2 * ((Nx + BP_TX - 1) / BP_TX), (Nz + BP_TZ - 1) / BP_TZ, (SG + 1) / 2)
                               : dim3((Nx + BP_TX - 1) / BP_TX, (Nz + BP_TZ - 1) / BP_TZ, SG);
        auto bp_launch = [&](int nt_) {
            if constexpr (std::is_same<ST, float>::value) {
                if (a.bulk) {
                    k_bp<0, ST, VT, true, true><<<bgrid, BP_THREADS, bp_smem(1), st>>>(a);
                    return;
                }
            }
            k_bp<0, ST, VT, true><<<bgrid, BP_THREADS, bp_smem(0), st>>>(a);
        };
        // first back-projection: all tilts, relax 1 (CTomoSart.cpp:68-69)
        a.sino = raw; a.t0 = 0; a.t1 = T; a.relax = 1.f; a.low_bit = kFlagRawLow;
        TB(p, st);
        bp_launch(T);
        TE(p, st, KK_BP_SART, es * S * (double)T * N + (2 * f4 + (vs < 4 ? vs : 0)) * vox, vox * T);
        a.sino = dif; a.relax = p->relax; a.low_bit = kFlagDiffLow;
        for (int it = 0; it < p->g.iterations; it++) {
            for (size_t s = 0; s < p->sub_start.size(); s++) {
                const int t0 = p->sub_start[s] + p->g.start_tilt, nt = p->sub_size[s];
                if (nt <= 0) continue;
                double samples = 0;
                for (int t = t0; t < t0 + nt; t++) samples += (double)p->ray_len[t];
                double* rfp = p->g.compute_rfactor ? p->d_rf + 2 * it : nullptr;
                TB(p, st);
                k_fp_diff<ST, VT, true><<<dim3((N + 255) / 256, nt, (S + fp_slices<VT>() - 1) / fp_slices<VT>()), 256,
                                          0, st>>>(
                    reinterpret_cast<const float*>(p->d_w), p->d_shadow, Nx, Nz, S, raw, dif, p->d_scale, p->d_cs, T,
                    N, t0, rfp, p->d_flags);
                TE(p, st, KK_FP_DIFF, vs * vox + 2.0 * es * S * nt * N, samples * N * S);
                a.t0 = t0; a.t1 = t0 + nt;
                TB(p, st);
                bp_launch(nt);
                TE(p, st, KK_BP_SART, es * S * (double)nt * N + (2 * f4 + (vs < 4 ? vs : 0)) * vox, vox * nt);
            }
        }
        TB(p, st);
        k_ungroup<<<dim3((unsigned)(((size_t)Nx * Nz + 255) / 256), SG), 256, 0, st>>>(p->d_w, vol, S,
                                                                                       (size_t)Nx * Nz);
        TE(p, st, KK_UNGROUP, 2 * f4 * vox, vox);
        // the empty-voxel fill (CTomoSart.cpp:88); only flagged slices do work
        const int fb = std::max(1, std::min((Nx * Nz + 255) / 256, (8 * 148 + S - 1) / S));
        TB(p, st);
        k_fill_mark<<<dim3(fb, S), 256, 0, st>>>(vol, Nx, Nz, p->d_flags, p->fill_seed, p->d_seen);
        TE(p, st, KK_FILL, f4 * S, 0);
        TB(p, st);
        k_fill_finish<<<S, 512, 0, st>>>(vol, Nx, Nz, p->d_flags, p->d_seen);
        TE(p, st, KK_FILL, f4 * S, 0);
        return AT3R_OK;
    }
    // WBP
    TB(p, st);
    dispatch_rs(p->fN.rs, [&](auto R) {
        k_rweight<ST, decltype(R)::value><<<dim3(((T + 1) / 2 + p->b_rweight - 1) / p->b_rweight, S), 512,
                                            p->smem_rweight, st>>>(proj, tilt_stride, p->nx, proj_y0, p->d_cs, T, N,
                                                                   Nz, p->d_h, p->fN.plan, p->b_rweight, filt,
                                                                   scale, flags);
    });
    TE(p, st, KK_RWEIGHT, (f4 + es) * S * T * N, (double)S * T * N);
    BpArgs a{};
    a.sino = filt; a.scale = scale; a.shadow = nullptr; a.T = T; a.N = N; a.t0 = 0; a.t1 = T; a.cs = p->d_cs;
    a.GX = 2 * Nx; a.GZ = 2 * Nz; a.S = S; a.relax = 1.f; a.out = g2; a.out_slice = (size_t)4 * Nx * Nz;
    a.ww = p->bp_ww_wbp; a.flags = flags; a.seen = p->d_seen; a.low_bit = kFlagRawLow; a.bulk = p->bp_bulk;
    TB(p, st);
    const dim3 wgrid((2 * Nx + BP_TX - 1) / BP_TX, (2 * Nz + BP_TZ - 1) / BP_TZ, SG);
    bool launched = false;
    if constexpr (std::is_same<ST, float>::value) {
        if (a.bulk) {
            k_bp<1, ST, float, false, true><<<wgrid, BP_THREADS, bp_smem(1), st>>>(a);
            launched = true;
        }
    }
    if (!launched) k_bp<1, ST, float, false><<<wgrid, BP_THREADS, bp_smem(0), st>>>(a);
    TE(p, st, KK_BP_WBP, es * S * (double)T * N + f4 * 4 * vox, 4 * vox * T);
    TB(p, st);
    dispatch_rs(p->f2x.rs, [&](auto R) {
        k_row_r2c<decltype(R)::value><<<dim3((Nz + p->b_row - 1) / p->b_row, S),
                                        fft_threads(decltype(R)::value, p->smem_row), p->smem_row, st>>>(
            g2, Nx, Nz, p->f2x.plan, p->b_row, yws);
    });
    TE(p, st, KK_ROW_R2C, f4 * 4 * vox + 8.0 * S * 2 * Nz * KX, 4 * vox);
    const float norm = (float)(1.0 / (2.0 * Nx) / (2.0 * Nz));
    float2* w = reinterpret_cast<float2*>(g2);
    TB(p, st);
    dispatch_rs(p->rs_zcrop, [&](auto R) {
        k_zcrop<decltype(R)::value><<<dim3((KX + p->zcrop_cb - 1) / p->zcrop_cb, S),
                                      fft_threads(decltype(R)::value, p->smem_zcrop), p->smem_zcrop, st>>>(
            yws, Nx, Nz, p->zcrop_cb, p->zcrop_pitch, p->f2z.plan, p->fz.plan, norm, w);
    });
    TE(p, st, KK_ZCROP, 8.0 * S * 3 * Nz * KX, (double)S * 2 * Nz * KX);
    TB(p, st);
    dispatch_rs(p->fx.rs, [&](auto R) {
        k_x_c2r<decltype(R)::value><<<dim3(((Nz + 1) / 2 + p->b_xc2r - 1) / p->b_xc2r, S), 512, p->smem_xc2r, st>>>(
            w, Nx, Nz, p->fx.plan, p->b_xc2r, p->c2r == AT3R_C2R_PACKED, vol, (size_t)Nx * Nz);
    });
    TE(p, st, KK_XC2R, 8.0 * S * Nz * KX + f4 * vox, vox);
    return AT3R_OK;
}

at3r_status run_slab(at3r_plan* p, const float* proj, size_t tilt_stride, int proj_y0, int S, float* vol,
                     cudaStream_t st, int lane = 0)
{
    switch (p->g.storage) {
        case AT3R_STORE_F16: return run_slab_t<__half, __half>(p, proj, tilt_stride, proj_y0, S, vol, st, lane);
        case AT3R_STORE_BF16:
            return run_slab_t<__nv_bfloat16, __nv_bfloat16>(p, proj, tilt_stride, proj_y0, S, vol, st, lane);
        default: return run_slab_t<float, float>(p, proj, tilt_stride, proj_y0, S, vol, st, lane);
    }
}

// The second WBP lane: allocated on first use (a run of two or more slabs).
at3r_status ensure_lane2(at3r_plan* p)
{
    if (p->s_lane2) return AT3R_OK;
    const size_t S = p->slab_cap, T = p->T, N = p->N, Nx = p->Nx, Nz = p->Nz, KX = p->KX;
    at3r_status rc;
    if ((rc = dalloc_bytes(p, &p->lane2.filt, S * T * N * p->esz))) return rc;
    if (p->g.storage != AT3R_STORE_F32 && (rc = dalloc(p, &p->lane2.scale, S * T))) return rc;
    if ((rc = dalloc(p, &p->lane2.flags, S))) return rc;
    if ((rc = dalloc(p, &p->lane2.g2, S * 4 * Nx * Nz))) return rc;
    if ((rc = dalloc(p, &p->lane2.y, S * 2 * Nz * KX))) return rc;
    for (cudaEvent_t& e : p->ev_lane) AT3R_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    AT3R_CUDA(cudaStreamCreateWithFlags(&p->s_lane2, cudaStreamNonBlocking));
    return AT3R_OK;
}

at3r_status begin_run(at3r_plan* p, cudaStream_t st)
{
    p->launches = 0;
    p->evused = 0;
    p->pending.clear();
    for (KStat& k : p->stats) k = KStat{};
    int dev = -1;
    AT3R_CUDA(cudaGetDevice(&dev));
    if (dev != p->device) return set_err(AT3R_ERR_INVALID_ARGUMENT, "plan was created on another device");
    AT3R_CUDA(cudaMemsetAsync(p->d_seen, 0, sizeof(int), st));
    if (p->g.method == AT3R_SART && p->g.compute_rfactor)
        AT3R_CUDA(cudaMemsetAsync(p->d_rf, 0, sizeof(double) * 2 * std::max(1, p->g.iterations), st));
    return AT3R_OK;
}

at3r_status end_run(at3r_plan* p, cudaStream_t st)
{
    if (p->g.method == AT3R_SART && p->g.compute_rfactor && p->g.iterations > 0)
        AT3R_CUDA(cudaMemcpyAsync(p->h_rf.data(), p->d_rf, sizeof(double) * 2 * p->g.iterations,
                                  cudaMemcpyDeviceToHost, st));
    return AT3R_OK;
}

}  // namespace

cudaMemPool_t at3r_device_pool(int dev)
{
    DevicePool* dp = device_pool(dev);
    return dp ? dp->pool : nullptr;
}

extern "C" {

void at3r_geom_init(at3r_geom* g, int method)
{
    if (!g) return;
    std::memset(g, 0, sizeof(*g));
    g->method = method;
    g->iterations = method == AT3R_SART ? 20 : 0;
    g->subsets = 1;
    g->relax = 0.f;
    g->storage = AT3R_STORE_F32;
    g->c2r = AT3R_C2R_MATCH_CUFFT;
    g->fill_seed = (unsigned long long)time(nullptr);   // as GGenRandoms::DoIt seeds it
}

at3r_status plan_create_impl(const at3r_geom* g, cudaStream_t alloc_stream, at3r_plan** out);

at3r_status at3r_plan_create(const at3r_geom* g, at3r_plan** out) { return plan_create_impl(g, nullptr, out); }

// Default slab (slices per launch).  SART: enough slice groups that one
// subset's forward projection (grid ceil(N/256) x tilts x groups) spans about
// 16 waves of 6 CTAs on every SM — measured on B200, the SART rate keeps
// rising with the slab up to the whole series (1024 x 1024 x 61: 37.9
// GVoxel*tilt/s at 58 slices, 55.2 at 1024) — with the workspace capped at
// 8 GB.  WBP: a 256 MB workspace (larger slabs gain under 3 %).
// per_slice: workspace bytes one slice adds.
int default_slab(const at3r_geom* g, size_t per_slice, int sms)
{
    long S;
    if (g->method == AT3R_SART) {
        const long N = g->nx & ~1;
        const long nt = std::max(1, (g->num_tilts + g->subsets - 1) / std::max(1, g->subsets));
        const long per_group = ((N + 255) / 256) * nt;
        const long target = (long)sms * 6 * 16;
        S = SB * ((target + per_group - 1) / per_group);
        S = std::min(S, (long)((size_t)(8ull << 30) / std::max<size_t>(per_slice, 1)));
    } else {
        S = (long)(((size_t)256 << 20) / std::max<size_t>(per_slice, 1));
    }
    S = std::max(S, 8L);
    return (int)std::min<long>(S, g->ny);
}

// Device bytes a plan and one at3r_run_host over it hold (workspace, FFT
// tables, the host path's two slab buffers), without allocating; an upper
// estimate the serving loop admits requests by.
size_t at3r_plan_estimate_bytes(const at3r_geom* g)
{
    if (!g || g->nx < 1 || g->ny < 1 || g->n_tilts < 1 || g->vol_z < 1) return 0;
    const size_t T = g->n_tilts, N = g->nx & ~1, Nx = N, Nz = g->vol_z, KX = Nx / 2 + 1, nx = g->nx;
    const size_t esz = g->storage == AT3R_STORE_F32 ? 4 : 2;
    size_t per_slice, tables = 0;
    if (g->method == AT3R_SART) {
        per_slice = 2 * T * N * esz + 4 * Nx * Nz + (esz < 4 ? 2 * Nx * Nz + 4 * T : 0);
    } else {
        per_slice = T * N * sizeof(float) + 16 * Nx * Nz + 2 * Nz * KX * sizeof(float2);
        tables = 4 * sizeof(float2) * 4 * (N + 2 * Nx + 3 * Nz + Nx);   // Bluestein can take 4x the length
    }
    size_t slab = g->slab_slices > 0 ? (size_t)g->slab_slices : (size_t)default_slab(g, per_slice, 148);
    slab = std::min<size_t>(slab, (size_t)g->ny);
    size_t work;
    if (g->method == AT3R_SART)
        work = (slab + 7) * (2 * T * N * esz + 4 * Nx * Nz + (esz < 4 ? 2 * Nx * Nz + T * 4 : 0)) + slab * 8;
    else   // two lanes of slab workspace when the series has more than one slab (device path)
        work = (slab < (size_t)g->ny ? 2 : 1) *
               slab * (T * N * esz + 16 * Nx * Nz + 2 * Nz * KX * sizeof(float2) + (esz < 4 ? T * 4 : 0) + 4);
    const size_t host_path = 2 * (T * slab * nx + slab * Nx * Nz) * sizeof(float);
    return work + host_path + tables + T * 8 + (1 << 20);
}

}  // extern "C"

// The serving loop's view of a request (csrc/at3r_server.cpp): its device
// bytes — the plan's workspace on one lane, FFT tables, the projections held
// on the device for the whole request, two volume slabs — and its slab.
size_t at3r_estimate_resident_bytes(const at3r_geom* g, int* slab_out)
{
    if (!g || g->nx < 1 || g->ny < 1 || g->n_tilts < 1 || g->vol_z < 1) return 0;
    const size_t T = g->n_tilts, N = g->nx & ~1, Nx = N, Nz = g->vol_z, KX = Nx / 2 + 1, nx = g->nx, ny = g->ny;
    const size_t esz = g->storage == AT3R_STORE_F32 ? 4 : 2;
    size_t per_slice, tables = 0, work;
    if (g->method == AT3R_SART) {
        per_slice = 2 * T * N * esz + 4 * Nx * Nz + (esz < 4 ? 2 * Nx * Nz + 4 * T : 0);
    } else {
        per_slice = T * N * sizeof(float) + 16 * Nx * Nz + 2 * Nz * KX * sizeof(float2);
        tables = 4 * sizeof(float2) * 4 * (N + 2 * Nx + 3 * Nz + Nx);
    }
    size_t slab = g->slab_slices > 0 ? (size_t)g->slab_slices : (size_t)default_slab(g, per_slice, 148);
    slab = std::min<size_t>(slab, ny);
    if (g->method == AT3R_SART)
        work = (slab + 7) * (2 * T * N * esz + 4 * Nx * Nz + (esz < 4 ? 2 * Nx * Nz + T * 4 : 0)) + slab * 8;
    else
        work = slab * (T * N * esz + 16 * Nx * Nz + 2 * Nz * KX * sizeof(float2) + (esz < 4 ? T * 4 : 0) + 4);
    if (slab_out) *slab_out = (int)slab;
    return work + tables + T * ny * nx * sizeof(float) + 2 * slab * Nx * Nz * sizeof(float) + T * 8 + (1 << 20);
}

// Rows [y0, y0 + n) of a series held on the device, proj[T][ny][nx], into
// vol_rows[n][Nz][Nx] on `st`: one slab of the plan's y loop, with none of a
// run's bookkeeping (timing, R-factor, the run summary).  n <= the plan's slab.
at3r_status at3r_plan_run_slab(at3r_plan* p, const float* proj, int y0, int n, float* vol_rows, cudaStream_t st)
{
    if (!p || !proj || !vol_rows || y0 < 0 || n < 1 || y0 + n > p->ny || n > p->slab_cap)
        return set_err(AT3R_ERR_INVALID_ARGUMENT, "slab outside the series or the plan's workspace");
    return run_slab(p, proj, (size_t)p->ny * p->nx, y0, n, vol_rows, st);
}

extern "C" {

at3r_status plan_create_impl(const at3r_geom* g, cudaStream_t alloc_stream, at3r_plan** out)
{
    if (!g || !out) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (g->nx < 4 || g->ny < 1 || g->n_tilts < 1 || g->vol_z < 2 || !g->tilts_deg)
        return set_err(AT3R_ERR_INVALID_ARGUMENT, "sizes must satisfy nx >= 4, ny >= 1, n_tilts >= 1, vol_z >= 2");
    if ((long long)(g->nx & ~1) * g->vol_z * 4 >= (1LL << 31))
        return set_err(AT3R_ERR_TOO_LARGE, "(nx & ~1) * vol_z must stay below 2^29 (32-bit in-slice offsets)");
    if (g->method != AT3R_WBP && g->method != AT3R_SART)
        return set_err(AT3R_ERR_INVALID_ARGUMENT, "method must be AT3R_WBP or AT3R_SART");
    if (g->storage != AT3R_STORE_F32 && g->storage != AT3R_STORE_F16 && g->storage != AT3R_STORE_BF16)
        return set_err(AT3R_ERR_INVALID_ARGUMENT, "storage must be AT3R_STORE_F32, _F16 or _BF16");
    if (g->method == AT3R_SART) {
        if (g->subsets < 1 || g->iterations < 0)
            return set_err(AT3R_ERR_INVALID_ARGUMENT, "SART needs subsets >= 1 and iterations >= 0");
        if (g->start_tilt < 0 || g->num_tilts < 0 || g->start_tilt + g->num_tilts > g->n_tilts)
            return set_err(AT3R_ERR_INVALID_ARGUMENT, "SART tilt range outside the series");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_err(AT3R_ERR_NO_DEVICE, "no CUDA device");
    }
    at3r_plan* p = new at3r_plan();
    p->alloc_stream = alloc_stream;
    p->pooled = alloc_stream == nullptr;
    p->g = *g;
    p->esz = g->storage == AT3R_STORE_F32 ? sizeof(float) : 2;
    p->tilts.assign(g->tilts_deg, g->tilts_deg + g->n_tilts);
    p->g.tilts_deg = p->tilts.data();
    p->nx = g->nx; p->ny = g->ny; p->T = g->n_tilts;
    p->fill_seed = g->fill_seed;
    p->bp_bulk = g->storage == AT3R_STORE_F32 && (g->nx & 3) == 0 && bp_bulk_from_env() ? 1 : 0;
    p->N = g->nx & ~1; p->Nx = p->N; p->Nz = g->vol_z; p->KX = p->Nx / 2 + 1;
    cudaGetDevice(&p->device);

    // geometry table exactly as CTomoBase::Setup builds it (CTomoBase.cpp:56-65)
    std::vector<float> cs(2 * p->T);
    for (int t = 0; t < p->T; t++) {
        const float a = 0.017453f * p->tilts[t];
        cs[2 * t] = std::cos(a);
        cs[2 * t + 1] = std::sin(a);
        if (!(cs[2 * t] > 1e-3f)) {
            delete p;
            return set_err(AT3R_ERR_INVALID_ARGUMENT, "tilt angles must satisfy |tilt| < 89.9 degrees");
        }
    }
    p->ray_len.resize(p->T);
    for (int t = 0; t < p->T; t++) p->ray_len[t] = (int)((float)p->Nz / cs[2 * t] + 1.5f);
    auto fail = [&](at3r_status s) { at3r_plan_destroy(p); return s; };
    at3r_status rc;
    if ((rc = dalloc(p, &p->d_cs, p->T))) return fail(rc);
    if ((rc = dalloc(p, &p->d_seen, 1))) return fail(rc);
    if (cudaMemcpy(p->d_cs, cs.data(), sizeof(float) * 2 * p->T, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(set_err(AT3R_ERR_CUDA, "geometry upload failed"));

    const size_t T = p->T, N = p->N, Nx = p->Nx, Nz = p->Nz, KX = p->KX;
    size_t per_slice;
    if (g->method == AT3R_SART) {
        p->relax = g->relax > 0.f ? g->relax : 1.0f / (float)g->subsets;
        // AreTomo/Util/CSplitItems.cpp:25-48
        const int n = g->num_tilts, k = g->subsets;
        p->sub_size.assign(k, n / k);
        p->sub_start.assign(k, 0);
        for (int i = 0; i < n % k; i++) p->sub_size[i]++;
        for (int i = 1; i < k; i++) p->sub_start[i] = p->sub_start[i - 1] + p->sub_size[i - 1];
        p->bp_ww_sart = bp_window(BP_TX, BP_TZ, 1.0, cs, p->T);
        if (p->bp_ww_sart > BP_WW) return fail(set_err(AT3R_ERR_TOO_LARGE, "back-projection window exceeds its stride"));
        for (const void* fn : {(const void*)k_bp<0, float, float, true>, (const void*)k_bp<0, __half, __half, true>,
                               (const void*)k_bp<0, __nv_bfloat16, __nv_bfloat16, true>})
            if ((rc = set_smem(fn, bp_smem(0)))) return fail(rc);
        if (p->bp_bulk && (rc = set_smem((const void*)k_bp<0, float, float, true, true>, bp_smem(1)))) return fail(rc);
        per_slice = 2 * T * N * p->esz + 4 * Nx * Nz + (p->esz < 4 ? 2 * Nx * Nz + 4 * T : 0);
    } else {
        if (g->c2r == AT3R_C2R_MATCH_CUFFT) {
            bool measured = false;
            p->c2r = probe_cufft_c2r(p->Nz, p->Nx, &measured);
            if (!measured)
                return fail(set_err(AT3R_ERR_UNSUPPORTED,
                                    "cannot ask cuFFT which C2R convention it uses for " + std::to_string(p->Nz) +
                                        " x " + std::to_string(p->Nx) +
                                        " (libcufft not loadable); pass c2r = AT3R_C2R_HERMITIAN or AT3R_C2R_PACKED"));
        } else {
            p->c2r = g->c2r;
        }
        if ((rc = make_fft(p, p->N, p->fN))) return fail(rc);
        if ((rc = make_fft(p, 2 * p->Nx, p->f2x))) return fail(rc);
        if ((rc = make_fft(p, 2 * p->Nz, p->f2z))) return fail(rc);
        if ((rc = make_fft(p, p->Nz, p->fz))) return fail(rc);
        if ((rc = make_fft(p, p->Nx, p->fx))) return fail(rc);
        // sequences per CTA: enough butterflies per stage for 512 threads,
        // two buffers of them within 96 KB (two CTAs per SM) where possible
        auto batch = [](int work) {
            int b = 1;
            while (b < 8 && (size_t)work * b * 2 <= 4096) b *= 2;
            while (b > 1 && 2 * sizeof(float2) * (size_t)fft_pitch(work) * b > (96u << 10)) b /= 2;
            return b;
        };
        p->b_rweight = batch(p->fN.plan.work);
        p->b_row = batch(p->f2x.plan.work);
        p->b_xc2r = batch(p->fx.plan.work);
        p->smem_rweight = 2 * sizeof(float2) * fft_pitch(p->fN.plan.work) * p->b_rweight;
        p->smem_row = 2 * sizeof(float2) * fft_pitch(p->f2x.plan.work) * p->b_row;
        p->smem_xc2r = 2 * sizeof(float2) * fft_pitch(p->fx.plan.work) * p->b_xc2r;
        p->zcrop_pitch = round_up(fft_pitch(std::max(p->f2z.plan.work, p->fz.plan.work)), 2) + 1;
        p->zcrop_cb = std::max(4, std::min(32, 4096 / (2 * p->Nz)));
        while (p->zcrop_cb > 1 && 2 * sizeof(float2) * p->zcrop_cb * p->zcrop_pitch > 227 * 1024) p->zcrop_cb /= 2;
        p->smem_zcrop = 2 * sizeof(float2) * p->zcrop_cb * p->zcrop_pitch;
        p->bp_ww_wbp = bp_window(BP_TX, BP_TZ, 0.5, cs, p->T);
        if (p->bp_ww_wbp > BP_WW) return fail(set_err(AT3R_ERR_TOO_LARGE, "back-projection window exceeds its stride"));
        p->rs_zcrop = std::max(p->f2z.rs, p->fz.rs);
        std::vector<std::pair<const void*, size_t>> fns;
        dispatch_rs(p->fN.rs, [&](auto R) {
            constexpr int r = decltype(R)::value;
            fns.push_back({(const void*)k_rweight<float, r>, p->smem_rweight});
            fns.push_back({(const void*)k_rweight<__half, r>, p->smem_rweight});
            fns.push_back({(const void*)k_rweight<__nv_bfloat16, r>, p->smem_rweight});
        });
        dispatch_rs(p->f2x.rs, [&](auto R) { fns.push_back({(const void*)k_row_r2c<decltype(R)::value>, p->smem_row}); });
        dispatch_rs(p->rs_zcrop, [&](auto R) { fns.push_back({(const void*)k_zcrop<decltype(R)::value>, p->smem_zcrop}); });
        dispatch_rs(p->fx.rs, [&](auto R) { fns.push_back({(const void*)k_x_c2r<decltype(R)::value>, p->smem_xc2r}); });
        for (auto& f : fns)
            if ((rc = set_smem(f.first, f.second))) return fail(rc);
        for (const void* fn : {(const void*)k_bp<1, float, float, false>, (const void*)k_bp<1, __half, float, false>,
                               (const void*)k_bp<1, __nv_bfloat16, float, false>})
            if ((rc = set_smem(fn, bp_smem(0)))) return fail(rc);
        if (p->bp_bulk && (rc = set_smem((const void*)k_bp<1, float, float, false, true>, bp_smem(1)))) return fail(rc);
        // R-weight transfer function (GRWeight.cu:15-20), 1/N folded in
        std::vector<float> h(N / 2 + 1);
        const double twopi = (double)6.2831852f;
        for (size_t k = 0; k <= N / 2; k++) {
            const double f = (double)k / (double)N;
            h[k] = (float)((1.0 / N) * 2.0 * f * (0.55 + 0.45 * std::cos(twopi * f)));
        }
        if ((rc = dalloc(p, &p->d_h, h.size()))) return fail(rc);
        cudaMemcpy(p->d_h, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice);
        per_slice = T * N * sizeof(float) + 16 * Nx * Nz + 2 * Nz * KX * sizeof(float2);
    }

    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
    int slab = g->slab_slices > 0 ? g->slab_slices : default_slab(g, per_slice, sms);
    p->slab = std::min(slab, p->ny);
    p->slab_cap = p->slab;
    const size_t S = p->slab;
    if (g->method == AT3R_SART) {
        if ((rc = dalloc_bytes(p, &p->d_raw, S * T * N * p->esz))) return fail(rc);
        if ((rc = dalloc_bytes(p, &p->d_diff, S * T * N * p->esz))) return fail(rc);
        if (g->storage != AT3R_STORE_F32) {
            if ((rc = dalloc(p, &p->d_scale, S * T))) return fail(rc);
            // eight 16-bit slices per voxel, the slab rounded up to whole groups of eight
            if ((rc = dalloc_bytes(p, &p->d_shadow, sizeof(uint4) * ((S + 7) / 8) * Nx * Nz))) return fail(rc);
        }
        if ((rc = dalloc_bytes(p, reinterpret_cast<void**>(&p->d_w), sizeof(float4) * ((S + SB - 1) / SB) * Nx * Nz)))
            return fail(rc);
        if ((rc = dalloc(p, &p->d_flags, S))) return fail(rc);
        if ((rc = dalloc(p, &p->d_rf, 2 * (size_t)std::max(1, g->iterations)))) return fail(rc);
        p->h_rf.assign(2 * std::max(1, g->iterations), 0.0);
    } else {
        if ((rc = dalloc_bytes(p, &p->d_filt, S * T * N * p->esz))) return fail(rc);
        if (g->storage != AT3R_STORE_F32 && (rc = dalloc(p, &p->d_scale, S * T))) return fail(rc);
        if ((rc = dalloc(p, &p->d_flags, S))) return fail(rc);
        if ((rc = dalloc(p, &p->d_g2, S * 4 * Nx * Nz))) return fail(rc);
        if ((rc = dalloc(p, &p->d_y, S * 2 * Nz * KX))) return fail(rc);
    }
    *out = p;
    return AT3R_OK;
}

void at3r_plan_destroy(at3r_plan* p)
{
    if (!p) return;
    // like cudaFree, wait for work that may still use the plan's memory
    if (p->pooled) cudaDeviceSynchronize();
    for (void* ptr : {(void*)p->d_cs, (void*)p->d_seen, (void*)p->d_raw, (void*)p->d_diff, (void*)p->d_scale, (void*)p->d_shadow,
                      (void*)p->d_w,
                      (void*)p->d_flags, (void*)p->d_rf, (void*)p->d_h, (void*)p->d_filt, (void*)p->d_g2,
                      (void*)p->d_y})
        dfree(p, ptr);
    for (void* ptr : {p->lane2.filt, (void*)p->lane2.scale, (void*)p->lane2.flags, (void*)p->lane2.g2,
                      (void*)p->lane2.y})
        dfree(p, ptr);
    if (p->s_lane2) cudaStreamDestroy(p->s_lane2);
    for (cudaEvent_t& e : p->ev_lane) if (e) cudaEventDestroy(e);
    for (HostFft* f : {&p->fN, &p->f2x, &p->f2z, &p->fz, &p->fx}) dfree(p, f->d_tables);
    for (int i = 0; i < 2; i++) { dfree(p, p->d_proj_slab[i]); dfree(p, p->d_vol_slab[i]); dfree(p, p->d_xyz_slab[i]); }
    if (p->s_copy_in) cudaStreamDestroy(p->s_copy_in);
    if (p->s_copy_out) cudaStreamDestroy(p->s_copy_out);
    for (cudaEvent_t& e : p->ev) if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : p->ev_stage) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : p->evpool) cudaEventDestroy(e);
    delete p;
}

at3r_status at3r_run_device(at3r_plan* p, const float* proj, float* vol, void* stream)
{
    if (!p || !proj || !vol) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    at3r_status rc;
    if ((rc = begin_run(p, st))) return rc;
    const size_t tilt_stride = (size_t)p->ny * p->nx;
    // (one lane while per-kernel timing is on: overlapping kernels would time each other)
    const bool two = p->g.method == AT3R_WBP && !p->timing && p->ny > p->slab && ensure_lane2(p) == AT3R_OK;
    if (two) {
        // alternate slabs on two streams: fork from st, join back at the end
        AT3R_CUDA(cudaEventRecord(p->ev_lane[0], st));
        AT3R_CUDA(cudaStreamWaitEvent(p->s_lane2, p->ev_lane[0], 0));
    }
    for (int k = 0, y0 = 0; y0 < p->ny; y0 += p->slab, k++) {
        const int S = std::min(p->slab, p->ny - y0), lane = two ? (k & 1) : 0;
        if ((rc = run_slab(p, proj, tilt_stride, y0, S, vol + (size_t)y0 * p->Nx * p->Nz, lane ? p->s_lane2 : st,
                           lane)))
            return rc;
    }
    if (two) {
        AT3R_CUDA(cudaEventRecord(p->ev_lane[1], p->s_lane2));
        AT3R_CUDA(cudaStreamWaitEvent(st, p->ev_lane[1], 0));
    }
    return end_run(p, st);
}

}  // extern "C"

namespace at3r {

// Host <-> device staging for pageable caller memory.  A copy between the
// device and pageable host memory runs at a fraction of the link's rate (the
// driver stages it itself, synchronously); instead, data passes through two
// pinned 64 MB ring slots, and the host side of each slot (pageable <->
// pinned) is a parallel memcpy that overlaps the GPU's work.
bool host_pinned(const void* ptr)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// memcpy of every piece, split over up to 8 host threads (4 MB or more each)
void parallel_copy(const std::vector<Piece>& pieces)
{
    size_t total = 0;
    for (const Piece& pc : pieces) total += pc.bytes;
    const unsigned hw = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    const size_t nt = std::min<size_t>(hw, std::max<size_t>(1, total >> 22));
    auto run = [&](size_t lo, size_t hi) {
        size_t off = 0;
        for (const Piece& pc : pieces) {
            const size_t a = std::max(lo, off), b = std::min(hi, off + pc.bytes);
            if (a < b) std::memcpy(pc.dst + (a - off), pc.src + (a - off), b - a);
            off += pc.bytes;
            if (off >= hi) break;
        }
    };
    if (nt <= 1) {
        run(0, total);
        return;
    }
    const size_t per = (total + nt - 1) / nt;
    std::vector<std::thread> th;
    for (size_t i = 1; i < nt; i++) th.emplace_back(run, i * per, std::min(total, (i + 1) * per));
    run(0, std::min(total, per));
    for (std::thread& t : th) t.join();
}

// Pieces of at most kStageBytes each, in order.
std::vector<Piece> split_pieces(const std::vector<Piece>& in)
{
    std::vector<Piece> out;
    for (const Piece& pc : in)
        for (size_t o = 0; o < pc.bytes; o += kStageBytes)
            out.push_back({pc.dst + o, pc.src + o, std::min(kStageBytes, pc.bytes - o)});
    return out;
}

// Pinned staging sets (four 64 MB slots) shared by all plans of the process:
// a run borrows one and returns it, so plans created per series do not pay
// for pinned allocations (256 MB of cudaHostAlloc took longer than a 512^3
// WBP).  The pool grows to the number of runs in flight at once.
static std::mutex g_stage_mu;
static std::vector<char*> g_stage_free;   // each entry: 4 * kStageBytes pinned

char* stage_acquire()
{
    {
        std::lock_guard<std::mutex> lk(g_stage_mu);
        if (!g_stage_free.empty()) {
            char* s = g_stage_free.back();
            g_stage_free.pop_back();
            return s;
        }
    }
    char* s = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void**>(&s), 4 * kStageBytes, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return s;
}

void stage_release(char* s)
{
    if (!s) return;
    std::lock_guard<std::mutex> lk(g_stage_mu);
    g_stage_free.push_back(s);
}

// Consecutive pieces whose source and destination both continue where the
// previous one ended, merged into one (fewer, larger copies).
std::vector<Piece> merge_pieces(const std::vector<Piece>& in)
{
    std::vector<Piece> out;
    for (const Piece& pc : in) {
        if (!out.empty() && out.back().dst + out.back().bytes == pc.dst && out.back().src + out.back().bytes == pc.src)
            out.back().bytes += pc.bytes;
        else
            out.push_back(pc);
    }
    return out;
}

}  // namespace at3r

extern "C" {

// Borrows a staging set for this run; the caller returns it with stage_return.
at3r_status ensure_stage(at3r_plan* p)
{
    char* s = stage_acquire();
    if (!s) return set_err(AT3R_ERR_OUT_OF_MEMORY, "pinned staging allocation failed");
    for (int i = 0; i < 2; i++) {
        p->h_stage_in[i] = s + i * kStageBytes;
        p->h_stage_out[i] = s + (2 + i) * kStageBytes;
    }
    if (!p->ev_stage[0])
        for (cudaEvent_t& e : p->ev_stage) AT3R_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    // the ring slots start free
    for (int i = 0; i < 2; i++) AT3R_CUDA(cudaEventRecord(p->ev_stage[i], p->s_copy_in));
    return AT3R_OK;
}

// Gives the borrowed set back once every copy through it has finished.
void stage_return(at3r_plan* p)
{
    if (!p->h_stage_in[0]) return;
    cudaStreamSynchronize(p->s_copy_in);
    cudaStreamSynchronize(p->s_copy_out);
    stage_release(p->h_stage_in[0]);
    for (int i = 0; i < 2; i++) p->h_stage_in[i] = p->h_stage_out[i] = nullptr;
}

// Pageable host -> device: pieces (host src, device dst) through the input
// ring on s_copy_in.  The host waits only for a ring slot's previous copy.
at3r_status stage_in(at3r_plan* p, const std::vector<Piece>& pieces, int& slot)
{
    std::vector<Piece> chunk;
    size_t used = 0;
    auto flush = [&]() -> at3r_status {
        if (chunk.empty()) return AT3R_OK;
        AT3R_CUDA(cudaEventSynchronize(p->ev_stage[slot]));
        char* st = p->h_stage_in[slot];
        std::vector<Piece> host;
        size_t o = 0;
        for (const Piece& pc : chunk) {
            host.push_back({st + o, pc.src, pc.bytes});
            o += pc.bytes;
        }
        parallel_copy(host);
        std::vector<Piece> dev;
        o = 0;
        for (const Piece& pc : chunk) {
            dev.push_back({pc.dst, st + o, pc.bytes});
            o += pc.bytes;
        }
        for (const Piece& pc : merge_pieces(dev))
            AT3R_CUDA(cudaMemcpyAsync(pc.dst, pc.src, pc.bytes, cudaMemcpyHostToDevice, p->s_copy_in));
        AT3R_CUDA(cudaEventRecord(p->ev_stage[slot], p->s_copy_in));
        slot ^= 1;
        chunk.clear();
        used = 0;
        return AT3R_OK;
    };
    at3r_status rc;
    for (const Piece& pc : split_pieces(pieces)) {
        if (used + pc.bytes > kStageBytes && (rc = flush())) return rc;
        chunk.push_back(pc);
        used += pc.bytes;
    }
    return flush();
}

// Device -> pageable host: pieces (device src, host dst) through the output
// ring on s_copy_out; each filled slot is copied out on the host while the
// next one fills.
at3r_status stage_out(at3r_plan* p, const std::vector<Piece>& pieces)
{
    struct Pending {
        int slot;
        std::vector<Piece> host;
    };
    std::vector<Pending> pend;
    auto drain = [&](Pending& d) -> at3r_status {
        AT3R_CUDA(cudaEventSynchronize(p->ev_stage[2 + d.slot]));
        parallel_copy(d.host);
        return AT3R_OK;
    };
    std::vector<Piece> chunk;
    size_t used = 0;
    int slot = 0;
    at3r_status rc;
    auto flush = [&]() -> at3r_status {
        if (chunk.empty()) return AT3R_OK;
        if (pend.size() == 2) {   // the slot about to be filled must be copied out first
            if ((rc = drain(pend.front()))) return rc;
            pend.erase(pend.begin());
        }
        char* st = p->h_stage_out[slot];
        Pending d{slot, {}};
        size_t o = 0;
        std::vector<Piece> dev;
        for (const Piece& pc : chunk) {
            dev.push_back({st + o, pc.src, pc.bytes});
            d.host.push_back({pc.dst, st + o, pc.bytes});
            o += pc.bytes;
        }
        for (const Piece& pc : merge_pieces(dev))
            AT3R_CUDA(cudaMemcpyAsync(pc.dst, pc.src, pc.bytes, cudaMemcpyDeviceToHost, p->s_copy_out));
        AT3R_CUDA(cudaEventRecord(p->ev_stage[2 + slot], p->s_copy_out));
        pend.push_back(std::move(d));
        slot ^= 1;
        chunk.clear();
        used = 0;
        return AT3R_OK;
    };
    for (const Piece& pc : split_pieces(pieces)) {
        if (used + pc.bytes > kStageBytes && (rc = flush())) return rc;
        chunk.push_back(pc);
        used += pc.bytes;
    }
    if ((rc = flush())) return rc;
    for (Pending& d : pend)
        if ((rc = drain(d))) return rc;
    return AT3R_OK;
}

// The host path: slabs of projections in on one copy stream, reconstruction
// on `stream`, volume out on another copy stream, two slabs in flight.  The
// volume goes out as XZ frames (vol_frames) or, when vol_xyz is set, as the
// XY frames of FlipVol(flip) in one contiguous buffer [Nz][ny][Nx].  Pinned
// caller memory is copied directly; pageable memory through the staging
// ring, the output of slab k drained on the host while slab k+1 computes.
at3r_status run_host_body(at3r_plan* p, const float* const* frames, float* const* vol_frames, float* vol_xyz,
                          int flip, void* stream)
{
    if (!p || !frames || (!vol_frames && !vol_xyz)) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    for (int t = 0; t < p->T; t++)
        if (!frames[t]) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null tilt frame");
    if (!vol_xyz)
        for (int y = 0; y < p->ny; y++)
            if (!vol_frames[y]) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null volume frame");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t S = p->slab, nx = p->nx, T = p->T, slice = (size_t)p->Nx * p->Nz;
    at3r_status rc;
    if (!p->d_proj_slab[0]) {
        for (int i = 0; i < 2; i++) {
            if ((rc = dalloc(p, &p->d_proj_slab[i], T * S * nx))) return rc;
            if ((rc = dalloc(p, &p->d_vol_slab[i], S * slice))) return rc;
        }
        AT3R_CUDA(cudaStreamCreateWithFlags(&p->s_copy_in, cudaStreamNonBlocking));
        AT3R_CUDA(cudaStreamCreateWithFlags(&p->s_copy_out, cudaStreamNonBlocking));
        for (cudaEvent_t& e : p->ev) AT3R_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    if (vol_xyz && !p->d_xyz_slab[0])
        for (int i = 0; i < 2; i++)
            if ((rc = dalloc(p, &p->d_xyz_slab[i], S * slice))) return rc;
    const bool in_pinned = host_pinned(frames[0]);
    const bool out_pinned = host_pinned(vol_xyz ? (const void*)vol_xyz : (const void*)vol_frames[0]);
    if ((!in_pinned || !out_pinned) && (rc = ensure_stage(p))) return rc;
    if ((rc = begin_run(p, st))) return rc;
    // ev[0,1]: input slab i copied; ev[2,3]: slab i computed; ev[4,5]: output slab i copied out
    const int nslab = (p->ny + p->slab - 1) / p->slab;
    int in_slot = 0;
    auto copy_in = [&](int k) -> at3r_status {
        const int b = k & 1, y0 = k * p->slab, n = std::min(p->slab, p->ny - y0);
        if (k >= 2) AT3R_CUDA(cudaStreamWaitEvent(p->s_copy_in, p->ev[2 + b], 0));
        if (in_pinned) {
            for (int t = 0; t < p->T; t++)
                AT3R_CUDA(cudaMemcpyAsync(p->d_proj_slab[b] + (size_t)t * S * nx, frames[t] + (size_t)y0 * nx,
                                          sizeof(float) * n * nx, cudaMemcpyHostToDevice, p->s_copy_in));
        } else {
            std::vector<Piece> pc;
            for (int t = 0; t < p->T; t++)
                pc.push_back({reinterpret_cast<char*>(p->d_proj_slab[b] + (size_t)t * S * nx),
                              reinterpret_cast<const char*>(frames[t] + (size_t)y0 * nx), sizeof(float) * n * nx});
            at3r_status r2 = stage_in(p, pc, in_slot);
            if (r2) return r2;
        }
        AT3R_CUDA(cudaEventRecord(p->ev[b], p->s_copy_in));
        return AT3R_OK;
    };
    // output of slab k: pieces (device src, host dst)
    auto out_pieces = [&](int k) {
        const int b = k & 1, y0 = k * p->slab, n = std::min(p->slab, p->ny - y0);
        std::vector<Piece> pc;
        if (vol_xyz) {
            for (int fz = 0; fz < p->Nz; fz++)
                pc.push_back({reinterpret_cast<char*>(vol_xyz + ((size_t)fz * p->ny + y0) * p->Nx),
                              reinterpret_cast<const char*>(p->d_xyz_slab[b] + (size_t)fz * n * p->Nx),
                              sizeof(float) * (size_t)n * p->Nx});
        } else {
            for (int j = 0; j < n; j++)
                pc.push_back({reinterpret_cast<char*>(vol_frames[y0 + j]),
                              reinterpret_cast<const char*>(p->d_vol_slab[b] + (size_t)j * slice),
                              sizeof(float) * slice});
        }
        return pc;
    };
    auto drain_out = [&](int k) -> at3r_status {
        const int b = k & 1;
        AT3R_CUDA(cudaStreamWaitEvent(p->s_copy_out, p->ev[2 + b], 0));
        at3r_status r2 = stage_out(p, out_pieces(k));
        if (r2) return r2;
        AT3R_CUDA(cudaEventRecord(p->ev[4 + b], p->s_copy_out));
        return AT3R_OK;
    };
    if ((rc = copy_in(0))) return rc;
    // one compute stream here: with slabs overlapping on two streams the
    // first slab would finish later, and the copies out (the bound of this
    // path) would start later
    for (int k = 0; k < nslab; k++) {
        const int b = k & 1, y0 = k * p->slab, n = std::min(p->slab, p->ny - y0);
        const int lane = 0;
        cudaStream_t cs = st;
        if (k + 1 < nslab && (rc = copy_in(k + 1))) return rc;
        AT3R_CUDA(cudaStreamWaitEvent(cs, p->ev[b], 0));
        if (k >= 2) AT3R_CUDA(cudaStreamWaitEvent(cs, p->ev[4 + b], 0));
        if ((rc = run_slab(p, p->d_proj_slab[b], S * nx, 0, n, p->d_vol_slab[b], cs, lane))) return rc;
        if (vol_xyz) {
            k_flip_rows<<<dim3(p->Nz, n), 256, 0, cs>>>(p->d_vol_slab[b], p->d_xyz_slab[b], p->Nz, p->Nx, flip,
                                                        (size_t)n * p->Nx);
            p->launches++;
        }
        AT3R_CUDA(cudaEventRecord(p->ev[2 + b], cs));
        if (!out_pinned) {
            // slab k computes while the host drains slab k - 1
            if (k >= 1 && (rc = drain_out(k - 1))) return rc;
            continue;
        }
        AT3R_CUDA(cudaStreamWaitEvent(p->s_copy_out, p->ev[2 + b], 0));
        if (vol_xyz) {
            // rows y0 .. y0+n of every XY frame: one strided copy
            AT3R_CUDA(cudaMemcpy2DAsync(vol_xyz + (size_t)y0 * p->Nx, sizeof(float) * (size_t)p->ny * p->Nx,
                                        p->d_xyz_slab[b], sizeof(float) * (size_t)n * p->Nx,
                                        sizeof(float) * (size_t)n * p->Nx, p->Nz, cudaMemcpyDeviceToHost,
                                        p->s_copy_out));
        } else {
            // frames that sit back to back in host memory go out as one copy
            std::vector<Piece> pc;
            for (int j = 0; j < n; j++)
                pc.push_back({reinterpret_cast<char*>(vol_frames[y0 + j]),
                              reinterpret_cast<const char*>(p->d_vol_slab[b] + (size_t)j * slice),
                              sizeof(float) * slice});
            for (const Piece& m : merge_pieces(pc))
                AT3R_CUDA(cudaMemcpyAsync(m.dst, m.src, m.bytes, cudaMemcpyDeviceToHost, p->s_copy_out));
        }
        AT3R_CUDA(cudaEventRecord(p->ev[4 + b], p->s_copy_out));
    }
    if (!out_pinned && (rc = drain_out(nslab - 1))) return rc;
    AT3R_CUDA(cudaStreamWaitEvent(st, p->ev[4 + ((nslab - 1) & 1)], 0));
    if ((rc = end_run(p, st))) return rc;
    AT3R_CUDA(cudaStreamSynchronize(st));
    return AT3R_OK;
}

at3r_status run_host_impl(at3r_plan* p, const float* const* frames, float* const* vol_frames, float* vol_xyz,
                          int flip, void* stream)
{
    const at3r_status rc = run_host_body(p, frames, vol_frames, vol_xyz, flip, stream);
    if (p) stage_return(p);
    return rc;
}

void at3r_release_cached_memory(void)
{
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (auto& kv : g_pools)
        if (kv.second.pool) {
            int dev = 0;
            cudaGetDevice(&dev);
            cudaSetDevice(kv.first);
            cudaStreamSynchronize(kv.second.stream);
            cudaMemPoolTrimTo(kv.second.pool, 0);
            cudaSetDevice(dev);
        }
    {
        std::lock_guard<std::mutex> lk2(g_stage_mu);
        for (char* st : g_stage_free) cudaFreeHost(st);
        g_stage_free.clear();
    }
    cudaGetLastError();
}

at3r_status at3r_run_host(at3r_plan* p, const float* const* frames, float* const* vol_frames, void* stream)
{
    if (!vol_frames) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    return run_host_impl(p, frames, vol_frames, nullptr, 0, stream);
}

at3r_status at3r_run_host_xyz(at3r_plan* p, const float* const* frames, float* vol_xyz, int flip, void* stream)
{
    if (!vol_xyz) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    return run_host_impl(p, frames, nullptr, vol_xyz, flip != 0, stream);
}

at3r_status at3r_volume_xyz(const float* vol_xzy, int nx, int ny, int vol_z, int flip, float* vol_xyz, void* stream)
{
    if (!vol_xzy || !vol_xyz || nx < 2 || ny < 1 || vol_z < 1)
        return set_err(AT3R_ERR_INVALID_ARGUMENT, "null buffer or empty volume");
    const int Nx = nx & ~1;
    if (Nx != nx) return set_err(AT3R_ERR_INVALID_ARGUMENT, "the volume width is even (nx & ~1 of the projections)");
    if (vol_z > 65535 || ny > 65535) return set_err(AT3R_ERR_TOO_LARGE, "ny and vol_z must stay below 65536");
    k_flip_rows<<<dim3(vol_z, ny), 256, 0, (cudaStream_t)stream>>>(vol_xzy, vol_xyz, vol_z, Nx, flip != 0,
                                                                   (size_t)ny * Nx);
    AT3R_CUDA(cudaGetLastError());
    return AT3R_OK;
}

at3r_status at3r_get_rfactor(const at3r_plan* p, double* out, int n)
{
    if (!p || !out) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    if (p->g.method != AT3R_SART || !p->g.compute_rfactor)
        return set_err(AT3R_ERR_INVALID_ARGUMENT, "plan does not compute the R-factor");
    const int m = std::min(n, 2 * p->g.iterations);
    for (int i = 0; i < m; i++) out[i] = p->h_rf[i];
    return AT3R_OK;
}

size_t at3r_plan_workspace_bytes(const at3r_plan* p) { return p ? p->ws_bytes : 0; }

at3r_status at3r_plan_set_timing(at3r_plan* p, int enable)
{
    if (!p) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null plan");
    p->timing = enable != 0;
    return AT3R_OK;
}

int at3r_plan_kernel_stats(at3r_plan* p, int kind, const char** name, int64_t* launches, double* ms, double* bytes,
                           double* units)
{
    if (!p) return 0;
    if (kind < 0 || kind >= KK_COUNT) return KK_COUNT;
    if (p->timing && !p->pending.empty()) {
        // resolve event pairs once the last one has completed
        cudaEventSynchronize(p->evpool[p->pending.back().second + 1]);
        for (KStat& k : p->stats) k.ms = 0;
        for (auto& pr : p->pending) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, p->evpool[pr.second], p->evpool[pr.second + 1]) == cudaSuccess)
                p->stats[pr.first].ms += t;
        }
        cudaGetLastError();
    }
    const KStat& k = p->stats[kind];
    if (name) *name = kKernelNames[kind];
    if (launches) *launches = k.launches;
    if (ms) *ms = k.ms;
    if (bytes) *bytes = k.bytes;
    if (units) *units = k.units;
    return KK_COUNT;
}
int64_t at3r_plan_last_launches(const at3r_plan* p) { return p ? p->launches : 0; }


int at3r_plan_c2r(const at3r_plan* p) { return p ? p->c2r : 0; }

int at3r_plan_flags_seen(const at3r_plan* p)
{
    if (!p) return 0;
    int v = 0;
    if (cudaDeviceSynchronize() != cudaSuccess || cudaMemcpy(&v, p->d_seen, sizeof(int), cudaMemcpyDeviceToHost) !=
                                                      cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return v;
}

at3r_status at3r_plan_fill_table(const at3r_plan* p, int* table, size_t n)
{
    if (!p || !table) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    if (p->g.method != AT3R_SART) return set_err(AT3R_ERR_INVALID_ARGUMENT, "only SART plans fill empty voxels");
    const size_t m = (size_t)p->Nx * p->Nz;
    if (n < m) return set_err(AT3R_ERR_INVALID_ARGUMENT, "table capacity below Nx * Nz entries");
    int* d = nullptr;
    AT3R_CUDA(cudaMalloc(&d, sizeof(int) * m));
    k_fill_table<<<(unsigned)((m + 255) / 256), 256>>>(d, (int)m, p->fill_seed);
    cudaError_t e = cudaMemcpy(table, d, sizeof(int) * m, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return set_err(AT3R_ERR_CUDA, std::string("fill table: ") + cudaGetErrorString(e));
    return AT3R_OK;
}

const char* at3r_status_str(at3r_status s)
{
    switch (s) {
        case AT3R_OK: return "ok";
        case AT3R_ERR_INVALID_ARGUMENT: return "invalid argument";
        case AT3R_ERR_CUDA: return "CUDA error";
        case AT3R_ERR_OUT_OF_MEMORY: return "out of device memory";
        case AT3R_ERR_UNSUPPORTED: return "unsupported option";
        case AT3R_ERR_TOO_LARGE: return "size exceeds a kernel limit";
        case AT3R_ERR_NO_DEVICE: return "no CUDA device";
        case AT3R_ERR_IO: return "file error";
    }
    return "unknown status";
}

const char* at3r_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"

void at3r_set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

extern "C" {

}  // extern "C"

// ===========================================================================
// SART without device allocation.
//
// Some callers cannot allocate device memory at the moment they reconstruct:
// a host application whose allocator has already reserved the device's
// memory (a cudaMalloc would fail or fragment its pool), or a pipeline that
// keeps several series in flight on other streams (cudaMalloc and cudaFree
// may synchronise the whole device and stall that work).  For them this
// entry point runs the plain-FP32 SART path with its scratch — the per-tilt
// cos/sin table, the weighted sinogram rows, the residual rows and the
// per-slice sentinel flags — in one fixed array that lives in this library's
// device image.  The caller passes the projections and the volume.
//
// The array is AT3R_NOALLOC_SCRATCH_BYTES (16 MiB) on every GPU the library
// is loaded on, held until the process exits.  Every call shares it and it
// keeps the last call's contents, so calls that overlap on the GPU (two
// streams, two threads) race; serialise them.  Every call looks up the
// array's device address; the first call on a device also raises the
// back-projection kernel's shared-memory limit; make that first call before
// any stream capture.
// ===========================================================================
namespace {

constexpr size_t kNoallocBytes = (size_t)16 << 20;
constexpr int kNoallocMaxTilts = 4096;   // cos/sin table capacity
constexpr int kNoallocMaxSlab = 8192;    // sentinel-flag capacity
constexpr size_t kNoallocHeader = sizeof(float2) * kNoallocMaxTilts + sizeof(int) * kNoallocMaxSlab;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

// The array's device address on the current device.  Looked up on every call
// (a cheap query), so it stays right if the device's context is rebuilt.  The
// first call on a device also raises the back-projection kernel's
// shared-memory limit (once per device and process).
at3r_status noalloc_scratch_address(unsigned char** out)
{
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
        cudaGetLastError();
        return set_err(AT3R_ERR_CUDA, std::string("cudaGetSymbolAddress(no-allocation scratch): ") +
                                          cudaGetErrorString(e));
    }
    at3r_status rc = set_smem((const void*)k_bp<0, float, float, false>, 0);
    if (rc != AT3R_OK) return rc;
    *out = (unsigned char*)ptr;
    return AT3R_OK;
}

// Writes a chunk of the cos/sin table into the scratch header: the values
// travel in the launch's parameters, so no host buffer has to outlive the call.
constexpr int kCsChunk = 448;   // 3.5 KB of parameters per launch
struct CsChunk {
    float2 v[kCsChunk];
};
__global__ void k_put_cs(CsChunk c, int n, float2* __restrict__ dst)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = c.v[i];
}

}  // namespace

extern "C" at3r_status at3r_sart_device_noalloc(const float* proj, int nx, int ny, int n_tilts,
                                                const float* tilts_deg, int vol_z, int start_tilt, int num_tilts,
                                                int iterations, int subsets, float relax, float* vol, void* stream)
{
    if (!proj || !vol || !tilts_deg) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    if (nx < 4 || ny < 1 || n_tilts < 1 || vol_z < 2)
        return set_err(AT3R_ERR_INVALID_ARGUMENT, "sizes must satisfy nx >= 4, ny >= 1, n_tilts >= 1, vol_z >= 2");
    if (subsets < 1 || iterations < 0)
        return set_err(AT3R_ERR_INVALID_ARGUMENT, "SART needs subsets >= 1 and iterations >= 0");
    if (start_tilt < 0 || num_tilts < 0 || start_tilt + num_tilts > n_tilts)
        return set_err(AT3R_ERR_INVALID_ARGUMENT, "SART tilt range outside the series");
    if ((long long)(nx & ~1) * vol_z * 4 >= (1LL << 31))
        return set_err(AT3R_ERR_TOO_LARGE, "(nx & ~1) * vol_z must stay below 2^29 (32-bit in-slice offsets)");
    const int T = n_tilts, N = nx & ~1, Nx = N, Nz = vol_z;
    if (T > kNoallocMaxTilts)
        return set_err(AT3R_ERR_TOO_LARGE, "the no-allocation entry point takes at most " +
                                               std::to_string(kNoallocMaxTilts) + " tilts");
    const size_t per_slice = 2 * sizeof(float) * (size_t)T * N;
    const size_t room = kNoallocBytes - kNoallocHeader;
    if (per_slice > room)
        return set_err(AT3R_ERR_TOO_LARGE,
                       "the no-allocation scratch (16 MiB) holds the weighted sinogram and residual of at least one "
                       "y-slice, 2 * n_tilts * (nx & ~1) floats; this series needs " +
                           std::to_string(per_slice) + " bytes per slice, at most " + std::to_string(room));
    std::vector<float> cs(2 * T);
    for (int t = 0; t < T; t++) {
        const float a = 0.017453f * tilts_deg[t];
        cs[2 * t] = std::cos(a);
        cs[2 * t + 1] = std::sin(a);
        if (!(cs[2 * t] > 1e-3f))
            return set_err(AT3R_ERR_INVALID_ARGUMENT, "tilt angles must satisfy |tilt| < 89.9 degrees");
    }
    const int ww = bp_window(BP_TX, BP_TZ, 1.0, cs, T);
    if (ww > BP_WW) return set_err(AT3R_ERR_TOO_LARGE, "back-projection window exceeds its stride");
    if (bp_smem(0) > 227 * 1024) return set_err(AT3R_ERR_TOO_LARGE, "back-projection window exceeds 227 KB");
    unsigned char* base = nullptr;
    at3r_status rc = noalloc_scratch_address(&base);
    if (rc != AT3R_OK) return rc;
    float2* d_cs = reinterpret_cast<float2*>(base);
    int* d_flags = reinterpret_cast<int*>(base + sizeof(float2) * kNoallocMaxTilts);
    const int slab = (int)std::min<size_t>({room / per_slice, (size_t)kNoallocMaxSlab, (size_t)ny});
    float* d_raw = reinterpret_cast<float*>(base + kNoallocHeader);
    float* d_diff = d_raw + (size_t)slab * T * N;
    cudaStream_t st = (cudaStream_t)stream;
    for (int t0 = 0; t0 < T; t0 += kCsChunk) {
        CsChunk c{};
        const int n = std::min(kCsChunk, T - t0);
        for (int i = 0; i < n; i++) c.v[i] = make_float2(cs[2 * (t0 + i)], cs[2 * (t0 + i) + 1]);
        k_put_cs<<<1, 256, 0, st>>>(c, n, d_cs + t0);
        AT3R_CUDA(cudaGetLastError());
    }

    // contiguous subsets of [start_tilt, start_tilt + num_tilts), the first n % k one larger
    std::vector<int> sub_start(subsets, 0), sub_size(subsets, num_tilts / subsets);
    for (int i = 0; i < num_tilts % subsets; i++) sub_size[i]++;
    for (int i = 1; i < subsets; i++) sub_start[i] = sub_start[i - 1] + sub_size[i - 1];
    const float rlx = relax > 0.f ? relax : 1.0f / (float)subsets;
    const size_t tilt_stride = (size_t)ny * nx;
    // the empty-voxel fill's table is drawn per call from the time, as the
    // reference draws it per series (GGenRandoms::DoIt)
    const unsigned long long fill_seed = (unsigned long long)time(nullptr);
    for (int y0 = 0; y0 < ny; y0 += slab) {
        const int S = std::min(slab, ny - y0);
        float* v = vol + (size_t)y0 * Nx * Nz;
        const int SG = (S + SB - 1) / SB;
        AT3R_CUDA(cudaMemsetAsync(d_flags, 0, sizeof(int) * S, st));
        k_gather_weight<float><<<dim3(T, S), 256, 0, st>>>(proj, tilt_stride, nx, y0, d_cs, T, N, Nz, d_raw, nullptr,
                                                           d_flags);
        AT3R_CUDA(cudaGetLastError());
        AT3R_CUDA(cudaMemsetAsync(v, 0, sizeof(float) * (size_t)S * Nx * Nz, st));
        BpArgs a{};
        a.T = T; a.N = N; a.cs = d_cs; a.GX = Nx; a.GZ = Nz; a.S = S;
        a.out = v; a.out_slice = (size_t)Nx * Nz; a.ww = ww; a.flags = d_flags;
        const dim3 bgrid((Nx + BP_TX - 1) / BP_TX, (Nz + BP_TZ - 1) / BP_TZ, SG);
        a.sino = d_raw; a.t0 = 0; a.t1 = T; a.relax = 1.f; a.low_bit = kFlagRawLow;
        k_bp<0, float, float, false><<<bgrid, BP_THREADS, bp_smem(0), st>>>(a);
        AT3R_CUDA(cudaGetLastError());
        a.sino = d_diff; a.relax = rlx; a.low_bit = kFlagDiffLow;
        for (int it = 0; it < iterations; it++) {
            for (int s = 0; s < subsets; s++) {
                const int t0 = sub_start[s] + start_tilt, nt = sub_size[s];
                if (nt <= 0) continue;
                k_fp_diff<float, float, false><<<dim3((N + 255) / 256, nt, SG), 256, 0, st>>>(v, nullptr, Nx, Nz, S, d_raw, d_diff,
                                                                                       nullptr, d_cs, T, N, t0, nullptr,
                                                                                       d_flags);
                AT3R_CUDA(cudaGetLastError());
                a.t0 = t0; a.t1 = t0 + nt;
                k_bp<0, float, float, false><<<bgrid, BP_THREADS, bp_smem(0), st>>>(a);
                AT3R_CUDA(cudaGetLastError());
            }
        }
        const int fb = std::max(1, std::min((Nx * Nz + 255) / 256, (8 * 148 + S - 1) / S));
        k_fill_mark<<<dim3(fb, S), 256, 0, st>>>(v, Nx, Nz, d_flags, fill_seed, nullptr);
        AT3R_CUDA(cudaGetLastError());
        k_fill_finish<<<S, 512, 0, st>>>(v, Nx, Nz, d_flags, nullptr);
        AT3R_CUDA(cudaGetLastError());
    }
    return AT3R_OK;
}

// ===========================================================================
// Batched form: many series in one CUDA graph, and the slab autotuner.
// ===========================================================================
struct at3r_batch {
    std::vector<at3r_plan*> plans;
    std::vector<const float*> proj;
    std::vector<float*> vol;
    int branches = 1;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    int mode_req = AT3R_BATCH_AUTO, mode = 0;   // requested and chosen form
    float ms_waves = 0.f, ms_branches = 0.f;    // the autotuner's timings (both forms possible)
    // WBP batches of one storage type: persistent stage kernels over waves
    bool waves = false;
    int storage = 0;
    int rs[kWbpStages] = {};            // radix set of each FFT stage over the batch
    size_t smem[kWbpStages] = {};       // dynamic shared memory of each stage
    int grid[kWbpStages] = {};          // persistent CTAs of each stage
    std::vector<int> wave_off, wave_n;  // per wave: first descriptor, descriptors
    std::vector<int> wave_start;        // per (wave, stage): offset of its block-start array
    WbpSlab* d_slabs = nullptr;
    int* d_start = nullptr;
    int* d_counters = nullptr;          // one per (wave, stage)
};

namespace {

// Slab sizes the autotuner tries (slices per device batch, up to the plan's
// workspace capacity) and the best one found per problem shape.
std::mutex g_tune_mu;
std::map<std::vector<int>, int> g_tune_cache;

std::vector<int> tune_key(const at3r_plan* p)
{
    return {p->g.method, p->nx, p->Nz, p->T, p->g.storage, p->g.iterations, (int)p->sub_size.size(), p->slab_cap};
}

// The five stage kernels of a wave for storage ST, each with the radix set the
// batch needs; fn[k] for stage k (0 rweight, 1 bp, 2 row_r2c, 3 zcrop, 4 x_c2r).
template <typename ST>
void wave_kernels(const int* rs, const void** fn)
{
    dispatch_rs(rs[0], [&](auto R) { fn[0] = (const void*)k_wbp_wave<0, ST, decltype(R)::value>; });
    fn[1] = (const void*)k_wbp_wave<1, ST, 0>;
    dispatch_rs(rs[2], [&](auto R) { fn[2] = (const void*)k_wbp_wave<2, float, decltype(R)::value>; });
    dispatch_rs(rs[3], [&](auto R) { fn[3] = (const void*)k_wbp_wave<3, float, decltype(R)::value>; });
    dispatch_rs(rs[4], [&](auto R) { fn[4] = (const void*)k_wbp_wave<4, float, decltype(R)::value>; });
}

void wave_kernels_of(int storage, const int* rs, const void** fn)
{
    if (storage == AT3R_STORE_F16) wave_kernels<__half>(rs, fn);
    else if (storage == AT3R_STORE_BF16) wave_kernels<__nv_bfloat16>(rs, fn);
    else wave_kernels<float>(rs, fn);
}

// Descriptors of every wave of a WBP batch: wave w holds slab w of every
// series that has one.  Uploads them with the block-start arrays.
at3r_status build_waves(at3r_batch* b)
{
    const int n = (int)b->plans.size();
    for (at3r_plan* p : b->plans)
        if (p->ny > p->slab) {
            at3r_status rc = ensure_lane2(p);
            if (rc) return rc;
        }
    // as many waves as the series with the most slabs has slabs; every other
    // series spreads its slabs evenly over them (slab j of n in wave
    // floor(j * waves / n)), so the waves carry similar work
    int nw = 0;
    for (at3r_plan* p : b->plans) nw = std::max(nw, (p->ny + p->slab - 1) / p->slab);
    std::vector<WbpSlab> slabs;
    std::vector<int> starts;
    for (int w = 0; w < nw; w++) {
        b->wave_off.push_back((int)slabs.size());
        int cnt = 0;
        for (int i = 0; i < n; i++) {
            at3r_plan* p = b->plans[i];
            const int ns = (p->ny + p->slab - 1) / p->slab;
            // the slab of series i in wave w, if any: the j with floor(j * nw / ns) == w
            const int j = (int)(((long long)w * ns + nw - 1) / nw);
            if (j >= ns || (long long)j * nw / ns != w) continue;
            const int y0 = j * p->slab;
            const int S = std::min(p->slab, p->ny - y0);
            const int Nx = p->Nx, Nz = p->Nz, T = p->T, N = p->N, KX = p->KX;
            // alternate waves use the plan's two workspaces, so two waves overlap
            const bool l2 = (w & 1) && p->s_lane2;
            void* const filt = l2 ? p->lane2.filt : p->d_filt;
            float* const scale = l2 ? p->lane2.scale : p->d_scale;
            int* const flags = l2 ? p->lane2.flags : p->d_flags;
            float* const g2 = l2 ? p->lane2.g2 : p->d_g2;
            float2* const yw = l2 ? p->lane2.y : p->d_y;
            WbpSlab d{};
            d.proj = b->proj[i];
            d.tilt_stride = (size_t)p->ny * p->nx;
            d.row_pitch = p->nx;
            d.y0 = y0;
            d.cs = p->d_cs;
            d.T = T; d.N = N; d.Nx = Nx; d.Nz = Nz; d.S = S;
            d.h = p->d_h;
            d.filt = filt;
            d.scale = scale;
            d.flags = flags;
            d.g2 = g2;
            d.y = yw;
            d.vol = b->vol[i] + (size_t)y0 * Nx * Nz;
            d.vol_slice = (size_t)Nx * Nz;
            d.b_rweight = p->b_rweight; d.b_row = p->b_row; d.b_xc2r = p->b_xc2r;
            d.zcrop_cb = p->zcrop_cb; d.zcrop_pitch = p->zcrop_pitch;
            d.packed = p->c2r == AT3R_C2R_PACKED;
            d.norm = (float)(1.0 / (2.0 * Nx) / (2.0 * Nz));
            BpArgs& a = d.bp;
            a.sino = filt; a.scale = scale; a.shadow = nullptr; a.T = T; a.N = N; a.t0 = 0; a.t1 = T;
            a.cs = p->d_cs; a.GX = 2 * Nx; a.GZ = 2 * Nz; a.S = S; a.relax = 1.f; a.out = g2;
            a.out_slice = (size_t)4 * Nx * Nz; a.ww = p->bp_ww_wbp; a.flags = flags; a.seen = p->d_seen;
            a.low_bit = kFlagRawLow; a.bulk = 0;
            d.fN = p->fN.plan; d.f2x = p->f2x.plan; d.f2z = p->f2z.plan; d.fz = p->fz.plan; d.fx = p->fx.plan;
            d.gx[0] = ((T + 1) / 2 + p->b_rweight - 1) / p->b_rweight;
            d.gx[1] = (2 * Nx + BP_TX - 1) / BP_TX;
            d.bp_gy = (2 * Nz + BP_TZ - 1) / BP_TZ;
            d.bp_gz = (S + SB - 1) / SB;
            d.gx[2] = (Nz + p->b_row - 1) / p->b_row;
            d.gx[3] = (KX + p->zcrop_cb - 1) / p->zcrop_cb;
            d.gx[4] = ((Nz + 1) / 2 + p->b_xc2r - 1) / p->b_xc2r;
            slabs.push_back(d);
            cnt++;
        }
        b->wave_n.push_back(cnt);
        // block starts of each stage over this wave's descriptors
        for (int k = 0; k < kWbpStages; k++) {
            b->wave_start.push_back((int)starts.size());
            int acc = 0;
            for (int j = 0; j < cnt; j++) {
                const WbpSlab& d = slabs[b->wave_off[w] + j];
                starts.push_back(acc);
                acc += k == 1 ? d.gx[1] * d.bp_gy * d.bp_gz : d.gx[k] * d.S;
            }
            starts.push_back(acc);
        }
    }
    AT3R_CUDA(cudaMalloc(&b->d_slabs, sizeof(WbpSlab) * slabs.size()));
    AT3R_CUDA(cudaMalloc(&b->d_start, sizeof(int) * starts.size()));
    AT3R_CUDA(cudaMalloc(&b->d_counters, sizeof(int) * (size_t)nw * kWbpStages));
    AT3R_CUDA(cudaMemcpy(b->d_slabs, slabs.data(), sizeof(WbpSlab) * slabs.size(), cudaMemcpyHostToDevice));
    AT3R_CUDA(cudaMemcpy(b->d_start, starts.data(), sizeof(int) * starts.size(), cudaMemcpyHostToDevice));
    // radix sets, shared memory and persistent grids of the stage kernels
    for (at3r_plan* p : b->plans) {
        b->rs[0] = std::max(b->rs[0], p->fN.rs);
        b->rs[2] = std::max(b->rs[2], p->f2x.rs);
        b->rs[3] = std::max(b->rs[3], p->rs_zcrop);
        b->rs[4] = std::max(b->rs[4], p->fx.rs);
        b->smem[0] = std::max(b->smem[0], p->smem_rweight);
        b->smem[2] = std::max(b->smem[2], p->smem_row);
        b->smem[3] = std::max(b->smem[3], p->smem_zcrop);
        b->smem[4] = std::max(b->smem[4], p->smem_xc2r);
    }
    b->smem[1] = bp_smem(0);
    const void* fn[kWbpStages];
    wave_kernels_of(b->storage, b->rs, fn);
    int dev = 0, sms = 148;
    AT3R_CUDA(cudaGetDevice(&dev));
    AT3R_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (int k = 0; k < kWbpStages; k++) {
        at3r_status rc = set_smem(fn[k], b->smem[k]);
        if (rc) return rc;
        int per_sm = 0;
        AT3R_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn[k], k == 1 ? BP_THREADS : 512, b->smem[k]));
        b->grid[k] = std::max(1, per_sm) * sms;
    }
    b->waves = true;
    return AT3R_OK;
}

// One run of a wave batch: per wave the flags, then the five stages; even
// waves on st0, odd ones on st1 (their own workspaces), which both start
// after the counters are cleared on st0.
at3r_status run_waves(at3r_batch* b, cudaStream_t st0, cudaStream_t st1, cudaEvent_t ev)
{
    const void* fn[kWbpStages];
    wave_kernels_of(b->storage, b->rs, fn);
    AT3R_CUDA(cudaMemsetAsync(b->d_counters, 0, sizeof(int) * b->wave_n.size() * kWbpStages, st0));
    if (st1 != st0) {
        AT3R_CUDA(cudaEventRecord(ev, st0));
        AT3R_CUDA(cudaStreamWaitEvent(st1, ev, 0));
    }
    for (size_t w = 0; w < b->wave_n.size(); w++) {
        const cudaStream_t st = (w & 1) ? st1 : st0;
        const int nw = b->wave_n[w];
        WbpSlab* ds = b->d_slabs + b->wave_off[w];
        k_wave_flags<<<nw, 128, 0, st>>>(ds);
        AT3R_CUDA(cudaGetLastError());
        for (int k = 0; k < kWbpStages; k++) {
            const int* start = b->d_start + b->wave_start[w * kWbpStages + k];
            int* counter = b->d_counters + w * kWbpStages + k;
            int nslabs = nw;
            void* args[] = {(void*)&ds, (void*)&start, (void*)&nslabs, (void*)&counter};
            AT3R_CUDA(cudaLaunchKernel(fn[k], dim3(b->grid[k]), dim3(k == 1 ? BP_THREADS : 512), args, b->smem[k], st));
        }
    }
    return AT3R_OK;
}

}  // namespace

extern "C" {

at3r_status at3r_plan_autotune(at3r_plan* p, const float* proj, float* vol, void* stream, int* chosen)
{
    if (!p || !proj || !vol) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    const auto key = tune_key(p);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            p->slab = it->second;
            if (chosen) *chosen = p->slab;
            return AT3R_OK;
        }
    }
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<int> cand;
    for (int s = SB; s < p->slab_cap; s *= 2) cand.push_back(s);
    cand.push_back(p->slab_cap);
    cudaEvent_t e0, e1;
    AT3R_CUDA(cudaEventCreate(&e0));
    AT3R_CUDA(cudaEventCreate(&e1));
    const bool timing = p->timing;
    p->timing = false;
    int best = p->slab_cap;
    float best_ms = 3.0e38f;
    at3r_status rc = AT3R_OK;
    // every candidate is timed on the same leading rows (slab cost is the
    // same along y), at most two of the largest slabs
    const int rows = std::min(p->ny, 2 * p->slab_cap);
    const size_t tilt_stride = (size_t)p->ny * p->nx;
    auto run_rows = [&]() -> at3r_status {
        at3r_status r;
        if ((r = begin_run(p, st))) return r;
        for (int y0 = 0; y0 < rows; y0 += p->slab) {
            const int S = std::min(p->slab, rows - y0);
            if ((r = run_slab(p, proj, tilt_stride, y0, S, vol + (size_t)y0 * p->Nx * p->Nz, st))) return r;
        }
        return end_run(p, st);
    };
    for (int s : cand) {
        p->slab = s;
        if ((rc = run_rows())) break;   // warm-up
        cudaEventRecord(e0, st);
        if ((rc = run_rows())) break;
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; best = s; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    p->timing = timing;
    p->slab = best;
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
    if (chosen) *chosen = best;
    return AT3R_OK;
}

at3r_status at3r_batch_create(at3r_plan* const* plans, const float* const* proj, float* const* vol, int n,
                              int branches, at3r_batch** out)
{
    if (!plans || !proj || !vol || !out || n < 1) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null argument or n < 1");
    for (int i = 0; i < n; i++) {
        if (!plans[i] || !proj[i] || !vol[i]) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null plan or buffer");
        if (plans[i]->g.method == AT3R_SART && plans[i]->g.compute_rfactor)
            return set_err(AT3R_ERR_UNSUPPORTED, "a batched SART plan cannot copy its R-factor to the host");
        if (plans[i]->timing) return set_err(AT3R_ERR_UNSUPPORTED, "disable per-kernel timing on batched plans");
    }
    at3r_batch* b = new at3r_batch();
    b->plans.assign(plans, plans + n);
    b->proj.assign(proj, proj + n);
    b->vol.assign(vol, vol + n);
    b->branches = std::max(1, std::min(branches, n));
    // WBP series of one storage type run as waves of persistent stage kernels
    bool waves = true;
    for (int i = 0; i < n; i++)
        waves = waves && plans[i]->g.method == AT3R_WBP && plans[i]->g.storage == plans[0]->g.storage;
    if (waves) {
        b->storage = plans[0]->g.storage;
        const at3r_status rc = build_waves(b);
        if (rc) {
            at3r_batch_destroy(b);
            return rc;
        }
    }
    *out = b;
    return AT3R_OK;
}

// Captures (on first use) every plan's launches into one graph — plan i on
// branch i % branches, forked from and joined back to `stream` — and then
// replays the whole batch as one graph launch.
// Captures the batch's work into one graph: the wave form (persistent stage
// kernels over all series) or the branch form (every plan's own launches,
// plan i on branch i % branches).
static at3r_status capture_batch(at3r_batch* b, bool waves, cudaGraph_t* graph, cudaGraphExec_t* exec)
{
    cudaStream_t cap = nullptr;
    AT3R_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    if (b->streams.empty()) {
        b->streams.assign(b->branches, nullptr);
        b->events.assign(b->branches + 2, nullptr);
        for (auto& s2 : b->streams) AT3R_CUDA(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
        for (auto& e : b->events) AT3R_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    AT3R_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    at3r_status rc = AT3R_OK;
    if (cudaEventRecord(b->events[0], cap) != cudaSuccess) rc = AT3R_ERR_CUDA;
    for (int k = 0; k < b->branches && !rc; k++)
        if (cudaStreamWaitEvent(b->streams[k], b->events[0], 0) != cudaSuccess) rc = AT3R_ERR_CUDA;
    if (!rc && waves) {
        // alternate waves on two branches (the plans' two workspaces)
        rc = run_waves(b, b->streams[0], b->streams[std::min(1, b->branches - 1)], b->events[b->branches + 1]);
    } else {
        for (size_t i = 0; i < b->plans.size() && !rc; i++)
            rc = at3r_run_device(b->plans[i], b->proj[i], b->vol[i], b->streams[i % b->branches]);
    }
    for (int k = 0; k < b->branches && !rc; k++) {
        if (cudaEventRecord(b->events[k + 1], b->streams[k]) != cudaSuccess ||
            cudaStreamWaitEvent(cap, b->events[k + 1], 0) != cudaSuccess)
            rc = AT3R_ERR_CUDA;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    if (rc || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return set_err(AT3R_ERR_CUDA, std::string("batch capture failed: ") +
                                          (rc ? at3r_last_error() : cudaGetErrorString(ce)));
    }
    *graph = g;
    AT3R_CUDA(cudaGraphInstantiate(exec, g, 0));
    return AT3R_OK;
}

// Device milliseconds of one launch of a captured batch (after one untimed launch).
static at3r_status time_graph(cudaGraphExec_t exec, cudaStream_t st, float* ms)
{
    cudaEvent_t e0, e1;
    AT3R_CUDA(cudaEventCreate(&e0));
    AT3R_CUDA(cudaEventCreate(&e1));
    cudaGraphLaunch(exec, st);
    cudaEventRecord(e0, st);
    cudaGraphLaunch(exec, st);
    cudaEventRecord(e1, st);
    const cudaError_t e = cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    AT3R_CUDA(e);
    return AT3R_OK;
}

at3r_status at3r_batch_run(at3r_batch* b, void* stream)
{
    if (!b) return set_err(AT3R_ERR_INVALID_ARGUMENT, "null batch");
    cudaStream_t st = (cudaStream_t)stream;
    if (!b->exec) {
        at3r_status rc;
        const bool try_waves = b->waves && b->mode_req != AT3R_BATCH_BRANCHES;
        const bool try_branches = !b->waves || b->mode_req != AT3R_BATCH_WAVES;
        cudaGraph_t gw = nullptr, gb = nullptr;
        cudaGraphExec_t xw = nullptr, xb = nullptr;
        if (try_waves && (rc = capture_batch(b, true, &gw, &xw))) return rc;
        if (try_branches && (rc = capture_batch(b, false, &gb, &xb))) {
            if (xw) cudaGraphExecDestroy(xw);
            if (gw) cudaGraphDestroy(gw);
            return rc;
        }
        b->mode = xw ? AT3R_BATCH_WAVES : AT3R_BATCH_BRANCHES;
        if (xw && xb) {
            // both forms were possible: keep the faster on this device
            float mw = 0.f, mb = 0.f;
            if ((rc = time_graph(xw, st, &mw)) || (rc = time_graph(xb, st, &mb))) return rc;
            b->ms_waves = mw;
            b->ms_branches = mb;
            b->mode = mw <= mb ? AT3R_BATCH_WAVES : AT3R_BATCH_BRANCHES;
        }
        if (b->mode == AT3R_BATCH_WAVES) {
            b->graph = gw; b->exec = xw;
            if (xb) { cudaGraphExecDestroy(xb); cudaGraphDestroy(gb); }
        } else {
            b->graph = gb; b->exec = xb;
            if (xw) { cudaGraphExecDestroy(xw); cudaGraphDestroy(gw); }
        }
    }
    AT3R_CUDA(cudaGraphLaunch(b->exec, st));
    return AT3R_OK;
}

at3r_status at3r_batch_set_mode(at3r_batch* b, int mode)
{
    if (!b || mode < AT3R_BATCH_AUTO || mode > AT3R_BATCH_WAVES)
        return set_err(AT3R_ERR_INVALID_ARGUMENT, "mode must be AT3R_BATCH_AUTO, _BRANCHES or _WAVES");
    if (b->exec) return set_err(AT3R_ERR_INVALID_ARGUMENT, "the batch has run already");
    if (mode == AT3R_BATCH_WAVES && !b->waves)
        return set_err(AT3R_ERR_UNSUPPORTED, "the wave form needs WBP plans of one storage type");
    b->mode_req = mode;
    return AT3R_OK;
}

int at3r_batch_mode(const at3r_batch* b, float* ms_waves, float* ms_branches)
{
    if (!b) return 0;
    if (ms_waves) *ms_waves = b->ms_waves;
    if (ms_branches) *ms_branches = b->ms_branches;
    return b->mode;
}

void at3r_batch_destroy(at3r_batch* b)
{
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (void* ptr : {(void*)b->d_slabs, (void*)b->d_start, (void*)b->d_counters})
        if (ptr) cudaFree(ptr);
    for (auto s2 : b->streams) if (s2) cudaStreamDestroy(s2);
    for (auto e : b->events) if (e) cudaEventDestroy(e);
    delete b;
}

int at3r_plan_slab(const at3r_plan* p) { return p ? p->slab : 0; }

}  // extern "C"
