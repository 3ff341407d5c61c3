// Projection-alignment re-projection: the image tilt proj_idx would have if
// the series' nearby tilts were back-projected and the result projected at
// tilt proj_idx.  Same results as AreTomo3's ProjAlign::CCalcReproj::DoIt
// (AreTomo/ProjAlign/CCalcReproj.cpp:36-58) with GReproj
// (AreTomo/ProjAlign/GReproj.cu), which walks the rows one at a time with a
// synchronous copy per tilt row and two launches per row; here every row of
// a slab goes through two launches:
//   k_reproj_bp : the tilts of the range, angle-weighted nearest-neighbour
//                 back-projection onto a (2 nx) x vol_z slice per row
//                 (GReproj.cu:22-60);
//   k_reproj_fp : nearest-neighbour rays at the projection angle, mean over
//                 the in-slice samples, -1e30 below 80 % coverage
//                 (GReproj.cu:64-110), one warp per ray summing in the
//                 reference's order (512 strided partial sums, then a tree).
// FP32 in the reference's operation order; trigonometry with the same CUDA
// cosf / sinf calls on the same arguments.
#include "at3r.h"
#include "at3r_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

namespace {

constexpr float kD2R = 0.01745f;   // s_fD2R of GReproj.cu and CCalcReproj.cpp
constexpr int kMaxRange = 10;      // CCalcReproj keeps at most 10 tilts

struct RangeTilts {
    float t[kMaxRange];
    int n;
};

// Row slab [S][VZ][VX] of back-projected slices.  Grid (ceil(VX/256), VZ, S).
__global__ void __launch_bounds__(256) k_reproj_bp(const float* __restrict__ proj, size_t tilt_stride, int nx,
                                                   int y0, int i0, RangeTilts rt, float proj_angle, int VX, int VZ,
                                                   float* __restrict__ vol)
{
    __shared__ float tw[kMaxRange], tc[kMaxRange], ts[kMaxRange];
    if (threadIdx.x < rt.n) {
        const float a = rt.t[threadIdx.x];
        tw[threadIdx.x] = cosf((proj_angle - a) * kD2R);
        const float v = a * kD2R;
        tc[threadIdx.x] = cosf(v);
        ts[threadIdx.x] = sinf(v);
    }
    __syncthreads();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y, s = blockIdx.z;
    if (x >= VX) return;
    const float fX = x + 0.5f - VX * 0.5f, fZ = z + 0.5f - VZ * 0.5f;
    const float cent = nx * 0.5f;
    const int iend = nx - 1;
    const float* row = proj + (size_t)(y0 + s) * nx;
    float sum = 0.f, cnt = 0.f;
    for (int k = 0; k < rt.n; k++) {
        const float p = __fadd_rn(__fmaf_rn(fX, tc[k], __fmul_rn(fZ, ts[k])), cent);
        if (p < 0 || p > iend) continue;
        float val = __ldg(row + (size_t)(i0 + k) * tilt_stride + (int)p);
        if (val < -1e10f) val = -1e30f;
        if (val < -1e20f) continue;
        sum = __fmaf_rn(__fmul_rn(val, tc[k]), tw[k], sum);
        cnt = __fadd_rn(cnt, tw[k]);
    }
    vol[((size_t)s * VZ + z) * VX + x] = cnt < 0.001f ? -1e30f : __fdiv_rn(sum, cnt);
}

// One warp per ray u of row s.  Lane l plays the reference's threads
// l + 32k (k < 16) of its 512-thread block: sample i goes to thread i mod 512,
// and the tree halves 256, 128, 64, 32 in registers, then 16 .. 1 across
// lanes.  Grid (ceil(nx / 8), S), 256 threads.
__global__ void __launch_bounds__(256) k_reproj_fp(const float* __restrict__ vol, int VX, int VZ, int nx, int L,
                                                   float c, float sn, float* __restrict__ out, size_t out_row)
{
    const int lane = threadIdx.x & 31;
    const int u = blockIdx.x * 8 + (threadIdx.x >> 5), s = blockIdx.y;
    if (u >= nx) return;   // whole warps leave together
    const float xp = u + 0.5f - nx * 0.5f;
    const float tx = __fadd_rn(__fadd_rn(VX * 0.5f, __fmul_rn(L * 0.5f, sn)), __fdiv_rn(xp, c));
    const float tz = __fsub_rn(VZ * 0.5f, __fmul_rn(L * 0.5f, c));
    const float* v = vol + (size_t)s * VZ * VX;
    float part[16];
    int pc[16];
#pragma unroll
    for (int k = 0; k < 16; k++) { part[k] = 0.f; pc[k] = 0; }
    for (int base = 0; base < L; base += 512) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int i = base + 32 * k + lane;
            if (i >= L) continue;
            const float fx = __fmaf_rn(-(float)i, sn, tx), fz = __fmaf_rn((float)i, c, tz);
            if (fx < 0 || fx >= VX || fz < 0 || fz >= VZ) continue;
            const float val = __ldg(v + (size_t)VX * (int)fz + (int)fx);
            if (val <= -1e10f) continue;
            part[k] = __fadd_rn(part[k], val);
            pc[k] += 1;
        }
    }
#pragma unroll
    for (int h = 8; h > 0; h >>= 1)
#pragma unroll
        for (int k = 0; k < h; k++) {
            part[k] = __fadd_rn(part[k], part[k + h]);
            pc[k] += pc[k + h];
        }
    float sum = part[0];
    int cnt = pc[0];
#pragma unroll
    for (int h = 16; h > 0; h >>= 1) {
        sum = __fadd_rn(sum, __shfl_down_sync(0xffffffffu, sum, h));
        cnt += __shfl_down_sync(0xffffffffu, cnt, h);
    }
    if (lane == 0) out[(size_t)s * out_row + u] = cnt < 0.8f * L ? -1e30f : __fdiv_rn(sum, (float)cnt);
}

// CCalcReproj::mFindProjRange (CCalcReproj.cpp:66-119).
void find_range(const float* tilts, const unsigned char* skip, int T, int proj, int* range)
{
    const float ref_range = 20.5f, ref_stretch = 1.20f;
    const float a = tilts[proj];
    const float cos_a = (float)std::cos((double)(a * kD2R));
    auto ok = [&](int i) {
        if (skip && skip[i]) return false;
        const float t = tilts[i];
        if (std::fabs(a - t) > ref_range) return false;
        const float stretch = (float)(std::cos((double)(t * kD2R)) / cos_a);
        return !(stretch > ref_stretch);
    };
    int start = -1, end = -1;
    for (int i = 0; i < T; i++)
        if (ok(i)) { start = i; break; }
    for (int i = start; i >= 0 && i < T; i++)
        if (ok(i)) end = i;
    if (start < 0 || end < 0) {
        const int sign = a > 0 ? 1 : -1;
        start = proj - sign;
        end = start;
    }
    if (end - start > 9) end = start + 9;
    range[0] = start;
    range[1] = end;
}

at3r_status check_args(int nx, int ny, int n_tilts, const float* tilts, int proj_idx, int vol_z)
{
    if (!tilts || nx < 2 || ny < 1 || n_tilts < 1 || vol_z < 1 || proj_idx < 0 || proj_idx >= n_tilts) {
        at3r_set_last_error("sizes must satisfy nx >= 2, ny >= 1, vol_z >= 1, 0 <= proj_idx < n_tilts");
        return AT3R_ERR_INVALID_ARGUMENT;
    }
    if (ny > 65535 || vol_z > 65535) {
        at3r_set_last_error("ny and vol_z must stay below 65536");
        return AT3R_ERR_TOO_LARGE;
    }
    const double c = std::cos(4.0 * std::atan(1.0) / 180.0 * tilts[proj_idx]);
    if (!(c > 1e-3)) {
        at3r_set_last_error("the projection angle must satisfy |tilt| < 89.9 degrees");
        return AT3R_ERR_INVALID_ARGUMENT;
    }
    return AT3R_OK;
}

// Stream-ordered workspace from the library's pool (cached between calls).
cudaError_t ws_alloc(void** ptr, size_t bytes, cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaMemPool_t pool = at3r_device_pool(dev)) return cudaMallocFromPoolAsync(ptr, bytes, pool, st);
    return cudaMallocAsync(ptr, bytes, st);
}

#define RP_CUDA(x)                                                                                         \
    do {                                                                                                   \
        cudaError_t e_ = (x);                                                                              \
        if (e_ != cudaSuccess) {                                                                           \
            at3r_set_last_error((std::string(#x) + ": " + cudaGetErrorString(e_)).c_str());               \
            return AT3R_ERR_CUDA;                                                                          \
        }                                                                                                  \
    } while (0)

// Re-projects rows through device slabs.  proj(y0 ... ) rows of tilt t at
// proj + t * tilt_stride + y * nx; out rows at out + y * nx (device).
at3r_status reproj_rows(const float* proj, size_t tilt_stride, int nx, int ny, const float* tilts, const int* range,
                        int proj_idx, int vol_z, float* out, cudaStream_t st)
{
    RangeTilts rt{};
    rt.n = range[1] - range[0] + 1;
    if (rt.n < 1 || rt.n > kMaxRange) {
        at3r_set_last_error("no tilt in the re-projection range");
        return AT3R_ERR_INVALID_ARGUMENT;
    }
    for (int k = 0; k < rt.n; k++) rt.t[k] = tilts[range[0] + k];
    const int VX = 2 * nx, VZ = vol_z;
    const float a = tilts[proj_idx];
    const double rad = 4.0 * std::atan(1.0) / 180.0;
    const float c = (float)std::cos(rad * a), sn = (float)std::sin(rad * a);
    const int L = (int)(VZ / c + 0.5f);
    const size_t slice = (size_t)VX * VZ;
    const int S = (int)std::max<size_t>(1, std::min<size_t>(ny, ((size_t)1 << 30) / (slice * sizeof(float))));
    float* vol = nullptr;
    RP_CUDA(ws_alloc(reinterpret_cast<void**>(&vol), sizeof(float) * slice * S, st));
    at3r_status rc = AT3R_OK;
    for (int y0 = 0; y0 < ny && rc == AT3R_OK; y0 += S) {
        const int n = std::min(S, ny - y0);
        k_reproj_bp<<<dim3((VX + 255) / 256, VZ, n), 256, 0, st>>>(proj, tilt_stride, nx, y0, range[0], rt, a, VX,
                                                                   VZ, vol);
        k_reproj_fp<<<dim3((nx + 7) / 8, n), 256, 0, st>>>(vol, VX, VZ, nx, L, c, sn, out + (size_t)y0 * nx,
                                                          (size_t)nx);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            at3r_set_last_error(cudaGetErrorString(e));
            rc = AT3R_ERR_CUDA;
        }
    }
    cudaFreeAsync(vol, st);
    return rc;
}

}  // namespace

extern "C" {

at3r_status at3r_reproj_range(const float* tilts_deg, const unsigned char* skip, int n_tilts, int proj_idx,
                              int* range)
{
    if (!tilts_deg || !range || n_tilts < 1 || proj_idx < 0 || proj_idx >= n_tilts) {
        at3r_set_last_error("null argument or projection index outside the series");
        return AT3R_ERR_INVALID_ARGUMENT;
    }
    find_range(tilts_deg, skip, n_tilts, proj_idx, range);
    return AT3R_OK;
}

at3r_status at3r_reproj_device(const float* proj, int nx, int ny, int n_tilts, const float* tilts_deg,
                               const unsigned char* skip, int proj_idx, int vol_z, float* reproj, void* stream)
{
    at3r_status rc = check_args(nx, ny, n_tilts, tilts_deg, proj_idx, vol_z);
    if (rc) return rc;
    if (!proj || !reproj) {
        at3r_set_last_error("null buffer");
        return AT3R_ERR_INVALID_ARGUMENT;
    }
    int range[2];
    find_range(tilts_deg, skip, n_tilts, proj_idx, range);
    if (range[0] < 0 || range[1] >= n_tilts) {
        at3r_set_last_error("no tilt in the re-projection range");
        return AT3R_ERR_INVALID_ARGUMENT;
    }
    return reproj_rows(proj, (size_t)ny * nx, nx, ny, tilts_deg, range, proj_idx, vol_z, reproj,
                       (cudaStream_t)stream);
}

at3r_status at3r_reproj_host(const float* const* frames, int nx, int ny, int n_tilts, const float* tilts_deg,
                             const unsigned char* skip, int proj_idx, int vol_z, float* reproj, void* stream)
{
    at3r_status rc = check_args(nx, ny, n_tilts, tilts_deg, proj_idx, vol_z);
    if (rc) return rc;
    if (!frames || !reproj) {
        at3r_set_last_error("null buffer");
        return AT3R_ERR_INVALID_ARGUMENT;
    }
    int range[2];
    find_range(tilts_deg, skip, n_tilts, proj_idx, range);
    if (range[0] < 0 || range[1] >= n_tilts) {
        at3r_set_last_error("no tilt in the re-projection range");
        return AT3R_ERR_INVALID_ARGUMENT;
    }
    for (int t = range[0]; t <= range[1]; t++)
        if (!frames[t]) {
            at3r_set_last_error("null tilt frame");
            return AT3R_ERR_INVALID_ARGUMENT;
        }
    cudaStream_t st = (cudaStream_t)stream;
    const int n = range[1] - range[0] + 1;
    const size_t frame = (size_t)nx * ny;
    float* d_proj = nullptr;
    float* d_out = nullptr;
    RP_CUDA(ws_alloc(reinterpret_cast<void**>(&d_proj), sizeof(float) * frame * n, st));
    RP_CUDA(ws_alloc(reinterpret_cast<void**>(&d_out), sizeof(float) * frame, st));
    // only the frames of the range travel; the kernels see them as tilts 0 .. n-1
    for (int k = 0; k < n; k++)
        RP_CUDA(cudaMemcpyAsync(d_proj + k * frame, frames[range[0] + k], sizeof(float) * frame,
                                cudaMemcpyHostToDevice, st));
    const int local[2] = {0, n - 1};
    std::vector<float> tl(tilts_deg + range[0], tilts_deg + range[1] + 1);
    // the projection angle is read from tilts[proj_idx]; give it a slot of its own
    tl.push_back(tilts_deg[proj_idx]);
    rc = reproj_rows(d_proj, frame, nx, ny, tl.data(), local, n, vol_z, d_out, st);
    if (rc == AT3R_OK) {
        RP_CUDA(cudaMemcpyAsync(reproj, d_out, sizeof(float) * frame, cudaMemcpyDeviceToHost, st));
        RP_CUDA(cudaStreamSynchronize(st));
    }
    cudaFreeAsync(d_proj, st);
    cudaFreeAsync(d_out, st);
    return rc;
}

}  // extern "C"
