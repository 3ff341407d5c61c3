// Input-stage kernels: the aligned stack of AreTomo/Correct/GCorrPatchShift.cu
// (nearest-neighbour shift + rotation + local patch shifts), the random fill
// of empty pixels (MaUtil/GFillEmpty2D.cu with the table of
// MaUtil/GGenRandoms.cu) and the Fourier-crop binning of
// AreTomo/Correct/CFourierCropImage.cpp:41-61 / CBinStack.cpp:61-106
// (2-D R2C normalised by 1/(nx ny), MaUtil/GFourierResize2D.cu:7-39 crop,
// 2-D C2R), plus the plane statistics of the thickness measurement
// (AreTomo/Recon/CCalcVolThick.cpp:172-197).
//
// Layouts (all on the device, every tilt of a chunk in one launch):
//   raw    [T][ny][nx]            input frames
//   aln    [T][ay][ax]            aligned frames (ax x ay = aligned size)
//   empty  [T][W * ay]            1 where the aligned pixel is empty (< -1e10)
//   Y      [T][ay][KXo]           row spectra, the KXo = bx/2 + 1 kept columns
//   Wc     [T][by][KXo]           cropped spectra after the column transforms
//   out    [T][by][bx]            binned frames
// W is the width the reference's kernels cover: (padX/2 - 1) * 2 with
// padX = (ax/2 + 1) * 2, i.e. ax when ax is even and ax - 1 when it is odd.
#pragma once
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <stdint.h>

#include "fft_smem.cuh"
#include "rand_table.cuh"

namespace at3r {

// Random table of the fill, MaUtil/GGenRandoms.cu:7-20 (rand_table.cuh).
__global__ void k_rand_table(int* __restrict__ r, int n, unsigned long long seed)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = rand_table_entry(seed, i, n);
}

// cos / sin of every tilt's rotation (radians), as GCorrPatchShift.cu:77-78
// evaluates them on the device.
__global__ void k_axis_cs(const float* __restrict__ rad, int T, float2* __restrict__ cs)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < T) cs[t] = make_float2(cosf(rad[t]), sinf(rad[t]));
}

// GCorrPatchShift.cu:61-104 (mGCorrect) with the local shift of :18-49: the
// raw pixel that aligned pixel (X, Y) of frame t takes — its centred
// coordinates rotated by the tilt axis, moved by the weighted patch shift and
// the global shift, then int() of coordinate + 0.5 — as an index into the raw
// frame, or -1 outside it.  The FP32 operations are the ones the reference's
// kernel executes, written out: nvcc contracts its rotation
// x*c - y*s, x*s + y*c into fma(x, c, -(y*s)), fma(y, c, x*s) (established
// on 4096^2 frames, where the other contractions pick a different raw pixel
// for about one pixel in 10^5).
// local: [5][P] of this tilt = patch centre x, centre y, shift x, shift y, good flag.
__device__ __forceinline__ long long corr_src(int X, int Y, int nx, int ny, int ay, int W, float2 r, float2 sh,
                                              const float* __restrict__ lp, int P)
{
    float fx = X + 0.5f - W * 0.5f;
    float fy = Y + 0.5f - ay * 0.5f;
    const float ft = __fmaf_rn(fx, r.x, -__fmul_rn(fy, r.y));
    fy = __fmaf_rn(fy, r.x, __fmul_rn(fx, r.y));
    fx = ft;
    if (P > 0 && lp) {
        int cnt = 0;
        float sx = 0.f, sy = 0.f, sw = 0.f;
        for (int p = 0; p < P; p++) {
            if (__ldg(lp + 4 * P + p) < 0.9f) continue;
            const float lx = __fdiv_rn(__fsub_rn(fx, __ldg(lp + p)), (float)nx);
            const float ly = __fdiv_rn(__fsub_rn(fy, __ldg(lp + P + p)), (float)ny);
            const float w = expf(__fmul_rn(-100.0f, __fmaf_rn(ly, ly, __fmul_rn(lx, lx))));
            sx = __fmaf_rn(__ldg(lp + 2 * P + p), w, sx);
            sy = __fmaf_rn(__ldg(lp + 3 * P + p), w, sy);
            sw = __fadd_rn(sw, w);
            cnt += 1;
        }
        float dx = 0.f, dy = 0.f;
        if (cnt > 0) {
            dx = sx / sw;
            dy = sy / sw;
        }
        fx += dx;
        fy += dy;
    }
    fx += (sh.x + nx * 0.5f);
    fy += (sh.y + ny * 0.5f);
    const int x = (int)(fx + 0.5f), y = (int)(fy + 0.5f);
    return (x >= 0 && x < nx && y >= 0 && y < ny) ? (long long)y * nx + x : -1;
}

// The aligned frames: pixel (X, Y) = the raw pixel corr_src picks, -1e30
// outside the raw frame; columns X >= W (the odd-width case) are 0.  With
// `fill`, the empty mask of the fill is written alongside.
// A CTA covers a 32 x 32 tile; each warp an 8 x 4 patch, four times (rows
// 8 apart), so the raw pixels a warp gathers lie within a few rows and
// columns whatever the rotation (a 32 x 1 warp on a frame rotated by ~90
// degrees would read 32 raw rows), and every thread has four independent
// gathers in flight.  Tiles are visited along x (grid (ceil(ax / 32),
// ceil(ay / 32), T)), or with `by_rows` along y (grid (ceil(ay / 32),
// ceil(ax / 32), T)): for an axis near 90 degrees aligned y runs along raw
// rows, so consecutive CTAs then read neighbouring pieces of the same raw
// rows.  256 threads.
__global__ void __launch_bounds__(256) k_corr(const float* __restrict__ raw, int nx, int ny, int ax, int ay, int W,
                                              const float2* __restrict__ shifts, const float2* __restrict__ cs,
                                              const float* __restrict__ local, int P, int fill, int by_rows,
                                              float* __restrict__ aln, uint8_t* __restrict__ empty)
{
    constexpr int K = 4;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tx = by_rows ? blockIdx.y : blockIdx.x, ty = by_rows ? blockIdx.x : blockIdx.y;
    const int X = tx * 32 + (warp & 3) * 8 + (lane & 7);
    const int Y0 = ty * 32 + (warp >> 2) * 4 + (lane >> 3);
    const int t = blockIdx.z;
    if (X >= ax) return;
    const float2 r = cs[t], sh = shifts[t];
    const float* lp = local ? local + (size_t)t * 5 * P : nullptr;
    const float* rt = raw + (size_t)t * ny * nx;
    long long src[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int Y = Y0 + 8 * k;
        src[k] = (Y < ay && X < W) ? corr_src(X, Y, nx, ny, ay, W, r, sh, lp, P) : -1;
    }
    float v[K];
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = src[k] >= 0 ? __ldg(rt + src[k]) : -1e30f;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int Y = Y0 + 8 * k;
        if (Y >= ay) continue;
        aln[((size_t)t * ay + Y) * ax + X] = X < W ? v[k] : 0.f;
        if (fill && X < W) empty[(size_t)t * W * ay + (size_t)Y * W + X] = v[k] < -1e10f ? 1 : 0;
    }
}

// GFillEmpty2D.cu:62-87: an empty pixel takes the value of the first
// non-empty pixel along its chain r[i], r[r[i]], ... (at most 100 links).  A
// pixel whose chain finds none keeps its value (below -1e10) and flags its
// frame for k_fill_mean, which gives it the frame mean as the reference does.
// Only empty pixels are written and only non-empty ones are used, so the
// result does not depend on thread order.  Each thread follows four chains
// (pixels 256 apart) in step, and reads a link's flag and value together, so
// that its random reads overlap.  Grid (ceil(W*ay / 1024), T), 256 threads.
__global__ void __launch_bounds__(256) k_fill(float* __restrict__ aln, const uint8_t* __restrict__ empty,
                                              const int* __restrict__ r, int W, int ax, int ay,
                                              int* __restrict__ flags)
{
    constexpr int K = 4;
    const int n = W * ay, t = blockIdx.y;
    const int base = blockIdx.x * (256 * K) + threadIdx.x;
    const uint8_t* e = empty + (size_t)t * n;
    float* f = aln + (size_t)t * ay * ax;
    int cur[K];
    bool act[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int i = base + 256 * k;
        act[k] = i < n && e[i];
        cur[k] = act[k] ? __ldg(r + i) : 0;
    }
    bool any = act[0] || act[1] || act[2] || act[3];
    for (int j = 0; j < 100 && any; j++) {
        any = false;
        uint8_t ek[K];
        float fv[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int yn = cur[k] / W;
            ek[k] = act[k] ? e[cur[k]] : 0;
            fv[k] = act[k] ? f[(size_t)yn * ax + (cur[k] - yn * W)] : 0.f;
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            if (!act[k]) continue;
            if (ek[k]) {
                cur[k] = __ldg(r + cur[k]);
                any = true;
            } else {
                const int i = base + 256 * k, yi = i / W;
                f[(size_t)yi * ax + (i - yi * W)] = fv[k];
                act[k] = false;
            }
        }
    }
    if (act[0] || act[1] || act[2] || act[3]) flags[t] = 1;
}

// GFillEmpty2D.cu:24-60 (mGCalcMean), for the frames k_fill flagged: the mean
// of the non-empty pixels summed as the reference's single 512-thread block
// sums them (thread j adds pixels j, j + 512, ... in float, then a halving
// tree), written to the empty pixels whose chain found no value.  Frames
// without a flag return at once.  Grid T, 512 threads.
__global__ void __launch_bounds__(512) k_fill_mean(float* __restrict__ aln, const uint8_t* __restrict__ empty, int W,
                                                   int ax, int ay, const int* __restrict__ flags)
{
    const int t = blockIdx.x;
    if (!flags[t]) return;
    __shared__ float s_sum[512], s_cnt[512];
    const int n = W * ay, tid = threadIdx.x;
    const uint8_t* e = empty + (size_t)t * n;
    float* f = aln + (size_t)t * ay * ax;
    float sum = 0.f, cnt = 0.f;
    for (int i = tid; i < n; i += 512) {
        if (e[i]) continue;
        const int y = i / W;
        sum += f[(size_t)y * ax + (i - y * W)];
        cnt += 1.0f;
    }
    s_sum[tid] = sum;
    s_cnt[tid] = cnt;
    __syncthreads();
    for (int off = 256; off > 0; off >>= 1) {
        if (tid < off) {
            s_sum[tid] += s_sum[tid + off];
            s_cnt[tid] += s_cnt[tid + off];
        }
        __syncthreads();
    }
    const float mean = s_cnt[0] <= 0.f ? 0.f : s_sum[0] / s_cnt[0];
    for (int i = tid; i < n; i += 512) {
        if (!e[i]) continue;
        const int y = i / W;
        float* v = f + (size_t)y * ax + (i - y * W);
        if (*v < -1e10f) *v = mean;
    }
}

// Binning, step 1: forward FFT of length n = ax along every row of the
// aligned frames, two real rows per complex sequence (a + ib), separated into
// the row spectra of both; the KXo lowest bins are kept.  B row pairs per
// CTA.  Grid (ceil(ceil(ay/2) / B), T).
template <int RS>
__global__ void __launch_bounds__(512, RS < 2 ? 2 : 1) k_bin_r2c(const float* __restrict__ aln, int n, int rows,
                                                                 int KXo, const __grid_constant__ FftPlan plan, int B,
                                                                 float2* __restrict__ Y)
{
    extern __shared__ float2 fsm[];
    const int pitch = fft_pitch(plan.work);
    float2* a = fsm;
    float2* b = fsm + (size_t)B * pitch;
    const int pr0 = blockIdx.x * B, t = blockIdx.y;
    const int nq = min(B, (rows + 1) / 2 - pr0);
    const float* src = aln + (size_t)t * rows * n;
    for (int q = 0; q < nq; q++) {
        const int r0 = 2 * (pr0 + q);
        const bool two = r0 + 1 < rows;
        const float* g0 = src + (size_t)r0 * n;
        float2* aq = a + (size_t)q * pitch;
        staged_copy<4>(n, [&](int x) { return make_float2(__ldg(g0 + x), two ? __ldg(g0 + n + x) : 0.f); },
                       [&](int x, float2 v) { aq[fft_pad(x)] = v; });
    }
    __syncthreads();
    const float2* Zs = fft_run<RS>(a, b, plan, nq, pitch, -1);
    for (int q = 0; q < nq; q++) {
        const int r0 = 2 * (pr0 + q);
        const bool two = r0 + 1 < rows;
        const float2* Z = Zs + (size_t)q * pitch;
        float2* y0 = Y + ((size_t)t * rows + r0) * KXo;
        for (int k = threadIdx.x; k < KXo; k += blockDim.x) {
            const float2 p = Z[fft_pad(k)], qv = Z[fft_pad(k == 0 ? 0 : n - k)];
            y0[k] = make_float2(0.5f * (p.x + qv.x), 0.5f * (p.y - qv.y));
            if (two) y0[KXo + k] = make_float2(0.5f * (p.y + qv.y), -0.5f * (p.x - qv.x));
        }
    }
}

// Binning, step 2: per kept column, forward FFT over the Lin = ay rows, scale
// by 1/(ax ay) (MaUtil/CCufft2D.cpp:65-86), keep rows kz <= Lout/2 from row
// kz and kz > Lout/2 from row kz + Lin - Lout (GFourierResize2D.cu:20-28),
// inverse FFT over Lout = by.  CB columns per CTA, pitch >= both plans' need.
// Grid (ceil(KXo / CB), T).
template <int RS>
__global__ void __launch_bounds__(512, RS < 2 ? 2 : 1) k_bin_cols(const float2* __restrict__ Y, int KXo, int Lin,
                                                                  int Lout, int CB, int pitch,
                                                                  const __grid_constant__ FftPlan pin,
                                                                  const __grid_constant__ FftPlan pout, float norm,
                                                                  float2* __restrict__ Wc)
{
    extern __shared__ float2 fsm[];
    const int kx0 = blockIdx.x * CB, t = blockIdx.y;
    const int nc = min(CB, KXo - kx0);
    float2* a = fsm;
    float2* b = fsm + (size_t)CB * pitch;
    const float2* ysl = Y + (size_t)t * Lin * KXo;
    staged_copy<4>(Lin * CB,
                   [&](int idx) {
                       const int Z = idx / CB, c = idx - Z * CB;
                       return c < nc ? __ldg(ysl + (size_t)Z * KXo + kx0 + c) : make_float2(0.f, 0.f);
                   },
                   [&](int idx, float2 v) {
                       const int Z = idx / CB, c = idx - Z * CB;
                       a[(size_t)c * pitch + fft_pad(Z)] = v;
                   });
    __syncthreads();
    float2* F = fft_run<RS>(a, b, pin, CB, pitch, -1);
    float2* G = (F == a) ? b : a;
    for (int idx = threadIdx.x; idx < Lout * CB; idx += blockDim.x) {
        const int c = idx / Lout, kz = idx - c * Lout;
        const int src = kz <= Lout / 2 ? kz : kz + Lin - Lout;
        const float2 v = F[(size_t)c * pitch + fft_pad(src)];
        G[(size_t)c * pitch + fft_pad(kz)] = make_float2(v.x * norm, v.y * norm);
    }
    __syncthreads();
    float2* H = fft_run<RS>(G, F, pout, CB, pitch, +1);
    float2* wsl = Wc + (size_t)t * Lout * KXo;
    for (int idx = threadIdx.x; idx < Lout * CB; idx += blockDim.x) {
        const int z = idx / CB, c = idx - z * CB;
        if (c < nc) wsl[(size_t)z * KXo + kx0 + c] = H[(size_t)c * pitch + fft_pad(z)];
    }
}

// Binning, step 3: C2R of length bx along every cropped row
// (MaUtil/CCufft2D.cpp:108-117, unnormalised), two rows per complex sequence:
// with the imaginary parts of their DC and Nyquist bins set aside, A + iB
// extended Hermitian-wise inverts to a + ib; packed != 0 adds what cuFFT's
// half-length packing makes of those imaginary parts (-(Im A0 + Im A_H) on
// even and (Im A0 - Im A_H) on odd samples, H = bx/2).  B row pairs per CTA.
// Grid (ceil(ceil(by/2) / B), T).
template <int RS>
__global__ void __launch_bounds__(512, RS < 2 ? 2 : 1) k_bin_c2r(const float2* __restrict__ Wc, int bx, int by,
                                                                 const __grid_constant__ FftPlan plan, int B,
                                                                 int packed, float* __restrict__ out)
{
    extern __shared__ float2 fsm[];
    const int pitch = fft_pitch(plan.work);
    float2* a = fsm;
    float2* b = fsm + (size_t)B * pitch;
    const int KXo = bx / 2 + 1, H = bx / 2;
    const int pz0 = blockIdx.x * B, t = blockIdx.y;
    const int nq = min(B, (by + 1) / 2 - pz0);
    for (int q = 0; q < nq; q++) {
        const int z0 = 2 * (pz0 + q);
        const bool two = z0 + 1 < by;
        const float2* A = Wc + ((size_t)t * by + z0) * KXo;
        const float2* Bv = A + KXo;
        float2* aq = a + (size_t)q * pitch;
        staged_copy<4>(bx,
                       [&](int k) {
                           const bool lo = k <= H;
                           const int kk = lo ? k : bx - k;
                           float2 av = __ldg(A + kk);
                           float2 bv = two ? __ldg(Bv + kk) : make_float2(0.f, 0.f);
                           if (kk == 0 || kk == H) {
                               av.y = 0.f;
                               bv.y = 0.f;
                           }
                           if (!lo) {
                               av.y = -av.y;
                               bv.y = -bv.y;
                           }
                           return make_float2(av.x - bv.y, av.y + bv.x);
                       },
                       [&](int k, float2 v) { aq[fft_pad(k)] = v; });
    }
    __syncthreads();
    const float2* rs = fft_run<RS>(a, b, plan, nq, pitch, +1);
    for (int q = 0; q < nq; q++) {
        const int z0 = 2 * (pz0 + q);
        const bool two = z0 + 1 < by;
        const float2* A = Wc + ((size_t)t * by + z0) * KXo;
        const float2* Bv = A + KXo;
        const float2* r = rs + (size_t)q * pitch;
        float ea = 0.f, oa = 0.f, eb = 0.f, ob = 0.f;
        if (packed) {
            const float ia0 = A[0].y, iah = A[H].y;
            ea = -(ia0 + iah);
            oa = ia0 - iah;
            if (two) {
                const float ib0 = Bv[0].y, ibh = Bv[H].y;
                eb = -(ib0 + ibh);
                ob = ib0 - ibh;
            }
        }
        float* o0 = out + ((size_t)t * by + z0) * bx;
        for (int x = threadIdx.x; x < bx; x += blockDim.x) {
            const float2 v = r[fft_pad(x)];
            o0[x] = v.x + ((x & 1) ? oa : ea);
            if (two) o0[bx + x] = v.y + ((x & 1) ? ob : eb);
        }
    }
}

// CCalcVolThick.cpp:172-197 (mMeasureStd) for every plane of the flipped
// volume at once: mean and variance in double of the central tile (samples
// below -1e20 skipped; squares formed in float as the reference forms them),
// standard deviation = sqrtf of the variance rounded to float.  Plane k of
// CTiltSeries::FlipVol(true) is row Nz-1-k of every XZ frame of vol
// [ny][Nz][Nx].  Grid n_planes, 256 threads.
__global__ void __launch_bounds__(256) k_plane_std(const float* __restrict__ vol, int Nx, int Nz, int x0, int y0,
                                                   int tx, int ty, float* __restrict__ out)
{
    const int k = blockIdx.x, zr = Nz - 1 - k;
    double s1 = 0.0, s2 = 0.0;
    int cnt = 0;
    for (int idx = threadIdx.x; idx < tx * ty; idx += blockDim.x) {
        const int j = idx / tx, i = idx - j * tx;
        const float v = __ldg(vol + ((size_t)(y0 + j) * Nz + zr) * Nx + x0 + i);
        if (v < -1e20f) continue;
        const float sq = __fmul_rn(v, v);
        s1 += (double)v;
        s2 += (double)sq;
        cnt += 1;
    }
    __shared__ double r1[8], r2[8];
    __shared__ int rc[8];
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        r1[w] = s1;
        r2[w] = s2;
        rc[w] = cnt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        int c = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
            a += r1[i];
            b += r2[i];
            c += rc[i];
        }
        const double mean = a / c;
        const double var = __dsub_rn(b / c, __dmul_rn(mean, mean));
        out[k] = var <= 0.0 ? 0.f : sqrtf((float)var);
    }
}

}  // namespace at3r
