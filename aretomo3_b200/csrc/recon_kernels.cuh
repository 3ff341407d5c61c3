// Reconstruction kernels for sm_100a: projection staging and weighting, the
// R-weight filter, SART and WBP back-projection, SART forward projection with
// the residual fused in, and the separable Fourier crop of the WBP 2x grid.
//
// Arithmetic mirrors AreTomo/Recon exactly where a rounding decides which
// samples are used: detector positions are formed with the same FP32
// operations in the same order as the reference kernels (the x*cos product is
// fused with the add, as nvcc contracts `fX*c + fZ*s`), and per-voxel tilt
// sums run in the reference's tilt order, so a voxel sees the same samples.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "fft_smem.cuh"

namespace at3r {

constexpr float kSentinelTest = -1e10f;   // "empty sample" threshold of the reference
constexpr float kSentinelValue = -1e30f;  // value the reference writes for "no sample"

// ---------------------------------------------------------------------------
// Storage of staged sinograms: FP32, or FP16/BF16 with a per-row scale.
// ---------------------------------------------------------------------------
template <typename S>
struct Store;
template <>
struct Store<float> {
    __device__ __forceinline__ static float load(const float* p, float) { return *p; }
    __device__ __forceinline__ static void store(float* p, float v, float) { *p = v; }
};
template <>
struct Store<__half> {
    __device__ __forceinline__ static float load(const __half* p, float inv) { return __half2float(*p) * inv; }
    __device__ __forceinline__ static void store(__half* p, float v, float scale) { *p = __float2half_rn(v * scale); }
};
template <>
struct Store<__nv_bfloat16> {
    __device__ __forceinline__ static float load(const __nv_bfloat16* p, float inv) { return __bfloat162float(*p) * inv; }
    __device__ __forceinline__ static void store(__nv_bfloat16* p, float v, float scale) { *p = __float2bfloat16_rn(v * scale); }
};

// ---------------------------------------------------------------------------
// SART staging: raw[ys][t][x] = proj[t][y0 + ys][x] * (cos_t / Nz), x < N.
// AreTomo/Recon/CDoSartRecon.cpp:100-117 (row gather) and
// AreTomo/Recon/GWeightProjs.cu:7-19 (weight).  Grid (T, slices).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_gather_weight(const float* __restrict__ proj, size_t tilt_stride,
                                                       int row_pitch, int y0, const float2* __restrict__ cs, int T,
                                                       int N, int Nz, float* __restrict__ raw)
{
    const int t = blockIdx.x, ys = blockIdx.y;
    const float w = __ldg(&cs[t].x) / (float)Nz;
    const float* src = proj + (size_t)t * tilt_stride + (size_t)(y0 + ys) * row_pitch;
    float* dst = raw + ((size_t)ys * T + t) * N;
    for (int x = threadIdx.x; x < N; x += blockDim.x) dst[x] = __ldg(src + x) * w;
}

// ---------------------------------------------------------------------------
// WBP staging + R-weight, two tilt rows per CTA packed as the real and
// imaginary parts of one complex sequence: the filter H(k) is real and even
// (H(N-k) = H(k)), so filtering a + ib filters a and b independently.
// AreTomo/Recon/GWeightProjs.cu:18, GRWeight.cu:7-23 (+ MaUtil/GFFT1D.cu R2C/C2R).
// Grid (ceil(T/2), slices).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_rweight(const float* __restrict__ proj, size_t tilt_stride, int row_pitch,
                                                 int y0, const float2* __restrict__ cs, int T, int N, int Nz,
                                                 const float* __restrict__ hhalf, FftPlan plan, float* __restrict__ out)
{
    extern __shared__ float2 fsm[];
    float2* a = fsm;
    float2* b = fsm + plan.work;
    const int t0 = 2 * blockIdx.x, t1 = t0 + 1, ys = blockIdx.y;
    const bool two = t1 < T;
    const float w0 = __ldg(&cs[t0].x) / (float)Nz;
    const float w1 = two ? __ldg(&cs[t1].x) / (float)Nz : 0.f;
    const float* s0 = proj + (size_t)t0 * tilt_stride + (size_t)(y0 + ys) * row_pitch;
    const float* s1 = proj + (size_t)(two ? t1 : t0) * tilt_stride + (size_t)(y0 + ys) * row_pitch;
    for (int x = threadIdx.x; x < N; x += blockDim.x)
        a[x] = make_float2(__ldg(s0 + x) * w0, two ? __ldg(s1 + x) * w1 : 0.f);
    __syncthreads();
    float2* r = fft_run(a, b, plan, 1, plan.work, -1);
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        const float h = __ldg(hhalf + (k <= N - k ? k : N - k));
        float2 v = r[k];
        r[k] = make_float2(v.x * h, v.y * h);
    }
    __syncthreads();
    float2* r2 = fft_run(r, r == a ? b : a, plan, 1, plan.work, +1);
    float* d0 = out + ((size_t)ys * T + t0) * N;
    for (int x = threadIdx.x; x < N; x += blockDim.x) {
        const float2 v = r2[x];
        d0[x] = v.x;
        if (two) d0[N + x] = v.y;
    }
}

// ---------------------------------------------------------------------------
// Back-projection.  MODE 0: SART update on the 1x grid
// (AreTomo/Recon/GBackProj.cu:12-60, bSart): the mean over tilts [t0, t1) of
// the lerped sinogram is scaled by relax, added, clamped at 0.  MODE 1: the
// WBP 2x grid (AreTomo/Recon/GBackProjWbp.cu:14-53): mean over all tilts,
// or 0 where no tilt contributes.
//
// A CTA covers BP_TX x BP_TZ voxels of one slice.  For every tilt it stages
// in shared memory only the detector window its voxels can reach (the
// sinogram position is affine in the voxel coordinates, so the window is
// bounded by the tile's corners).  Voxels are written warp-contiguous in x.
// ---------------------------------------------------------------------------
constexpr int BP_TX = 64, BP_TZ = 32, BP_THREADS = 256;
constexpr int BP_CX = BP_TX / 32, BP_CZ = BP_TZ / (BP_THREADS / 32);

struct BpArgs {
    const float* sino;       // [slices][T][N]
    int T, N, t0, t1;
    const float2* cs;
    int GX, GZ;              // voxel grid of this mode
    float relax;
    float* out;              // MODE 0: vol slab [slices][GZ][GX] (z flipped); MODE 1: [slices][GZ][GX]
    size_t out_slice;
    int ww;                  // staged window width (floats)
    int* flags;              // MODE 0: per-slice "wrote a sentinel" flag
};

template <int MODE>
__device__ __forceinline__ float bp_xp(float fX, float fZs, float c, float cent)
{
    // MODE 0: fX*c + fZ*s + N/2.0f            (GBackProj.cu:35-36)
    // MODE 1: (fX*c + fZ*s)/2 + (N/2) + 0.5f  (GBackProjWbp.cu:34-35)
    const float a = __fmaf_rn(fX, c, fZs);
    if (MODE == 0) return __fadd_rn(a, cent);
    return __fadd_rn(__fadd_rn(__fmul_rn(a, 0.5f), cent), 0.5f);
}

template <int MODE>
__global__ void __launch_bounds__(BP_THREADS) k_bp(BpArgs p)
{
    extern __shared__ float bsm[];
    const int nt = p.t1 - p.t0;
    int* ws = reinterpret_cast<int*>(bsm);
    float* win = bsm + ((nt + 3) & ~3);
    const int ys = blockIdx.z, X0 = blockIdx.x * BP_TX, Z0 = blockIdx.y * BP_TZ;
    const float* sino = p.sino + (size_t)ys * p.T * p.N;
    const float cent = MODE == 0 ? (float)p.N / 2.0f : (float)(p.N / 2);
    const float hx = MODE == 0 ? (float)p.GX * 0.5f : (float)p.GX / 2.0f;
    const float hz = MODE == 0 ? (float)p.GZ * 0.5f : (float)p.GZ / 2.0f;

    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
        const float2 c = __ldg(&p.cs[p.t0 + t]);
        float lo = 3.0e38f;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float fX = (float)(X0 + ((k & 1) ? BP_TX - 1 : 0)) - hx;
            const float fZ = (float)(Z0 + ((k & 2) ? BP_TZ - 1 : 0)) - hz;
            lo = fminf(lo, bp_xp<MODE>(fX, __fmul_rn(fZ, c.y), c.x, cent));
        }
        ws[t] = (int)floorf(lo) - 1;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < nt * p.ww; idx += blockDim.x) {
        const int t = idx / p.ww, k = idx - t * p.ww;
        const int x = ws[t] + k;
        win[idx] = (x >= 0 && x < p.N) ? __ldg(sino + (size_t)(p.t0 + t) * p.N + x) : 0.f;
    }
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float fX[BP_CX], fZ[BP_CZ];
#pragma unroll
    for (int i = 0; i < BP_CX; i++) fX[i] = (float)(X0 + lane + 32 * i) - hx;
#pragma unroll
    for (int j = 0; j < BP_CZ; j++) fZ[j] = (float)(Z0 + warp + (BP_THREADS / 32) * j) - hz;
    float sum[BP_CZ][BP_CX];
    int cnt[BP_CZ][BP_CX];
#pragma unroll
    for (int j = 0; j < BP_CZ; j++)
#pragma unroll
        for (int i = 0; i < BP_CX; i++) { sum[j][i] = 0.f; cnt[j][i] = 0; }
    const float endX = (float)(p.N - 2);
    const int wmax = p.ww - 2;

    for (int t = 0; t < nt; t++) {
        const float2 c = __ldg(&p.cs[p.t0 + t]);
        const float* w = win + t * p.ww;
        const int st = ws[t];
#pragma unroll
        for (int j = 0; j < BP_CZ; j++) {
            const float fzs = __fmul_rn(fZ[j], c.y);
#pragma unroll
            for (int i = 0; i < BP_CX; i++) {
                const float xp = bp_xp<MODE>(fX[i], fzs, c.x, cent);
                if (xp >= 0.f && xp <= endX) {
                    const int ii = (int)xp;
                    const float fr = __fsub_rn(xp, (float)ii);
                    const int k = min(max(ii - st, 0), wmax);
                    const float v = __fmaf_rn(w[k], __fsub_rn(1.f, fr), __fmul_rn(w[k + 1], fr));
                    if (v > kSentinelTest) {
                        sum[j][i] = __fadd_rn(sum[j][i], v);
                        cnt[j][i] += 1;
                    }
                }
            }
        }
    }

    float* out = p.out + (size_t)ys * p.out_slice;
#pragma unroll
    for (int j = 0; j < BP_CZ; j++) {
        const int Z = Z0 + warp + (BP_THREADS / 32) * j;
        if (Z >= p.GZ) continue;
#pragma unroll
        for (int i = 0; i < BP_CX; i++) {
            const int X = X0 + lane + 32 * i;
            if (X >= p.GX) continue;
            if (MODE == 0) {
                if (cnt[j][i] <= 0) continue;
                float* v = out + (size_t)(p.GZ - 1 - Z) * p.GX + X;
                const float f = __fadd_rn(__fdiv_rn(__fmul_rn(p.relax, sum[j][i]), (float)cnt[j][i]), *v);
                if (f > kSentinelTest) {
                    *v = fmaxf(f, 0.f);
                } else {
                    *v = kSentinelValue;
                    p.flags[ys] = 1;
                }
            } else {
                out[(size_t)Z * p.GX + X] = cnt[j][i] > 0 ? __fdiv_rn(sum[j][i], (float)cnt[j][i]) : 0.f;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// SART forward projection of tilts [t0, t0 + grid.y) with the residual fused:
// AreTomo/Recon/GForProj.cu:10-76 (ray of L = int(Nz/cos + 1.5) samples,
// bilinear, mean over in-volume samples, -1e30 if none) followed by
// AreTomo/Recon/GDiffProj.cu:7-21 (d = raw - fp, 0 where either is empty).
// One ray per thread; a warp walks 32 neighbouring rays in lock-step, so each
// step reads two short runs of two volume rows.  Optional residual sums for
// the per-iteration R-factor are reduced per CTA and added in FP64.
// Grid (ceil(N/256), tilts, slices).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_fp_diff(const float* __restrict__ vol, int Nx, int Nz,
                                                 const float* __restrict__ raw, float* __restrict__ diff,
                                                 const float2* __restrict__ cs, int T, int N, int t0,
                                                 double* __restrict__ rf)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = t0 + blockIdx.y, ys = blockIdx.z;
    float ad = 0.f, ar = 0.f;
    if (u < N) {
        const float2 c = __ldg(&cs[t]);
        const float fCos = c.x, fSin = c.y;
        const int L = (int)((float)Nz / fCos + 1.5f);
        const float fXp = (float)u - 0.5f * (float)N;
        const float fTempX = fXp / fCos + (float)Nx * 0.5f;
        const float fTempZ = (float)Nz * 0.5f;
        const float halfL = (float)L * 0.5f;
        const float endX = (float)(Nx - 2), endZ = (float)(Nz - 2);
        // the volume slab is stored z flipped: voxel (X, Z) at row Nz-1-Z
        const float* v0 = vol + (size_t)ys * Nx * Nz + (size_t)(Nz - 1) * Nx;
        float fSum = 0.f, fCount = 0.f;
        for (int i = 0; i < L; i++) {
            const float z0 = (float)i - halfL;
            const float fX = __fmaf_rn(-z0, fSin, fTempX);
            const float fZ = __fmaf_rn(z0, fCos, fTempZ);
            if (fX < 0.f || fZ < 0.f || fX > endX || fZ > endZ) continue;
            const int iX = (int)fX, iZ = (int)fZ;
            const float wx = fX - (float)iX, wz = fZ - (float)iZ;
            const float* q = v0 - (size_t)iZ * Nx + iX;
            const float a00 = __ldg(q), a10 = __ldg(q + 1), a01 = __ldg(q - Nx), a11 = __ldg(q - Nx + 1);
            const float val = a00 * (1.f - wx) * (1.f - wz) + a10 * wx * (1.f - wz) + a01 * (1.f - wx) * wz +
                              a11 * wx * wz;
            if (val < kSentinelTest) continue;
            fSum += val;
            fCount += 1.f;
        }
        const float fp = fCount <= 0.f ? kSentinelValue : fSum / fCount;
        const size_t o = ((size_t)ys * T + t) * N + u;
        const float r = __ldg(raw + o);
        float d = 0.f;
        if (!(fp < kSentinelTest) && !(r < kSentinelTest)) {
            d = r - fp;
            ad = fabsf(d);
            ar = fabsf(r);
        }
        diff[o] = d;
    }
    if (rf) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ad += __shfl_xor_sync(0xffffffffu, ad, o);
            ar += __shfl_xor_sync(0xffffffffu, ar, o);
        }
        __shared__ float red[2][8];
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 0) { red[0][warp] = ad; red[1][warp] = ar; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double sd = 0, sr = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); k++) { sd += red[0][k]; sr += red[1][k]; }
            atomicAdd(rf, sd);
            atomicAdd(rf + 1, sr);
        }
    }
}

// ---------------------------------------------------------------------------
// Replace any "-1e30" voxel of a flagged slice (MaUtil/GFillEmpty2D.cu runs
// after SART, AreTomo/Recon/CTomoSart.cpp:88).  The reference copies a
// time-seeded random valid voxel; this fills the slice's valid mean, which is
// deterministic.  From a zero start no voxel reaches the sentinel unless the
// input holds values near -1e10, so this is a guard.  Grid (slices).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_fill_empty(float* __restrict__ vol, size_t slice_elems,
                                                    const int* __restrict__ flags)
{
    const int ys = blockIdx.x;
    if (flags[ys] == 0) return;
    float* v = vol + (size_t)ys * slice_elems;
    float s = 0.f, n = 0.f;
    for (size_t i = threadIdx.x; i < slice_elems; i += blockDim.x)
        if (!(v[i] < kSentinelTest)) { s += v[i]; n += 1.f; }
    __shared__ float rs[256], rn[256];
    rs[threadIdx.x] = s;
    rn[threadIdx.x] = n;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) { rs[threadIdx.x] += rs[threadIdx.x + o]; rn[threadIdx.x] += rn[threadIdx.x + o]; }
        __syncthreads();
    }
    const float mean = rn[0] > 0.f ? rs[0] / rn[0] : 0.f;
    for (size_t i = threadIdx.x; i < slice_elems; i += blockDim.x)
        if (v[i] < kSentinelTest) v[i] = mean;
}

// ---------------------------------------------------------------------------
// WBP Fourier crop, step 1: forward real FFT of the 2x-grid rows, keeping
// bins kx in [0, Nx/2].  Two rows per CTA as one complex sequence z = a + ib:
// A[k] = (Z[k] + conj Z[-k]) / 2, B[k] = (Z[k] - conj Z[-k]) / 2i.
// g: [slices][2Nz][2Nx]; y: [slices][2Nz][KX] with KX = Nx/2 + 1.
// Grid (Nz, slices): CTA r handles rows 2r, 2r+1.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_row_r2c(const float* __restrict__ g, int Nx, int Nz, FftPlan plan,
                                                 float2* __restrict__ y)
{
    extern __shared__ float2 fsm[];
    float2* a = fsm;
    float2* b = fsm + plan.work;
    const int X2 = 2 * Nx, KX = Nx / 2 + 1;
    const int r0 = 2 * blockIdx.x, ys = blockIdx.y;
    const float* g0 = g + ((size_t)ys * 2 * Nz + r0) * X2;
    for (int x = threadIdx.x; x < X2; x += blockDim.x) a[x] = make_float2(__ldg(g0 + x), __ldg(g0 + X2 + x));
    __syncthreads();
    const float2* Z = fft_run(a, b, plan, 1, plan.work, -1);
    float2* y0 = y + ((size_t)ys * 2 * Nz + r0) * KX;
    for (int k = threadIdx.x; k < KX; k += blockDim.x) {
        const float2 p = Z[k], q = Z[k == 0 ? 0 : X2 - k];
        // A = (p + conj q)/2 ; B = (p - conj q)/(2i) = -i (p - conj q)/2
        y0[k] = make_float2(0.5f * (p.x + q.x), 0.5f * (p.y - q.y));
        y0[KX + k] = make_float2(0.5f * (p.y + q.y), -0.5f * (p.x - q.x));
    }
}

// ---------------------------------------------------------------------------
// WBP Fourier crop, step 2 (AreTomo/Recon/GBackProjWbp.cu:126-136,
// MaUtil/GFourierResize2D.cu:7-39): per column kx, forward FFT over the 2Nz
// rows, keep kz in [0, Nz/2] from row kz and kz in (Nz/2, Nz) from row
// kz + Nz, scale by 1/(2Nx * 2Nz) (the forward normalisation of
// MaUtil/CCufft2D.cpp:65-86), inverse FFT over Nz.  CB columns per CTA.
// y: [slices][2Nz][KX] -> w: [slices][Nz][KX].  Grid (ceil(KX/CB), slices).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_zcrop(const float2* __restrict__ y, int Nx, int Nz, int CB, int pitch,
                                               FftPlan p2, FftPlan p1, float norm, float2* __restrict__ w)
{
    extern __shared__ float2 fsm[];
    const int KX = Nx / 2 + 1, Z2 = 2 * Nz;
    const int kx0 = blockIdx.x * CB, ys = blockIdx.y;
    const int nc = min(CB, KX - kx0);
    float2* a = fsm;
    float2* b = fsm + (size_t)CB * pitch;
    const float2* ysl = y + (size_t)ys * Z2 * KX;
    for (int idx = threadIdx.x; idx < Z2 * CB; idx += blockDim.x) {
        const int Z = idx / CB, c = idx - Z * CB;
        a[(size_t)c * pitch + Z] = c < nc ? ysl[(size_t)Z * KX + kx0 + c] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* F = fft_run(a, b, p2, CB, pitch, -1);
    float2* G = (F == a) ? b : a;
    for (int idx = threadIdx.x; idx < Nz * CB; idx += blockDim.x) {
        const int c = idx / Nz, kz = idx - c * Nz;
        const int src = kz <= Nz / 2 ? kz : kz + Nz;
        const float2 v = F[(size_t)c * pitch + src];
        G[(size_t)c * pitch + kz] = make_float2(v.x * norm, v.y * norm);
    }
    __syncthreads();
    float2* H = fft_run(G, F, p1, CB, pitch, +1);
    float2* wsl = w + (size_t)ys * Nz * KX;
    for (int idx = threadIdx.x; idx < Nz * CB; idx += blockDim.x) {
        const int z = idx / CB, c = idx - z * CB;
        if (c < nc) wsl[(size_t)z * KX + kx0 + c] = H[(size_t)c * pitch + z];
    }
}

// ---------------------------------------------------------------------------
// WBP Fourier crop, step 3 (MaUtil/CCufft2D.cpp:108-117, C2R over Nx,
// unnormalised; MaUtil/CPad2D.cpp:29-39 unpad; AreTomo/Recon/
// CDoWbpRecon.cpp:115-122 z flip).  Two rows per CTA: with the imaginary
// parts of their DC and Nyquist bins set aside, A + iB extended
// Hermitian-wise inverts to a + ib.  packed != 0 then adds what cuFFT's
// half-length packing algorithm makes of those imaginary parts:
// -(Im A0 + Im A_{Nx/2}) on even and (Im A0 - Im A_{Nx/2}) on odd samples.
// w: [slices][Nz][KX] -> vol: [slices][Nz][Nx] (row Nz-1-z).  Grid (ceil(Nz/2), slices).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_x_c2r(const float2* __restrict__ w, int Nx, int Nz, FftPlan plan,
                                               int packed, float* __restrict__ vol, size_t vol_slice)
{
    extern __shared__ float2 fsm[];
    float2* a = fsm;
    float2* b = fsm + plan.work;
    const int KX = Nx / 2 + 1, H = Nx / 2;
    const int z0 = 2 * blockIdx.x, z1 = z0 + 1, ys = blockIdx.y;
    const bool two = z1 < Nz;
    const float2* A = w + ((size_t)ys * Nz + z0) * KX;
    const float2* B = A + KX;
    for (int k = threadIdx.x; k < Nx; k += blockDim.x) {
        const bool lo = k <= H;
        const int kk = lo ? k : Nx - k;
        float2 av = A[kk];
        float2 bv = two ? B[kk] : make_float2(0.f, 0.f);
        if (kk == 0 || kk == H) { av.y = 0.f; bv.y = 0.f; }
        if (!lo) { av.y = -av.y; bv.y = -bv.y; }
        a[k] = make_float2(av.x - bv.y, av.y + bv.x);   // A + iB
    }
    __syncthreads();
    const float2* r = fft_run(a, b, plan, 1, plan.work, +1);
    float ea = 0.f, oa = 0.f, eb = 0.f, ob = 0.f;
    if (packed) {
        const float ia0 = A[0].y, iah = A[H].y;
        ea = -(ia0 + iah); oa = ia0 - iah;
        if (two) { const float ib0 = B[0].y, ibh = B[H].y; eb = -(ib0 + ibh); ob = ib0 - ibh; }
    }
    float* o0 = vol + (size_t)ys * vol_slice + (size_t)(Nz - 1 - z0) * Nx;
    for (int x = threadIdx.x; x < Nx; x += blockDim.x) {
        const float2 v = r[x];
        o0[x] = v.x + ((x & 1) ? oa : ea);
        if (two) o0[x - Nx] = v.y + ((x & 1) ? ob : eb);
    }
}

}  // namespace at3r
