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
#include <climits>
#include <type_traits>

#include "fft_smem.cuh"
#include "rand_table.cuh"

namespace at3r {

constexpr float kSentinelTest = -1e10f;   // "empty sample" threshold of the reference
constexpr float kSentinelValue = -1e30f;  // value the reference writes for "no sample"
// 16-bit storage keeps the -1e30 "no sample" class as a marker (NaN) instead
// of a value: every value at or below this (the weighted -1e30 lies far
// below it) is stored as the marker; every other value keeps its magnitude,
// so a value between -1e20 and -1e10 still lerps as the reference lerps it.
constexpr float kStoreMissing = -1e20f;

// floor without the conversion units: for 0 <= x < 2^23, x + 2^23 rounded
// down is 2^23 + floor(x) exactly, so its bit pattern minus kMagicBits is
// floor(x) and subtracting 2^23 again gives floor(x) as a float.
constexpr float kMagic = 8388608.0f;
constexpr int kMagicBits = 0x4B000000;

// ---------------------------------------------------------------------------
// Storage of staged sinograms.  FP32 as is; FP16 / BF16 as value / scale with
// one scale per (slice, tilt) row (the row's largest magnitude, the -1e30
// "no sample" markers left out), so a row spans [-1, 1] whatever its level.
// Accumulation is always FP32.  A row keeps 2^-24 (FP16) or 2^-133 (BF16) of
// its largest magnitude: FP16 loses the ordinary values of a row that also
// holds a value ten orders of magnitude larger (as near-threshold test inputs
// do); BF16 does not.
// ---------------------------------------------------------------------------
template <typename ST>
struct Stor;
template <>
struct Stor<float> {
    __device__ __forceinline__ static float ld(const float* p, float) { return __ldg(p); }
    __device__ __forceinline__ static void st(float* p, float v, float) { *p = v; }
};
// An empty value is stored as NaN, which no stored number equals; it reads
// back as the reference's -1e30 (a lerp with a zero weight then stays exact).
__device__ __forceinline__ float unscale(float x, float scale) { return x != x ? kSentinelValue : x * scale; }

template <>
struct Stor<__half> {
    __device__ __forceinline__ static float ld(const __half* p, float scale) { return unscale(__half2float(__ldg(p)), scale); }
    __device__ __forceinline__ static void st(__half* p, float v, float inv)
    {
        *p = __float2half_rn(v <= kStoreMissing ? __int_as_float(0x7fc00000) : v * inv);
    }
};
template <>
struct Stor<__nv_bfloat16> {
    __device__ __forceinline__ static float ld(const __nv_bfloat16* p, float scale)
    {
        return unscale(__bfloat162float(__ldg(p)), scale);
    }
    __device__ __forceinline__ static void st(__nv_bfloat16* p, float v, float inv)
    {
        *p = __float2bfloat16_rn(v <= kStoreMissing ? __int_as_float(0x7fc00000) : v * inv);
    }
};

// Four slices of the SART working volume at one voxel (the slice-group
// layout): FP32 as float4; the 16-bit shadow as four 16-bit values in 8 bytes.
template <typename VT>
struct Quad;
template <>
struct Quad<float> {
    using T4 = float4;
    __device__ __forceinline__ static float4 ld(const float4* p) { return __ldg(p); }
};
template <typename T2>
__device__ __forceinline__ uint32_t bits_of(T2 v)
{
    return *reinterpret_cast<uint32_t*>(&v);
}
template <typename T2>
__device__ __forceinline__ T2 from_bits(uint32_t u)
{
    return *reinterpret_cast<T2*>(&u);
}
template <>
struct Quad<__half> {
    using T4 = uint2;
    __device__ __forceinline__ static float4 ld(const uint2* p)
    {
        const uint2 u = __ldg(p);
        const float2 a = __half22float2(from_bits<__half2>(u.x)), b = __half22float2(from_bits<__half2>(u.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
    __device__ __forceinline__ static uint2 make(float4 v)
    {
        return make_uint2(bits_of(__floats2half2_rn(v.x, v.y)), bits_of(__floats2half2_rn(v.z, v.w)));
    }
    __device__ __forceinline__ static void st1(uint2* p, int q, float v)
    {
        reinterpret_cast<__half*>(p)[q] = __float2half_rn(v);
    }
};
template <>
struct Quad<__nv_bfloat16> {
    using T4 = uint2;
    __device__ __forceinline__ static float4 ld(const uint2* p)
    {
        const uint2 u = __ldg(p);
        const float2 a = __bfloat1622float2(from_bits<__nv_bfloat162>(u.x));
        const float2 b = __bfloat1622float2(from_bits<__nv_bfloat162>(u.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
    __device__ __forceinline__ static uint2 make(float4 v)
    {
        return make_uint2(bits_of(__floats2bfloat162_rn(v.x, v.y)), bits_of(__floats2bfloat162_rn(v.z, v.w)));
    }
    __device__ __forceinline__ static void st1(uint2* p, int q, float v)
    {
        reinterpret_cast<__nv_bfloat16*>(p)[q] = __float2bfloat16_rn(v);
    }
};

// acc + h in one mixed-precision add (FP16 operand, FP32 result); the same
// value as converting h to FP32 (exact) and adding.
__device__ __forceinline__ float add_f32_f16(float acc, __half h)
{
    float r;
    asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(r) : "h"(__half_as_ushort(h)), "f"(acc));
    return r;
}

__device__ __forceinline__ float comp(const float4& v, int q)
{
    return q == 0 ? v.x : q == 1 ? v.y : q == 2 ? v.z : v.w;
}

// Largest magnitude over a CTA's values (non-empty ones only); every thread
// gets the result.  Uses red[32] of shared memory.
__device__ __forceinline__ float block_absmax(float v, float* red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    float m = 0.f;
    for (int k = 0; k < (int)((blockDim.x + 31) >> 5); k++) m = fmaxf(m, red[k]);
    return m;
}

__device__ __forceinline__ float row_scale(float absmax) { return absmax > 0.f ? absmax : 1.f; }

// Per-slice flag bits (one int per slice of a slab).  A set bit only sends
// work to the fully tested path, so a conservative (sticky) bit is harmless.
constexpr int kFlagVolEmpty = 1;    // the volume holds a -1e30 voxel (AreTomo's "empty")
constexpr int kFlagRawLow = 2;      // the staged sinogram holds values <= kLowValue
constexpr int kFlagDiffLow = 4;     // the residual holds values <= kLowValue
constexpr float kLowValue = -5.0e9f;  // far from any lerp of values above it reaching -1e10

// y-slices one thread carries: every slice has the same geometry (single
// tilt axis), so positions, weights, indices and bounds are formed once and
// only the loads and the accumulation repeat per slice.
constexpr int SB = 4;

// ---------------------------------------------------------------------------
// SART staging: raw[ys][t][x] = proj[t][y0 + ys][x] * (cos_t / Nz), x < N.
// AreTomo/Recon/CDoSartRecon.cpp:100-117 (row gather) and
// AreTomo/Recon/GWeightProjs.cu:7-19 (weight).  Grid (T, slices).
// ---------------------------------------------------------------------------
template <typename ST>
__global__ void __launch_bounds__(256) k_gather_weight(const float* __restrict__ proj, size_t tilt_stride,
                                                       int row_pitch, int y0, const float2* __restrict__ cs, int T,
                                                       int N, int Nz, ST* __restrict__ raw, float* __restrict__ scale,
                                                       int* __restrict__ flags)
{
    const int t = blockIdx.x, ys = blockIdx.y;
    const float w = __ldg(&cs[t].x) / (float)Nz;
    const float* src = proj + (size_t)t * tilt_stride + (size_t)(y0 + ys) * row_pitch;
    ST* dst = raw + ((size_t)ys * T + t) * N;
    bool low = false;
    float inv = 1.f;
    if constexpr (!std::is_same<ST, float>::value) {
        __shared__ float red[32];
        float m = 0.f;
        for (int x = threadIdx.x; x < N; x += blockDim.x) {
            const float v = __ldg(src + x) * w;
            if (v > kStoreMissing) m = fmaxf(m, fabsf(v));
        }
        const float sc = row_scale(block_absmax(m, red));
        inv = 1.f / sc;
        if (threadIdx.x == 0) scale[(size_t)ys * T + t] = sc;
    }
    for (int x = threadIdx.x; x < N; x += blockDim.x) {
        const float v = __ldg(src + x) * w;
        Stor<ST>::st(dst + x, v, inv);
        low |= v <= kLowValue;
    }
    if (low) atomicOr(flags + ys, kFlagRawLow);
}

// ---------------------------------------------------------------------------
// WBP staging + R-weight, two tilt rows per CTA packed as the real and
// imaginary parts of one complex sequence: the filter H(k) is real and even
// (H(N-k) = H(k)), so filtering a + ib filters a and b independently.
// AreTomo/Recon/GWeightProjs.cu:18, GRWeight.cu:7-23 (+ MaUtil/GFFT1D.cu R2C/C2R).
// B such pairs per CTA, transformed as one batch (B <= 8: one warp per row
// for the 16-bit row scales).  Grid (ceil(ceil(T/2) / B), slices).
// ---------------------------------------------------------------------------
template <typename ST, int RS>
__device__ __forceinline__ void rweight_block(const float* __restrict__ proj, size_t tilt_stride, int row_pitch,
                                                 int y0, const float2* __restrict__ cs, int T, int N, int Nz,
                                                 const float* __restrict__ hhalf, const FftPlan& plan, int B,
                                                 ST* __restrict__ out, float* __restrict__ scale,
                                                 int* __restrict__ flags, int bx, int by)
{
    extern __shared__ float2 fsm[];
    __shared__ float rsc[16];   // per row of the CTA: 1 / scale
    const int pitch = fft_pitch(plan.work);
    float2* a = fsm;
    float2* b = fsm + (size_t)B * pitch;
    const int ys = by, pair0 = bx * B;
    const int nq = min(B, (T + 1) / 2 - pair0);   // tilt pairs in this CTA
    const float* srow = proj + (size_t)(y0 + ys) * row_pitch;
    for (int q = 0; q < nq; q++) {
        const int t0 = 2 * (pair0 + q), t1 = t0 + 1;
        const bool two = t1 < T;
        const float w0 = __ldg(&cs[t0].x) / (float)Nz;
        const float w1 = two ? __ldg(&cs[t1].x) / (float)Nz : 0.f;
        const float* s0 = srow + (size_t)t0 * tilt_stride;
        const float* s1 = srow + (size_t)(two ? t1 : t0) * tilt_stride;
        float2* aq = a + (size_t)q * pitch;
        staged_copy<4>(N, [&](int x) { return make_float2(__ldg(s0 + x) * w0, two ? __ldg(s1 + x) * w1 : 0.f); },
                       [&](int x, float2 v) { aq[fft_pad(x)] = v; });
    }
    __syncthreads();
    float2* r = fft_run<RS>(a, b, plan, nq, pitch, -1);
    for (int q = 0; q < nq; q++) {
        float2* rq = r + (size_t)q * pitch;
        for (int k = threadIdx.x; k < N; k += blockDim.x) {
            const float h = __ldg(hhalf + (k <= N - k ? k : N - k));
            const float2 v = rq[fft_pad(k)];
            rq[fft_pad(k)] = make_float2(v.x * h, v.y * h);
        }
    }
    __syncthreads();
    float2* r2 = fft_run<RS>(r, r == a ? b : a, plan, nq, pitch, +1);
    // row 2q + c of the CTA is tilt 2(pair0 + q) + c, component c of sequence q
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if constexpr (!std::is_same<ST, float>::value) {
        // one warp per row: the row's largest non-empty magnitude is its scale
        if (warp < 2 * nq) {
            const int q = warp >> 1, c = warp & 1, t = 2 * (pair0 + q) + c;
            const float2* rq = r2 + (size_t)q * pitch;
            float m = 0.f;
            for (int x = lane; x < N; x += 32) {
                const float2 w2 = rq[fft_pad(x)];
                const float v = c ? w2.y : w2.x;
                if (v > kStoreMissing) m = fmaxf(m, fabsf(v));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            const float sc = row_scale(m);
            if (lane == 0) {
                rsc[warp] = 1.f / sc;
                if (t < T) scale[(size_t)ys * T + t] = sc;
            }
        }
        __syncthreads();
    }
    bool low = false;
    for (int q = 0; q < nq; q++) {
        const int t0 = 2 * (pair0 + q);
        const bool two = t0 + 1 < T;
        const float2* rq = r2 + (size_t)q * pitch;
        ST* d0 = out + ((size_t)ys * T + t0) * N;
        const float inv0 = std::is_same<ST, float>::value ? 1.f : rsc[2 * q];
        const float inv1 = std::is_same<ST, float>::value ? 1.f : rsc[2 * q + 1];
        for (int x = threadIdx.x; x < N; x += blockDim.x) {
            const float2 v = rq[fft_pad(x)];
            Stor<ST>::st(d0 + x, v.x, inv0);
            low |= v.x <= kLowValue;
            if (two) {
                Stor<ST>::st(d0 + N + x, v.y, inv1);
                low |= v.y <= kLowValue;
            }
        }
    }
    if (low) atomicOr(flags + ys, kFlagRawLow);
}

template <typename ST, int RS>
__global__ void __launch_bounds__(512, RS < 2 ? 2 : 1) k_rweight(const float* __restrict__ proj, size_t tilt_stride, int row_pitch,
                                                 int y0, const float2* __restrict__ cs, int T, int N, int Nz,
                                                 const float* __restrict__ hhalf, const __grid_constant__ FftPlan plan, int B,
                                                 ST* __restrict__ out, float* __restrict__ scale,
                                                 int* __restrict__ flags)
{
    rweight_block<ST, RS>(proj, tilt_stride, row_pitch, y0, cs, T, N, Nz, hhalf, plan, B, out, scale, flags, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// Back-projection.  MODE 0: SART update on the 1x grid
// (AreTomo/Recon/GBackProj.cu:12-60, bSart): the mean over tilts [t0, t1) of
// the lerped sinogram is scaled by relax, added, clamped at 0.  MODE 1: the
// WBP 2x grid (AreTomo/Recon/GBackProjWbp.cu:14-53): mean over all tilts,
// or 0 where no tilt contributes.
//
// A CTA covers BP_TX x BP_TZ voxels of SB slices; each thread keeps 2 x 4
// voxel positions (x warp-contiguous) for all SB slices.  Tilts go in chunks
// of BP_CHUNK: for each tilt the CTA stages in shared memory only the
// detector window its voxels reach (the detector position is affine in the
// voxel coordinates, so the tile's corners bound it), as (p[i], p[i+1]) pairs
// so that one 8-byte load feeds a lerp.  Positions, indices, weights and the
// in-detector test are computed once per voxel and tilt and serve all SB
// slices; a chunk whose tilts keep the whole tile strictly inside [0, N-2]
// skips the test.  Slices whose staged data hold values near the -1e10
// "empty" marker (flag bit) go through the per-slice path that tests every
// sample as the reference does.  Sums run in the reference's (tilt) order;
// the fast paths fold the lerp into the sum with fused multiply-adds.
// ---------------------------------------------------------------------------
constexpr int BP_TX = 64, BP_TZ = 32, BP_THREADS = 256, BP_CHUNK = 16;
// Shared-memory stride of one tilt's staged window (pairs).  A window spans
// at most |cos|(BP_TX - 1) + |sin|(BP_TZ - 1) + 6 <= sqrt(63^2 + 31^2) + 6 < 77
// samples (cos^2 + sin^2 = 1; the WBP grid halves it), so a fixed stride
// holds every case and makes the per-slice offsets immediates.
constexpr int BP_WW = 80;
constexpr int BP_PSLAB = BP_CHUNK * BP_WW;   // pairs per slice
constexpr int BP_CX = BP_TX / 32, BP_CZ = BP_TZ / (BP_THREADS / 32);

struct BpArgs {
    const void* sino;        // [slices][T][N] of the storage type
    const float* scale;      // [slices][T] row scales (16-bit storage), else null
    int T, N, t0, t1;
    const float2* cs;
    int GX, GZ;              // voxel grid of this mode
    int S;                   // slices in this launch
    float relax;
    float* out;              // MODE 0: vol slab [slices][GZ][GX] (z flipped), or the slice-group volume
                             // [groups][GZ][GX] float4; MODE 1: [slices][GZ][GX]
    size_t out_slice;
    int ww;                  // staged window width (samples)
    int* flags;              // per-slice flag bits
    int low_bit;             // the flag bit that marks this sinogram as holding low values
    void* shadow;            // MODE 0, 16-bit volume type: [ceil(slices/8)][GZ][GX] of eight 16-bit values
                             // beside the slice-group volume (shadow_half)
    int* seen;               // run summary: the flags of every slice ORed in (may be null)
    int bulk;                // FP32 storage, N % 4 == 0: launch the bulk-copy staging form (bp_smem_bytes(1))
};

template <int MODE>
__device__ __forceinline__ float bp_xp(float fX, float fZs, float c, float cent)
{
    // MODE 0: fX*c + fZ*s + N/2.0f            (GBackProj.cu:35-36)
    // MODE 1: (fX*c + fZ*s)/2 + (N/2) + 0.5f  (GBackProjWbp.cu:34-35); a/2 is
    //         exact, so fl(a/2 + cent) is one fused multiply-add.
    const float a = __fmaf_rn(fX, c, fZs);
    if (MODE == 0) return __fadd_rn(a, cent);
    return __fadd_rn(__fmaf_rn(a, 0.5f, cent), 0.5f);
}

// Raw window rows of the bulk-copy staging: a row is copied from the 16-byte
// boundary at or below its window start, so it spans at most 3 + 81 floats.
constexpr int BP_RAW_W = 88;
constexpr int kFlagStageTimeout = 16;   // a bulk staging wait ran out (the tile was not written)

__host__ __device__ inline size_t bp_smem_bytes(int bulk)
{
    const size_t base = (sizeof(int) + sizeof(float2)) * BP_CHUNK + sizeof(float2) * (size_t)SB * BP_PSLAB;
    return bulk ? base + 16 + sizeof(float) * (size_t)SB * BP_CHUNK * BP_RAW_W : base;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Waits for phase `parity` of the mbarrier at `bar`, at most `limit` polls;
// false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit)
{
    for (int i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Writes one voxel and returns its value afterwards (the old value where no
// tilt contributed).
// k: relax / cnt (MODE 0) or 1 / cnt (MODE 1), one division per voxel for
// all its slices.
template <int MODE>
__device__ __forceinline__ float bp_store(const BpArgs& p, int ys, int Z, int X, float sum, int cnt, float k)
{
    float* out = p.out + (size_t)ys * p.out_slice;
    if (MODE == 0) {
        float* v = out + (size_t)(p.GZ - 1 - Z) * p.GX + X;
        if (cnt <= 0) return *v;
        const float f = __fadd_rn(__fmul_rn(sum, k), *v);
        if (f > kSentinelTest) {
            const float r = fmaxf(f, 0.f);
            *v = r;
            return r;
        }
        *v = kSentinelValue;
        atomicOr(p.flags + ys, kFlagVolEmpty);
        return kSentinelValue;
    } else {
        const float r = cnt > 0 ? __fmul_rn(sum, k) : 0.f;
        out[(size_t)Z * p.GX + X] = r;
        return r;
    }
}

// The 16-bit shadow of the SART working volume holds eight slices per voxel
// ([ceil(S/8)][GZ][GX] x 16 bytes, rows z flipped), so that one forward-
// projection load gives a tap of eight slices; slice group g (four slices)
// is the half g & 1 of element g >> 1.  Index of that half, in 8-byte units.
__device__ __forceinline__ size_t shadow_half(const BpArgs& p, int g, int Z, int X)
{
    return 2 * (((size_t)(g >> 1) * p.GZ + (p.GZ - 1 - Z)) * p.GX + X) + (g & 1);
}

// SART update of one voxel of the slice-group working volume
// ([groups][GZ][GX] float4, component q = slice 4g + q, rows z flipped): all
// four slices at once, and the 16-bit shadow beside it.  Components past the
// slab's last slice are computed from zero rows and never read back.
static_assert(SB == 4, "the slice-group layout holds four slices per voxel");
template <typename VT>
__device__ __forceinline__ void bp_store_grp(const BpArgs& p, int g, int ys0, int nsl, int Z, int X, float4 sum,
                                             int cnt)
{
    if (cnt <= 0) return;
    const size_t idx = ((size_t)g * p.GZ + (p.GZ - 1 - Z)) * p.GX + X;
    float4* v4 = reinterpret_cast<float4*>(p.out) + idx;
    const float4 o = *v4;
    const float k = __fdiv_rn(p.relax, (float)cnt);
    const float sm[4] = {sum.x, sum.y, sum.z, sum.w}, old[4] = {o.x, o.y, o.z, o.w};
    float r[4];
    int empty = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float f = __fadd_rn(__fmul_rn(sm[q], k), old[q]);
        if (f > kSentinelTest) {
            r[q] = fmaxf(f, 0.f);
        } else {
            r[q] = kSentinelValue;
            if (q < nsl) empty |= 1 << q;
        }
    }
    const float4 nv = make_float4(r[0], r[1], r[2], r[3]);
    *v4 = nv;
    if (empty) {
#pragma unroll
        for (int q = 0; q < 4; q++)
            if ((empty >> q) & 1) atomicOr(p.flags + ys0 + q, kFlagVolEmpty);
    }
    if constexpr (!std::is_same<VT, float>::value) reinterpret_cast<uint2*>(p.shadow)[shadow_half(p, g, Z, X)] =
        Quad<VT>::make(nv);
}
template <typename VT>
__device__ __forceinline__ void bp_store1_grp(const BpArgs& p, int g, int q, int ys, int Z, int X, float sum, int cnt)
{
    if (cnt <= 0) return;
    const size_t idx = ((size_t)g * p.GZ + (p.GZ - 1 - Z)) * p.GX + X;
    float* v = reinterpret_cast<float*>(p.out) + 4 * idx + q;
    const float f = __fadd_rn(__fmul_rn(sum, __fdiv_rn(p.relax, (float)cnt)), *v);
    float r;
    if (f > kSentinelTest) {
        r = fmaxf(f, 0.f);
    } else {
        r = kSentinelValue;
        atomicOr(p.flags + ys, kFlagVolEmpty);
    }
    *v = r;
    if constexpr (!std::is_same<VT, float>::value)
        Quad<VT>::st1(reinterpret_cast<uint2*>(p.shadow) + shadow_half(p, g, Z, X), q, r);
}

// GRP (MODE 0 only): the volume is the slice-group working volume above;
// otherwise MODE 0 updates a plain [slices][GZ][GX] volume (z flipped).
// BULK (FP32 storage, N a multiple of 4): window rows staged by bulk
// asynchronous copies, the comparison form; the default form has none of its code.
template <int MODE, typename ST, typename VT, bool GRP, bool BULK = false>
__device__ __forceinline__ void bp_tile(BpArgs p, int bx, int by, int bz)
{
    // FP16 WBP (MODE 1) stages FP16 values and differences (below); SART keeps
    // the FP32 pairs, where the per-sample conversion of the fraction to FP16
    // cost more than the halved shared-memory bytes saved
    constexpr bool H2 = std::is_same<ST, __half>::value && MODE == 1;
    static_assert(!GRP || MODE == 0, "the slice-group layout is the SART working volume");
    static_assert(GRP || std::is_same<VT, float>::value, "the 16-bit shadow exists in the slice-group layout only");
    extern __shared__ float2 bsm[];
    float2* cs_s = bsm;                                               // [BP_CHUNK]
    float2* pw = bsm + BP_CHUNK;                                      // [SB][BP_CHUNK][BP_WW]
    int* ws = reinterpret_cast<int*>(pw + SB * BP_PSLAB);             // [BP_CHUNK]
    // bulk staging: an mbarrier and the raw rows [SB][BP_CHUNK][BP_RAW_W]
    uint64_t* mbar = reinterpret_cast<uint64_t*>(ws + BP_CHUNK);
    float* raw = reinterpret_cast<float*>(reinterpret_cast<char*>(mbar) + 16);
    constexpr bool bulk = BULK && std::is_same<ST, float>::value;
    uint32_t phase = 0;
    bool stage_ok = true;
    if (bulk) {
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
    }
    const int ys0 = bz * SB, nsl = min(SB, p.S - ys0);
    const int X0 = bx * BP_TX, Z0 = by * BP_TZ;
    const float cent = MODE == 0 ? (float)p.N / 2.0f : (float)(p.N / 2);
    const float hx = MODE == 0 ? (float)p.GX * 0.5f : (float)p.GX / 2.0f;
    const float hz = MODE == 0 ? (float)p.GZ * 0.5f : (float)p.GZ / 2.0f;
    const float endX = (float)(p.N - 2);
    const unsigned wmax = (unsigned)(p.ww - 2);

    bool low = false;
    for (int q = 0; q < nsl; q++) low |= (__ldg(p.flags + ys0 + q) & p.low_bit) != 0;
    if (p.seen && bx == 0 && by == 0 && (int)threadIdx.x < nsl)
        atomicOr(p.seen, __ldg(p.flags + ys0 + threadIdx.x));

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // H2: the fast path stages each window position as FP16 values and
    // differences in a common scale per slice (2^-12 of the largest row scale
    // of the launch's tilts), so a sample interpolates two slices per fma.f16x2
    __shared__ float ssc[SB];
    __shared__ float rq[SB][BP_CHUNK];
    float slice_scale[SB];
    if constexpr (H2) {
        if (warp < SB) {
            float m = 0.f;
            if (warp < nsl)
                for (int t = p.t0 + lane; t < p.t1; t += 32) m = fmaxf(m, __ldg(p.scale + (size_t)(ys0 + warp) * p.T + t));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            // 2^-12 of the largest row scale: the largest values stage as up to
            // 4096 (FP16 holds 65504), and rows far weaker than the strongest
            // stay above FP16's subnormal range
            if (lane == 0) ssc[warp] = m > 0.f ? m * 0x1p-12f : 1.f;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < SB; q++) slice_scale[q] = ssc[q];
    }
    float fX[BP_CX], fZ[BP_CZ];
#pragma unroll
    for (int i = 0; i < BP_CX; i++) fX[i] = (float)(X0 + lane + 32 * i) - hx;
#pragma unroll
    for (int j = 0; j < BP_CZ; j++) fZ[j] = (float)(Z0 + warp + (BP_THREADS / 32) * j) - hz;

    // stage chunk [c0, c0 + nc) of slices [ys0, ys0 + ns) into pw; returns
    // whether the whole tile stays strictly inside the detector for it
    auto stage = [&](int c0, int nc, int ysA, int ns, bool h2) -> bool {
        int inside = 1;
        if (H2 && h2 && threadIdx.x < nc) {
#pragma unroll
            for (int q = 0; q < SB; q++)
                rq[q][threadIdx.x] =
                    q < ns ? __fdiv_rn(__ldg(p.scale + (size_t)(ysA + q) * p.T + c0 + threadIdx.x), ssc[q]) : 0.f;
        }
        if (threadIdx.x < nc) {
            const float2 c = __ldg(&p.cs[c0 + threadIdx.x]);
            float lo = 3.0e38f, hi = -3.0e38f;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float cX = (float)(X0 + ((k & 1) ? BP_TX - 1 : 0)) - hx;
                const float cZ = (float)(Z0 + ((k & 2) ? BP_TZ - 1 : 0)) - hz;
                const float xp = bp_xp<MODE>(cX, __fmul_rn(cZ, c.y), c.x, cent);
                lo = fminf(lo, xp);
                hi = fmaxf(hi, xp);
            }
            ws[threadIdx.x] = (int)floorf(lo) - 1;
            cs_s[threadIdx.x] = c;
            inside = (lo >= 0.01f) && (hi <= endX - 0.01f);
        }
        inside = __syncthreads_and(inside);
        if constexpr (H2) {
            if (h2) {
                // entry (t, k) = {v0 v1, v2 v3, d0 d1, d2 d3} (FP16): v_q the value of
                // slice q at window position k, d_q = v_q(k + 1) - v_q(k), both in
                // units of the slice's scale; slices past the slab stay zero.  One
                // warp per tilt, lanes along the window.  (No value here is a
                // missing-value marker: a row holding one flags its slice, which
                // takes the per-slice path.)
                uint4* ph = reinterpret_cast<uint4*>(pw);
                constexpr int NW = BP_THREADS / 32;
                for (int t = warp; t < nc; t += NW) {
                    const int x0 = ws[t];
                    const bool on = x0 >= 0 && x0 + p.ww + 1 <= p.N;   // warp-uniform
                    for (int k = lane; k < p.ww; k += 32) {
                        const int x = x0 + k;
                        float v[SB], d[SB];
#pragma unroll
                        for (int q = 0; q < SB; q++) {
                            float a = 0.f, b = 0.f;
                            if (q < ns) {
                                const __half* src =
                                    reinterpret_cast<const __half*>(p.sino) + ((size_t)(ysA + q) * p.T + c0 + t) * p.N;
                                if (on || (x >= 0 && x < p.N)) a = __half2float(__ldg(src + x));
                                if (on || (x + 1 >= 0 && x + 1 < p.N)) b = __half2float(__ldg(src + x + 1));
                            }
                            const float r = rq[q][t];
                            v[q] = __fmul_rn(a, r);
                            d[q] = __fmul_rn(__fsub_rn(b, a), r);
                        }
                        ph[t * BP_WW + k] = make_uint4(bits_of(__floats2half2_rn(v[0], v[1])),
                                                       bits_of(__floats2half2_rn(v[2], v[3])),
                                                       bits_of(__floats2half2_rn(d[0], d[1])),
                                                       bits_of(__floats2half2_rn(d[2], d[3])));
                    }
                }
                __syncthreads();
                return inside != 0;
            }
        }
        // bulk staging (FP32): a row whose copy range — from the 16-byte boundary
        // at or below its window start through the window's last sample, rounded
        // up to 16 bytes — lies on the detector is fetched by one bulk
        // asynchronous copy (warp 0, one row per lane, completion counted by
        // the mbarrier); other rows take the load path below
        auto bulk_row = [&](int t, int& xa, int& nf) {
            const int x0 = ws[t];
            xa = x0 & ~3;
            nf = (x0 + p.ww + 1 - xa + 3) & ~3;
            return xa >= 0 && xa + nf <= p.N;
        };
        if (bulk && warp == 0) {
            uint32_t bytes = 0;
            for (int r = lane; r < ns * nc; r += 32) {
                int xa, nf;
                if (bulk_row(r % nc, xa, nf)) bytes += 4u * nf;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
            if (lane == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes)
                             : "memory");
            }
            __syncwarp();
            for (int r = lane; r < ns * nc; r += 32) {
                const int q = r / nc, t = r - q * nc;
                int xa, nf;
                if (!bulk_row(t, xa, nf)) continue;
                const float* src = reinterpret_cast<const float*>(p.sino) + ((size_t)(ysA + q) * p.T + c0 + t) * p.N + xa;
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        smem_u32(raw + (q * BP_CHUNK + t) * BP_RAW_W)),
                    "l"(src), "r"(4u * nf), "r"(smem_u32(mbar))
                    : "memory");
            }
        }
        // one warp per (slice, tilt) row, lanes along the window; a lane issues
        // all its loads of the row before its first store, so a warp waits for
        // the L2 once per row rather than once per load
        constexpr int NW = BP_THREADS / 32, KS = (BP_WW + 31) / 32;
        // rows (slice q, tilt t) of the chunk, warp `warp` takes every NW-th;
        // q and t advance without a division
        int q = warp / nc, t = warp - (warp / nc) * nc;
        for (int row = warp; row < ns * nc; row += NW) {
            const int x0 = ws[t];
            if (bulk) {
                int xa, nf;
                if (bulk_row(t, xa, nf)) {
                    t += NW;
                    while (t >= nc) { t -= nc; q++; }
                    continue;
                }
            }
            const size_t row_id = (size_t)(ysA + q) * p.T + c0 + t;
            const float sc = std::is_same<ST, float>::value ? 1.f : __ldg(p.scale + row_id);
            const ST* src = reinterpret_cast<const ST*>(p.sino) + row_id * p.N + x0 + lane;
            float2* dst = pw + q * BP_PSLAB + t * BP_WW + lane;
            float va[KS], vb[KS];
            if (x0 >= 0 && x0 + p.ww + 1 <= p.N) {
                // the whole window lies on the detector (warp-uniform)
#pragma unroll
                for (int u = 0; u < KS; u++) {
                    const bool kv = lane + 32 * u < p.ww;
                    va[u] = kv ? Stor<ST>::ld(src + 32 * u, sc) : 0.f;
                    vb[u] = kv ? Stor<ST>::ld(src + 32 * u + 1, sc) : 0.f;
                }
            } else {
#pragma unroll
                for (int u = 0; u < KS; u++) {
                    const int k = lane + 32 * u, x = x0 + k;
                    const bool kv = k < p.ww;
                    va[u] = (kv && x >= 0 && x < p.N) ? Stor<ST>::ld(src + 32 * u, sc) : 0.f;
                    vb[u] = (kv && x + 1 >= 0 && x + 1 < p.N) ? Stor<ST>::ld(src + 32 * u + 1, sc) : 0.f;
                }
            }
#pragma unroll
            for (int u = 0; u < KS; u++)
                if (lane + 32 * u < p.ww) dst[32 * u] = make_float2(va[u], vb[u]);
            t += NW;
            while (t >= nc) { t -= nc; q++; }
        }
        if (bulk) {
            // every thread waits for the copies (a bounded wait: on timeout the
            // tile is flagged and left unwritten), then the raw rows become pairs
            const bool ok = mbar_wait(smem_u32(mbar), phase, 1 << 22);
            stage_ok = __syncthreads_and(ok && stage_ok) != 0;
            if (stage_ok) phase ^= 1;
            for (int e = threadIdx.x; stage_ok && e < ns * nc * p.ww; e += BP_THREADS) {
                const int r = e / p.ww, k = e - r * p.ww;
                const int q = r / nc, t = r - q * nc;
                int xa, nf;
                if (!bulk_row(t, xa, nf)) continue;
                const float* rr = raw + (q * BP_CHUNK + t) * BP_RAW_W + (ws[t] - xa) + k;
                pw[q * BP_PSLAB + t * BP_WW + k] = make_float2(rr[0], rr[1]);
            }
        }
        __syncthreads();
        return inside != 0;
    };

    // a bulk staging wait that ran out: wait once more (bounded) for the
    // copies still in flight, flag the slab, write nothing
    auto give_up = [&]() {
        mbar_wait(smem_u32(mbar), phase, 1 << 22);
        if (threadIdx.x == 0) atomicOr(p.flags + ys0, kFlagStageTimeout);
    };

    if (!low) {
        if (!H2 && GRP && nsl < SB) {
            // rows of slices past the slab's end stay zero (staging never writes them)
            for (int k = threadIdx.x; k < (SB - nsl) * BP_PSLAB; k += BP_THREADS)
                pw[nsl * BP_PSLAB + k] = make_float2(0.f, 0.f);
        }
        float sum[SB][BP_CZ][BP_CX];
        int cnt[BP_CZ][BP_CX];
#pragma unroll
        for (int j = 0; j < BP_CZ; j++)
#pragma unroll
            for (int i = 0; i < BP_CX; i++) {
                cnt[j][i] = 0;
#pragma unroll
                for (int q = 0; q < SB; q++) sum[q][j][i] = 0.f;
            }
        for (int c0 = p.t0; c0 < p.t1; c0 += BP_CHUNK) {
            const int nc = min(BP_CHUNK, p.t1 - c0);
            const bool inside = stage(c0, nc, ys0, nsl, true);
            if (!stage_ok) break;
            if (H2 && inside) {
                const uint4* ph = reinterpret_cast<const uint4*>(pw);
                for (int t = 0; t < nc; t++) {
                    const float2 c = cs_s[t];
                    const int wb = t * BP_WW - ws[t] - kMagicBits;
#pragma unroll
                    for (int j = 0; j < BP_CZ; j++) {
                        const float fzs = __fmul_rn(fZ[j], c.y);
#pragma unroll
                        for (int i = 0; i < BP_CX; i++) {
                            const float xp = bp_xp<MODE>(fX[i], fzs, c.x, cent);
                            const float tr = __fadd_rd(xp, kMagic);
                            const float fr = __fsub_rn(xp, __fsub_rn(tr, kMagic));
                            const uint4 e = ph[__float_as_int(tr) + wb];
                            const __half2 f2 = __float2half2_rn(fr);
                            const __half2 v01 = __hfma2(from_bits<__half2>(e.z), f2, from_bits<__half2>(e.x));
                            const __half2 v23 = __hfma2(from_bits<__half2>(e.w), f2, from_bits<__half2>(e.y));
                            sum[0][j][i] = add_f32_f16(sum[0][j][i], __low2half(v01));
                            sum[1][j][i] = add_f32_f16(sum[1][j][i], __high2half(v01));
                            sum[2][j][i] = add_f32_f16(sum[2][j][i], __low2half(v23));
                            sum[3][j][i] = add_f32_f16(sum[3][j][i], __high2half(v23));
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < BP_CZ; j++)
#pragma unroll
                    for (int i = 0; i < BP_CX; i++) cnt[j][i] += nc;
            } else if (H2) {
                const uint4* ph = reinterpret_cast<const uint4*>(pw);
                for (int t = 0; t < nc; t++) {
                    const float2 c = cs_s[t];
                    const uint4* w = ph + t * BP_WW;
                    const int st = ws[t];
#pragma unroll
                    for (int j = 0; j < BP_CZ; j++) {
                        const float fzs = __fmul_rn(fZ[j], c.y);
#pragma unroll
                        for (int i = 0; i < BP_CX; i++) {
                            const float xp = bp_xp<MODE>(fX[i], fzs, c.x, cent);
                            const bool in = xp >= 0.f && xp <= endX;
                            const int ii = (int)xp;
                            const float fr = __fsub_rn(xp, (float)ii);
                            const uint4 e = w[min((unsigned)(ii - st), wmax)];
                            const __half2 f2 = __float2half2_rn(fr);
                            const __half2 v01 = __hfma2(from_bits<__half2>(e.z), f2, from_bits<__half2>(e.x));
                            const __half2 v23 = __hfma2(from_bits<__half2>(e.w), f2, from_bits<__half2>(e.y));
                            if (in) {
                                sum[0][j][i] = add_f32_f16(sum[0][j][i], __low2half(v01));
                                sum[1][j][i] = add_f32_f16(sum[1][j][i], __high2half(v01));
                                sum[2][j][i] = add_f32_f16(sum[2][j][i], __low2half(v23));
                                sum[3][j][i] = add_f32_f16(sum[3][j][i], __high2half(v23));
                                cnt[j][i] += 1;
                            }
                        }
                    }
                }
            } else if (inside) {
                // the whole tile lands inside the detector for every tilt of the chunk
                for (int t = 0; t < nc; t++) {
                    const float2 c = cs_s[t];
                    // window index of sample xp: floor(xp) - st, from the bits of xp + 2^23
                    const int wb = t * BP_WW - ws[t] - kMagicBits;
#pragma unroll
                    for (int j = 0; j < BP_CZ; j++) {
                        const float fzs = __fmul_rn(fZ[j], c.y);
#pragma unroll
                        for (int i = 0; i < BP_CX; i++) {
                            const float xp = bp_xp<MODE>(fX[i], fzs, c.x, cent);
                            const float tr = __fadd_rd(xp, kMagic);
                            const float fr = __fsub_rn(xp, __fsub_rn(tr, kMagic));
                            const float om = __fsub_rn(1.f, fr);
                            const float2* wq = pw + (__float_as_int(tr) + wb);
#pragma unroll
                            for (int q = 0; q < SB; q++) {
                                const float2 v = wq[q * BP_PSLAB];
                                sum[q][j][i] = __fmaf_rn(v.y, fr, __fmaf_rn(v.x, om, sum[q][j][i]));
                            }
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < BP_CZ; j++)
#pragma unroll
                    for (int i = 0; i < BP_CX; i++) cnt[j][i] += nc;
            } else {
                for (int t = 0; t < nc; t++) {
                    const float2 c = cs_s[t];
                    const float2* w = pw + t * BP_WW;
                    const int st = ws[t];
#pragma unroll
                    for (int j = 0; j < BP_CZ; j++) {
                        const float fzs = __fmul_rn(fZ[j], c.y);
#pragma unroll
                        for (int i = 0; i < BP_CX; i++) {
                            const float xp = bp_xp<MODE>(fX[i], fzs, c.x, cent);
                            const bool in = xp >= 0.f && xp <= endX;
                            const int ii = (int)xp;
                            const float fr = __fsub_rn(xp, (float)ii);
                            const float om = __fsub_rn(1.f, fr);
                            const float2* wq = w + min((unsigned)(ii - st), wmax);
#pragma unroll
                            for (int q = 0; q < SB; q++) {
                                const float2 v = wq[q * BP_PSLAB];
                                const float acc = __fmaf_rn(v.y, fr, __fmaf_rn(v.x, om, sum[q][j][i]));
                                sum[q][j][i] = in ? acc : sum[q][j][i];
                            }
                            cnt[j][i] += in ? 1 : 0;
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (!stage_ok) {
            give_up();
            return;
        }
#pragma unroll
        for (int j = 0; j < BP_CZ; j++) {
            const int Z = Z0 + warp + (BP_THREADS / 32) * j;
#pragma unroll
            for (int i = 0; i < BP_CX; i++) {
                const int X = X0 + lane + 32 * i;
                if (Z >= p.GZ || X >= p.GX) continue;
                if constexpr (H2) {
#pragma unroll
                    for (int q = 0; q < SB; q++) sum[q][j][i] = __fmul_rn(sum[q][j][i], slice_scale[q]);
                }
                if constexpr (GRP) {
                    bp_store_grp<VT>(p, bz, ys0, nsl, Z, X,
                                     make_float4(sum[0][j][i], sum[1][j][i], sum[2][j][i], sum[3][j][i]), cnt[j][i]);
                } else {
                    const float k = cnt[j][i] > 0 ? __fdiv_rn(MODE == 0 ? p.relax : 1.f, (float)cnt[j][i]) : 0.f;
#pragma unroll
                    for (int q = 0; q < SB; q++)
                        if (q < nsl) bp_store<MODE>(p, ys0 + q, Z, X, sum[q][j][i], cnt[j][i], k);
                }
            }
        }
        return;
    }

    // per-slice path: every sample tested as the reference does
    for (int q = 0; q < nsl; q++) {
        float sum[BP_CZ][BP_CX];
        int cnt[BP_CZ][BP_CX];
#pragma unroll
        for (int j = 0; j < BP_CZ; j++)
#pragma unroll
            for (int i = 0; i < BP_CX; i++) { sum[j][i] = 0.f; cnt[j][i] = 0; }
        for (int c0 = p.t0; c0 < p.t1; c0 += BP_CHUNK) {
            const int nc = min(BP_CHUNK, p.t1 - c0);
            stage(c0, nc, ys0 + q, 1, false);
            if (!stage_ok) break;
            for (int t = 0; t < nc; t++) {
                const float2 c = cs_s[t];
                const float2* w = pw + t * BP_WW;
                const int st = ws[t];
#pragma unroll
                for (int j = 0; j < BP_CZ; j++) {
                    const float fzs = __fmul_rn(fZ[j], c.y);
#pragma unroll
                    for (int i = 0; i < BP_CX; i++) {
                        const float xp = bp_xp<MODE>(fX[i], fzs, c.x, cent);
                        const int ii = (int)xp;
                        const float fr = __fsub_rn(xp, (float)ii);
                        const float2 v2 = w[min((unsigned)(ii - st), wmax)];
                        const float v = __fmaf_rn(v2.x, __fsub_rn(1.f, fr), __fmul_rn(v2.y, fr));
                        // the reference skips v <= -1e10 (a NaN sample is summed)
                        if (xp >= 0.f && xp <= endX && !(v <= kSentinelTest)) {
                            sum[j][i] = __fadd_rn(sum[j][i], v);
                            cnt[j][i] += 1;
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (!stage_ok) {
            give_up();
            return;
        }
#pragma unroll
        for (int j = 0; j < BP_CZ; j++) {
            const int Z = Z0 + warp + (BP_THREADS / 32) * j;
#pragma unroll
            for (int i = 0; i < BP_CX; i++) {
                const int X = X0 + lane + 32 * i;
                if (Z < p.GZ && X < p.GX) {
                    if constexpr (GRP) {
                        bp_store1_grp<VT>(p, bz, q, ys0 + q, Z, X, sum[j][i], cnt[j][i]);
                    } else {
                        const float k = cnt[j][i] > 0 ? __fdiv_rn(MODE == 0 ? p.relax : 1.f, (float)cnt[j][i]) : 0.f;
                        bp_store<MODE>(p, ys0 + q, Z, X, sum[j][i], cnt[j][i], k);
                    }
                }
            }
        }
    }
}

// Grid (tiles x, tiles z, slice groups).  With a 16-bit shadow the two slice
// groups that share its 16-byte elements run as neighbouring CTAs instead —
// grid (2 * tiles x, tiles z, ceil(groups / 2)), the group's low bit fastest
// (k_bp_grid) — so both halves of an element reach L2 together and leave it
// as whole sectors.
template <typename VT>
__host__ __device__ constexpr bool bp_paired() { return !std::is_same<VT, float>::value; }

template <int MODE, typename ST, typename VT, bool GRP, bool BULK = false>
__global__ void __launch_bounds__(BP_THREADS, 3) k_bp(BpArgs p)
{
    if constexpr (GRP && bp_paired<VT>()) {
        const int g = 2 * (int)blockIdx.z + (int)(blockIdx.x & 1);
        if (g * SB >= p.S) return;
        bp_tile<MODE, ST, VT, GRP, BULK>(p, blockIdx.x >> 1, blockIdx.y, g);
    } else {
        bp_tile<MODE, ST, VT, GRP, BULK>(p, blockIdx.x, blockIdx.y, blockIdx.z);
    }
}

// ---------------------------------------------------------------------------
// SART forward projection of tilts [t0, t0 + grid.y) with the residual fused:
// AreTomo/Recon/GForProj.cu:10-76 (ray of L = int(Nz/cos + 1.5) samples,
// bilinear, mean over in-volume samples, -1e30 if none) followed by
// AreTomo/Recon/GDiffProj.cu:7-21 (d = raw - fp, 0 where either is empty).
// One ray per thread, for SB slices at once; the lanes of a warp are
// neighbouring rays and step through sample index i in lock-step, so every
// step reads two short runs of two volume rows per slice.
//
// The sample positions x_i = fma(-z0_i, sin, tx), z_i = fma(z0_i, cos, tz)
// (z0_i = i - L/2) are monotonic in i after FP32 rounding too, so the samples
// the reference keeps (0 <= x <= Nx-2, 0 <= z <= Nz-2) form one contiguous
// range of i per ray.  Each ray finds that range exactly (an estimate, then
// a walk to the first/last index that passes the reference's own test) and
// samples it without per-sample bounds tests; positions and weights serve
// all SB slices.  Slices whose volume may hold "empty" voxels (flag bit) are
// projected one at a time with the per-sample value test kept.
// Grid (ceil(N/256), tilts, ceil(slices/SB)).
// ---------------------------------------------------------------------------
struct RayPos {
    float tx, tz, c, s, halfL;
    __device__ __forceinline__ float x(int i) const { return __fmaf_rn(-((float)i - halfL), s, tx); }
    __device__ __forceinline__ float z(int i) const { return __fmaf_rn((float)i - halfL, c, tz); }
};

// First index in [lo, hi + 1] where a predicate that is monotonic false -> true
// over [lo, hi] holds, starting the walk from an estimate.
template <class P>
__device__ __forceinline__ int first_true(int lo, int hi, int est, P pred)
{
    est = min(max(est, lo), hi + 1);
    while (est > lo && pred(est - 1)) est--;
    while (est <= hi && !pred(est)) est++;
    return est;
}

__device__ __forceinline__ int est_index(float v) { return (int)fminf(fmaxf(v, -1.0e8f), 1.0e8f); }

// Ray set-up: position of ray u of tilt (c, s), and the in-volume sample
// range [lo, hi] (empty when lo > hi).
__device__ __forceinline__ void fp_ray_setup(int u, int N, int Nx, int Nz, float c, float s, RayPos& r, int& lo,
                                             int& hi)
{
    r.c = c;
    r.s = s;
    const int L = (int)((float)Nz / c + 1.5f);
    const float fXp = (float)u - 0.5f * (float)N;
    r.tx = fXp / c + (float)Nx * 0.5f;
    r.tz = (float)Nz * 0.5f;
    r.halfL = (float)L * 0.5f;
    const float endX = (float)(Nx - 2), endZ = (float)(Nz - 2);
    lo = first_true(0, L - 1, est_index(ceilf(r.halfL - r.tz / c)), [&](int i) { return r.z(i) >= 0.f; });
    hi = first_true(lo, L - 1, est_index(floorf(r.halfL + (endZ - r.tz) / c)) + 1,
                    [&](int i) { return r.z(i) > endZ; }) - 1;
    if (s > 0.f) {
        lo = first_true(lo, hi, est_index(ceilf(r.halfL + (r.tx - endX) / s)), [&](int i) { return r.x(i) <= endX; });
        hi = first_true(lo, hi, est_index(floorf(r.halfL + r.tx / s)) + 1, [&](int i) { return r.x(i) < 0.f; }) - 1;
    } else if (s < 0.f) {
        lo = first_true(lo, hi, est_index(ceilf(r.halfL + r.tx / s)), [&](int i) { return r.x(i) >= 0.f; });
        hi = first_true(lo, hi, est_index(floorf(r.halfL + (r.tx - endX) / s)) + 1,
                        [&](int i) { return r.x(i) > endX; }) - 1;
    } else if (!(r.tx >= 0.f && r.tx <= endX)) {
        hi = lo - 1;
    }
}

__device__ __forceinline__ float bilerp(float a00, float a10, float a01, float a11, float wx, float wz)
{
    const float A = __fmaf_rn(wz, a01 - a00, a00);
    const float B = __fmaf_rn(wz, a11 - a10, a10);
    return __fmaf_rn(wx, B - A, A);
}

// Slices one forward-projection thread carries: four of the FP32 volume (one
// float4 tap); eight of the 16-bit shadow (one 16-byte tap), which halves the
// per-slice cost of the sample positions, weights and loads.
template <typename VT>
__host__ __device__ constexpr int fp_slices()
{
    return std::is_same<VT, float>::value ? 4 : 8;
}

// bf16 pair -> two floats: a bf16 is the upper half of an FP32 word.
__device__ __forceinline__ float bf_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf_hi(uint32_t u) { return __uint_as_float(u & 0xffff0000u); }

// ST: storage of raw / diff rows; VT: float reads the FP32 volume, __half /
// __nv_bfloat16 read its 16-bit shadow — the FP32 volume is then read only
// for slices that may hold "empty" voxels.  GRP: the volume is in the
// slice-group layout (one float4 load gives a tap of four slices) and the
// shadow holds eight slices per voxel (one 16-byte load gives a tap of
// eight); otherwise (FP32 only) the volume is plain [slices][Nz][Nx].
// Grid (ceil(N/256), tilts, ceil(slices / fp_slices<VT>())).  Six CTAs per SM
// with FP32 taps (40 registers), five with the 16-bit shadow (48): the loop
// waits on L1 and L2, so resident warps are what hides it.
template <typename ST, typename VT, bool GRP>
__global__ void __launch_bounds__(256, std::is_same<VT, float>::value ? 6 : 5) k_fp_diff(const float* __restrict__ vol, const void* __restrict__ shadow,
                                                 int Nx, int Nz, int S, const ST* __restrict__ raw,
                                                 ST* __restrict__ diff, const float* __restrict__ scale,
                                                 const float2* __restrict__ cs, int T, int N, int t0,
                                                 double* __restrict__ rf, int* __restrict__ flags)
{
    static_assert(GRP || std::is_same<VT, float>::value, "the 16-bit shadow exists in the slice-group layout only");
    constexpr int NS = fp_slices<VT>();
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = t0 + blockIdx.y, ys0 = blockIdx.z * NS, nsl = min(NS, S - ys0);
    const bool active = u < N;
    const float2 cc = __ldg(&cs[t]);
    RayPos r;
    int lo, hi;
    fp_ray_setup(active ? u : N - 1, N, Nx, Nz, cc.x, cc.y, r, lo, hi);
    if (!active) { lo = 1; hi = 0; }
    // the warp walks one common index range so its lanes read the same rows
    const int wlo = __reduce_min_sync(0xffffffffu, lo <= hi ? lo : INT_MAX);
    const int whi = __reduce_max_sync(0xffffffffu, lo <= hi ? hi : INT_MIN);
    const size_t slice = (size_t)Nx * Nz;
    const float* vbase = vol + (size_t)(Nz - 1) * Nx;   // voxel (X, Z) at row Nz-1-Z
    bool empty_vox = false;
    for (int q = 0; q < nsl; q++) empty_vox |= (__ldg(flags + ys0 + q) & kFlagVolEmpty) != 0;

    float fSum[NS], fCount[NS];
#pragma unroll
    for (int q = 0; q < NS; q++) { fSum[q] = 0.f; fCount[q] = 0.f; }
    if (GRP && !empty_vox) {
        // cell offset iX - iZ*Nx from the bits of x + 2^23 and z + 2^23
        // (wrapping 32-bit arithmetic; the true value fits an int)
        const unsigned kx = (unsigned)kMagicBits * (unsigned)(Nx - 1);
        float fi = (float)wlo;   // i as a float, exact below 2^24
        if constexpr (std::is_same<VT, float>::value) {
            // slice group: one float4 load per tap; rows of voxel Z and Z + 1 as bases
            const float4* g0 = reinterpret_cast<const float4*>(vol) + (size_t)blockIdx.z * slice + (size_t)(Nz - 1) * Nx;
            const float4* g1 = g0 - Nx;
            for (int i = wlo; i <= whi; i++, fi += 1.f) {
                if (i < lo || i > hi) continue;
                const float fd = fi - r.halfL;   // exact: the sample index of RayPos
                const float fX = __fmaf_rn(-fd, r.s, r.tx), fZ = __fmaf_rn(fd, r.c, r.tz);
                const float tX = __fadd_rd(fX, kMagic), tZ = __fadd_rd(fZ, kMagic);
                const float wx = fX - (tX - kMagic), wz = fZ - (tZ - kMagic);
                const int o = (int)((unsigned)__float_as_int(tX) - (unsigned)__float_as_int(tZ) * (unsigned)Nx + kx);
                const float ux = 1.f - wx, uz = 1.f - wz;
                const float w00 = ux * uz, w10 = wx * uz, w01 = ux * wz, w11 = wx * wz;
                const float4 a00 = __ldg(g0 + o), a10 = __ldg(g0 + o + 1);
                const float4 a01 = __ldg(g1 + o), a11 = __ldg(g1 + o + 1);
                fSum[0] = __fmaf_rn(w11, a11.x, __fmaf_rn(w01, a01.x, __fmaf_rn(w10, a10.x, __fmaf_rn(w00, a00.x, fSum[0]))));
                fSum[1] = __fmaf_rn(w11, a11.y, __fmaf_rn(w01, a01.y, __fmaf_rn(w10, a10.y, __fmaf_rn(w00, a00.y, fSum[1]))));
                fSum[2] = __fmaf_rn(w11, a11.z, __fmaf_rn(w01, a01.z, __fmaf_rn(w10, a10.z, __fmaf_rn(w00, a00.z, fSum[2]))));
                fSum[3] = __fmaf_rn(w11, a11.w, __fmaf_rn(w01, a01.w, __fmaf_rn(w10, a10.w, __fmaf_rn(w00, a00.w, fSum[3]))));
            }
        } else {
            // 16-bit shadow, eight slices per 16-byte tap
            const uint4* g0 = reinterpret_cast<const uint4*>(shadow) + (size_t)blockIdx.z * slice + (size_t)(Nz - 1) * Nx;
            const uint4* g1 = g0 - Nx;
            for (int i = wlo; i <= whi; i++, fi += 1.f) {
                if (i < lo || i > hi) continue;
                const float fd = fi - r.halfL;
                const float fX = __fmaf_rn(-fd, r.s, r.tx), fZ = __fmaf_rn(fd, r.c, r.tz);
                const float tX = __fadd_rd(fX, kMagic), tZ = __fadd_rd(fZ, kMagic);
                const float wx = fX - (tX - kMagic), wz = fZ - (tZ - kMagic);
                const int o = (int)((unsigned)__float_as_int(tX) - (unsigned)__float_as_int(tZ) * (unsigned)Nx + kx);
                const float ux = 1.f - wx, uz = 1.f - wz;
                const float w00 = ux * uz, w10 = wx * uz, w01 = ux * wz, w11 = wx * wz;
                const uint4 b00 = __ldg(g0 + o), b10 = __ldg(g0 + o + 1);
                const uint4 b01 = __ldg(g1 + o), b11 = __ldg(g1 + o + 1);
                const uint32_t p00[4] = {b00.x, b00.y, b00.z, b00.w}, p10[4] = {b10.x, b10.y, b10.z, b10.w};
                const uint32_t p01[4] = {b01.x, b01.y, b01.z, b01.w}, p11[4] = {b11.x, b11.y, b11.z, b11.w};
                if constexpr (std::is_same<VT, __half>::value) {
                    // the sample value of two slices per half2 instruction,
                    // added to the FP32 sums by mixed-precision adds
                    const __half2 h00 = __float2half2_rn(w00), h10 = __float2half2_rn(w10);
                    const __half2 h01 = __float2half2_rn(w01), h11 = __float2half2_rn(w11);
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        __half2 v = __hmul2(h00, from_bits<__half2>(p00[k]));
                        v = __hfma2(h10, from_bits<__half2>(p10[k]), v);
                        v = __hfma2(h01, from_bits<__half2>(p01[k]), v);
                        v = __hfma2(h11, from_bits<__half2>(p11[k]), v);
                        fSum[2 * k] = add_f32_f16(fSum[2 * k], __low2half(v));
                        fSum[2 * k + 1] = add_f32_f16(fSum[2 * k + 1], __high2half(v));
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        fSum[2 * k] = __fmaf_rn(w11, bf_lo(p11[k]), __fmaf_rn(w01, bf_lo(p01[k]),
                                      __fmaf_rn(w10, bf_lo(p10[k]), __fmaf_rn(w00, bf_lo(p00[k]), fSum[2 * k]))));
                        fSum[2 * k + 1] = __fmaf_rn(w11, bf_hi(p11[k]), __fmaf_rn(w01, bf_hi(p01[k]),
                                          __fmaf_rn(w10, bf_hi(p10[k]), __fmaf_rn(w00, bf_hi(p00[k]), fSum[2 * k + 1]))));
                    }
                }
            }
        }
        const float n = (float)max(hi - lo + 1, 0);
#pragma unroll
        for (int q = 0; q < NS; q++) fCount[q] = n;
    } else if (!empty_vox) {
        // plain layout (FP32): per slice, the rows of voxel Z and Z + 1 as
        // loop-invariant bases; a sample then costs one 32-bit cell offset
        // and one wide add per row
        const float* r0[NS];
        const float* r1[NS];
#pragma unroll
        for (int q = 0; q < NS; q++) {
            r0[q] = vbase + (size_t)(ys0 + min(q, nsl - 1)) * slice;
            r1[q] = r0[q] - Nx;
        }
        for (int i = wlo; i <= whi; i++) {
            if (i < lo || i > hi) continue;
            const float fX = r.x(i), fZ = r.z(i);
            const int iX = (int)fX, iZ = (int)fZ;
            const float wx = fX - (float)iX, wz = fZ - (float)iZ;
            const int o = iX - iZ * Nx;   // within one slice: |o| < Nx * Nz
#pragma unroll
            for (int q = 0; q < NS; q++) {
                const float* p0 = r0[q] + o;
                const float* p1 = r1[q] + o;
                fSum[q] += bilerp(__ldg(p0), __ldg(p0 + 1), __ldg(p1), __ldg(p1 + 1), wx, wz);
            }
        }
        const float n = (float)max(hi - lo + 1, 0);
#pragma unroll
        for (int q = 0; q < NS; q++) fCount[q] = n;
    } else {
        // slices that may hold empty voxels: one at a time from the FP32
        // volume (slice-group layout: group (ys0+q)/4, component (ys0+q)%4)
        // with the reference's per-sample test
        constexpr int E = GRP ? 4 : 1;
        for (int q = 0; q < nsl; q++) {
            const int ys = ys0 + q;
            const float* v0 = GRP ? vol + E * ((size_t)(ys >> 2) * slice + (size_t)(Nz - 1) * Nx) + (ys & 3)
                                  : vbase + (size_t)ys * slice;
            float s0 = 0.f, n0 = 0.f;
            for (int i = wlo; i <= whi; i++) {
                if (i < lo || i > hi) continue;
                const float fX = r.x(i), fZ = r.z(i);
                const int iX = (int)fX, iZ = (int)fZ;
                const float* p = v0 + E * (iX - (ptrdiff_t)iZ * Nx);
                const float val = bilerp(__ldg(p), __ldg(p + E), __ldg(p - E * Nx), __ldg(p - E * Nx + E),
                                         fX - (float)iX, fZ - (float)iZ);
                if (val < kSentinelTest) continue;
                s0 += val;
                n0 += 1.f;
            }
#pragma unroll
            for (int k = 0; k < NS; k++)
                if (k == q) { fSum[k] = s0; fCount[k] = n0; }
        }
    }

    float ad = 0.f, ar = 0.f;
    if (active) {
#pragma unroll
        for (int q = 0; q < NS; q++) {
            if (q >= nsl) continue;
            const float fp = fCount[q] <= 0.f ? kSentinelValue : fSum[q] / fCount[q];
            const size_t row = (size_t)(ys0 + q) * T + t;
            const size_t o = row * N + u;
            const float sc = std::is_same<ST, float>::value ? 1.f : __ldg(scale + row);
            const float rw = Stor<ST>::ld(raw + o, sc);
            float d = 0.f;
            if (!(fp < kSentinelTest) && !(rw < kSentinelTest)) {
                d = rw - fp;
                ad += fabsf(d);
                ar += fabsf(rw);
                if (d <= kLowValue) atomicOr(flags + ys0 + q, kFlagDiffLow);
            }
            Stor<ST>::st(diff + o, d, 1.f / sc);
        }
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
            for (int k = 0; k < 8; k++) { sd += red[0][k]; sr += red[1][k]; }
            atomicAdd(rf, sd);
            atomicAdd(rf + 1, sr);
        }
    }
}

// ---------------------------------------------------------------------------
// Slice-group working volume -> output slices: vol[4g + q][r][x] =
// W[g][r][x].q for the slab's S slices (rows already z flipped).
// Grid (ceil(Nx*Nz / 256), groups).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_ungroup(const float4* __restrict__ w, float* __restrict__ vol, int S,
                                                 size_t slice)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    if (i >= slice) return;
    const float4 v = __ldg(w + (size_t)g * slice + i);
    const int n = min(4, S - 4 * g);
    float* o = vol + (size_t)4 * g * slice + i;
    o[0] = v.x;
    if (n > 1) o[slice] = v.y;
    if (n > 2) o[2 * slice] = v.z;
    if (n > 3) o[3 * slice] = v.w;
}

// ---------------------------------------------------------------------------
// Volume output stage, DataUtil/CTiltSeries.cpp:286-305 (FlipVol): the
// reconstruction's XZ frames become XY frames.  in: S frames [Nz][Nx] (row zr
// of frame s); out frame fz = (flip ? Nz-1-zr : zr) gets row s = in frame s
// row zr, out[fz * frame_pitch + s * Nx + x].  Nx is even; rows move as
// float2.  Grid (Nz, S).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_flip_rows(const float* __restrict__ in, float* __restrict__ out, int Nz,
                                                   int Nx, int flip, size_t frame_pitch)
{
    const int zr = blockIdx.x, s = blockIdx.y;
    const int fz = flip ? Nz - 1 - zr : zr;
    const float2* src = reinterpret_cast<const float2*>(in + ((size_t)s * Nz + zr) * Nx);
    float2* dst = reinterpret_cast<float2*>(out + (size_t)fz * frame_pitch + (size_t)s * Nx);
    for (int x = threadIdx.x; x < Nx / 2; x += blockDim.x) dst[x] = __ldg(src + x);
}

// ---------------------------------------------------------------------------
// Empty-voxel fill after SART (AreTomo/Recon/CTomoSart.cpp:88 ->
// MaUtil/GFillEmpty2D.cu:7-143, table of MaUtil/GGenRandoms.cu): on every
// slice with empty voxels (value below -1e10, flag bit), an empty voxel
// follows its chain through the random table — at most 100 links — to the
// first non-empty voxel and takes its value; a chain that finds none takes the
// mean of the slice's non-empty voxels, summed as the reference's single
// 512-thread block sums it.  Voxel indices are the reference's, i = Z*Nx + X
// in its unflipped slice; here voxel (X, Z) lives in row Nz-1-Z of
// vol[S][Nz][Nx].  Table entries are drawn on the fly (rand_table.cuh), so no
// table is stored.
//
// Two passes, in place.  k_fill_mark: each empty voxel finds its source and
// is overwritten with a marker, a float below -1e10 whose bits encode the
// source index (kFillMark + k) or the mean (kFillMarkMean); markers still
// read as empty, so chains walked at the same time see the state before the
// fill, as the reference's separate emptiness pass gives them.
// k_fill_finish: the mean of the non-empty voxels (markers excluded), then
// every marker is replaced by its source voxel's value (never a marker) or
// the mean.
// ---------------------------------------------------------------------------
constexpr unsigned kFillMark = 0xD0200000u;       // -1.07e10: marker of source 0
constexpr unsigned kFillMarkMean = 0xF0200000u;   // -1.98e29: beyond every source (< 2^29 voxels)
constexpr int kFlagFillMean = 8;                  // a chain found no non-empty voxel (run summary bit)

__device__ __forceinline__ size_t fill_addr(int i, int Nx, int Nz)
{
    const int Z = i / Nx;
    return (size_t)(Nz - 1 - Z) * Nx + (i - Z * Nx);
}

// Grid (blocks, S), 256 threads; blocks stride over the slice.
__global__ void __launch_bounds__(256) k_fill_mark(float* __restrict__ vol, int Nx, int Nz,
                                                   const int* __restrict__ flags, unsigned long long seed,
                                                   int* __restrict__ seen)
{
    const int ys = blockIdx.y;
    if ((flags[ys] & kFlagVolEmpty) == 0) return;
    const int n = Nx * Nz;
    float* v = vol + (size_t)ys * n;
    bool mean_used = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t a = fill_addr(i, Nx, Nz);
        if (!(v[a] < kSentinelTest)) continue;
        int next = rand_table_entry(seed, i, n);
        unsigned mark = kFillMarkMean;
        for (int j = 0; j < 100; j++) {
            if (v[fill_addr(next, Nx, Nz)] < kSentinelTest) {
                next = rand_table_entry(seed, next, n);
                continue;
            }
            mark = kFillMark + (unsigned)next;
            break;
        }
        mean_used |= mark == kFillMarkMean;
        v[a] = __uint_as_float(mark);
    }
    if (mean_used && seen) atomicOr(seen, kFlagFillMean);
}

// Grid S, 512 threads (the reference's mean is one 512-thread block's sum).
// Also ORs every slice's flags into the run summary `seen` (may be null).
__global__ void __launch_bounds__(512) k_fill_finish(float* __restrict__ vol, int Nx, int Nz,
                                                     const int* __restrict__ flags, int* __restrict__ seen)
{
    const int ys = blockIdx.x, tid = threadIdx.x;
    const int f = flags[ys];
    if (tid == 0 && seen) atomicOr(seen, f);
    if ((f & kFlagVolEmpty) == 0) return;
    const int n = Nx * Nz;
    float* v = vol + (size_t)ys * n;
    __shared__ float s_sum[512], s_cnt[512];
    float sum = 0.f, cnt = 0.f;
    for (int i = tid; i < n; i += 512) {
        const float x = v[fill_addr(i, Nx, Nz)];
        if (x < kSentinelTest) continue;
        sum = __fadd_rn(sum, x);
        cnt = __fadd_rn(cnt, 1.0f);
    }
    s_sum[tid] = sum;
    s_cnt[tid] = cnt;
    __syncthreads();
    for (int off = 256; off > 0; off >>= 1) {
        if (tid < off) {
            s_sum[tid] = __fadd_rn(s_sum[tid], s_sum[tid + off]);
            s_cnt[tid] = __fadd_rn(s_cnt[tid], s_cnt[tid + off]);
        }
        __syncthreads();
    }
    const float mean = s_cnt[0] <= 0.f ? 0.f : __fdiv_rn(s_sum[0], s_cnt[0]);
    for (int i = tid; i < n; i += 512) {
        const size_t a = fill_addr(i, Nx, Nz);
        const unsigned u = __float_as_uint(v[a]);
        if (u < kFillMark || u > kFillMarkMean) continue;
        v[a] = u == kFillMarkMean ? mean : v[fill_addr((int)(u - kFillMark), Nx, Nz)];
    }
}

// The fill's random table itself, for introspection (the oracle is driven by it).
__global__ void k_fill_table(int* __restrict__ r, int n, unsigned long long seed)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = rand_table_entry(seed, i, n);
}

// ---------------------------------------------------------------------------
// WBP Fourier crop, step 1: forward real FFT of the 2x-grid rows, keeping
// bins kx in [0, Nx/2].  Two rows per CTA as one complex sequence z = a + ib:
// A[k] = (Z[k] + conj Z[-k]) / 2, B[k] = (Z[k] - conj Z[-k]) / 2i.
// g: [slices][2Nz][2Nx]; y: [slices][2Nz][KX] with KX = Nx/2 + 1.
// B row pairs per CTA.  Grid (ceil(Nz / B), slices).
// ---------------------------------------------------------------------------
template <int RS>
__device__ __forceinline__ void row_r2c_block(const float* __restrict__ g, int Nx, int Nz, const FftPlan& plan, int B,
                                                 float2* __restrict__ y, int bx, int by)
{
    extern __shared__ float2 fsm[];
    const int pitch = fft_pitch(plan.work);
    float2* a = fsm;
    float2* b = fsm + (size_t)B * pitch;
    const int X2 = 2 * Nx, KX = Nx / 2 + 1;
    const int pr0 = bx * B, ys = by;   // row pairs (2 pr, 2 pr + 1) of the 2Nz rows
    const int nq = min(B, Nz - pr0);
    for (int q = 0; q < nq; q++) {
        const float* g0 = g + ((size_t)ys * 2 * Nz + 2 * (pr0 + q)) * X2;
        float2* aq = a + (size_t)q * pitch;
        staged_copy<4>(X2, [&](int x) { return make_float2(__ldg(g0 + x), __ldg(g0 + X2 + x)); },
                       [&](int x, float2 v) { aq[fft_pad(x)] = v; });
    }
    __syncthreads();
    const float2* Zs = fft_run<RS>(a, b, plan, nq, pitch, -1);
    for (int q = 0; q < nq; q++) {
        const float2* Z = Zs + (size_t)q * pitch;
        float2* y0 = y + ((size_t)ys * 2 * Nz + 2 * (pr0 + q)) * KX;
        for (int k = threadIdx.x; k < KX; k += blockDim.x) {
            const float2 p = Z[fft_pad(k)], qv = Z[fft_pad(k == 0 ? 0 : X2 - k)];
            // A = (p + conj q)/2 ; B = (p - conj q)/(2i) = -i (p - conj q)/2
            y0[k] = make_float2(0.5f * (p.x + qv.x), 0.5f * (p.y - qv.y));
            y0[KX + k] = make_float2(0.5f * (p.y + qv.y), -0.5f * (p.x - qv.x));
        }
    }
}

// Threads per CTA of the row and column FFT kernels: up to 1024 for the radix
// sets that fit 64 registers (where a CTA's two buffers fill an SM's shared
// memory, one CTA of 32 warps in place of 16; two CTAs of 512 otherwise), 512
// for the generic radices.  The transforms do not depend on the block size.
template <int RS>
__host__ __device__ constexpr int fft_threads_max()
{
    return RS < 2 ? 1024 : 512;
}

template <int RS>
__global__ void __launch_bounds__(fft_threads_max<RS>(), 1) k_row_r2c(const float* __restrict__ g, int Nx, int Nz, const __grid_constant__ FftPlan plan, int B,
                                                 float2* __restrict__ y)
{
    row_r2c_block<RS>(g, Nx, Nz, plan, B, y, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// WBP Fourier crop, step 2 (AreTomo/Recon/GBackProjWbp.cu:126-136,
// MaUtil/GFourierResize2D.cu:7-39): per column kx, forward FFT over the 2Nz
// rows, keep kz in [0, Nz/2] from row kz and kz in (Nz/2, Nz) from row
// kz + Nz, scale by 1/(2Nx * 2Nz) (the forward normalisation of
// MaUtil/CCufft2D.cpp:65-86), inverse FFT over Nz.  CB columns per CTA.
// y: [slices][2Nz][KX] -> w: [slices][Nz][KX].  Grid (ceil(KX/CB), slices).
// ---------------------------------------------------------------------------
template <int RS>
__device__ __forceinline__ void zcrop_block(const float2* __restrict__ y, int Nx, int Nz, int CB, int pitch,
                                               const FftPlan& p2, const FftPlan& p1, float norm, float2* __restrict__ w, int bx, int by)
{
    extern __shared__ float2 fsm[];
    const int KX = Nx / 2 + 1, Z2 = 2 * Nz;
    const int kx0 = bx * CB, ys = by;
    const int nc = min(CB, KX - kx0);
    float2* a = fsm;
    float2* b = fsm + (size_t)CB * pitch;
    const float2* ysl = y + (size_t)ys * Z2 * KX;
    staged_copy<4>(Z2 * CB,
                   [&](int idx) {
                       const int Z = idx / CB, c = idx - Z * CB;
                       return c < nc ? __ldg(ysl + (size_t)Z * KX + kx0 + c) : make_float2(0.f, 0.f);
                   },
                   [&](int idx, float2 v) {
                       const int Z = idx / CB, c = idx - Z * CB;
                       a[(size_t)c * pitch + fft_pad(Z)] = v;
                   });
    __syncthreads();
    float2* F = fft_run<RS>(a, b, p2, CB, pitch, -1);
    float2* G = (F == a) ? b : a;
    for (int idx = threadIdx.x; idx < Nz * CB; idx += blockDim.x) {
        const int c = idx / Nz, kz = idx - c * Nz;
        const int src = kz <= Nz / 2 ? kz : kz + Nz;
        const float2 v = F[(size_t)c * pitch + fft_pad(src)];
        G[(size_t)c * pitch + fft_pad(kz)] = make_float2(v.x * norm, v.y * norm);
    }
    __syncthreads();
    float2* H = fft_run<RS>(G, F, p1, CB, pitch, +1);
    float2* wsl = w + (size_t)ys * Nz * KX;
    for (int idx = threadIdx.x; idx < Nz * CB; idx += blockDim.x) {
        const int z = idx / CB, c = idx - z * CB;
        if (c < nc) wsl[(size_t)z * KX + kx0 + c] = H[(size_t)c * pitch + fft_pad(z)];
    }
}

template <int RS>
__global__ void __launch_bounds__(fft_threads_max<RS>(), 1) k_zcrop(const float2* __restrict__ y, int Nx, int Nz, int CB, int pitch,
                                               const __grid_constant__ FftPlan p2, const __grid_constant__ FftPlan p1, float norm, float2* __restrict__ w)
{
    zcrop_block<RS>(y, Nx, Nz, CB, pitch, p2, p1, norm, w, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// WBP Fourier crop, step 3 (MaUtil/CCufft2D.cpp:108-117, C2R over Nx,
// unnormalised; MaUtil/CPad2D.cpp:29-39 unpad; AreTomo/Recon/
// CDoWbpRecon.cpp:115-122 z flip).  Two rows per CTA: with the imaginary
// parts of their DC and Nyquist bins set aside, A + iB extended
// Hermitian-wise inverts to a + ib.  packed != 0 then adds what cuFFT's
// half-length packing algorithm makes of those imaginary parts:
// -(Im A0 + Im A_{Nx/2}) on even and (Im A0 - Im A_{Nx/2}) on odd samples.
// w: [slices][Nz][KX] -> vol: [slices][Nz][Nx] (row Nz-1-z).  B row pairs per
// CTA.  Grid (ceil(ceil(Nz/2) / B), slices).
// ---------------------------------------------------------------------------
template <int RS>
__device__ __forceinline__ void x_c2r_block(const float2* __restrict__ w, int Nx, int Nz, const FftPlan& plan, int B,
                                               int packed, float* __restrict__ vol, size_t vol_slice, int bx, int by)
{
    extern __shared__ float2 fsm[];
    const int pitch = fft_pitch(plan.work);
    float2* a = fsm;
    float2* b = fsm + (size_t)B * pitch;
    const int KX = Nx / 2 + 1, H = Nx / 2;
    const int pz0 = bx * B, ys = by;   // z pairs (2 pz, 2 pz + 1)
    const int nq = min(B, (Nz + 1) / 2 - pz0);
    for (int q = 0; q < nq; q++) {
        const int z0 = 2 * (pz0 + q);
        const bool two = z0 + 1 < Nz;
        const float2* A = w + ((size_t)ys * Nz + z0) * KX;
        const float2* Bv = A + KX;
        float2* aq = a + (size_t)q * pitch;
        staged_copy<4>(Nx,
                       [&](int k) {
                           const bool lo = k <= H;
                           const int kk = lo ? k : Nx - k;
                           float2 av = __ldg(A + kk);
                           float2 bv = two ? __ldg(Bv + kk) : make_float2(0.f, 0.f);
                           if (kk == 0 || kk == H) { av.y = 0.f; bv.y = 0.f; }
                           if (!lo) { av.y = -av.y; bv.y = -bv.y; }
                           return make_float2(av.x - bv.y, av.y + bv.x);   // A + iB
                       },
                       [&](int k, float2 v) { aq[fft_pad(k)] = v; });
    }
    __syncthreads();
    const float2* rs = fft_run<RS>(a, b, plan, nq, pitch, +1);
    for (int q = 0; q < nq; q++) {
        const int z0 = 2 * (pz0 + q);
        const bool two = z0 + 1 < Nz;
        const float2* A = w + ((size_t)ys * Nz + z0) * KX;
        const float2* Bv = A + KX;
        const float2* r = rs + (size_t)q * pitch;
        float ea = 0.f, oa = 0.f, eb = 0.f, ob = 0.f;
        if (packed) {
            const float ia0 = A[0].y, iah = A[H].y;
            ea = -(ia0 + iah); oa = ia0 - iah;
            if (two) { const float ib0 = Bv[0].y, ibh = Bv[H].y; eb = -(ib0 + ibh); ob = ib0 - ibh; }
        }
        float* o0 = vol + (size_t)ys * vol_slice + (size_t)(Nz - 1 - z0) * Nx;
        for (int x = threadIdx.x; x < Nx; x += blockDim.x) {
            const float2 v = r[fft_pad(x)];
            o0[x] = v.x + ((x & 1) ? oa : ea);
            if (two) o0[x - Nx] = v.y + ((x & 1) ? ob : eb);
        }
    }
}

template <int RS>
__global__ void __launch_bounds__(512, RS < 2 ? 2 : 1) k_x_c2r(const float2* __restrict__ w, int Nx, int Nz, const __grid_constant__ FftPlan plan, int B,
                                               int packed, float* __restrict__ vol, size_t vol_slice)
{
    x_c2r_block<RS>(w, Nx, Nz, plan, B, packed, vol, vol_slice, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// Batched WBP: persistent stage kernels over many series.  A wave holds one
// slab of every series in the batch (series of fewer slabs drop out of later
// waves); each of the five WBP stages runs as one launch over the whole wave,
// whose persistent CTAs pull virtual blocks — (series' slab, block of that
// stage) — from a counter until none is left, and run the same block body
// the per-series kernels run, so every result is bit-identical to the
// per-series launches.
// ---------------------------------------------------------------------------
struct WbpSlab {
    const float* proj;        // series projections [T][ny][nx]
    size_t tilt_stride;
    int row_pitch, y0;        // nx; first row of the slab
    const float2* cs;
    int T, N, Nx, Nz, S;
    const float* h;           // R-weight transfer function
    void* filt;               // staged, filtered sinogram (storage type of the batch)
    float* scale;
    int* flags;
    float* g2;                // 2x grid, then the cropped spectrum
    float2* y;                // row spectra
    float* vol;               // the slab's first output slice
    size_t vol_slice;
    int b_rweight, b_row, b_xc2r, zcrop_cb, zcrop_pitch, packed;
    float norm;
    BpArgs bp;
    FftPlan fN, f2x, f2z, fz, fx;
    int gx[5];                // virtual grid x of each stage (y is the slab's slices; the BP's y, z below)
    int bp_gy, bp_gz;
};

constexpr int kWbpStages = 5;   // rweight, bp, row_r2c, zcrop, x_c2r

// Flags of every slab of the wave to zero (run_slab_t's memset); grid = slabs.
__global__ void k_wave_flags(const WbpSlab* __restrict__ w)
{
    const WbpSlab& d = w[blockIdx.x];
    for (int i = threadIdx.x; i < d.S; i += blockDim.x) d.flags[i] = 0;
}

// Stage STAGE of a wave: start[k] is the first virtual block of slab k
// (start[nslabs] the total); counter starts at 0.
template <int STAGE, typename ST, int RS>
__global__ void __launch_bounds__(STAGE == 1 ? BP_THREADS : 512, STAGE == 1 ? 3 : (RS < 2 ? 2 : 1))
    k_wbp_wave(const WbpSlab* __restrict__ w, const int* __restrict__ start, int nslabs, int* __restrict__ counter)
{
    __shared__ int s_item;
    const int total = start[nslabs];
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= total) return;
        int lo = 0, hi = nslabs - 1;   // the slab whose block range holds item
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (start[mid] <= item) lo = mid;
            else hi = mid - 1;
        }
        const WbpSlab& d = w[lo];
        const int v = item - start[lo];
        const int bx = v % d.gx[STAGE], by = v / d.gx[STAGE];
        if constexpr (STAGE == 0) {
            rweight_block<ST, RS>(d.proj, d.tilt_stride, d.row_pitch, d.y0, d.cs, d.T, d.N, d.Nz, d.h, d.fN,
                                  d.b_rweight, static_cast<ST*>(d.filt), d.scale, d.flags, bx, by);
        } else if constexpr (STAGE == 1) {
            bp_tile<1, ST, float, false>(d.bp, bx, by % d.bp_gy, by / d.bp_gy);
        } else if constexpr (STAGE == 2) {
            row_r2c_block<RS>(d.g2, d.Nx, d.Nz, d.f2x, d.b_row, d.y, bx, by);
        } else if constexpr (STAGE == 3) {
            const float2* yv = d.y;
            zcrop_block<RS>(yv, d.Nx, d.Nz, d.zcrop_cb, d.zcrop_pitch, d.f2z, d.fz, d.norm,
                            reinterpret_cast<float2*>(d.g2), bx, by);
        } else {
            x_c2r_block<RS>(reinterpret_cast<const float2*>(d.g2), d.Nx, d.Nz, d.fx, d.b_xc2r, d.packed, d.vol,
                            d.vol_slice, bx, by);
        }
        __syncthreads();   // shared memory is reused by the next block
    }
}

}  // namespace at3r
