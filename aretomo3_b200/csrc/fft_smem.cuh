// Shared-memory FFT engine for the reconstruction kernels.
//
// Complex FFTs of any length run inside one CTA on sequences staged in
// shared memory.  Lengths whose prime factors are all in {2, 3, 5, 7, 11, 13}
// use a mixed-radix Stockham autosort iteration (the formulation of
// Govindaraju et al., "High Performance Discrete Fourier Transforms on
// Graphics Processors", SC'08: butterfly j reads in[j + r*n/R], twiddles by
// exp(sign 2 pi i r (j mod Ns) / (Ns R)), writes out[(j/Ns)*Ns*R + j mod Ns + r*Ns]).
// Every other length goes through Bluestein's chirp-z transform on a
// power-of-two length m >= 2n - 1.  Twiddle and chirp tables are computed in
// double on the host and stored as float2 in device memory.
//
// Transforms are unnormalised; sign -1 is the forward (e^{-i...}) direction.
#pragma once
#include <cuda_runtime.h>

#include "fast_div.h"

namespace at3r {

constexpr int kMaxFftStages = 32;

// Sequences sit in shared memory with one spare element after every 16, so
// that the stride-R writes of the early Stockham stages (and other strided
// patterns) spread over the banks: element i of a sequence is at fft_pad(i).
__host__ __device__ constexpr int fft_pad(int i) { return i + (i >> 4); }
// Elements one padded sequence of length n occupies.
__host__ __device__ constexpr int fft_pitch(int n) { return n + ((n - 1) >> 4) + 1; }

struct FftDirect {
    int n;                       // length
    int nst;                     // number of stages
    int radix[kMaxFftStages];    // radix of each stage (product = n)
    FastDiv by_nb[kMaxFftStages];   // division by n / radix[s]
    FastDiv by_ns[kMaxFftStages];   // division by the product of the radices before stage s
    const float2* tw;            // exp(-2 pi i k / n), k in [0, n)
};

struct FftPlan {
    int n;              // logical length
    int work;           // complex elements one sequence occupies while transforming (n, or m)
    int bluestein;      // 0 direct, 1 chirp-z
    FftDirect d;        // plan of length n (direct) or m (Bluestein)
    const float2* chirp;  // [n]  exp(-i pi k^2 / n)
    const float2* bhat;   // [m]  FFT_m(conj chirp, wrapped) / m
};

// for (i = threadIdx.x; i < n; i += blockDim.x) st(i, ld(i)), U iterations at
// a time with their loads issued before their stores, so a thread waits for
// global memory once per U elements rather than once per element.
template <int U, class Ld, class St>
__device__ __forceinline__ void staged_copy(int n, Ld ld, St st)
{
    for (int i0 = threadIdx.x; i0 < n; i0 += U * blockDim.x) {
        decltype(ld(0)) v[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int i = i0 + u * blockDim.x;
            if (i < n) v[u] = ld(i);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int i = i0 + u * blockDim.x;
            if (i < n) st(i, v[u]);
        }
    }
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(__fmaf_rn(a.x, b.x, -a.y * b.y), __fmaf_rn(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i*sign... helpers: i*a and -i*a
__device__ __forceinline__ float2 mul_i(float2 a) { return make_float2(-a.y, a.x); }
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }

__device__ __forceinline__ float2 twiddle(const float2* tw, int idx, int sign)
{
    float2 w = __ldg(tw + idx);
    return sign < 0 ? w : make_float2(w.x, -w.y);
}

// R-point DFTs on registers, unnormalised, direction `sign`.
template <int R>
struct Dft;

template <>
struct Dft<2> {
    __device__ __forceinline__ static void run(float2* v, int, const float2*, int)
    {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <>
struct Dft<4> {
    __device__ __forceinline__ static void run(float2* v, int sign, const float2*, int)
    {
        float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        float2 b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
        // forward: v1 = a1 - i b1, v3 = a1 + i b1
        float2 jb1 = sign < 0 ? mul_mi(b1) : mul_i(b1);
        v[0] = cadd(a0, b0);
        v[2] = csub(a0, b0);
        v[1] = cadd(a1, jb1);
        v[3] = csub(a1, jb1);
    }
};

template <>
struct Dft<8> {
    __device__ __forceinline__ static void run(float2* v, int sign, const float2* tw, int n)
    {
        // two radix-4 on even/odd samples, then combine with W8^k
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4>::run(e, sign, tw, n);
        Dft<4>::run(o, sign, tw, n);
        const float r = 0.70710678118654752f;
        // W8^1 = (r, -r*sign'), W8^2 = -i (forward), W8^3 = (-r, -r)
        float2 w1 = make_float2(r, sign < 0 ? -r : r);
        float2 w3 = make_float2(-r, sign < 0 ? -r : r);
        float2 t0 = o[0];
        float2 t1 = cmul(o[1], w1);
        float2 t2 = sign < 0 ? mul_mi(o[2]) : mul_i(o[2]);
        float2 t3 = cmul(o[3], w3);
        v[0] = cadd(e[0], t0); v[4] = csub(e[0], t0);
        v[1] = cadd(e[1], t1); v[5] = csub(e[1], t1);
        v[2] = cadd(e[2], t2); v[6] = csub(e[2], t2);
        v[3] = cadd(e[3], t3); v[7] = csub(e[3], t3);
    }
};

template <>
struct Dft<3> {
    __device__ __forceinline__ static void run(float2* v, int sign, const float2*, int)
    {
        const float c1 = -0.5f, s1 = (sign < 0 ? -1.f : 1.f) * 0.86602540378443865f;
        float2 a = v[0], b = v[1], c = v[2];
        float2 t = cadd(b, c), d = csub(b, c);
        v[0] = cadd(a, t);
        float2 m = make_float2(__fmaf_rn(c1, t.x, a.x), __fmaf_rn(c1, t.y, a.y));
        float2 jd = make_float2(-s1 * d.y, s1 * d.x);  // i*s1*d
        v[1] = cadd(m, jd);
        v[2] = csub(m, jd);
    }
};

template <>
struct Dft<5> {
    __device__ __forceinline__ static void run(float2* v, int sign, const float2*, int)
    {
        const float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;
        const float sg = sign < 0 ? -1.f : 1.f;
        const float s1 = sg * 0.95105651629515357f, s2 = sg * 0.58778525229247313f;
        float2 a = v[0];
        float2 t1 = cadd(v[1], v[4]), d1 = csub(v[1], v[4]);
        float2 t2 = cadd(v[2], v[3]), d2 = csub(v[2], v[3]);
        v[0] = cadd(a, cadd(t1, t2));
        float2 m1 = make_float2(a.x + c1 * t1.x + c2 * t2.x, a.y + c1 * t1.y + c2 * t2.y);
        float2 m2 = make_float2(a.x + c2 * t1.x + c1 * t2.x, a.y + c2 * t1.y + c1 * t2.y);
        // i*(s1 d1 + s2 d2) and i*(s2 d1 - s1 d2)
        float2 n1 = make_float2(-(s1 * d1.y + s2 * d2.y), s1 * d1.x + s2 * d2.x);
        float2 n2 = make_float2(-(s2 * d1.y - s1 * d2.y), s2 * d1.x - s1 * d2.x);
        v[1] = cadd(m1, n1);
        v[4] = csub(m1, n1);
        v[2] = cadd(m2, n2);
        v[3] = csub(m2, n2);
    }
};

// Generic odd radix through the length-n twiddle table: W_R^k = tw[k * n/R].
template <int R>
struct DftGeneric {
    __device__ __forceinline__ static void run(float2* v, int sign, const float2* tw, int n)
    {
        float2 o[R];
        const int step = n / R;
#pragma unroll
        for (int k = 0; k < R; k++) {
            float2 acc = v[0];
#pragma unroll
            for (int r = 1; r < R; r++) {
                const int e = (r * k) % R;
                acc = cadd(acc, cmul(v[r], twiddle(tw, e * step, sign)));
            }
            o[k] = acc;
        }
#pragma unroll
        for (int k = 0; k < R; k++) v[k] = o[k];
    }
};
template <> struct Dft<7> : DftGeneric<7> {};
template <> struct Dft<11> : DftGeneric<11> {};
template <> struct Dft<13> : DftGeneric<13> {};

// One Stockham stage of radix R over `batch` sequences of length d.n stored
// with pitch `pitch` (complex elements), element i at fft_pad(i).
template <int R>
__device__ __forceinline__ void stockham_stage(const float2* __restrict__ in, float2* __restrict__ out,
                                               const FftDirect& d, int st, int Ns, int batch, int pitch, int sign)
{
    const int nb = d.n / R;
    const int total = nb * batch;
    const int twbase = d.n / (Ns * R);
    const FastDiv dnb = d.by_nb[st], dns = d.by_ns[st];
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int q = (int)fast_div((unsigned)idx, dnb);
        const int j = idx - q * nb;
        const float2* src = in + (size_t)q * pitch;
        float2* dst = out + (size_t)q * pitch;
        const int jq = (int)fast_div((unsigned)j, dns);
        const int jm = j - jq * Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = src[fft_pad(j + r * nb)];
        if (Ns > 1) {
            // one table load; the higher twiddles as its powers
            const float2 w1 = twiddle(d.tw, twbase * jm, sign);
            float2 w = w1;
#pragma unroll
            for (int r = 1; r < R; r++) {
                v[r] = cmul(v[r], w);
                if (r + 1 < R) w = cmul(w, w1);
            }
        }
        Dft<R>::run(v, sign, d.tw, d.n);
        const int od = jq * Ns * R + jm;
#pragma unroll
        for (int r = 0; r < R; r++) dst[fft_pad(od + r * Ns)] = v[r];
    }
}

// Radix sets a kernel is compiled for (fewer radices, fewer registers):
// 0 = {2, 4, 8}; 1 = {2, 3, 4, 5, 8}; 2 = every radix of the planner.
__host__ __device__ constexpr int radix_set_of(int r) { return (r == 2 || r == 4 || r == 8) ? 0 : (r == 3 || r == 5) ? 1 : 2; }

// Runs all stages, ping-ponging between a and b.  Returns the buffer that
// holds the result.  All threads of the CTA must call it.
template <int RS>
__device__ inline float2* stockham(float2* a, float2* b, const FftDirect& d, int batch, int pitch, int sign)
{
    int Ns = 1;
    for (int s = 0; s < d.nst; s++) {
        const int R = d.radix[s];
        switch (R) {
            case 2: stockham_stage<2>(a, b, d, s, Ns, batch, pitch, sign); break;
            case 4: stockham_stage<4>(a, b, d, s, Ns, batch, pitch, sign); break;
            case 8: stockham_stage<8>(a, b, d, s, Ns, batch, pitch, sign); break;
            default:
                if constexpr (RS >= 1) {
                    if (R == 3) { stockham_stage<3>(a, b, d, s, Ns, batch, pitch, sign); break; }
                    if (R == 5) { stockham_stage<5>(a, b, d, s, Ns, batch, pitch, sign); break; }
                }
                if constexpr (RS >= 2) {
                    if (R == 7) { stockham_stage<7>(a, b, d, s, Ns, batch, pitch, sign); break; }
                    if (R == 11) { stockham_stage<11>(a, b, d, s, Ns, batch, pitch, sign); break; }
                    if (R == 13) { stockham_stage<13>(a, b, d, s, Ns, batch, pitch, sign); break; }
                }
                break;  // the host launches the radix set that holds every stage
        }
        __syncthreads();
        float2* t = a; a = b; b = t;
        Ns *= R;
    }
    return a;
}

// FFT of `batch` sequences of length p.n, each starting at a + q*pitch
// (pitch >= fft_pitch(p.work)), element i at fft_pad(i).  b is scratch of the same shape.  The first p.n
// elements of each sequence of the returned buffer hold the transform.
// Caller must __syncthreads() between writing a and calling this.
template <int RS>
__device__ inline float2* fft_run(float2* a, float2* b, const FftPlan& p, int batch, int pitch, int sign)
{
    if (!p.bluestein) return stockham<RS>(a, b, p.d, batch, pitch, sign);
    const int n = p.n, m = p.d.n;
    // x_k -> x_k * c_k (forward) or conj(x_k) * c_k (inverse = conj of forward of conj), zero pad
    for (int idx = threadIdx.x; idx < m * batch; idx += blockDim.x) {
        const int q = idx / m, k = idx - q * m;
        float2* s = a + (size_t)q * pitch;
        if (k < n) {
            float2 x = s[fft_pad(k)];
            if (sign > 0) x = cconj(x);
            s[fft_pad(k)] = cmul(x, __ldg(p.chirp + k));
        } else {
            s[fft_pad(k)] = make_float2(0.f, 0.f);
        }
    }
    __syncthreads();
    float2* r = stockham<RS>(a, b, p.d, batch, pitch, -1);
    float2* o = (r == a) ? b : a;
    for (int idx = threadIdx.x; idx < m * batch; idx += blockDim.x) {
        const int q = idx / m, k = idx - q * m;
        float2* s = r + (size_t)q * pitch;
        s[fft_pad(k)] = cmul(s[fft_pad(k)], __ldg(p.bhat + k));
    }
    __syncthreads();
    r = stockham<RS>(r, o, p.d, batch, pitch, +1);
    for (int idx = threadIdx.x; idx < n * batch; idx += blockDim.x) {
        const int q = idx / n, k = idx - q * n;
        float2* s = r + (size_t)q * pitch;
        float2 y = cmul(s[fft_pad(k)], __ldg(p.chirp + k));
        s[fft_pad(k)] = sign > 0 ? cconj(y) : y;
    }
    __syncthreads();
    return r;
}

}  // namespace at3r
