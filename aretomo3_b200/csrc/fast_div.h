// Multiply-shift division by a run-time constant, for index arithmetic in
// the shared-memory FFT (host planning and device code).
#pragma once
#ifndef __CUDACC__
#ifndef __host__
#define __host__
#define __device__
#endif
#endif

namespace at3r {

// Division by a stage constant d as a multiply and shift: for x < 2^24,
// floor(x / d) = (x * m) >> (24 + l) with l = ceil(log2 d), m = ceil(2^(24+l) / d)
// (the error x (m d - 2^(24+l)) / (d 2^(24+l)) stays below 2^-l <= 1/d); on
// the device (x * m) >> 24 is the high word of (x << 8) * m.
struct FastDiv {
    unsigned m;
    int l;
};
__host__ __device__ inline unsigned fast_div(unsigned x, FastDiv d)
{
#ifdef __CUDA_ARCH__
    return __umulhi(x << 8, d.m) >> d.l;
#else
    return (unsigned)(((unsigned long long)x * d.m) >> (24 + d.l));
#endif
}
inline FastDiv make_fast_div(unsigned d)
{
    int l = 0;
    while ((1u << l) < d) l++;
    const unsigned long long p = 1ull << (24 + l);
    return FastDiv{(unsigned)((p + d - 1) / d), l};
}

}  // namespace at3r
