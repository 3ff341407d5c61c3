// The random table of the empty-pixel / empty-voxel fill, MaUtil/GGenRandoms.cu:7-20:
// entry i is drawn from subsequence i of the XORWOW generator seeded with `seed`
// (curand_init(seed, i, 0), one curand_uniform), scaled to [0, n) as
// (int)(u * n + 0.5f) % n.  Shared by the input stage's fill and SART's.
#pragma once
#include <curand_kernel.h>

namespace at3r {

__device__ __forceinline__ int rand_table_entry(unsigned long long seed, int i, int n)
{
    curandState_t st;
    curand_init(seed, (unsigned long long)i, 0ull, &st);
    const float u = curand_uniform(&st);
    const int v = (int)(u * n + 0.5f);
    return v % n;
}

}  // namespace at3r
