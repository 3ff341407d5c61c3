// Host-side FFT planning shared by the reconstruction and input-stage
// sources: factorisation, twiddle and Bluestein tables for fft_smem.cuh, the
// radix-set dispatch of the FFT kernels, and the probe of the system cuFFT's
// complex-to-real convention.
#pragma once
#include "at3r.h"
#include "fft_smem.cuh"

#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

namespace at3r {

// ---------------------------------------------------------------------------
// FFT planning: factor n into radices {8, 4, 2, 3, 5, 7, 11, 13}; any other
// prime factor sends the length through Bluestein on m = 2^k >= 2n - 1.
// ---------------------------------------------------------------------------
inline bool factor_direct(int n, std::vector<int>& rad)
{
    rad.clear();
    int m = n;
    while (m % 8 == 0) { rad.push_back(8); m /= 8; }
    if (m % 4 == 0) { rad.push_back(4); m /= 4; }
    if (m % 2 == 0) { rad.push_back(2); m /= 2; }
    for (int p : {3, 5, 7, 11, 13})
        while (m % p == 0) { rad.push_back(p); m /= p; }
    if (n == 1) rad.push_back(1);
    return m == 1 && (int)rad.size() <= kMaxFftStages;
}

struct HostFft {
    int rs = 0;          // radix set of its stages (radix_set_of)
    size_t n_tw = 0, n_chirp = 0;   // table lengths, for bind_fft
    FftPlan plan{};
    float2* d_tables = nullptr;  // twiddles, chirp, bhat in one allocation
    size_t bytes = 0;
};

inline void fill_twiddles(std::vector<float2>& v, int n)
{
    v.resize(n);
    for (int k = 0; k < n; k++) {
        const double a = -2.0 * M_PI * (double)k / (double)n;
        v[k] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
}

// Reference FFT in double for the Bluestein kernel spectrum (host only).
inline void host_fft_pow2(std::vector<std::complex<double>>& a, int sign)
{
    const int n = (int)a.size();
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (int len = 2; len <= n; len <<= 1) {
        const double ang = sign * 2.0 * M_PI / len;
        for (int i = 0; i < n; i += len)
            for (int k = 0; k < len / 2; k++) {
                std::complex<double> w(std::cos(ang * k), std::sin(ang * k));
                auto u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
    }
}

// Calls f with std::integral_constant<int, rs> for the kernels compiled for
// radix set rs (see radix_set_of).
template <class F>
void dispatch_rs(int rs, F&& f)
{
    switch (rs) {
        case 0: f(std::integral_constant<int, 0>{}); break;
        case 1: f(std::integral_constant<int, 1>{}); break;
        default: f(std::integral_constant<int, 2>{}); break;
    }
}

// Per-stage divisors of the Stockham index arithmetic.
inline void set_stage_divs(FftDirect& d)
{
    int ns = 1;
    for (int i = 0; i < d.nst; i++) {
        d.by_nb[i] = make_fast_div((unsigned)(d.n / d.radix[i]));
        d.by_ns[i] = make_fast_div((unsigned)ns);
        ns *= d.radix[i];
    }
}

// Host half of a plan of length n: radices, stage divisors and the twiddle /
// chirp / Bluestein-kernel tables, laid out [tw | chirp | bhat] in `tables`
// for one device allocation of h.bytes.
inline void plan_fft(int n, HostFft& h, std::vector<float2>& tables)
{
    std::vector<int> rad;
    FftPlan& p = h.plan;
    p.n = n;
    std::vector<float2> tw, chirp, bhat;
    if (factor_direct(n, rad)) {
        p.bluestein = 0;
        p.work = n;
        p.d.n = n;
        p.d.nst = (n == 1) ? 0 : (int)rad.size();
        for (int i = 0; i < p.d.nst; i++) p.d.radix[i] = rad[i];
        set_stage_divs(p.d);
        h.rs = 0;
        for (int i = 0; i < p.d.nst; i++) h.rs = std::max(h.rs, radix_set_of(p.d.radix[i]));
        fill_twiddles(tw, n);
    } else {
        int m = 1;
        while (m < 2 * n - 1) m <<= 1;
        factor_direct(m, rad);
        p.bluestein = 1;
        p.work = m;
        p.d.n = m;
        p.d.nst = (int)rad.size();
        for (int i = 0; i < p.d.nst; i++) p.d.radix[i] = rad[i];
        set_stage_divs(p.d);
        h.rs = 0;   // a power of two
        fill_twiddles(tw, m);
        chirp.resize(n);
        std::vector<std::complex<double>> cd(n);
        for (int k = 0; k < n; k++) {
            const long long k2 = ((long long)k * k) % (2LL * n);
            const double a = -M_PI * (double)k2 / n;
            cd[k] = {std::cos(a), std::sin(a)};
            chirp[k] = make_float2((float)cd[k].real(), (float)cd[k].imag());
        }
        std::vector<std::complex<double>> b(m, 0.0);
        b[0] = std::conj(cd[0]);
        for (int k = 1; k < n; k++) b[k] = b[m - k] = std::conj(cd[k]);
        host_fft_pow2(b, -1);
        bhat.resize(m);
        for (int k = 0; k < m; k++) bhat[k] = make_float2((float)(b[k].real() / m), (float)(b[k].imag() / m));
    }
    h.n_tw = tw.size();
    h.n_chirp = chirp.size();
    tables.clear();
    tables.reserve(tw.size() + chirp.size() + bhat.size());
    tables.insert(tables.end(), tw.begin(), tw.end());
    tables.insert(tables.end(), chirp.begin(), chirp.end());
    tables.insert(tables.end(), bhat.begin(), bhat.end());
    h.bytes = tables.size() * sizeof(float2);
}

// Points the plan at its tables once they sit at h.d_tables.
inline void bind_fft(HostFft& h)
{
    FftPlan& p = h.plan;
    p.d.tw = h.d_tables;
    p.chirp = p.bluestein ? h.d_tables + h.n_tw : nullptr;
    p.bhat = p.bluestein ? h.d_tables + h.n_tw + h.n_chirp : nullptr;
}

// ---------------------------------------------------------------------------
// Which convention does the system cuFFT use for a 2-D C2R of (nz x nx)?
// A pure-imaginary DC bin is invisible under the Hermitian reading and shows
// up as -1/+1 on even/odd samples under half-length packing.  libcufft is
// opened at run time, only for this question, once per size and process.
// The probe runs on a stream of its own with stream-ordered memory and keeps
// its cuFFT plan (destroying one frees cuFFT's tables with a cudaFree, which
// would wait for the whole device), so it never synchronises other streams.
// *measured (may be null) tells whether cuFFT answered; when it cannot be
// loaded the Hermitian reading is assumed.
// ---------------------------------------------------------------------------
inline int probe_cufft_c2r(int nz, int nx, bool* measured = nullptr)
{
    static std::mutex mu;
    static std::map<std::pair<int, int>, std::pair<int, bool>> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair(nz, nx);
    auto it = cache.find(key);
    if (it != cache.end()) {
        if (measured) *measured = it->second.second;
        return it->second.first;
    }
    typedef int (*create_t)(int*);
    typedef int (*setauto_t)(int, int);
    typedef int (*make2d_t)(int, int, int, int, size_t*);
    typedef int (*setwork_t)(int, void*);
    typedef int (*setstream_t)(int, cudaStream_t);
    typedef int (*exec_t)(int, void*, float*);
    static void* lib = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        for (const char* name : {"/usr/local/cuda/lib64/libcufft.so.11", "libcufft.so.11", "libcufft.so.12", "libcufft.so"}) {
            lib = dlopen(name, RTLD_NOW | RTLD_LOCAL);
            if (lib) break;
        }
    }
    int result = AT3R_C2R_HERMITIAN;
    bool ok = false;
    if (lib) {
        auto create = (create_t)dlsym(lib, "cufftCreate");
        auto setauto = (setauto_t)dlsym(lib, "cufftSetAutoAllocation");
        auto make2d = (make2d_t)dlsym(lib, "cufftMakePlan2d");
        auto setwork = (setwork_t)dlsym(lib, "cufftSetWorkArea");
        auto setstream = (setstream_t)dlsym(lib, "cufftSetStream");
        auto exec = (exec_t)dlsym(lib, "cufftExecC2R");
        cudaStream_t st = nullptr;
        int plan = 0;
        size_t work = 0;
        if (create && setauto && make2d && setwork && setstream && exec &&
            cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess && create(&plan) == 0 &&
            setauto(plan, 0) == 0 && make2d(plan, nz, nx, 0x2c /* CUFFT_C2R */, &work) == 0) {
            const size_t elems = (size_t)nz * (nx / 2 + 1);
            const size_t data_bytes = (elems * sizeof(float2) + 255) / 256 * 256;
            char* d = nullptr;
            if (cudaMallocAsync(reinterpret_cast<void**>(&d), data_bytes + work, st) == cudaSuccess) {
                static const float2 one_i = make_float2(0.f, 1.f);
                float o[2] = {0.f, 0.f};
                if (cudaMemsetAsync(d, 0, elems * sizeof(float2), st) == cudaSuccess &&
                    cudaMemcpyAsync(d, &one_i, sizeof(float2), cudaMemcpyHostToDevice, st) == cudaSuccess &&
                    setwork(plan, work ? d + data_bytes : nullptr) == 0 && setstream(plan, st) == 0 &&
                    exec(plan, d, reinterpret_cast<float*>(d)) == 0 &&
                    cudaMemcpyAsync(o, d, sizeof(o), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
                    cudaStreamSynchronize(st) == cudaSuccess) {
                    ok = true;
                    if (std::fabs(o[0]) > 0.5f) result = AT3R_C2R_PACKED;
                }
                cudaFreeAsync(d, st);
                cudaStreamSynchronize(st);
            }
        }
        if (st) cudaStreamDestroy(st);
        cudaGetLastError();
    }
    cache[key] = {result, ok};
    if (measured) *measured = ok;
    return result;
}

}  // namespace at3r
