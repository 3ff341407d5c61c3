// TEST INFRASTRUCTURE — NOT THE PRODUCT.  CPU restatement of AreTomo3's
// AreTomo/Recon path, used only as the checker (FP64) and as the timed CPU
// baseline (FP32).  See recon_oracle.h for the conventions.
//
// Each function cites the reference code it restates (paths relative to the
// AreTomo3 source tree).
#include "recon_oracle.h"

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

int g_c2r_mode = 0;
// Threads the loops inside one y-slice use.  The *_run entry points spread
// slices over the threads when there are at least as many slices as threads,
// and otherwise run the slices one after another with the threads inside each
// (a 4096-wide SART slice is tens of seconds on one core).
int g_inner = 1;
constexpr float kSentinelTest = -1e10f;   // "empty" test used throughout the reference
constexpr float kSentinelValue = -1e30f;  // value written for an empty result

// ---------------------------------------------------------------------------
// FFT: iterative radix-2 for powers of two, Bluestein's chirp-z for every
// other length (L. Bluestein, "A linear filtering approach to the computation
// of the discrete Fourier transform", 1970).  Tables are built in double.
// The reference uses cuFFT (MaUtil/GFFT1D.cu:45-88, MaUtil/CCufft2D.cpp:23-117);
// only the mathematical transform matters here.
// ---------------------------------------------------------------------------
struct PlanD {
    int n = 0, m = 0;
    bool pow2 = false;
    std::vector<std::complex<double>> tw;      // exp(-2 pi i j / size), size = n or m
    std::vector<std::complex<double>> chirp;   // exp(-i pi k^2 / n)
    std::vector<std::complex<double>> bhat;    // FFT_m of conj(chirp) wrapped
};

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

template <class R>
void fft_pow2(std::complex<R>* a, int n, int sign, const std::vector<std::complex<double>>& tw)
{
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    const int tsz = (int)tw.size();
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1, step = (2 * tsz) / len;
        for (int i = 0; i < n; i += len)
            for (int k = 0; k < half; k++) {
                std::complex<double> w = tw[(size_t)k * step];
                if (sign > 0) w = std::conj(w);
                std::complex<R> wr((R)w.real(), (R)w.imag());
                std::complex<R> u = a[i + k], v = a[i + k + half] * wr;
                a[i + k] = u + v;
                a[i + k + half] = u - v;
            }
    }
}

std::shared_ptr<PlanD> get_plan(int n)
{
    static std::mutex mu;
    static std::map<int, std::shared_ptr<PlanD>> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(n);
    if (it != cache.end()) return it->second;
    auto p = std::make_shared<PlanD>();
    p->n = n;
    p->pow2 = is_pow2(n);
    int sz = n;
    if (!p->pow2) {
        int m = 1;
        while (m < 2 * n - 1) m <<= 1;
        p->m = m;
        sz = m;
    }
    p->tw.resize(sz / 2 > 0 ? sz / 2 : 1);
    for (int j = 0; j < (int)p->tw.size(); j++) {
        double a = -2.0 * M_PI * j / sz;
        p->tw[j] = {std::cos(a), std::sin(a)};
    }
    if (!p->pow2) {
        p->chirp.resize(n);
        for (int k = 0; k < n; k++) {
            int64_t k2 = ((int64_t)k * k) % (2 * (int64_t)n);
            double a = -M_PI * (double)k2 / n;
            p->chirp[k] = {std::cos(a), std::sin(a)};
        }
        std::vector<std::complex<double>> b(p->m, 0.0);
        b[0] = std::conj(p->chirp[0]);
        for (int k = 1; k < n; k++) b[k] = b[p->m - k] = std::conj(p->chirp[k]);
        fft_pow2<double>(b.data(), p->m, -1, p->tw);
        p->bhat = std::move(b);
    }
    cache[n] = p;
    return p;
}

// Complex FFT of length n in place, unnormalised.  sign -1: forward.
template <class R>
void fft(std::complex<R>* a, int n, int sign)
{
    if (n <= 1) return;
    auto p = get_plan(n);
    if (p->pow2) { fft_pow2<R>(a, n, sign, p->tw); return; }
    // forward uses the chirp, inverse its conjugate: X = c_k (a c) * conj(c)
    const int m = p->m;
    std::vector<std::complex<R>> buf(m, std::complex<R>(0, 0));
    for (int k = 0; k < n; k++) {
        std::complex<double> c = sign < 0 ? p->chirp[k] : std::conj(p->chirp[k]);
        buf[k] = a[k] * std::complex<R>((R)c.real(), (R)c.imag());
    }
    fft_pow2<R>(buf.data(), m, -1, p->tw);
    for (int k = 0; k < m; k++) {
        std::complex<double> b = sign < 0 ? p->bhat[k] : std::conj(p->bhat[(m - k) % m]);
        buf[k] *= std::complex<R>((R)b.real(), (R)b.imag());
    }
    fft_pow2<R>(buf.data(), m, +1, p->tw);
    const R inv = (R)(1.0 / m);
    for (int k = 0; k < n; k++) {
        std::complex<double> c = sign < 0 ? p->chirp[k] : std::conj(p->chirp[k]);
        a[k] = buf[k] * inv * std::complex<R>((R)c.real(), (R)c.imag());
    }
}

// Real inverse FFT of even length n from bins [0, n/2], unnormalised, under
// the selected treatment of imaginary parts in the DC and Nyquist bins.
template <class R>
void c2r(const std::complex<R>* X, int n, R* out, int mode)
{
    if (mode == 1 && n % 2 == 0) {
        // half-length complex packing: Z[k] = (X[k] + conj X[M-k]) + i e^{+2 pi i k/n} (X[k] - conj X[M-k])
        const int M = n / 2;
        std::vector<std::complex<R>> z(M);
        for (int k = 0; k < M; k++) {
            std::complex<R> a = X[k], b = std::conj(X[M - k]);
            double ang = 2.0 * M_PI * k / n;
            std::complex<R> w((R)std::cos(ang), (R)std::sin(ang));
            z[k] = (a + b) + std::complex<R>(0, 1) * (w * (a - b));
        }
        fft<R>(z.data(), M, +1);
        for (int k = 0; k < M; k++) {
            out[2 * k] = z[k].real();
            out[2 * k + 1] = z[k].imag();
        }
        return;
    }
    std::vector<std::complex<R>> full(n);
    for (int k = 0; k <= n / 2; k++) full[k] = X[k];
    for (int k = n / 2 + 1; k < n; k++) full[k] = std::conj(X[n - k]);
    fft<R>(full.data(), n, +1);
    for (int k = 0; k < n; k++) out[k] = full[k].real();
}

// ---------------------------------------------------------------------------
// Geometry table: AreTomo/Recon/CTomoBase.cpp:56-65.  The angle is the float
// product with the truncated constant 0.017453f; cos/sin of a float argument
// resolve to the float overloads in the reference's C++ build.
// ---------------------------------------------------------------------------
void cos_sin_table(const float* tilts, int n, float* cs)
{
    const float fRad = 0.017453f;
    for (int i = 0; i < n; i++) {
        float a = fRad * tilts[i];
        cs[2 * i] = std::cos(a);
        cs[2 * i + 1] = std::sin(a);
    }
}

// R-weight transfer function, AreTomo/Recon/GRWeight.cu:7-23 (normalisation
// 1/N folded in; the reference's 2*pi constant 6.2831852f).
template <class R>
void rweight_filter(int N, std::vector<R>& h)
{
    h.resize(N / 2 + 1);
    const double twopi = (double)6.2831852f;
    for (int k = 0; k <= N / 2; k++) {
        double f = (double)k / N;
        h[k] = (R)((1.0 / N) * 2.0 * f * (0.55 + 0.45 * std::cos(twopi * f)));
    }
}

// One row of the R-weight: R2C, multiply, C2R (GRWeight.cu:62-69, GFFT1D.cu:62-88).
template <class R>
void rweight_row(R* row, int N, const std::vector<R>& h, std::vector<std::complex<R>>& work)
{
    work.assign(N, std::complex<R>(0, 0));
    for (int x = 0; x < N; x++) work[x] = std::complex<R>(row[x], 0);
    fft<R>(work.data(), N, -1);
    for (int k = 0; k <= N / 2; k++) work[k] *= h[k];
    // the spectrum of a real row is Hermitian: its DC/Nyquist bins are real
    work[0] = std::complex<R>(work[0].real(), 0);
    work[N / 2] = std::complex<R>(work[N / 2].real(), 0);
    c2r<R>(work.data(), N, row, 0);
}

// 2x-grid weighted back-projection, AreTomo/Recon/GBackProjWbp.cu:14-53.
// sino: [T][N] filtered rows; g: [2Nz][2Nx].  Which samples enter a voxel
// (the bounds test and the integer index) is decided in FP32 exactly as the
// reference's kernel evaluates xp (the x*cos product fused with the add); the
// interpolation weight and the sums are carried in R.
template <class R>
void bp_wbp_2x(const R* sino, int N, int T, const float* cs, int Nx, int Nz, R* g)
{
    const int X2 = 2 * Nx, Z2 = 2 * Nz;
    const R cent = (R)(N / 2);
    const float centf = (float)(N / 2);
    const int endX = N - 2;
#pragma omp parallel for schedule(static) num_threads(g_inner) if (g_inner > 1)
    for (int Z = 0; Z < Z2; Z++) {
        const R fZ = (R)(Z - Nz);
        const float fZf = (float)Z - (float)Z2 / 2.0f;
        for (int X = 0; X < X2; X++) {
            const R fX = (R)(X - Nx);
            const float fXf = (float)X - (float)X2 / 2.0f;
            R sum = 0;
            int cnt = 0;
            for (int t = 0; t < T; t++) {
                const float c = cs[2 * t], s = cs[2 * t + 1];
                const float xf = std::fma(fXf, c, fZf * s) / 2.0f + centf + 0.5f;
                if (xf < 0 || xf > endX) continue;
                const int i = (int)xf;
                const R xp = (fX * (R)c + fZ * (R)s) / (R)2 + cent + (R)0.5;
                // where the reference's FP32 fraction is exactly 0 the second
                // sample has weight 0 (a -1e30 there contributes nothing)
                const R w = xf == (float)i ? (R)0 : xp - i;
                const R* p = sino + (size_t)t * N + i;
                R v = p[0] * (1 - w) + p[1] * w;
                if (v <= (R)kSentinelTest) continue;
                sum += v;
                cnt++;
            }
            g[(size_t)Z * X2 + X] = cnt > 0 ? sum / (R)cnt : (R)0;
        }
    }
}

// 2x -> 1x Fourier crop, AreTomo/Recon/GBackProjWbp.cu:124-142:
// R2C 2-D forward on (2Nz x 2Nx) normalised by 1/(4 Nx Nz) (MaUtil/CCufft2D.cpp:65-86),
// low-frequency block copy (MaUtil/GFourierResize2D.cu:7-39), C2R 2-D inverse
// on (Nz x Nx), unnormalised (MaUtil/CCufft2D.cpp:108-117), unpad (MaUtil/CPad2D.cpp:29-39).
template <class R>
void fourier_crop(const R* g, int Nx, int Nz, R* f, int mode)
{
    const int X2 = 2 * Nx, Z2 = 2 * Nz, KX = Nx / 2 + 1;
    std::vector<std::complex<R>> rows((size_t)Z2 * KX);
#pragma omp parallel num_threads(g_inner) if (g_inner > 1)
    {
        std::vector<std::complex<R>> line(X2);
#pragma omp for schedule(static)
        for (int Z = 0; Z < Z2; Z++) {
            for (int X = 0; X < X2; X++) line[X] = std::complex<R>(g[(size_t)Z * X2 + X], 0);
            fft<R>(line.data(), X2, -1);
            for (int k = 0; k < KX; k++) rows[(size_t)Z * KX + k] = line[k];
        }
    }
    const R norm = (R)(1.0 / X2 / Z2);
    std::vector<std::complex<R>> crop((size_t)Nz * KX);
#pragma omp parallel num_threads(g_inner) if (g_inner > 1)
    {
        std::vector<std::complex<R>> col(Z2), col2(Nz);
#pragma omp for schedule(static)
        for (int k = 0; k < KX; k++) {
            for (int Z = 0; Z < Z2; Z++) col[Z] = rows[(size_t)Z * KX + k];
            fft<R>(col.data(), Z2, -1);
            for (int kz = 0; kz < Nz; kz++) {
                int src = kz <= Nz / 2 ? kz : kz + Nz;
                col2[kz] = col[src] * norm;
            }
            fft<R>(col2.data(), Nz, +1);
            for (int z = 0; z < Nz; z++) crop[(size_t)z * KX + k] = col2[z];
        }
    }
#pragma omp parallel for schedule(static) num_threads(g_inner) if (g_inner > 1)
    for (int z = 0; z < Nz; z++) c2r<R>(&crop[(size_t)z * KX], Nx, f + (size_t)z * Nx, mode);
}

template <class R>
void wbp_slice(const float* frames, int nx, int ny, int T, const float* cs, int Nz, int y,
               const std::vector<R>& h, R* out)
{
    const int N = nx & ~1, Nx = N;
    std::vector<R> sino((size_t)T * N);
#pragma omp parallel num_threads(g_inner) if (g_inner > 1)
    {
        std::vector<std::complex<R>> work;
#pragma omp for schedule(static)
        for (int t = 0; t < T; t++) {
            const float* src = frames + ((size_t)t * ny + y) * nx;
            R* row = sino.data() + (size_t)t * N;
            // AreTomo/Recon/GWeightProjs.cu:18
            const R wgt = (R)cs[2 * t] / (R)Nz;
            for (int x = 0; x < N; x++) row[x] = (R)src[x] * wgt;
            rweight_row<R>(row, N, h, work);
        }
    }
    std::vector<R> g((size_t)4 * Nx * Nz), f((size_t)Nx * Nz);
    bp_wbp_2x<R>(sino.data(), N, T, cs, Nx, Nz, g.data());
    fourier_crop<R>(g.data(), Nx, Nz, f.data(), g_c2r_mode);
    // z flip, AreTomo/Recon/CDoWbpRecon.cpp:115-122
    for (int z = 0; z < Nz; z++)
        std::memcpy(out + (size_t)(Nz - 1 - z) * Nx, f.data() + (size_t)z * Nx, sizeof(R) * Nx);
}

// SART back-projection, AreTomo/Recon/GBackProj.cu:12-60 (bSart = true).
// Sample selection in FP32 as the reference's kernel does it; values in R.
template <class R>
void bp_sart(const R* sino, int N, const float* cs, int start, int end, R relax, int Nx, int Nz, R* vol)
{
    const R cent = (R)N / (R)2;
    const float centf = (float)N / 2.0f;
    const int endX = N - 2;
#pragma omp parallel for schedule(static) num_threads(g_inner) if (g_inner > 1)
    for (int Z = 0; Z < Nz; Z++) {
        const R fZ = (R)Z - (R)Nz * (R)0.5;
        const float fZf = (float)Z - (float)Nz * 0.5f;
        for (int X = 0; X < Nx; X++) {
            const R fX = (R)X - (R)Nx * (R)0.5;
            const float fXf = (float)X - (float)Nx * 0.5f;
            R sum = 0;
            int cnt = 0;
            for (int t = start; t < end; t++) {
                const float c = cs[2 * t], s = cs[2 * t + 1];
                const float xf = std::fma(fXf, c, fZf * s) + centf;
                if (xf < 0 || xf > endX) continue;
                const int i = (int)xf;
                const R xp = fX * (R)c + fZ * (R)s + cent;
                const R w = xf == (float)i ? (R)0 : xp - i;   // as in bp_wbp_2x
                const R* p = sino + (size_t)t * N + i;
                R v = p[0] * (1 - w) + p[1] * w;
                if (v <= (R)kSentinelTest) continue;
                sum += v;
                cnt++;
            }
            if (cnt <= 0) continue;
            R& vox = vol[(size_t)Z * Nx + X];
            R nv = relax * sum / (R)cnt + vox;
            vox = nv > (R)kSentinelTest ? std::max(nv, (R)0) : (R)kSentinelValue;
        }
    }
}

// Forward projection of tilts [start, end), AreTomo/Recon/GForProj.cu:10-76.
// The ray length, the in-volume test and the cell index are computed in FP32
// as the reference does; sample positions' fractions (zero where the FP32
// fraction is zero) and the sums in R.
template <class R>
void forward_project(const R* vol, int Nx, int Nz, int N, const float* cs, int start, int end, R* fp)
{
    const int endX = Nx - 2, endZ = Nz - 2;
    for (int t = start; t < end; t++) {
        const float fc = cs[2 * t], fs = cs[2 * t + 1];
        const int L = (int)((float)Nz / fc + 1.5f);
        const R c = (R)fc, s = (R)fs;
        const R halfL = (R)L * (R)0.5;
        const float halfLf = (float)L * 0.5f;
        const float tzf = (float)Nz * 0.5f;
#pragma omp parallel for schedule(static) num_threads(g_inner) if (g_inner > 1)
        for (int u = 0; u < N; u++) {
            const float fXpf = (float)u - 0.5f * (float)N;
            const float txf = fXpf / fc + (float)Nx * 0.5f;
            const R fXp = (R)u - (R)0.5 * (R)N;
            const R tx = fXp / c + (R)Nx * (R)0.5;
            const R tz = (R)Nz * (R)0.5;
            R sum = 0, cnt = 0;
            for (int i = 0; i < L; i++) {
                const float z0f = (float)i - halfLf;
                const float xf = std::fma(-z0f, fs, txf);
                const float zf = std::fma(z0f, fc, tzf);
                if (xf < 0 || zf < 0 || xf > endX || zf > endZ) continue;
                const int ix = (int)xf, iz = (int)zf;
                const R z0 = (R)i - halfL;
                // zero where the reference's FP32 fraction is exactly zero, so a
                // -1e30 voxel of weight 0 adds nothing, as in the reference
                const R wx = xf == (float)ix ? (R)0 : (tx - z0 * s) - ix;
                const R wz = zf == (float)iz ? (R)0 : (tz + z0 * c) - iz;
                const R* v = vol + (size_t)iz * Nx + ix;
                R val = v[0] * (1 - wx) * (1 - wz) + v[1] * wx * (1 - wz) + v[Nx] * (1 - wx) * wz +
                        v[Nx + 1] * wx * wz;
                if (val < (R)kSentinelTest) continue;
                sum += val;
                cnt += 1;
            }
            fp[(size_t)t * N + u] = cnt <= 0 ? (R)kSentinelValue : sum / cnt;
        }
    }
}

// The fill's random table (MaUtil/GGenRandoms.cu, drawn once per series by
// CTomoBase::Setup -> GFillEmpty2D::SetSize): entry i = the voxel index the
// chain of voxel i starts at, for the Nx*Nz voxels of an XZ slice in the
// reference's order (i = Z*Nx + X, before the z flip).  Set by the caller
// from the table the device drew (the oracle has no cuRAND); without one,
// every empty voxel takes the slice mean.
std::vector<int> g_fill_table;

// MaUtil/GFillEmpty2D.cu:7-143 on one slice vol[Z][X]: voxels below -1e10
// are empty (mGFindEmpty); the mean of the others is summed in float by one
// 512-thread block, thread t taking voxels t, t+512, ... in index order, then
// a tree over the threads (mGCalcMean); an empty voxel follows its chain
// through the table (at most 100 links) to the first non-empty voxel and
// takes its value, else the mean (mGFillEmpty2D).  Only empty voxels are
// written and only non-empty ones read, so the result is order-free.
template <class R>
void fill_empty(R* vol, int Nx, int Nz)
{
    const int n = Nx * Nz;
    std::vector<unsigned char> empty(n);
    bool any = false;
    for (int i = 0; i < n; i++) {
        empty[i] = vol[i] < (R)kSentinelTest;
        any |= empty[i] != 0;
    }
    if (!any) return;
    float s[512], c[512];
    for (int t = 0; t < 512; t++) {
        float sum = 0.f, cnt = 0.f;
        for (int i = t; i < n; i += 512) {
            if (empty[i]) continue;
            sum += (float)vol[i];
            cnt += 1.0f;
        }
        s[t] = sum;
        c[t] = cnt;
    }
    for (int off = 256; off > 0; off >>= 1)
        for (int t = 0; t < off; t++) {
            s[t] += s[t + off];
            c[t] += c[t + off];
        }
    const R mean = c[0] <= 0.f ? (R)0 : (R)(s[0] / c[0]);
    const bool chains = (int)g_fill_table.size() == n;
    std::vector<R> out(vol, vol + n);
    for (int i = 0; i < n; i++) {
        if (!empty[i]) continue;
        R v = mean;
        if (chains) {
            int next = g_fill_table[i];
            for (int j = 0; j < 100; j++) {
                if (empty[next]) {
                    next = g_fill_table[next];
                    continue;
                }
                v = vol[next];
                break;
            }
        }
        out[i] = v;
    }
    std::copy(out.begin(), out.end(), vol);
}

// AreTomo/Util/CSplitItems.cpp:25-48
void split_items(int n, int k, std::vector<int>& starts, std::vector<int>& sizes)
{
    starts.assign(k, 0);
    sizes.assign(k, n / k);
    for (int i = 0; i < n % k; i++) sizes[i] += 1;
    for (int i = 1; i < k; i++) starts[i] = starts[i - 1] + sizes[i - 1];
}

// AreTomo/Recon/CTomoSart.cpp:54-125 for one y-slice.
template <class R>
void sart_slice(const float* frames, int nx, int ny, int T, const float* cs, int Nz, int y, int start_tilt,
                int num_tilts, int iters, int subsets, R relax, R* out, double* rf)
{
    const int N = nx & ~1, Nx = N;
    std::vector<R> raw((size_t)T * N), fp((size_t)T * N, (R)0), vol((size_t)Nx * Nz, (R)0);
    for (int t = 0; t < T; t++) {
        const float* src = frames + ((size_t)t * ny + y) * nx;
        const R wgt = (R)cs[2 * t] / (R)Nz;
        for (int x = 0; x < N; x++) raw[(size_t)t * N + x] = (R)src[x] * wgt;
    }
    std::vector<int> starts, sizes;
    split_items(num_tilts, subsets, starts, sizes);
    bp_sart<R>(raw.data(), N, cs, 0, T, (R)1, Nx, Nz, vol.data());
    for (int it = 0; it < iters; it++) {
        for (int s = 0; s < subsets; s++) {
            const int t0 = starts[s] + start_tilt, t1 = t0 + sizes[s];
            if (t1 <= t0) continue;  // an empty subset changes nothing
            forward_project<R>(vol.data(), Nx, Nz, N, cs, t0, t1, fp.data());
            // AreTomo/Recon/GDiffProj.cu:17-20, in place over the forward projections
            double sd = 0, sr = 0;
            for (int t = t0; t < t1; t++)
                for (int u = 0; u < N; u++) {
                    R& d = fp[(size_t)t * N + u];
                    const R r = raw[(size_t)t * N + u];
                    if (d < (R)kSentinelTest || r < (R)kSentinelTest) { d = 0; continue; }
                    d = r - d;
                    sd += std::fabs((double)d);
                    sr += std::fabs((double)r);
                }
            if (rf) { rf[2 * it] += sd; rf[2 * it + 1] += sr; }
            bp_sart<R>(fp.data(), N, cs, t0, t1, relax, Nx, Nz, vol.data());
        }
    }
    // CTomoSart.cpp:88: the empty-voxel fill of the slice
    fill_empty<R>(vol.data(), Nx, Nz);
    for (int z = 0; z < Nz; z++)
        std::memcpy(out + (size_t)(Nz - 1 - z) * Nx, vol.data() + (size_t)z * Nx, sizeof(R) * Nx);
}

int check_common(const float* frames, int nx, int ny, int T, const float* tilts, int vol_z, int y0, int y1,
                 const void* out)
{
    if (!frames || !tilts || !out) return -1;
    if (nx < 2 || ny < 1 || T < 1 || vol_z < 1) return -2;
    if (y0 < 0 || y1 > ny || y0 >= y1) return -3;
    return 0;
}

template <class R>
int wbp_run(const float* frames, int nx, int ny, int T, const float* tilts, int vol_z, int y0, int y1, R* out,
            int nthreads)
{
    int rc = check_common(frames, nx, ny, T, tilts, vol_z, y0, y1, out);
    if (rc) return rc;
    std::vector<float> cs(2 * T);
    cos_sin_table(tilts, T, cs.data());
    const int Nx = nx & ~1;
    std::vector<R> h;
    rweight_filter<R>(Nx, h);
    get_plan(Nx); get_plan(2 * Nx); get_plan(2 * vol_z); get_plan(vol_z); get_plan(Nx / 2);
    const int nth = nthreads > 0 ? nthreads : 1;
    g_inner = (y1 - y0) < nth ? nth : 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_inner > 1 ? 1 : nth)
    for (int y = y0; y < y1; y++)
        wbp_slice<R>(frames, nx, ny, T, cs.data(), vol_z, y, h, out + (size_t)(y - y0) * Nx * vol_z);
    g_inner = 1;
    return 0;
}

template <class R>
int sart_run(const float* frames, int nx, int ny, int T, const float* tilts, int vol_z, int start, int num,
             int iters, int subsets, double relax, int y0, int y1, R* out, double* rf, int nthreads)
{
    int rc = check_common(frames, nx, ny, T, tilts, vol_z, y0, y1, out);
    if (rc) return rc;
    if (subsets < 1 || iters < 0 || start < 0 || num < 0 || start + num > T) return -4;
    std::vector<float> cs(2 * T);
    cos_sin_table(tilts, T, cs.data());
    const int Nx = nx & ~1;
    // CTomoSart.cpp:71 — the float 1/nSubsets unless overridden
    const R rlx = relax > 0 ? (R)relax : (R)(1.0f / (float)subsets);
    if (rf) std::memset(rf, 0, sizeof(double) * 2 * iters);
    const int nth = nthreads > 0 ? nthreads : 1;
    std::vector<std::vector<double>> rfs(nth, std::vector<double>(2 * (iters > 0 ? iters : 1), 0.0));
    g_inner = (y1 - y0) < nth ? nth : 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_inner > 1 ? 1 : nth)
    for (int y = y0; y < y1; y++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        sart_slice<R>(frames, nx, ny, T, cs.data(), vol_z, y, start, num, iters, subsets, rlx,
                      out + (size_t)(y - y0) * Nx * vol_z, rf ? rfs[tid].data() : nullptr);
    }
    g_inner = 1;
    if (rf)
        for (auto& v : rfs)
            for (int i = 0; i < 2 * iters; i++) rf[i] += v[i];
    return 0;
}


// ---------------------------------------------------------------------------
// Projection-alignment re-projection (AreTomo/ProjAlign/CCalcReproj.cpp,
// GReproj.cu).  FP32 throughout, in the reference kernels' operation order
// (nvcc contracts a*b + c*d to fma(a, b, c*d) and x + y*z to fma(y, z, x)).
// ---------------------------------------------------------------------------
constexpr float kReprojD2R = 0.01745f;   // s_fD2R of GReproj.cu / CCalcReproj.cpp

// CCalcReproj::mFindProjRange (CCalcReproj.cpp:66-119)
void reproj_range(const float* tilts, const unsigned char* skip, int T, int proj, int* range)
{
    const float ref_range = 20.5f, ref_stretch = 1.20f;
    const float a = tilts[proj];
    const float cos_a = (float)std::cos((double)(a * kReprojD2R));
    auto ok = [&](int i) {
        if (skip && skip[i]) return false;
        const float t = tilts[i];
        if (std::fabs(a - t) > ref_range) return false;
        const float stretch = (float)(std::cos((double)(t * kReprojD2R)) / cos_a);
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

// GReproj mGBackProj + mGForProj for one row (GReproj.cu:22-110).  sino:
// [T][nx] rows of the tilts in range; vol: scratch of (2 nx) x vz.
void reproj_row(const float* const* rows, const float* tilts, const int* range, float proj_angle, int nx, int vz,
                float* vol, float* out)
{
    const int VX = 2 * nx, VZ = vz;
    const float cent = nx * 0.5f;
    const int iend = nx - 1;
    for (int z = 0; z < VZ; z++) {
        const float fZ = z + 0.5f - VZ * 0.5f;
        for (int x = 0; x < VX; x++) {
            const float fX = x + 0.5f - VX * 0.5f;
            float sum = 0.f, cnt = 0.f;
            for (int i = range[0]; i <= range[1]; i++) {
                const float w = cosf((proj_angle - tilts[i]) * kReprojD2R);
                const float v = tilts[i] * kReprojD2R;
                const float c = cosf(v), sn = sinf(v);
                const float p = std::fmaf(fX, c, fZ * sn) + cent;
                if (p < 0 || p > iend) continue;
                float val = rows[i][(int)p];
                if (val < -1e10f) val = -1e30f;
                if (val < -1e20f) continue;
                sum = std::fmaf(val * c, w, sum);
                cnt += w;
            }
            vol[(size_t)z * VX + x] = cnt < 0.001f ? -1e30f : sum / cnt;
        }
    }
    const double rad = 4.0 * std::atan(1.0) / 180.0;
    const float c = (float)std::cos(rad * proj_angle), sn = (float)std::sin(rad * proj_angle);
    const int L = (int)(VZ / c + 0.5f);
    // a*b + c*d contracts to fma(a, b, c*d): the second product is rounded
    const float tz = VZ * 0.5f - (L * 0.5f) * c;
    constexpr int kT = 512;   // the reference's threads per ray
    for (int u = 0; u < nx; u++) {
        const float xp = u + 0.5f - nx * 0.5f;
        const float tx = (VX * 0.5f + (L * 0.5f) * sn) + xp / c;
        float part[kT];
        int pcnt[kT];
        for (int t = 0; t < kT; t++) {
            float s = 0.f;
            int n = 0;
            for (int i = t; i < L; i += kT) {
                const float fx = std::fmaf(-(float)i, sn, tx), fz = std::fmaf((float)i, c, tz);
                if (fx < 0 || fx >= VX || fz < 0 || fz >= VZ) continue;
                const float v = vol[(size_t)VX * (int)fz + (int)fx];
                if (v <= -1e10f) continue;
                s += v;
                n += 1;
            }
            part[t] = s;
            pcnt[t] = n;
        }
        for (int h = kT / 2; h > 0; h /= 2)
            for (int t = 0; t < h; t++) {
                part[t] += part[t + h];
                pcnt[t] += pcnt[t + h];
            }
        out[u] = pcnt[0] < 0.8f * L ? -1e30f : part[0] / pcnt[0];
    }
}

// ---------------------------------------------------------------------------
// Input stage (AreTomo/Correct): aligned frame, random fill, Fourier binning.
// ---------------------------------------------------------------------------

// CCorrectUtil::CalcAlignedSize (AreTomo/Correct/CCorrectUtil.cpp:11-21).
void stack_aligned_size(int nx, int ny, float axis_deg, int* a)
{
    a[0] = nx;
    a[1] = ny;
    const double rot = std::fabs(std::sin(axis_deg * 3.14 / 180.0));
    if (rot <= 0.707) return;
    a[0] = ny;
    a[1] = nx;
}

// GFourierResize2D::GetBinnedImgSize (MaUtil/GFourierResize2D.cu:75-88).
void stack_binned_size(const int* a, float bin, int* b)
{
    b[0] = a[0];
    b[1] = a[1];
    if (bin == 1.0f) return;
    b[0] = (int)(a[0] / bin) / 2 * 2;
    b[1] = (int)(a[1] / bin) / 2 * 2;
}

// GCorrPatchShift.cu:61-104 (mGCorrect) and :18-49 (mGCalcLocalShift), in
// FP32 with the fused multiply-adds the reference's compiled kernel executes:
// the rotation x*c - y*s, x*s + y*c as fma(x, c, -(y*s)), fma(y, c, x*s)
// (measured against the reference's output on 4096^2 frames), the squared
// patch distance as fma(ly, ly, lx*lx), s += a*b as fma(a, b, s).  W: the
// width the reference's grid covers; columns >= W are 0.
void stack_corr_frame(const float* raw, int nx, int ny, int ax, int ay, int W, float shx, float shy, float c,
                      float s, const float* local, int P, float* out)
{
    for (int Y = 0; Y < ay; Y++) {
        for (int X = 0; X < ax; X++) {
            float* o = out + (size_t)Y * ax + X;
            if (X >= W) {
                *o = 0.f;
                continue;
            }
            float fx = ((float)X + 0.5f) - (float)W * 0.5f;
            float fy = ((float)Y + 0.5f) - (float)ay * 0.5f;
            const float ft = std::fmaf(fx, c, -(fy * s));
            fy = std::fmaf(fy, c, fx * s);
            fx = ft;
            if (P > 0 && local) {
                int cnt = 0;
                float sx = 0.f, sy = 0.f, sw = 0.f;
                for (int p = 0; p < P; p++) {
                    if (local[4 * P + p] < 0.9f) continue;
                    const float lx = (fx - local[p]) / (float)nx;
                    const float ly = (fy - local[P + p]) / (float)ny;
                    const float w = std::exp(-100.0f * std::fmaf(ly, ly, lx * lx));
                    sx = std::fmaf(local[2 * P + p], w, sx);
                    sy = std::fmaf(local[3 * P + p], w, sy);
                    sw += w;
                    cnt++;
                }
                float dx = 0.f, dy = 0.f;
                if (cnt > 0) {
                    dx = sx / sw;
                    dy = sy / sw;
                }
                fx += dx;
                fy += dy;
            }
            fx += (shx + (float)nx * 0.5f);
            fy += (shy + (float)ny * 0.5f);
            const int x = (int)(fx + 0.5f), y = (int)(fy + 0.5f);
            *o = (x >= 0 && x < nx && y >= 0 && y < ny) ? raw[(size_t)y * nx + x] : kSentinelValue;
        }
    }
}

// GFillEmpty2D.cu:7-87: empty = value < -1e10; the mean of the non-empty
// pixels as one 512-thread block sums it (strided float partial sums, then a
// halving tree); every empty pixel follows its random chain (at most 100
// links) to the first non-empty pixel, else takes the mean.
void stack_fill_frame(float* img, int W, int ax, int ay, const int* table)
{
    const int n = W * ay;
    std::vector<unsigned char> empty(n);
    for (int i = 0; i < n; i++) empty[i] = img[(size_t)(i / W) * ax + i % W] < kSentinelTest;
    float psum[512], pcnt[512];
    for (int t = 0; t < 512; t++) {
        float sum = 0.f, cnt = 0.f;
        for (int i = t; i < n; i += 512) {
            if (empty[i]) continue;
            sum += img[(size_t)(i / W) * ax + i % W];
            cnt += 1.0f;
        }
        psum[t] = sum;
        pcnt[t] = cnt;
    }
    for (int off = 256; off > 0; off /= 2)
        for (int t = 0; t < off; t++) {
            psum[t] += psum[t + off];
            pcnt[t] += pcnt[t + off];
        }
    const float mean = pcnt[0] <= 0.f ? 0.f : psum[0] / pcnt[0];
    std::vector<float> src(img, img + (size_t)ay * ax);
    for (int i = 0; i < n; i++) {
        if (!empty[i]) continue;
        float v = mean;
        int next = table[i];
        for (int j = 0; j < 100; j++) {
            if (empty[next]) {
                next = table[next];
                continue;
            }
            v = src[(size_t)(next / W) * ax + next % W];
            break;
        }
        img[(size_t)(i / W) * ax + i % W] = v;
    }
}

// Fourier-crop binning (CFourierCropImage.cpp:41-61 = CBinStack::DoFFT per
// frame): 2-D R2C of (ay x ax) scaled by 1/(ax ay) (MaUtil/CCufft2D.cpp:65-86),
// crop to (by x bx) as GFourierResize2D.cu:7-39 does, 2-D C2R unnormalised
// under the selected C2R convention.  A binned size equal to the aligned size
// is a copy (CFourierCropImage::mCopy).
template <class R>
void stack_bin_frame(const float* img, int ax, int ay, int bx, int by, R* out)
{
    if (ax == bx && ay == by) {
        for (size_t i = 0; i < (size_t)ax * ay; i++) out[i] = img[i];
        return;
    }
    const int KX = bx / 2 + 1;
    std::vector<std::complex<R>> rows((size_t)ay * KX), line(ax);
    for (int y = 0; y < ay; y++) {
        for (int x = 0; x < ax; x++) line[x] = std::complex<R>((R)img[(size_t)y * ax + x], 0);
        fft<R>(line.data(), ax, -1);
        for (int k = 0; k < KX; k++) rows[(size_t)y * KX + k] = line[k];
    }
    const R norm = (R)(1.0 / ax / ay);
    std::vector<std::complex<R>> crop((size_t)by * KX), col(ay), col2(by);
    for (int k = 0; k < KX; k++) {
        for (int y = 0; y < ay; y++) col[y] = rows[(size_t)y * KX + k];
        fft<R>(col.data(), ay, -1);
        for (int ky = 0; ky < by; ky++) {
            const int src = ky <= by / 2 ? ky : ky + ay - by;
            col2[ky] = col[src] * norm;
        }
        fft<R>(col2.data(), by, +1);
        for (int y = 0; y < by; y++) crop[(size_t)y * KX + k] = col2[y];
    }
    for (int y = 0; y < by; y++) c2r<R>(&crop[(size_t)y * KX], bx, out + (size_t)y * bx, g_c2r_mode);
}

// CCalcVolThick::mMeasureStd (CCalcVolThick.cpp:172-197) on plane k of
// FlipVol(true) of vol[ny][Nz][Nx]: rows j in [0, ty) (from row 0, as the
// reference indexes them), columns x0 .. x0 + tx - 1; sums in double in the
// reference's order.
float thick_plane_std(const float* vol, int Nx, int Nz, int k, int x0, int tx, int ty)
{
    const int zr = Nz - 1 - k;
    double s1 = 0.0, s2 = 0.0;
    int cnt = 0;
    for (int j = 0; j < ty; j++) {
        const float* row = vol + ((size_t)j * Nz + zr) * Nx + x0;
        for (int i = 0; i < tx; i++) {
            const float v = row[i];
            if (v < (float)-1e20) continue;
            s1 += v;
            s2 += (v * v);
            cnt += 1;
        }
    }
    s1 = s1 / cnt;
    s2 = s2 / cnt - s1 * s1;
    if (s2 <= 0) s2 = 0.0f;
    else s2 = sqrtf((float)s2);
    return (float)s2;
}
}  // namespace

extern "C" {

void oracle_set_fill_table(const int* table, int n)
{
    if (table && n > 0) g_fill_table.assign(table, table + n);
    else g_fill_table.clear();
}

void oracle_set_c2r_mode(int mode) { g_c2r_mode = mode; }
int oracle_get_c2r_mode(void) { return g_c2r_mode; }

void oracle_cos_sin(const float* tilts_deg, int n_tilts, float* cos_sin) { cos_sin_table(tilts_deg, n_tilts, cos_sin); }

int oracle_wbp_f64(const float* frames, int nx, int ny, int n_tilts, const float* tilts_deg, int vol_z, int y0,
                   int y1, double* out, int n_threads)
{
    return wbp_run<double>(frames, nx, ny, n_tilts, tilts_deg, vol_z, y0, y1, out, n_threads);
}

int oracle_wbp_f32(const float* frames, int nx, int ny, int n_tilts, const float* tilts_deg, int vol_z, int y0,
                   int y1, float* out, int n_threads)
{
    return wbp_run<float>(frames, nx, ny, n_tilts, tilts_deg, vol_z, y0, y1, out, n_threads);
}

int oracle_sart_f64(const float* frames, int nx, int ny, int n_tilts, const float* tilts_deg, int vol_z,
                    int start_tilt, int num_tilts, int iters, int subsets, double relax, int y0, int y1,
                    double* out, double* rfactor, int n_threads)
{
    return sart_run<double>(frames, nx, ny, n_tilts, tilts_deg, vol_z, start_tilt, num_tilts, iters, subsets,
                            relax, y0, y1, out, rfactor, n_threads);
}

int oracle_sart_f32(const float* frames, int nx, int ny, int n_tilts, const float* tilts_deg, int vol_z,
                    int start_tilt, int num_tilts, int iters, int subsets, double relax, int y0, int y1,
                    float* out, double* rfactor, int n_threads)
{
    return sart_run<float>(frames, nx, ny, n_tilts, tilts_deg, vol_z, start_tilt, num_tilts, iters, subsets,
                           relax, y0, y1, out, rfactor, n_threads);
}

int oracle_fft_f64(const double* in, int n, int sign, double* out)
{
    if (!in || !out || n < 1) return -1;
    std::vector<std::complex<double>> a(n);
    for (int i = 0; i < n; i++) a[i] = {in[2 * i], in[2 * i + 1]};
    fft<double>(a.data(), n, sign < 0 ? -1 : 1);
    for (int i = 0; i < n; i++) { out[2 * i] = a[i].real(); out[2 * i + 1] = a[i].imag(); }
    return 0;
}

int oracle_rweight_row_f64(const double* in, int n, double* out)
{
    if (!in || !out || n < 2 || (n & 1)) return -1;
    std::vector<double> h;
    rweight_filter<double>(n, h);
    std::vector<std::complex<double>> work;
    std::memcpy(out, in, sizeof(double) * n);
    rweight_row<double>(out, n, h, work);
    return 0;
}

void oracle_rweight_filter_f64(int n, double* h)
{
    std::vector<double> v;
    rweight_filter<double>(n, v);
    std::memcpy(h, v.data(), sizeof(double) * v.size());
}

int oracle_fourier_crop_f64(const double* g, int nx_vol, int nz_vol, double* f)
{
    if (!g || !f || nx_vol < 2 || (nx_vol & 1) || nz_vol < 1) return -1;
    fourier_crop<double>(g, nx_vol, nz_vol, f, g_c2r_mode);
    return 0;
}

int oracle_c2r_f64(const double* in_cplx, int n, double* out)
{
    if (!in_cplx || !out || n < 2 || (n & 1)) return -1;
    std::vector<std::complex<double>> X(n / 2 + 1);
    for (int k = 0; k <= n / 2; k++) X[k] = {in_cplx[2 * k], in_cplx[2 * k + 1]};
    c2r<double>(X.data(), n, out, g_c2r_mode);
    return 0;
}

int oracle_reproj_range(const float* tilts_deg, const unsigned char* skip, int n_tilts, int proj_idx, int* range)
{
    if (!tilts_deg || !range || n_tilts < 1 || proj_idx < 0 || proj_idx >= n_tilts) return -1;
    reproj_range(tilts_deg, skip, n_tilts, proj_idx, range);
    return 0;
}

int oracle_reproj_f32(const float* frames, int nx, int ny, int n_tilts, const float* tilts_deg,
                      const unsigned char* skip, int proj_idx, int vol_z, float* out, int n_threads)
{
    if (!frames || !tilts_deg || !out || nx < 2 || ny < 1 || vol_z < 1 || proj_idx < 0 || proj_idx >= n_tilts)
        return -1;
    int range[2];
    reproj_range(tilts_deg, skip, n_tilts, proj_idx, range);
    if (range[0] < 0 || range[1] >= n_tilts) return -2;
    const int nth = n_threads > 0 ? n_threads : 1;
#pragma omp parallel num_threads(nth)
    {
        std::vector<float> vol((size_t)2 * nx * vol_z);
        std::vector<const float*> rows(n_tilts);
#pragma omp for schedule(dynamic, 1)
        for (int y = 0; y < ny; y++) {
            for (int t = 0; t < n_tilts; t++) rows[t] = frames + ((size_t)t * ny + y) * nx;
            reproj_row(rows.data(), tilts_deg, range, tilts_deg[proj_idx], nx, vol_z, vol.data(),
                       out + (size_t)y * nx);
        }
    }
    return 0;
}

/* ---- input stage and thickness ------------------------------------------ */

int oracle_stack_sizes(int nx, int ny, int correct, float size_axis_deg, float bin, int* sizes)
{
    if (!sizes || nx < 2 || ny < 2) return -1;
    int a[2] = {nx, ny}, b[2];
    if (correct) stack_aligned_size(nx, ny, size_axis_deg, a);
    stack_binned_size(a, bin, b);
    sizes[0] = a[0];
    sizes[1] = a[1];
    sizes[2] = b[0];
    sizes[3] = b[1];
    return 0;
}

int oracle_stack_f64(const float* raw, int nx, int ny, int n_tilts, int correct, const float* shifts,
                     const float* axes_deg, float size_axis_deg, int num_patches, const float* local,
                     int rand_fill, const int* table, float bin, double* out, float* aligned, int n_threads)
{
    int sz[4];
    if (!raw || !out || oracle_stack_sizes(nx, ny, correct, size_axis_deg, bin, sz)) return -1;
    if (correct && rand_fill && !table) return -2;
    const int ax = sz[0], ay = sz[1], bx = sz[2], by = sz[3];
    const int W = ((ax / 2 + 1) * 2 / 2 - 1) * 2;
    const float d2r = 3.141592654f / 180.0f;
    const int nth = n_threads > 0 ? n_threads : 1;
#pragma omp parallel for num_threads(nth) schedule(dynamic, 1)
    for (int t = 0; t < n_tilts; t++) {
        std::vector<float> img((size_t)ax * ay);
        const float* src = raw + (size_t)t * nx * ny;
        if (correct) {
            const float rad = axes_deg ? axes_deg[t] * d2r : 0.f;
            const float c = std::cos(rad), s = std::sin(rad);
            stack_corr_frame(src, nx, ny, ax, ay, W, shifts ? shifts[2 * t] : 0.f, shifts ? shifts[2 * t + 1] : 0.f,
                             c, s, local ? local + (size_t)t * 5 * num_patches : nullptr, num_patches, img.data());
            if (rand_fill) stack_fill_frame(img.data(), W, ax, ay, table);
        } else {
            std::memcpy(img.data(), src, sizeof(float) * img.size());
        }
        if (aligned) std::memcpy(aligned + (size_t)t * ax * ay, img.data(), sizeof(float) * img.size());
        stack_bin_frame<double>(img.data(), ax, ay, bx, by, out + (size_t)t * bx * by);
    }
    return 0;
}

int oracle_stack_fill_f32(float* img, int W, int ax, int ay, const int* table)
{
    if (!img || !table || W < 1 || W > ax || ay < 1) return -1;
    stack_fill_frame(img, W, ax, ay, table);
    return 0;
}

int oracle_thickness_profile(const float* vol, int Nx, int ny, int vol_z, float* profile)
{
    if (!vol || !profile || Nx < 2 || ny < 1 || vol_z < 2) return -1;
    const int tx = (int)(Nx * 0.4f) / 2 * 2, ty = (int)(ny * 0.4f) / 2 * 2;
    const int x0 = (Nx - tx) / 2;
    for (int k = 0; k < vol_z - 1; k++) profile[k] = thick_plane_std(vol, Nx, vol_z, k, x0, tx, ty);
    return 0;
}

int oracle_thickness_edges(const float* profile, int n, float bin, float* smoothed, int* result)
{
    if (!profile || !result || n < 10) return -1;
    // CCalcVolThick::mSmooth (CCalcVolThick.cpp:114-132)
    std::vector<float> cc(n);
    for (int i = 0; i < n; i++) {
        const int start = i - 5;
        double sum = 0.0;
        for (int j = 0; j < 11; j++) {
            const int k = std::min(std::max(j + start, 0), n - 1);
            sum += profile[k];
        }
        cc[i] = (float)sum / 11;
    }
    if (smoothed) std::memcpy(smoothed, cc.data(), sizeof(float) * n);
    // CCalcVolThick::mDetectEdges (CCalcVolThick.cpp:209-284); an edge that
    // no sample reaches stays at its search bound
    const int half = n / 2, bot = (int)(n * 0.1), top = n - bot;
    float mean = 0.f;
    for (int i = bot; i < top; i++) mean += cc[i];
    mean = mean / (top - bot);
    int e0 = bot, e1 = top;
    for (int i = bot; i < half; i++)
        if (cc[i] >= mean) { e0 = i; break; }
    float minv = mean;
    int imin = e0;
    for (int i = bot; i < e0; i++)
        if (cc[i] < minv) { minv = cc[i]; imin = i; }
    e0 = (e0 + imin) / 2;
    for (int i = top; i > half; i--)
        if (cc[i] >= mean) { e1 = i; break; }
    minv = mean;
    imin = e1;
    for (int i = top; i > e1; i--)
        if (cc[i] < minv) { minv = cc[i]; imin = i; }
    e1 = (e1 + imin) / 2;
    e0 = (int)(e0 * bin);
    e1 = (int)(e1 * bin);
    result[0] = e0;
    result[1] = e1;
    result[2] = e1 - e0;
    result[3] = (e0 + e1) / 2 - (int)(half * bin);
    return 0;
}

}  // extern "C"
