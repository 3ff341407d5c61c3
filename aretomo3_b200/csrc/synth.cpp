// Seeded synthetic tilt series: random ellipsoids + gold beads, projected
// analytically (exact chord lengths) in the single-axis parallel-beam geometry
// the reconstruction assumes, plus Gaussian or Poisson noise.
//
// Geometry.  A voxel (X, Y, Z) of an Nx x ny x Nz volume sits at
// x = X - Nx/2, y = Y - ny/2, z = Z - Nz/2.  At tilt theta it projects to the
// detector coordinate u = x cos(theta) + z sin(theta), which is detector
// pixel i = u + Nx/2 of row j = Y.  This is the mapping the back-projector of
// AreTomo/Recon/GBackProj.cu:35-36 uses (xp = fX*cos + fZ*sin + projX/2), so a
// phantom reconstructed from these projections lands where it was placed.
// The ray through pixel (i, j) runs along (-sin, 0, cos).
//
// Random numbers come from this file's own SplitMix64 / xoshiro256** streams
// and Box-Muller / inversion / PTRS samplers, so a seed gives the same bytes on
// every machine and for every thread count: object parameters are drawn from
// one sequential stream, and each pixel's noise from a stream keyed by
// (seed, pixel index).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

extern "C" {

typedef struct at3r_phantom_spec {
    uint64_t seed;
    int vol_x, vol_y, vol_z;       // phantom box (voxels): Nx, ny, thickness
    int n_ellipsoids;
    float axis_min, axis_max;      // semi-axes drawn U[axis_min, axis_max]
    float dens_min, dens_max;      // ellipsoid density U[dens_min, dens_max]
    int n_beads;
    float bead_radius, bead_density;
    int noise_kind;                // 0 none, 1 gaussian, 2 poisson
    float noise_param;             // gaussian: sigma / mean; poisson: electrons per pixel at the mean
} at3r_phantom_spec;

}

namespace {

inline uint64_t splitmix64(uint64_t& s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Xoshiro {
    uint64_t s[4];
    explicit Xoshiro(uint64_t seed)
    {
        uint64_t sm = seed;
        for (auto& v : s) v = splitmix64(sm);
    }
    static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    inline uint64_t next()
    {
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t; s[3] = rotl(s[3], 45);
        return r;
    }
    // uniform in [0, 1) with 53 random bits
    inline double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    inline double uniform(double a, double b) { return a + (b - a) * uniform(); }
    inline double gaussian()
    {   // Box-Muller, one value per call
        double u1 = uniform();
        double u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
    // Poisson: inversion for small means, Hormann's PTRS above (W. Hormann,
    // "The transformed rejection method for generating Poisson random
    // variables", Insurance: Mathematics and Economics 12, 1993).
    inline double poisson(double lam)
    {
        if (lam <= 0) return 0;
        if (lam < 30.0) {
            double L = std::exp(-lam), p = 1.0;
            int k = 0;
            do { k++; p *= uniform(); } while (p > L);
            return k - 1;
        }
        double slam = std::sqrt(lam), loglam = std::log(lam);
        double b = 0.931 + 2.53 * slam;
        double a = -0.059 + 0.02483 * b;
        double invalpha = 1.1239 + 1.1328 / (b - 3.4);
        double vr = 0.9277 - 3.6224 / (b - 2);
        for (;;) {
            double U = uniform() - 0.5;
            double V = uniform();
            double us = 0.5 - std::fabs(U);
            double k = std::floor((2 * a / us + b) * U + lam + 0.43);
            if (us >= 0.07 && V <= vr) return k;
            if (k < 0 || (us < 0.013 && V > us)) continue;
            if (std::log(V) + std::log(invalpha) - std::log(a / (us * us) + b) <=
                -lam + k * loglam - std::lgamma(k + 1))
                return k;
        }
    }
};

struct Ellipsoid {
    double c[3];     // centre (x, y, z), voxel units about the volume centre
    double A[3][3];  // R diag(a^2) R^T  (support-function matrix)
    double M[3][3];  // R diag(1/a^2) R^T (quadratic form)
    double dens;
};

void make_ellipsoid(Ellipsoid& e, const double c[3], const double ax[3], const double q_in[4], double dens)
{
    double q[4];
    double n = std::sqrt(q_in[0] * q_in[0] + q_in[1] * q_in[1] + q_in[2] * q_in[2] + q_in[3] * q_in[3]);
    if (n < 1e-12) { q[0] = 1; q[1] = q[2] = q[3] = 0; }
    else for (int i = 0; i < 4; i++) q[i] = q_in[i] / n;
    double w = q[0], x = q[1], y = q[2], z = q[3];
    double R[3][3] = {
        {1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)},
        {2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)},
        {2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)}};
    for (int i = 0; i < 3; i++) e.c[i] = c[i];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double sa = 0, sm = 0;
            for (int k = 0; k < 3; k++) {
                sa += R[i][k] * R[j][k] * ax[k] * ax[k];
                sm += R[i][k] * R[j][k] / (ax[k] * ax[k]);
            }
            e.A[i][j] = sa;
            e.M[i][j] = sm;
        }
    e.dens = dens;
}

inline double quad(const double M[3][3], const double a[3], const double b[3])
{
    double s = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) s += a[i] * M[i][j] * b[j];
    return s;
}

}  // namespace

extern "C" {

// Fills frames[T][ny][nx] (float32, row-major, x fastest).  Returns 0 on
// success, a negative number on invalid arguments.
int at3r_synth_tilt_series(const at3r_phantom_spec* sp, const float* tilts_deg, int n_tilts,
                           int nx, int ny, float* frames)
{
    if (!sp || !tilts_deg || !frames || n_tilts <= 0 || nx <= 1 || ny <= 0) return -1;
    const int NX = nx & ~1;
    Xoshiro rng(sp->seed);
    std::vector<Ellipsoid> objs;
    objs.reserve(sp->n_ellipsoids + sp->n_beads);
    const double hx = 0.5 * sp->vol_x, hy = 0.5 * sp->vol_y, hz = 0.5 * sp->vol_z;
    for (int i = 0; i < sp->n_ellipsoids; i++) {
        double c[3] = {rng.uniform(-hx, hx), rng.uniform(-hy, hy), rng.uniform(-hz, hz)};
        double ax[3];
        for (auto& a : ax) a = rng.uniform(sp->axis_min, sp->axis_max);
        double q[4];
        for (auto& v : q) v = rng.gaussian();
        double d = rng.uniform(sp->dens_min, sp->dens_max);
        Ellipsoid e;
        make_ellipsoid(e, c, ax, q, d);
        objs.push_back(e);
    }
    for (int i = 0; i < sp->n_beads; i++) {
        double r = sp->bead_radius;
        double c[3] = {rng.uniform(-hx + r, hx - r), rng.uniform(-hy + r, hy - r), rng.uniform(-hz + r, hz - r)};
        double ax[3] = {r, r, r};
        double q[4] = {1, 0, 0, 0};
        Ellipsoid e;
        make_ellipsoid(e, c, ax, q, sp->bead_density);
        objs.push_back(e);
    }

    const size_t frame_px = (size_t)nx * ny;
    std::memset(frames, 0, sizeof(float) * frame_px * n_tilts);

#pragma omp parallel for schedule(dynamic, 1)
    for (int t = 0; t < n_tilts; t++) {
        float* fr = frames + frame_px * t;
        const double th = tilts_deg[t] * (M_PI / 180.0);
        const double cs = std::cos(th), sn = std::sin(th);
        const double wu[3] = {cs, 0.0, sn};       // detector u direction
        const double d[3] = {-sn, 0.0, cs};       // ray direction
        std::vector<double> acc(frame_px, 0.0);
        for (const Ellipsoid& e : objs) {
            const double uc = e.c[0] * cs + e.c[2] * sn;
            const double vc = e.c[1];
            const double ue = std::sqrt(std::max(0.0, quad(e.A, wu, wu)));
            const double ve = std::sqrt(std::max(0.0, e.A[1][1]));
            const int i0 = std::max(0, (int)std::floor(uc - ue + 0.5 * NX));
            const int i1 = std::min(nx - 1, (int)std::ceil(uc + ue + 0.5 * NX));
            const int j0 = std::max(0, (int)std::floor(vc - ve + 0.5 * ny));
            const int j1 = std::min(ny - 1, (int)std::ceil(vc + ve + 0.5 * ny));
            if (i0 > i1 || j0 > j1) continue;
            const double dMd = quad(e.M, d, d);
            for (int j = j0; j <= j1; j++) {
                const double v = j - 0.5 * ny;
                for (int i = i0; i <= i1; i++) {
                    const double u = i - 0.5 * NX;
                    // ray point at parameter 0, relative to the centre
                    const double p[3] = {u * cs - e.c[0], v - e.c[1], u * sn - e.c[2]};
                    const double b = quad(e.M, d, p);
                    const double cq = quad(e.M, p, p) - 1.0;
                    const double disc = b * b - dMd * cq;
                    if (disc <= 0) continue;
                    acc[(size_t)j * nx + i] += e.dens * 2.0 * std::sqrt(disc) / dMd;
                }
            }
        }
        for (size_t k = 0; k < frame_px; k++) fr[k] = (float)acc[k];
    }

    if (sp->noise_kind == 0) return 0;
    double sum = 0;
    for (size_t k = 0; k < frame_px * n_tilts; k++) sum += frames[k];
    const double mean = sum / (double)(frame_px * n_tilts);
    const int64_t total = (int64_t)(frame_px * n_tilts);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < total; k++) {
        Xoshiro prng(sp->seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(k + 1)));
        double p = frames[k];
        if (sp->noise_kind == 1) {
            p += sp->noise_param * mean * prng.gaussian();
        } else if (sp->noise_kind == 2 && mean > 0) {
            double lam = sp->noise_param * std::max(p, 0.0) / mean;
            p = prng.poisson(lam) * mean / sp->noise_param;
        }
        frames[k] = (float)p;
    }
    return 0;
}

}  // extern "C"
