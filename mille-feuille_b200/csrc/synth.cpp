// synth.cpp -- seeded synthetic matrices of the benchmark configurations.
//
// The paper's SuiteSparse inputs are not available, so every configuration is
// a generated matrix with fixed shape, size and value distribution.  One
// counter-based generator is used everywhere: the i-th output of SplitMix64
// (Steele, Lea, Flood 2014) started from a per-(seed, stream) key, mapped to
// [0,1) with 53 bits.  A Python mirror (tests/synth_mirror.py) reproduces
// every generator for the parity tests.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mf.h"

namespace {

constexpr uint64_t GAMMA = 0x9E3779B97F4A7C15ull;

inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline uint64_t stream_key(uint64_t seed, uint64_t stream) { return mix64(seed * GAMMA ^ mix64(stream + GAMMA)); }

inline double u01(uint64_t key, uint64_t i) { return (double)(mix64(key + (i + 1) * GAMMA) >> 11) * 0x1.0p-53; }

inline double normal01(uint64_t key, uint64_t m)
{
    const double a = u01(key, 2 * m), b = u01(key, 2 * m + 1);
    return std::sqrt(-2.0 * std::log(1.0 - a)) * std::cos(6.283185307179586 * b);
}

enum Stream : uint64_t { S_XSTAR = 1, S_ROWSCALE = 2, S_SIZE = 3, S_ROWLEN = 4, S_COL = 5, S_VAL = 6, S_FIELD = 7 };

struct CsrOut {
    std::vector<int> rp, ci;
    std::vector<double> v;
};

mf_status emit(const CsrOut &c, int n, int *n_out, int *nnz_out, int **rowptr, int **colidx, double **val)
{
    const size_t nnz = c.ci.size();
    int *rp = (int *)malloc(sizeof(int) * (n + 1));
    int *ci = (int *)malloc(sizeof(int) * (nnz ? nnz : 1));
    double *v = (double *)malloc(sizeof(double) * (nnz ? nnz : 1));
    if (!rp || !ci || !v) {
        free(rp);
        free(ci);
        free(v);
        return MF_ERR_NO_MEMORY;
    }
    memcpy(rp, c.rp.data(), sizeof(int) * (n + 1));
    if (nnz) {
        memcpy(ci, c.ci.data(), sizeof(int) * nnz);
        memcpy(v, c.v.data(), sizeof(double) * nnz);
    }
    *n_out = n;
    *nnz_out = (int)nnz;
    *rowptr = rp;
    *colidx = ci;
    *val = v;
    return MF_OK;
}

// 7-point stencil assembly on a g^3 grid: off(i, nb, dir) gives the
// off-diagonal value, diag(i, offsum) the diagonal.  Columns ascending.
template <class Off, class Diag>
void stencil3d(int g, CsrOut &c, Off off, Diag diag)
{
    const long long n = (long long)g * g * g;
    c.rp.assign(n + 1, 0);
    c.ci.reserve(n * 7);
    c.v.reserve(n * 7);
    const long long st[3] = {(long long)g * g, g, 1};  // z, y, x strides
    for (long long i = 0; i < n; i++) {
        const int x = (int)(i % g), y = (int)((i / g) % g), z = (int)(i / ((long long)g * g));
        const int co[3] = {z, y, x};
        double offsum = 0.0;
        const size_t row0 = c.ci.size();
        // lower neighbours z-1, y-1, x-1
        for (int d = 0; d < 3; d++)
            if (co[d] > 0) {
                double a = off(i, i - st[d], d, 0);
                c.ci.push_back((int)(i - st[d]));
                c.v.push_back(a);
                offsum += std::fabs(a);
            }
        const size_t dpos = c.ci.size();
        c.ci.push_back((int)i);
        c.v.push_back(0.0);
        for (int d = 2; d >= 0; d--)
            if (co[d] < g - 1) {
                double a = off(i, i + st[d], d, 1);
                c.ci.push_back((int)(i + st[d]));
                c.v.push_back(a);
                offsum += std::fabs(a);
            }
        (void)row0;
        c.v[dpos] = diag(i, offsum, co);
        c.rp[i + 1] = (int)c.ci.size();
    }
}

}  // namespace

extern "C" {

double mf_rng_u01(uint64_t seed, uint64_t stream, uint64_t i) { return u01(stream_key(seed, stream), i); }

double mf_rng_normal(uint64_t seed, uint64_t stream, uint64_t m) { return normal01(stream_key(seed, stream), m); }

// x*_i = U[-1, 1] from (seed, stream 1).
mf_status mf_synth_xstar(uint64_t seed, int n, double *out)
{
    if (!out || n < 0) return MF_ERR_INVALID_ARG;
    const uint64_t k = stream_key(seed, S_XSTAR);
    for (int i = 0; i < n; i++) out[i] = -1.0 + 2.0 * u01(k, i);
    return MF_OK;
}

// 2D 5-point Laplacian, Dirichlet: 4 on the diagonal, -1 to the neighbours.
mf_status mf_synth_laplace2d(int nx, int ny, int *n_out, int *nnz_out, int **rowptr, int **colidx, double **val)
{
    if (nx <= 0 || ny <= 0) return MF_ERR_INVALID_ARG;
    const int n = nx * ny;
    CsrOut c;
    c.rp.assign(n + 1, 0);
    for (int i = 0; i < n; i++) {
        const int x = i % nx, y = i / nx;
        if (y > 0) c.ci.push_back(i - nx), c.v.push_back(-1.0);
        if (x > 0) c.ci.push_back(i - 1), c.v.push_back(-1.0);
        c.ci.push_back(i), c.v.push_back(4.0);
        if (x < nx - 1) c.ci.push_back(i + 1), c.v.push_back(-1.0);
        if (y < ny - 1) c.ci.push_back(i + nx), c.v.push_back(-1.0);
        c.rp[i + 1] = (int)c.ci.size();
    }
    return emit(c, n, n_out, nnz_out, rowptr, colidx, val);
}

// 3D 7-point pattern on g^3; off-diagonals -(f_i + f_j)/2 with per-row
// factors f = 10^U[-3,0] (the symmetrized row-scaled Laplacian), diagonal
// = sum |off| + 1e-3.
mf_status mf_synth_poisson3d_scaled(int g, uint64_t seed, int *n_out, int *nnz_out, int **rowptr, int **colidx,
                                    double **val)
{
    if (g <= 0 || (long long)g * g * g > 0x3fffffff) return MF_ERR_INVALID_ARG;
    const long long n = (long long)g * g * g;
    std::vector<double> f(n);
    const uint64_t k = stream_key(seed, S_ROWSCALE);
    for (long long i = 0; i < n; i++) f[i] = std::pow(10.0, -3.0 + 3.0 * u01(k, i));
    CsrOut c;
    stencil3d(
        g, c, [&](long long i, long long j, int, int) { return -(f[i] + f[j]) * 0.5; },
        [&](long long, double offsum, const int *) { return offsum + 1e-3; });
    return emit(c, (int)n, n_out, nnz_out, rowptr, colidx, val);
}

// 3D convection-diffusion on g^3: 7-point diffusion plus first-order upwind
// convection with velocity (vx, vy, vz) > 0.  Scaled by h^2/D, the upwind
// (lower) neighbour in direction d gets -(1 + gamma v_d), the downwind one
// -1, the diagonal 6 + gamma (vx + vy + vz), with gamma = 2 Pe / max(v) so
// that the cell Peclet number of the fastest direction is Pe.
mf_status mf_synth_convdiff3d(int g, double peclet, double vx, double vy, double vz, int *n_out, int *nnz_out,
                              int **rowptr, int **colidx, double **val)
{
    if (g <= 0 || (long long)g * g * g > 0x3fffffff || vx < 0 || vy < 0 || vz < 0) return MF_ERR_INVALID_ARG;
    const double vmax = std::max(vx, std::max(vy, vz));
    const double gam = vmax > 0 ? 2.0 * peclet / vmax : 0.0;
    const double vel[3] = {vz, vy, vx};  // indexed like stencil3d's dims (z, y, x)
    CsrOut c;
    stencil3d(
        g, c, [&](long long, long long, int d, int upper) { return upper ? -1.0 : -(1.0 + gam * vel[d]); },
        [&](long long, double, const int *) { return 6.0 + gam * (vx + vy + vz); });
    const long long n = (long long)g * g * g;
    return emit(c, (int)n, n_out, nnz_out, rowptr, colidx, val);
}

// Size of batched system `seed`: round(exp(U[ln 1000, ln 64000])).
int mf_synth_random_spd_size(uint64_t seed)
{
    const double u = u01(stream_key(seed, S_SIZE), 0);
    return (int)std::llround(std::exp(std::log(1000.0) + u * (std::log(64000.0) - std::log(1000.0))));
}

// Random symmetric SPD system: row i draws k_i = 8 + floor(25 U) column
// indices uniform in [0, n) (self-references dropped) with values N(0,1)
// times the row scale 10^U[-4,4]; A = (B + B^T)/2 with duplicates summed in
// draw order; diagonal = row |sum| + 1.  n <= 0 uses the seeded size.
mf_status mf_synth_random_spd(int n, uint64_t seed, int *n_out, int *nnz_out, int **rowptr, int **colidx,
                              double **val)
{
    if (n <= 0) n = mf_synth_random_spd_size(seed);
    const uint64_t kl = stream_key(seed, S_ROWLEN), ks = stream_key(seed, S_ROWSCALE), kc = stream_key(seed, S_COL),
                   kv = stream_key(seed, S_VAL);
    struct Trip {
        long long key;
        long long ord;
        double v;
    };
    std::vector<Trip> tr;
    tr.reserve((size_t)n * 40);
    long long ord = 0;
    for (int i = 0; i < n; i++) {
        const int k = 8 + (int)std::floor(25.0 * u01(kl, i));
        const double sc = std::pow(10.0, -4.0 + 8.0 * u01(ks, i));
        for (int e = 0; e < k; e++) {
            int j = (int)std::floor(u01(kc, (uint64_t)i * 32 + e) * n);
            if (j >= n) j = n - 1;
            if (j == i) continue;
            const double a = normal01(kv, (uint64_t)i * 32 + e) * sc * 0.5;
            tr.push_back({(long long)i * n + j, ord++, a});
            tr.push_back({(long long)j * n + i, ord++, a});
        }
    }
    std::sort(tr.begin(), tr.end(), [](const Trip &a, const Trip &b) { return a.key != b.key ? a.key < b.key : a.ord < b.ord; });
    CsrOut c;
    c.rp.assign(n + 1, 0);
    std::vector<double> rowabs(n, 0.0);
    // merge duplicates
    std::vector<long long> keys;
    std::vector<double> vals;
    for (size_t q = 0; q < tr.size(); q++) {
        if (!keys.empty() && keys.back() == tr[q].key) vals.back() += tr[q].v;
        else keys.push_back(tr[q].key), vals.push_back(tr[q].v);
    }
    for (size_t q = 0; q < keys.size(); q++) rowabs[keys[q] / n] += std::fabs(vals[q]);
    size_t q = 0;
    for (int i = 0; i < n; i++) {
        bool diag_done = false;
        while (q < keys.size() && keys[q] / n == i) {
            const int j = (int)(keys[q] % n);
            if (!diag_done && j > i) {
                c.ci.push_back(i), c.v.push_back(rowabs[i] + 1.0);
                diag_done = true;
            }
            c.ci.push_back(j), c.v.push_back(vals[q]);
            q++;
        }
        if (!diag_done) c.ci.push_back(i), c.v.push_back(rowabs[i] + 1.0);
        c.rp[i + 1] = (int)c.ci.size();
    }
    return emit(c, n, n_out, nnz_out, rowptr, colidx, val);
}

// Anisotropic lognormal diffusion on g^3 (cell-centred, Dirichlet).
// w ~ N(0,1) per cell; f = periodic separable convolution of w with
// h(d) = exp(-d^2 / l^2), |d| <= ceil(3 l), divided by (sum_d h(d)^2)^(3/2)
// so that f has unit variance (Gaussian covariance with correlation length
// l); cell coefficient k = exp(sigma f).  Face coefficient = harmonic mean of
// the two cells (k of the cell for a boundary face), times `aniso` on z
// faces.  Off-diagonal = -face, diagonal = sum of the cell's faces.
mf_status mf_synth_aniso3d(int g, uint64_t seed, double log_sigma, double corr_len, double aniso, int *n_out,
                           int *nnz_out, int **rowptr, int **colidx, double **val)
{
    if (g <= 0 || (long long)g * g * g > 0x3fffffff || corr_len <= 0) return MF_ERR_INVALID_ARG;
    const long long n = (long long)g * g * g;
    const uint64_t kf = stream_key(seed, S_FIELD);
    std::vector<double> w(n), t(n);
    for (long long i = 0; i < n; i++) w[i] = normal01(kf, i);
    const int R = (int)std::ceil(3.0 * corr_len);
    std::vector<double> h(2 * R + 1);
    double h2 = 0.0;
    for (int d = -R; d <= R; d++) {
        h[d + R] = std::exp(-(double)d * d / (corr_len * corr_len));
        h2 += h[d + R] * h[d + R];
    }
    auto idx = [g](long long x, long long y, long long z) { return x + (long long)g * (y + (long long)g * z); };
    auto wrap = [g](int a) { a %= g; return a < 0 ? a + g : a; };
    // x pass: w -> t, y pass: t -> w, z pass: w -> t
    for (int pass = 0; pass < 3; pass++) {
        std::vector<double> &src = (pass == 1) ? t : w;
        std::vector<double> &dst = (pass == 1) ? w : t;
        for (int z = 0; z < g; z++)
            for (int y = 0; y < g; y++)
                for (int x = 0; x < g; x++) {
                    double s = 0.0;
                    for (int d = -R; d <= R; d++) {
                        long long j = (pass == 0) ? idx(wrap(x + d), y, z) : (pass == 1) ? idx(x, wrap(y + d), z) : idx(x, y, wrap(z + d));
                        s += h[d + R] * src[j];
                    }
                    dst[idx(x, y, z)] = s;
                }
    }
    const double norm = std::pow(h2, 1.5);
    std::vector<double> kc(n);
    for (long long i = 0; i < n; i++) kc[i] = std::exp(log_sigma * t[i] / norm);
    const double an[3] = {aniso, 1.0, 1.0};  // dims (z, y, x)
    CsrOut c;
    stencil3d(
        g, c,
        [&](long long i, long long j, int d, int) { return -an[d] * 2.0 * kc[i] * kc[j] / (kc[i] + kc[j]); },
        [&](long long i, double offsum, const int *co) {
            double bnd = 0.0;
            for (int d = 0; d < 3; d++) {
                if (co[d] == 0) bnd += an[d] * kc[i];
                if (co[d] == g - 1) bnd += an[d] * kc[i];
            }
            return offsum + bnd;
        });
    return emit(c, (int)n, n_out, nnz_out, rowptr, colidx, val);
}

}  // extern "C"
