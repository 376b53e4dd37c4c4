/*
 * inputs.cpp -- seeded synthetic particle sets for the workloads this library is measured
 * and tested on.  Host-only; nothing here runs on the device.
 *
 *   lattice        the reference driver's close-packed lattice (src/main.cu:84-109)
 *   jiggle_ref     the reference driver's jiggle (src/main.cu:47-63), std::mt19937
 *   jiggle_frac    a fraction of particles picked uniformly without replacement, h scaled
 *                  by U[lo, hi]  (the lattice-100 workload: 1%, [0.65, 1.35])
 *   plummer        Plummer sphere, scale radius 1, truncated at rmax, h from the local
 *                  density times a log-normal factor, isotropic velocities at a fraction
 *                  of the circular speed
 *   uniform_box    uniform random positions in a box
 *   gaussian       i.i.d. normal values
 * Random streams are std::mt19937_64 seeded by the caller, except jiggle_ref, which uses
 * std::mt19937 as the reference driver does.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>

extern "C" {

// Number of particles lattice(npartx) produces.
long cin_lattice_count(int npartx)
{
    if (npartx < 4) return 0;
    const double dx = 1.0 / npartx;
    const double dy = dx * std::sqrt(3.0) / 2.0;
    const double dz = dx * std::sqrt(6.0) / 3.0;
    return long(npartx) * int(1.0 / dy) * int(1.0 / dz);
}

// Close-packed lattice in the unit box; h = 1.2 * dx.  Returns pmass = 1/N.
double cin_lattice(int npartx, double* x, double* y, double* z, double* h)
{
    const double dx = 1.0 / npartx;
    const double dy = dx * std::sqrt(3.0) / 2.0;
    const double dz = dx * std::sqrt(6.0) / 3.0;
    const int ny = int(1.0 / dy), nz = int(1.0 / dz);
    long p = 0;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < npartx; ++i, ++p)
            {
                x[p] = i * dx + ((j + k) % 2) * 0.5 * dx;
                y[p] = j * dy + (k % 2) * dy / 3.0;
                z[p] = k * dz;
                h[p] = 1.2 * dx;
            }
    return 1.0 / double(p);
}

// The reference driver's jiggle: ~1% of particles, h *= 1 + 0.5*sign(r-1/2)*r^30.
long cin_jiggle_ref(long n, double* h, unsigned seed)
{
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    long count = 0;
    for (long i = 0; i < n; ++i)
    {
        if (u(rng) < 0.99) continue;
        const double r = u(rng);
        h[i] *= 1.0 + 0.5 * std::copysign(std::pow(r, 30.0), r - 0.5);
        ++count;
    }
    return count;
}

// round(frac*n) distinct particles picked uniformly (partial Fisher-Yates); each h scaled
// by an independent U[lo, hi].  Returns the number changed.
long cin_jiggle_frac(long n, double* h, double frac, double lo, double hi, uint64_t seed)
{
    std::mt19937_64 rng(seed);
    const long m = std::lround(frac * double(n));
    std::vector<long> idx(n);
    for (long i = 0; i < n; ++i) idx[i] = i;
    std::uniform_real_distribution<double> f(lo, hi);
    for (long k = 0; k < m; ++k)
    {
        std::uniform_int_distribution<long> pick(k, n - 1);
        std::swap(idx[k], idx[pick(rng)]);
        h[idx[k]] *= f(rng);
    }
    return m;
}

void cin_gaussian(long n, double* out, double mean, double sigma, uint64_t seed)
{
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> g(mean, sigma);
    for (long i = 0; i < n; ++i) out[i] = g(rng);
}

void cin_uniform(long n, double* out, double lo, double hi, uint64_t seed)
{
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(lo, hi);
    for (long i = 0; i < n; ++i) out[i] = u(rng);
}

// Uniform random positions in [0,1)^3 (one stream, x y z interleaved per particle);
// h = hfac * (1/n)^(1/3) * U[hlo, hhi].  Returns pmass = 1/n.
double cin_uniform_box(long n, double* x, double* y, double* z, double* h, double hfac, double hlo,
                       double hhi, uint64_t seed)
{
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(0.0, 1.0), f(hlo, hhi);
    const double dx = std::cbrt(1.0 / double(n));
    for (long i = 0; i < n; ++i)
    {
        x[i] = u(rng);
        y[i] = u(rng);
        z[i] = u(rng);
        h[i] = hfac * dx * f(rng);
    }
    return 1.0 / double(n);
}

// Plummer sphere (a = 1, M = 1, G = 1) truncated at rmax.  r from the inverse of the
// cumulative mass, redrawn when r >= rmax; isotropic position and velocity directions.
// h = hfact * (m / rho(r))^(1/3) * hmul, with hmul = exp(lnsigma * N(0,1)) when lnsigma > 0,
// else U[ulo, uhi].  |v| = vfrac * sqrt(M(<r)/r).  u_out (optional) = uval.
double cin_plummer(long n, double* x, double* y, double* z, double* h, double* vx, double* vy,
                   double* vz, double rmax, double hfact, double lnsigma, double ulo, double uhi,
                   double vfrac, uint64_t seed)
{
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(0.0, 1.0), fu(ulo, uhi);
    std::normal_distribution<double> g(0.0, 1.0);
    const double pi = 3.141592653589793;
    const double m = 1.0 / double(n);
    auto dir = [&](double& a, double& b, double& c) {
        const double ct = 2.0 * u(rng) - 1.0;
        const double st = std::sqrt(std::max(0.0, 1.0 - ct * ct));
        const double ph = 2.0 * pi * u(rng);
        a = st * std::cos(ph); b = st * std::sin(ph); c = ct;
    };
    for (long i = 0; i < n; ++i)
    {
        double r;
        do
        {
            double U = u(rng);
            while (U <= 0.0) U = u(rng);
            r = 1.0 / std::sqrt(std::pow(U, -2.0 / 3.0) - 1.0);
        } while (!(r < rmax));
        double a, b, c;
        dir(a, b, c);
        x[i] = r * a; y[i] = r * b; z[i] = r * c;
        const double rho = 3.0 / (4.0 * pi) * std::pow(1.0 + r * r, -2.5);
        const double hm = (lnsigma > 0.0) ? std::exp(lnsigma * g(rng)) : fu(rng);
        h[i] = hfact * std::cbrt(m / rho) * hm;
        const double menc = r * r * r / std::pow(r * r + 1.0, 1.5);
        const double vmag = vfrac * std::sqrt(menc / r);
        dir(a, b, c);
        if (vx) { vx[i] = vmag * a; vy[i] = vmag * b; vz[i] = vmag * c; }
    }
    return m;
}

} // extern "C"
