// A recording stand-in for the library the reference's driver (src/main.cu) links.
// It implements the calls the driver makes -- cosmo_arrays_init, cosmo_upload,
// cosmo_download and solveDensH -- and writes what the driver uploads (positions and
// h, after its lattice generator and optional jiggle) to the file named by the
// environment variable COSMO_CAPTURE, as raw float64: n, pmass, x[n], y[n], z[n], h[n].
// Nothing is solved; the downloads return the uploaded h and zeros.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "arrays.hpp"
#include "density.hpp"

static int gN = 0;
static std::vector<double> gPos, gH;
static int gSolves = 0;

extern "C" void cosmo_arrays_init(int n) { gN = n; }
extern "C" int cosmo_slot_ncomp(int slot) { return slot == COSMO_POS ? 3 : 1; }
extern "C" void cosmo_upload(int slot, const double* host, int n)
{
    if (slot == COSMO_POS) gPos.assign(host, host + 3 * (size_t)n);
    if (slot == COSMO_HSML) gH.assign(host, host + (size_t)n);
}
extern "C" void cosmo_upload_sorted(int, const double*, int) {}
extern "C" void cosmo_download(int slot, double* host, int n)
{
    for (int i = 0; i < n; ++i) host[i] = (slot == COSMO_HSML) ? gH[i] : 0.0;
    if (slot == COSMO_DENS_OUT)
        for (int i = 0; i < 2 * n; ++i) host[i] = 0.0;
}
extern "C" void cosmo_pin_host(void*, std::size_t) {}
extern "C" void cosmo_unpin_host(void*) {}
extern "C" double cosmo_kernel_radius(void) { return 2.0; }

DensTimings solveDensH(int n, double pmass, KernelMode mode, bool, const double*, double, double)
{
    // The driver solves three times on the same input (warm-up, flat, warp-per-leaf);
    // the first is recorded.
    if (gSolves++ == 0)
    {
        if (const char* path = std::getenv("COSMO_CAPTURE"))
        {
            if (std::FILE* f = std::fopen(path, "wb"))
            {
                const double hdr[2] = {double(n), pmass};
                std::fwrite(hdr, sizeof(double), 2, f);
                std::fwrite(gPos.data(), sizeof(double), gPos.size(), f);
                std::fwrite(gH.data(), sizeof(double), gH.size(), f);
                std::fclose(f);
            }
        }
    }
    DensTimings t{};
    t.kernelMode = mode;
    t.nParticles = n;
    return t;
}
