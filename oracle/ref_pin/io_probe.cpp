// Test infrastructure: exposes the reference's own particle-file reader and h.txt writer
// (include/io.hpp, compiled where it lies) through a C-ABI, so the golden-fixture
// script can record what the reference parses from a file and what it writes.
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "io.hpp"

extern "C" {

// Reads path; fills n, pmass and, when xyzh is not null, xyzh (x[n] y[n] z[n] h[n]).
// Returns 0, or -1 with the reader's message in err.
int ref_read_particles(const char* path, int* n, double* pmass, double* xyzh, char* err, int errlen)
{
    try
    {
        const io::ParticleData pd = io::readCosmoFile(path);
        *n = pd.ngas;
        *pmass = pd.pmass;
        if (xyzh)
        {
            const size_t m = size_t(pd.ngas);
            std::memcpy(xyzh, pd.x.data(), m * sizeof(double));
            std::memcpy(xyzh + m, pd.y.data(), m * sizeof(double));
            std::memcpy(xyzh + 2 * m, pd.z.data(), m * sizeof(double));
            std::memcpy(xyzh + 3 * m, pd.h.data(), m * sizeof(double));
        }
        return 0;
    }
    catch (const std::exception& e)
    {
        if (err && errlen > 0)
        {
            std::strncpy(err, e.what(), size_t(errlen) - 1);
            err[errlen - 1] = '\0';
        }
        return -1;
    }
}

// Writes h (n values) with the reference's h.txt writer.
int ref_write_h(const char* path, int n, const double* h)
{
    try
    {
        io::writeH(path, std::vector<double>(h, h + n));
        return 0;
    }
    catch (const std::exception&)
    {
        return -1;
    }
}

} // extern "C"
