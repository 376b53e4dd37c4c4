/*
 * noalloc.cu -- Hilbert keys and their sort order for callers that cannot allocate
 * device memory.
 *
 * Who needs this: a caller that reserves its whole device-memory budget when it starts
 * and treats any later allocation as a failure (a long simulation run under a fixed
 * memory cap), and a caller that keeps its own GPU work in flight while it calls us --
 * cudaMalloc and cudaFree synchronise the whole device, which stalls that work.  The
 * regular entry points size their buffers on first use (cosmo_arrays_init and the
 * density solve grow persistent allocations); this one allocates nothing.
 *
 * Its scratch is one file-scope device array of fixed size, g_noallocScratch below,
 * which every GPU that loads the library holds until the process exits.  Host code
 * cannot use the array's name as a device address (on the host it names a stand-in
 * object), so the address is looked up once per device, with that device current, by
 * cudaGetSymbolAddress, on the first call made on that device; make that first call
 * before any stream capture.
 */
#include <cstdio>

#include "state.hpp"
#include "../../include/cosmosphere.h"

namespace cosmo {

size_t keysort_scratch_bytes(int n);
int keysort_raw(int n, const double* x, const double* y, const double* z, const double* h,
                const double* periodicBox, uint64_t* keysOut, int* orderOut, void* scratch, int numSMs,
                cudaStream_t st);

namespace {

// Largest particle count the fixed scratch serves, and the scratch itself (7.06 MiB:
// the sort's key/index ping-pong partners, its look-back flags and histograms, the
// bounding-box partials).
constexpr int kNoallocMaxN = 1 << 19;
constexpr size_t kNoallocScratchBytes = (size_t(7) << 20) + (size_t(64) << 10);

static __device__ __align__(256) unsigned char g_noallocScratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratchAddr[kMaxDevices] = {};
int g_numSMs[kMaxDevices] = {};

// Per-device set-up: resolve the array's device address with that device current.
int scratch_for_current_device(void** addr, int* sms)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    {
        std::fprintf(stderr, "cosmo_hilbert_order_noalloc: no usable current device\n");
        return -2;
    }
    if (!g_scratchAddr[dev])
    {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noallocScratch);
        if (e != cudaSuccess || p == nullptr)
        {
            std::fprintf(stderr, "cosmo_hilbert_order_noalloc: cudaGetSymbolAddress failed: %s\n",
                         cudaGetErrorString(e));
            return -2;
        }
        int sm = 0;
        if (cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -2;
        g_numSMs[dev] = sm;
        g_scratchAddr[dev] = p;
    }
    *addr = g_scratchAddr[dev];
    *sms = g_numSMs[dev];
    return 0;
}

} // namespace
} // namespace cosmo

extern "C" int cosmo_hilbert_order_noalloc(int n, const double* d_x, const double* d_y, const double* d_z,
                                           const double* d_h, int periodic, const double* box6,
                                           unsigned long long* d_keys, int* d_order)
{
    using namespace cosmo;
    if (n < 1 || n > kNoallocMaxN || keysort_scratch_bytes(n) > kNoallocScratchBytes)
    {
        std::fprintf(stderr,
                     "cosmo_hilbert_order_noalloc: n=%d is outside [1, %d], the most its fixed %zu-byte "
                     "scratch serves\n",
                     n, kNoallocMaxN, kNoallocScratchBytes);
        return -1;
    }
    if (periodic && box6 == nullptr)
    {
        std::fprintf(stderr, "cosmo_hilbert_order_noalloc: periodic=%d needs box6 (xmin,xmax,ymin,ymax,zmin,zmax)\n",
                     periodic);
        return -1;
    }
    // An error left pending by the caller's own earlier CUDA calls is not this call's to
    // report or to clear: refuse before launching, and leave it in place.
    if (const cudaError_t pending = cudaPeekAtLastError(); pending != cudaSuccess)
    {
        std::fprintf(stderr, "cosmo_hilbert_order_noalloc: a CUDA error is pending from before this call (%s)\n",
                     cudaGetErrorString(pending));
        return -2;
    }
    void* scratch = nullptr;
    int sms = 0;
    if (const int e = scratch_for_current_device(&scratch, &sms)) return e;
    // The calling thread's default stream: it does not wait for, or hold up, work on the
    // caller's other streams (the legacy default stream would serialise with them).
    return keysort_raw(n, d_x, d_y, d_z, d_h, periodic ? box6 : nullptr, reinterpret_cast<uint64_t*>(d_keys),
                       d_order, scratch, sms, cudaStreamPerThread);
}
