/*
 * common.cuh -- constants, the SPH kernel, the Hilbert curve, the device box and the
 * error handling shared by every translation unit of libcosmoSPHere.
 *
 * The plain FP64 path is compiled with -fmad=false: every multiply and add rounds on
 * its own, as the CPU oracle does, except where a kernel writes fma() explicitly (r^2
 * in the pair loops).  That keeps the plain form bit-for-bit equal to the oracle.
 */
#pragma once

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include <cuda_runtime.h>

namespace cosmo {

// Abort the process with a "FATAL:" line, the reference's only error channel
// (src/dens_c_api.cu:60-67, src/density_base.cu:905-911).
[[noreturn]] void fatal(const char* fmt, ...);

#define COSMO_CUDA(call)                                                                   \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            ::cosmo::fatal("CUDA error %s (%s:%d): %s", #call, __FILE__, __LINE__,         \
                           cudaGetErrorString(e_));                                        \
    } while (0)

// Every launch site calls this right after <<<...>>>: it checks the launch and counts it
// (the count is reported by the harness as the number of the library's kernel launches).
extern std::atomic<unsigned long long> g_launches;
#define COSMO_LAUNCHED()                                                                   \
    do {                                                                                   \
        ++::cosmo::g_launches;                                                             \
        COSMO_CUDA(cudaGetLastError());                                                    \
    } while (0)

constexpr int      kMaxLevel = 21;              // 21 bits per axis, 63-bit keys
constexpr uint64_t kKeyEnd   = 1ull << 63;      // one past the largest live key
constexpr uint64_t kDeadKey  = ~0ull;           // h <= 0: sorted to the end (tree.cuh:99-104)
constexpr uint32_t kBucket   = 64;              // leaf capacity, BUCKET_SIZE (tree.cuh:53)
constexpr int kWalkScratch   = 512;             // list entries per leaf a count walk keeps for its fill

inline int iceil(long a, long b) { return int((a + b - 1) / b); }

// --------------------------------------------------------------------------------------
// SPH smoothing kernel (include/kernel.hpp:35-99), fixed at compile time as in the
// reference: -DCOSMO_KERNEL_QUINTIC selects M6, otherwise M4.
// --------------------------------------------------------------------------------------
#ifdef COSMO_KERNEL_QUINTIC
constexpr double kRadKernel = 3.0;
constexpr double kRadK2     = 9.0;
constexpr double kCnormk    = 1.0 / (120.0 * 3.141592653589793);
constexpr double kHfactDefault = 1.0;
constexpr bool   kQuintic   = true;
#else
constexpr double kRadKernel = 2.0;
constexpr double kRadK2     = 4.0;
constexpr double kCnormk    = 1.0 / 3.141592653589793;
constexpr double kHfactDefault = 1.2;
constexpr bool   kQuintic   = false;
#endif

// W(q) and dW/dq, unnormalised (the caller applies cnormk / h^3 and / h^4).
__host__ __device__ inline void sph_kernel(double q2, double q, double& w, double& dw)
{
    if constexpr (kQuintic)
    {
        if (q < 1.0)
        {
            const double q4 = q2 * q2;
            w  = -10.0 * q4 * q + 30.0 * q4 - 60.0 * q2 + 66.0;
            dw = q * (-50.0 * q2 * q + 120.0 * q2 - 120.0);
        }
        else if (q < 2.0)
        {
            const double a = q - 3.0, b = q - 2.0;
            const double a2 = a * a, b2 = b * b;
            w  = -(a2 * a2 * a) + 6.0 * (b2 * b2 * b);
            dw = -5.0 * (a2 * a2) + 30.0 * (b2 * b2);
        }
        else if (q < 3.0)
        {
            const double a = q - 3.0, a2 = a * a;
            w  = -(a2 * a2 * a);
            dw = -5.0 * (a2 * a2);
        }
        else { w = 0.0; dw = 0.0; }
    }
    else
    {
        (void)q2;
        const double a  = (2.0 - q > 0.0) ? (2.0 - q) : 0.0;
        const double b  = (1.0 - q > 0.0) ? (1.0 - q) : 0.0;
        const double a2 = a * a, a3 = a2 * a;
        const double b2 = b * b, b3 = b2 * b;
        w  = 0.25 * (a3 - 4.0 * b3);
        dw = 0.25 * (-3.0 * a2 + 12.0 * b2);
    }
}

// --------------------------------------------------------------------------------------
// Hilbert curve: J. Skilling, "Programming the Hilbert curve", AIP Conf. Proc. 707
// (2004), restated.  Integer arithmetic only, so host and device agree bit for bit.
// An aligned cube of 2^s cells per side is one contiguous key range of length 8^s.
// --------------------------------------------------------------------------------------
__host__ __device__ inline uint64_t hilbert_key(uint32_t ix, uint32_t iy, uint32_t iz)
{
    uint32_t X0 = ix, X1 = iy, X2 = iz;
    for (uint32_t Q = 1u << (kMaxLevel - 1); Q > 1; Q >>= 1)
    {
        const uint32_t P = Q - 1;
        if (X0 & Q) X0 ^= P;
        if (X1 & Q) X0 ^= P;
        else { const uint32_t t = (X0 ^ X1) & P; X0 ^= t; X1 ^= t; }
        if (X2 & Q) X0 ^= P;
        else { const uint32_t t = (X0 ^ X2) & P; X0 ^= t; X2 ^= t; }
    }
    X1 ^= X0;
    X2 ^= X1;
    uint32_t t = 0;
    for (uint32_t Q = 1u << (kMaxLevel - 1); Q > 1; Q >>= 1)
        if (X2 & Q) t ^= Q - 1;
    X0 ^= t; X1 ^= t; X2 ^= t;
    uint64_t key = 0;
#pragma unroll
    for (int b = kMaxLevel - 1; b >= 0; --b)
        key = (key << 3) | (uint64_t((X0 >> b) & 1u) << 2) | (uint64_t((X1 >> b) & 1u) << 1)
                         | uint64_t((X2 >> b) & 1u);
    return key;
}

__host__ __device__ inline void hilbert_cell(uint64_t key, uint32_t& ox, uint32_t& oy, uint32_t& oz)
{
    uint32_t X0 = 0, X1 = 0, X2 = 0;
#pragma unroll
    for (int b = kMaxLevel - 1; b >= 0; --b)
    {
        const uint32_t o = uint32_t(key >> (3 * b)) & 7u;
        X0 |= ((o >> 2) & 1u) << b;
        X1 |= ((o >> 1) & 1u) << b;
        X2 |= (o & 1u) << b;
    }
    const uint32_t N = 2u << (kMaxLevel - 1);
    const uint32_t t = X2 >> 1;
    X2 ^= X1;
    X1 ^= X0;
    X0 ^= t;
    for (uint32_t Q = 2; Q != N; Q <<= 1)
    {
        const uint32_t P = Q - 1;
        if (X2 & Q) X0 ^= P;
        else { const uint32_t s = (X0 ^ X2) & P; X0 ^= s; X2 ^= s; }
        if (X1 & Q) X0 ^= P;
        else { const uint32_t s = (X0 ^ X1) & P; X0 ^= s; X1 ^= s; }
        if (X0 & Q) X0 ^= P;
    }
    ox = X0; oy = X1; oz = X2;
}

// Cornerstone-style node bookkeeping: a node at level L spans 8^(21-L) keys; its
// placeholder-bit prefix sorts level-major, key-minor.
__host__ __device__ inline uint64_t node_range(int level) { return 1ull << (3 * (kMaxLevel - level)); }
__host__ __device__ inline int level_of_range(uint64_t len)
{
#ifdef __CUDA_ARCH__
    return kMaxLevel - (__ffsll((long long)len) - 1) / 3;
#else
    return kMaxLevel - __builtin_ctzll(len) / 3;
#endif
}
__host__ __device__ inline uint64_t encode_prefix(uint64_t start, int level)
{
    return (start >> (3 * (kMaxLevel - level))) | (1ull << (3 * level));
}
__host__ __device__ inline int prefix_level(uint64_t p)
{
#ifdef __CUDA_ARCH__
    return (63 - __clzll((long long)p)) / 3;
#else
    return (63 - __builtin_clzll(p)) / 3;
#endif
}
__host__ __device__ inline uint64_t prefix_start(uint64_t p)
{
    const int L = prefix_level(p);
    return (p ^ (1ull << (3 * L))) << (3 * (kMaxLevel - L));
}

// --------------------------------------------------------------------------------------
// The root box as the kernels see it.  lo/hi are the box; len, scale (2^21/len) and unit
// (len/2^21) are derived on the device with the same operations the oracle uses.
// --------------------------------------------------------------------------------------
struct DevBox
{
    double lo[3], hi[3], len[3], scale[3], unit[3];
    int periodic;
};

__host__ __device__ inline void box_finish(DevBox& b)
{
    for (int d = 0; d < 3; ++d)
    {
        b.len[d]   = b.hi[d] - b.lo[d];
        b.scale[d] = 2097152.0 / b.len[d];
        b.unit[d]  = b.len[d] / 2097152.0;
    }
}

__device__ inline uint32_t quantise(double x, double lo, double scale)
{
    const double v = (x - lo) * scale;
    if (!(v >= 0.0)) return 0u;
    if (v >= 2097151.0) return 2097151u;
    return uint32_t(floor(v));
}

// Nearest periodic image of a pair separation (include/tree.cuh:75-84).
template<bool Periodic>
__device__ __forceinline__ void nearest_image(double& dx, double& dy, double& dz, double lx,
                                              double ly, double lz)
{
    if constexpr (Periodic)
    {
        if (fabs(dx) > 0.5 * lx) dx = dx - lx * copysign(1.0, dx);
        if (fabs(dy) > 0.5 * ly) dy = dy - ly * copysign(1.0, dy);
        if (fabs(dz) > 0.5 * lz) dz = dz - lz * copysign(1.0, dz);
    }
}

// Read-only 32-byte load as two 128-bit loads through the non-coherent path.
__device__ __forceinline__ double4 ldg4(const double4* p)
{
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ double pair_r2(double dx, double dy, double dz)
{
    return fma(dz, dz, fma(dy, dy, dx * dx));
}

// Device error word bits (State::devErr).
enum DevErr : int
{
    kErrSortSpin  = 1,      // radix sort look-back gave up waiting
    kErrListCap   = 2,      // a j-list fill found more entries than its count pass
    kErrStageWait = 4,      // a TMA staging wait gave up
    kErrFlagWait  = 8,      // a wait on a flag another block sets gave up (the wait test hook)
    kErrListFull  = 16,     // a j-list build needed more than the preallocated capacity
};

} // namespace cosmo
