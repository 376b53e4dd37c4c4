/*
 * sort.cuh -- scans and the onesweep LSD radix sort shared by the single-set and the
 * batched (forest) tree builds.  Internal-linkage kernels: each translation unit that
 * includes this gets its own copy.
 */
#pragma once

#include "common.cuh"
#include "tma.cuh"

namespace cosmo {
namespace {

constexpr int kBlk = 256;

__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.volatile.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// ------------------------------------------------------------------ scan (3 phase)
constexpr int kScanThreads = 1024;
constexpr int kScanItems   = 4;
constexpr int kScanTile    = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive prefix and
// the block total in *total.
__device__ uint32_t block_excl_scan(uint32_t v, uint32_t* total)
{
    __shared__ uint32_t sw[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    const uint32_t inc = warp_incl_scan(v);
    if (lane == 31) sw[warp] = inc;
    __syncthreads();
    if (warp == 0)
    {
        uint32_t s = lane < nw ? sw[lane] : 0;
        s = warp_incl_scan(s);
        sw[lane] = s;
    }
    __syncthreads();
    const uint32_t before = warp ? sw[warp - 1] : 0;
    *total = sw[nw - 1];
    __syncthreads();
    return before + inc - v;
}

// nPtr (when given): the element count on the device, n then being a bound on it (a scan
// issued before its count is known, as a captured graph does).
__global__ void scan_reduce_kernel(const uint32_t* __restrict__ in, int n, uint32_t* __restrict__ bsum,
                                   const int* __restrict__ nPtr = nullptr)
{
    if (nPtr) n = *nPtr;
    const long base = long(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) s += in[base + k];
    uint32_t tot;
    block_excl_scan(s, &tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void scan_blocks_kernel(uint32_t* bsum, int nb, uint32_t* totalOut, uint32_t* out = nullptr,
                                   const int* __restrict__ nPtr = nullptr)
{
    if (nPtr) totalOut = out + *nPtr;   // the total goes after the last element
    // one block of kScanThreads; nb <= kScanTile
    const int base = threadIdx.x * kScanItems;
    uint32_t v[kScanItems], s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        v[k] = (base + k < nb) ? bsum[base + k] : 0;
        s += v[k];
    }
    uint32_t tot;
    uint32_t run = block_excl_scan(s, &tot);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < nb)
        {
            bsum[base + k] = run;
            run += v[k];
        }
    if (threadIdx.x == 0) *totalOut = tot;
}

__global__ void scan_apply_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int n,
                                  const uint32_t* __restrict__ boff, const int* __restrict__ nPtr = nullptr)
{
    if (nPtr) n = *nPtr;
    const long base = long(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems], s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    uint32_t tot;
    uint32_t run = block_excl_scan(s, &tot) + boff[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n)
        {
            out[base + k] = run;
            run += v[k];
        }
}

// ------------------------------------------------------------------ onesweep radix sort
constexpr int kSortThreads = 256;
constexpr int kSortIpt     = 16;
constexpr int kSortTile    = kSortThreads * kSortIpt;
constexpr int kSortWarps   = kSortThreads / 32;
constexpr int kSortPasses  = 8;
constexpr uint32_t kLbAgg  = 1u << 30, kLbInc = 2u << 30, kLbMask = (1u << 30) - 1;

__global__ void digit_hist_kernel(const uint64_t* __restrict__ keys, int n, uint32_t* __restrict__ hist)
{
    __shared__ uint32_t s[kSortPasses][256];
    for (int i = threadIdx.x; i < kSortPasses * 256; i += blockDim.x) (&s[0][0])[i] = 0;
    __syncthreads();
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
    {
        const uint64_t k = keys[i];
#pragma unroll
        for (int p = 0; p < kSortPasses; ++p) atomicAdd(&s[p][(k >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kSortPasses * 256; i += blockDim.x)
        if ((&s[0][0])[i]) atomicAdd(&hist[i], (&s[0][0])[i]);
}

__global__ void digit_base_kernel(const uint32_t* __restrict__ hist, uint32_t* __restrict__ base)
{
    // block p scans the 256 bins of pass p
    const uint32_t v = hist[blockIdx.x * 256 + threadIdx.x];
    uint32_t tot;
    base[blockIdx.x * 256 + threadIdx.x] = block_excl_scan(v, &tot);
}

// One stable counting pass of an LSD radix sort of (key, value) pairs, single pass per
// digit with decoupled look-back between tiles.  The digit is byte `shift/8` of the key,
// or -- when SetDigit -- of setOf[value] (the set id of the element's original index),
// which turns a finished key sort into a stable (set, key) segmented sort.
template<bool SetDigit>
__device__ __forceinline__ void
onesweep_body(const uint64_t* __restrict__ kin, const int* __restrict__ vin, uint64_t* __restrict__ kout,
                  int* __restrict__ vout, int n, int shift, const uint32_t* __restrict__ binBase,
                  uint32_t* lookback, unsigned int* tileTicket, int* err, const int* __restrict__ setOf,
                  long long waitNs)
{
    __shared__ uint32_t sHist[kSortWarps][256];
    __shared__ uint32_t sBase[256];
    __shared__ int sTile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < kSortWarps * 256; i += kSortThreads) (&sHist[0][0])[i] = 0;
    if (tid == 0) sTile = int(atomicAdd(tileTicket, 1u));
    __syncthreads();
    const int tile = sTile;
    const long base = long(tile) * kSortTile + long(warp) * 32 * kSortIpt;

    uint64_t k[kSortIpt];
    int v[kSortIpt];
    uint32_t rank[kSortIpt];
#pragma unroll
    for (int it = 0; it < kSortIpt; ++it)
    {
        const long idx = base + it * 32 + lane;
        if (idx < n) { k[it] = kin[idx]; v[it] = vin ? vin[idx] : int(idx); }
        else { k[it] = 0; v[it] = 0; }
    }
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int it = 0; it < kSortIpt; ++it)
    {
        const bool valid = (base + it * 32 + lane) < n;
        const uint32_t d = valid ? (SetDigit ? (uint32_t(setOf[v[it]]) >> shift) & 255u
                                             : uint32_t(k[it] >> shift) & 255u)
                                 : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t c = 0;
        if (valid) c = sHist[warp][d];
        __syncwarp();
        rank[it] = c + __popc(peers & lt);
        if (valid && (peers & lt) == 0u) sHist[warp][d] = c + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        const int d = tid;
        uint32_t total = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w)
        {
            const uint32_t c = sHist[w][d];
            sHist[w][d] = total;
            total += c;
        }
        uint32_t* mine = lookback + size_t(tile) * 256 + d;
        if (tile == 0)
        {
            atomicExch(mine, kLbInc | total);
            sBase[d] = binBase[d];
        }
        else
        {
            atomicExch(mine, kLbAgg | total);
            uint32_t excl = 0;
            int p = tile - 1;
            WaitClock clk;
            while (p >= 0)
            {
                const uint32_t s = ld_volatile_u32(lookback + size_t(p) * 256 + d);
                if ((s & ~kLbMask) == 0u)
                {
                    if (clk.over(waitNs)) { atomicOr(err, int(kErrSortSpin)); break; }
                    continue;
                }
                excl += s & kLbMask;
                if (s & kLbInc) break;
                --p;
            }
            atomicExch(mine, kLbInc | (excl + total));
            sBase[d] = binBase[d] + excl;
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kSortIpt; ++it)
    {
        const long idx = base + it * 32 + lane;
        if (idx < n)
        {
            const uint32_t d = SetDigit ? (uint32_t(setOf[v[it]]) >> shift) & 255u : uint32_t(k[it] >> shift) & 255u;
            const uint32_t pos = sBase[d] + sHist[warp][d] + rank[it];
            kout[pos] = k[it];
            vout[pos] = v[it];
        }
    }
}


__global__ void __launch_bounds__(kSortThreads, 3)
onesweep_kernel(const uint64_t* __restrict__ kin, const int* __restrict__ vin, uint64_t* __restrict__ kout,
                int* __restrict__ vout, int n, int shift, const uint32_t* __restrict__ binBase,
                uint32_t* lookback, unsigned int* tileTicket, int* err, long long waitNs)
{
    onesweep_body<false>(kin, vin, kout, vout, n, shift, binBase, lookback, tileTicket, err, nullptr, waitNs);
}

__global__ void __launch_bounds__(kSortThreads)
onesweep_set_kernel(const uint64_t* __restrict__ kin, const int* __restrict__ vin, uint64_t* __restrict__ kout,
                    int* __restrict__ vout, int n, int shift, const uint32_t* __restrict__ binBase,
                    uint32_t* lookback, unsigned int* tileTicket, int* err, const int* __restrict__ setOf,
                    long long waitNs)
{
    onesweep_body<true>(kin, vin, kout, vout, n, shift, binBase, lookback, tileTicket, err, setOf, waitNs);
}

} // namespace
} // namespace cosmo
