/*
 * rows.cuh -- neighbour rows: each particle's accepted j, in ascending order, written once
 * by a group pass so that the heavy pair passes run with one lane per particle.
 *
 * The group pass streams a leaf's list through the group filter into the warp's ring and
 * tests each batch with j on the lanes (for each group particle in turn, every lane tests
 * its candidate with a conservative FP32 prefilter); the ballot of a group particle's
 * tests is its lane's mask over the batch, and the owner lane applies the exact FP64 test
 * to the masked j, lowest lane first, and appends the accepted ones -- ascending j.  A
 * pass that then walks a row applies the same exact test to the same candidates in the
 * same order as a walk of the whole list would, so its sums are the same bit for bit.
 *
 * An entry is j (the symmetric rows of the gradient and force passes), or r^2 of the pair
 * (the Newton rows: positions do not move during a density solve, so the later Newton
 * iterations need only r^2 and h_i, and read no j data at all).  The Newton rows are flat
 * (kNbl consecutive entries per particle, FP64, or FP32 in the mixed form): their reader
 * streams its own row 16-32 bytes at a time, so the sectors it touches hold only its own
 * entries whichever particles share its warp.
 *
 * Row layout: kNbl entries per particle, interleaved over blocks of 32 particles -- entry
 * k of particle i at nbl[(i / 32) * 32 kNbl + 32 k + i % 32] -- so that the lanes of a warp
 * over 32 consecutive particles read entry k of all their rows from one 128-byte line.  A
 * count above kNbl marks a row that overflowed, whose particle keeps the group path.
 */
#pragma once

#include <type_traits>

#include "pairstream.cuh"

namespace cosmo {

constexpr int kNbl = kQuintic ? 256 : 128;
constexpr int kRowStride = 32;   // distance between consecutive entries of one row

// Entries the row buffer of n particles holds.
inline size_t row_buffer_entries(size_t n) { return ((n + 31) / 32) * size_t(32) * kNbl; }

// Entry 0 of particle i's row; entry k is at [k * kRowStride].
template<class T>
__device__ __forceinline__ T* row_of(T* nbl, uint32_t i)
{
    return nbl + (size_t(i >> 5) * kNbl << 5) + (i & 31u);
}

// An exact test's verdict on a pair and the entry an accepted pair writes.
template<class T>
struct RowEntry
{
    bool ok;
    T v;
};

// Four consecutive j of a flat row in one vector store (the row's first entry and every
// fourth are aligned to four entries).
__device__ __forceinline__ void store4(int* p, int a, int b, int c, int d)
{
    *reinterpret_cast<int4*>(p) = make_int4(a, b, c, d);
}

// Per-warp shared scratch of rows_group: the double ring, its indices, the group's data
// and its FP32 offsets and prefilter bounds.
constexpr int kRowsScratch = kRing * 32 + kRing * 4 + 32 * 32 + 4 * 32 * 4;

// Rows of one group.  Lanes [0, ng) own the group's particles, whose per-particle data gi
// (a double4: position and one test value) the caller passes.  A conservative FP32
// prefilter picks the candidates each particle must test: the pair's float distance
// against fp32_bound2 of max(Bi, candB(pj)), where Bi (the particle's) and candB (the
// candidate's, 0 for a gather row) bound the exact test's distance.  exact(gi, pj, j)
// then applies the exact acceptance of the pair on the FP64 positions and returns it with
// the entry the owner writes for an accepted j (j itself, or r^2).  row is the lane's own row
// (row_of with Stride kRowStride, or row_flat with Stride 1; nullptr if not mine); rowLen
// receives its length (kNbl + 1 when it overflowed).  Entries come in ascending j.  rowJ,
// when given (the lane's own row in a second buffer of the same layout), receives each
// accepted j beside the entry, so that a row of r^2 is also a row of neighbour indices.
// Prefilter = false: no FP32 prefilter; every lane applies exact(gi of particle k, its
// candidate, j) in lockstep over the group particles, and the ballots are the masks (the
// symmetric rows, whose candidate-dependent bound makes the prefilter pass most pairs).
template<int Stride, bool Periodic, bool Prefilter = true, class T, class Ranges, class Filter, class CandB,
         class Exact>
__device__ __forceinline__ void rows_group(unsigned char* scr, bool mine, int ng, const double4& gi, double Bi,
                                           const GroupBox& bx, double lx, double ly, double lz, uint32_t jb,
                                           uint32_t nj, const int* __restrict__ jlist, Ranges ranges,
                                           const double4* __restrict__ xyzh, Filter filter, CandB candB, Exact exact,
                                           T* row, int& rowLen, int* rowJ = nullptr)
{
    const int lane = threadIdx.x & 31;
    double4* ring = reinterpret_cast<double4*>(scr);
    int* ringIdx = reinterpret_cast<int*>(ring + kRing);
    double4* grp = reinterpret_cast<double4*>(ringIdx + kRing);
    float* gfx = reinterpret_cast<float*>(grp + 32);
    float* gfy = gfx + 32;
    float* gfz = gfy + 32;
    float* gfT = gfz + 32;
    const double eps = fp32_margin(bx, Periodic ? fmax(lx, fmax(ly, lz)) : 0.0);
    if (mine) grp[lane] = gi;
    gfx[lane] = mine ? float(gi.x - bx.cx) : 0.0f;
    gfy[lane] = mine ? float(gi.y - bx.cy) : 0.0f;
    gfz[lane] = mine ? float(gi.z - bx.cz) : 0.0f;
    gfT[lane] = mine ? fp32_bound2(Bi, eps) : -1.0f;
    __syncwarp();
    const float Lx = float(lx), Ly = float(ly), Lz = float(lz);
    int len = 0;
    int k0 = 0, k1 = 0, k2 = 0, k3 = 0;   // a flat row's last four j, not yet written
    stream_ranges<true, false, true>(
        ring, nullptr, ringIdx, bx.cx, bx.cy, bx.cz, 0.0, 0.0, 0.0, jb, nj, jlist, ranges, xyzh, filter,
        [&](const double4* rg, const float4*, const int* ri, int head, int count) {
            const int mySlot = (head + (lane < count ? lane : 0)) & (kRing - 1);
            const double4 pj = rg[mySlot];
            if constexpr (!Prefilter)
            {
                uint32_t mask = 0;
                for (int i0 = 0; i0 < ng; i0 += 4)
                {
                    bool a[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        a[u] = lane < count && i0 + u < ng && exact(grp[min(i0 + u, 31)], pj, ri[mySlot]).ok;
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                    {
                        const uint32_t m = __ballot_sync(0xffffffffu, a[u]);
                        if (lane == i0 + u) mask = m;
                    }
                }
                while (mask)
                {
                    const int b = __ffs(mask) - 1;
                    mask &= mask - 1;
                    const int sl = (head + b) & (kRing - 1);
                    if (len < kNbl)
                    {
                        if constexpr (std::is_same<T, int>::value) row[size_t(len) * Stride] = ri[sl];   // j itself
                        else row[size_t(len) * Stride] = exact(gi, rg[sl], ri[sl]).v;
                        if (rowJ) rowJ[size_t(len) * Stride] = ri[sl];
                    }
                    ++len;
                }
                return;
            }
            const float px = float(image_offset(pj.x, bx.cx, lx)), py = float(image_offset(pj.y, bx.cy, ly));
            const float pz = float(image_offset(pj.z, bx.cz, lz));
            const double bj = candB(pj);
            const float tj = bj > 0.0 ? fp32_bound2(bj, eps) : 0.0f;
            const float2 nx = make_float2(-px, -px), ny = make_float2(-py, -py), nz = make_float2(-pz, -pz);
            uint32_t myMask = 0;
            for (int i0 = 0; i0 < ng; i0 += 4)
            {
                float r2u[4];
                if (!Periodic || Lx == 0.0f)
                {
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                    {
                        const int k = i0 + 2 * h;
                        const float2 dx = __fadd2_rn(*reinterpret_cast<const float2*>(gfx + k), nx);
                        const float2 dy = __fadd2_rn(*reinterpret_cast<const float2*>(gfy + k), ny);
                        const float2 dz = __fadd2_rn(*reinterpret_cast<const float2*>(gfz + k), nz);
                        float2 r2 = __fmul2_rn(dx, dx);
                        r2 = __ffma2_rn(dy, dy, r2);
                        r2 = __ffma2_rn(dz, dz, r2);
                        r2u[2 * h] = r2.x;
                        r2u[2 * h + 1] = r2.y;
                    }
                }
                else
                {
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                    {
                        const int k = i0 + u;
                        const float dx = axis_df<true>(gfx[k], px, Lx);
                        const float dy = axis_df<true>(gfy[k], py, Ly);
                        const float dz = axis_df<true>(gfz[k], pz, Lz);
                        r2u[u] = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                {
                    const bool a = lane < count && i0 + u < ng && r2u[u] < fmaxf(gfT[i0 + u], tj);
                    const uint32_t m = __ballot_sync(0xffffffffu, a);
                    if (lane == i0 + u) myMask = m;
                }
            }
            // the owner tests its prefiltered candidates exactly, lowest lane (j) first
            while (myMask)
            {
                const int b = __ffs(myMask) - 1;
                myMask &= myMask - 1;
                const int sl = (head + b) & (kRing - 1);
                const RowEntry<T> e = exact(gi, rg[sl], ri[sl]);
                if (e.ok)
                {
                    if constexpr (Stride == 1)
                    {
                        // a flat row: the entry stored at once; its j (when asked for) kept
                        // with the last three in registers and written as one vector store
                        // when the fourth arrives
                        if (len < kNbl) row[len] = e.v;
                        if (rowJ)
                        {
                            k0 = k1; k1 = k2; k2 = k3; k3 = ri[sl];
                            if ((len & 3) == 3 && len < kNbl) store4(rowJ + (len - 3), k0, k1, k2, k3);
                        }
                    }
                    else if (len < kNbl)
                    {
                        row[size_t(len) * Stride] = e.v;
                        if (rowJ) rowJ[size_t(len) * Stride] = ri[sl];
                    }
                    ++len;
                }
            }
        });
    if constexpr (Stride == 1)
    {
        // the last, partial group of four j (its unused slots hold nothing a reader uses)
        const int m = len & 3;
        if (rowJ != nullptr && m != 0 && len < kNbl)
        {
            const int ja = m == 1 ? k3 : (m == 2 ? k2 : k1), jb = m == 1 ? k3 : (m == 2 ? k3 : k2);
            store4(rowJ + (len - m), ja, jb, k3, k3);
        }
    }
    rowLen = len > kNbl ? kNbl + 1 : len;
}

// Entry 0 of particle i's row in the flat layout (kNbl consecutive entries per particle).
template<class T>
__device__ __forceinline__ T* row_flat(T* nbl, uint32_t i)
{
    return nbl + size_t(i) * kNbl;
}

// f(r2) for the cnt entries of a flat row of doubles, in order, 32 bytes per load (the
// rows are 32-byte aligned and kNbl is a multiple of 4, so the last load stays in the row).
template<class F>
__device__ __forceinline__ void for_flat_row(const double* __restrict__ row, int cnt, F&& f)
{
    const double4* r4 = reinterpret_cast<const double4*>(row);
    int k = 0;
    for (; k + 4 <= cnt; k += 4)
    {
        const double4 v = ldg4(r4 + (k >> 2));
        f(v.x); f(v.y); f(v.z); f(v.w);
    }
    if (k < cnt)
    {
        const double4 v = ldg4(r4 + (k >> 2));
        f(v.x);
        if (k + 1 < cnt) f(v.y);
        if (k + 2 < cnt) f(v.z);
    }
}

// The same over a flat row of floats (the mixed form's r^2 rows), 16 bytes per load.
template<class F>
__device__ __forceinline__ void for_flat_row(const float* __restrict__ row, int cnt, F&& f)
{
    const float4* r4 = reinterpret_cast<const float4*>(row);
    int k = 0;
    for (; k + 4 <= cnt; k += 4)
    {
        const float4 v = __ldg(r4 + (k >> 2));
        f(v.x); f(v.y); f(v.z); f(v.w);
    }
    if (k < cnt)
    {
        const float4 v = __ldg(r4 + (k >> 2));
        f(v.x);
        if (k + 1 < cnt) f(v.y);
        if (k + 2 < cnt) f(v.z);
    }
}

// f(entry) for the cnt entries of a row (row_of), in order, four loads ahead of their use.
template<class T, class F>
__device__ __forceinline__ void for_row(const T* __restrict__ row, int cnt, F&& f)
{
    int k = 0;
    for (; k + 4 <= cnt; k += 4)
    {
        const T a = __ldg(row + size_t(k) * kRowStride), b = __ldg(row + size_t(k + 1) * kRowStride);
        const T c = __ldg(row + size_t(k + 2) * kRowStride), d = __ldg(row + size_t(k + 3) * kRowStride);
        f(a); f(b); f(c); f(d);
    }
    for (; k < cnt; ++k) f(__ldg(row + size_t(k) * kRowStride));
}

// Whether particle i's row is usable (written and not overflowed).
__device__ __forceinline__ bool row_ok(const int* __restrict__ nblCount, uint32_t i)
{
    return unsigned(nblCount[i]) <= unsigned(kNbl);
}

} // namespace cosmo
