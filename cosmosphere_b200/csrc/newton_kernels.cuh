/*
 * newton_kernels.cuh -- the Newton-Raphson kernels of the single-set density solve
 * (the reference's src/density_base.cu:237-334): the group-engine iteration over work
 * items, the r^2 Newton rows and the row iterations.
 *
 * Included by density.cu, which instantiates the plain FP64 form (built with -fmad=false,
 * for bit parity with the oracle), and by density_mixed.cu, which instantiates the mixed
 * form (built with contraction into fused multiply-adds; nothing there is bit-compared).
 */
#pragma once

#include <type_traits>

#include "pairstream.cuh"
#include "state.hpp"
#include "workitems.cuh"
#include "densengine.cuh"
#include "rows.cuh"

namespace cosmo {
namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kThreads = 32 * kWarpsPerBlock;

constexpr double kListMargin = 1.15;            // gather-radius widening of the Newton lists
// Newton rows: each still-active particle's j within kRowMargin of its support at its h
// after an update, built once, after the first update that leaves at least 80% of the
// still-active particles settling (moved by less than kSettle), for the iterations after
// it; while fewer settle, too many rows would go stale before use.
constexpr double kRowMargin = 1.1;
constexpr double kSettle = 0.15;

// Newton-Raphson step of one particle from its un-normalised sums (src/density_base.cu:
// 294-333): rho, d(rho)/dh, the new h (clamped to +-20%) and whether |dh/h| < tolh.
// Returns true while the particle stays unconverged.
__device__ __forceinline__ bool newton_step(double rhoi, double gradhi, double hi, double pmass, double hfact,
                                           double tolh, double& rhoOut, double& gradOut, double& hOut, int& conv)
{
    const double hi1 = 1.0 / hi;
    const double hi31 = hi1 * hi1 * hi1;
    const double hi41 = hi31 * hi1;
    const double rho_i = rhoi * kCnormk * pmass * hi31;
    const double grad_i = gradhi * kCnormk * pmass * hi41;
    if (!(rho_i > 0.0))
    {
        rhoOut = 0.0;
        gradOut = 0.0;
        hOut = hi;
        conv = 0;
        return true;
    }
    const double rhoh_i = pmass * (hfact * hi1) * (hfact * hi1) * (hfact * hi1);
    const double funci = rhoh_i - rho_i;
    const double dhdrhoi = -hi / (3.0 * rhoh_i);
    const double omegai = 1.0 - dhdrhoi * grad_i;
    const double safe = (omegai > 0.0) ? omegai : fabs(omegai + 1e-300);
    const double hraw = hi - funci * dhdrhoi / safe;
    double hnew;
    if (hraw > 1.2 * hi) hnew = 1.2 * hi;
    else if (hraw < 0.8 * hi) hnew = 0.8 * hi;
    else hnew = hraw;
    rhoOut = rho_i;
    gradOut = grad_i;
    hOut = hnew;
    conv = (fabs((hnew - hi) / hi) < tolh) ? 1 : 0;
    return !conv;
}

// One Newton iteration over the work items, taken dynamically by a persistent grid of
// warps: each item's group sums come from density_group (plain FP64, bit for bit the
// oracle's; or mixed), then the FP64 Newton-Raphson step of src/density_base.cu:294-333.
// A warp whose group keeps an unconverged particle queues the leaf for the next
// iteration (once per leaf), and flags the lists stale when an updated h outgrows the
// radius its leaf's list covers.
// One Newton iteration over the work items, taken dynamically by a persistent grid of
// warps: each item's group sums come from density_group (plain FP64, bit for bit the
// oracle's; or mixed), then the FP64 Newton-Raphson step of src/density_base.cu:294-333.
// A warp whose group keeps an unconverged particle queues the leaf for the next
// iteration (once per leaf), and flags the lists stale when an updated h outgrows the
// radius its leaf's list covers.  Staged: the group's j-stream is staged into shared
// memory by bulk copies (the WarpStage of its warp) instead of loaded directly.
template<bool Periodic, bool Mixed, bool Staged>
__global__ void __launch_bounds__(kThreads, Mixed ? 6 : 5)
density_nr_kernel(const int4* __restrict__ items, int cap, const uint32_t* __restrict__ layout,
                  const uint32_t* __restrict__ jOffset, const uint32_t* __restrict__ jcount,
                  const int* __restrict__ jlist, double4* __restrict__ xyzh, double* __restrict__ rho,
                  double* __restrict__ gradh, int* __restrict__ converged, double pmass, double tolh,
                  double hfact, const DevBox* __restrict__ box, const double* __restrict__ listH,
                  int* __restrict__ leafNext, int* __restrict__ nextLeaves, PreorderTree tree,
                  const int* __restrict__ leafToInternal, const double* __restrict__ centers,
                  const double* __restrict__ sizes, DevScalars* __restrict__ ds, long long waitNs)
{
    __shared__ __align__(16) unsigned char sScr[kWarpsPerBlock][DensScratch<Mixed>::kBytes];
    __shared__ __align__(128) WarpStage sStage[Staged ? kWarpsPerBlock : 1];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    if constexpr (Staged) stage_init(sStage[wib]);
    double lx = 0, ly = 0, lz = 0;
    if (Periodic) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }
    // lists that outgrew their storage in a graph-run loop are incomplete: the solve is
    // redone on the host loop, so nothing reads them
    if (ds->err & kErrListFull) return;
    const int nHeavy = ds->itemsHeavy, nItems = nHeavy + ds->itemsLight;
    unsigned long long pairs = 0, cand = 0;

    for (;;)
    {
        const int w = next_item(ds, nHeavy, nItems, cap);
        if (w < 0) break;
        const Item d = decode_item(items[w], layout);
        const int leaf = d.leaf;
        const int slot = group_slot(d.m0, d.m1, d.nAct, d.grp, d.G, lane);
        const bool mine = slot >= 0;
        const uint32_t i = d.g0 + uint32_t(mine ? slot : 0);
        const double4 pi = xyzh[i];
        const double hi = pi.w;
        double rhoi, gradhi;
        unsigned int gp, gc;
        // a cut group (its leaf's list streams far more than it needs) scans the tree for
        // its own box instead, within the region its leaf's list covers
        auto src = list_source(jlist, jOffset[leaf], jcount[leaf], LayoutRanges{layout}, xyzh);
        if constexpr (Staged) src.stage = StageRef{&sStage[wib], &ds->err, waitNs};   // bulk-copy staging
        if (w < nHeavy)
        {
            const int in = leafToInternal[leaf];
            const double ext = kRadKernel * listH[leaf];
            src.walk = true;
            src.tree = tree;
            src.rc = make_double3(centers[3 * in], centers[3 * in + 1], centers[3 * in + 2]);
            src.re = make_double3(sizes[3 * in] + ext, sizes[3 * in + 1] + ext, sizes[3 * in + 2] + ext);
        }
        density_group<Periodic, Mixed, Staged>(sScr[wib], mine, d.ng, pi, lx, ly, lz, src, rhoi, gradhi, gp, gc);
        bool stillActive = false, settle = false;
        if (mine)
        {
            pairs += gp;
            cand += gc;
            double ro, go, ho;
            int conv;
            stillActive = newton_step(rhoi, gradhi, hi, pmass, hfact, tolh, ro, go, ho, conv);
            rho[i] = ro;
            gradh[i] = go;
            reinterpret_cast<double*>(xyzh + i)[3] = ho;
            converged[i] = conv;
            if (stillActive && ho > listH[leaf]) ds->listStale = 1;
            settle = stillActive && fabs(ho - hi) < kSettle * hi;
        }
        const uint32_t still = __ballot_sync(0xffffffffu, stillActive);
        const uint32_t settled = __ballot_sync(0xffffffffu, settle);
        if (still && lane == 0)
        {
            atomicAdd(&ds->settling, __popc(settled));
            atomicAdd(&ds->unconverged, __popc(still));
            if (atomicExch(&leafNext[leaf], 1) == 0) nextLeaves[atomicAdd(&ds->nextActive, 1)] = leaf;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
        cand += __shfl_xor_sync(0xffffffffu, cand, o);
    }
    if (lane == 0)
    {
        atomicAdd(&ds->pairs[0], pairs);
        atomicAdd(&ds->pairs[3], cand);
    }
}

// Newton rows of the still-active particles at their current h: r^2 of every j within
// kRowMargin of the particle's support, in ascending j.  A row is complete while the
// particle's h stays within kRowMargin of the h it was built at and within the radius its
// leaf's list covers; rowH records that bound.  With rowsJ given, each row's j are also
// written (flat, beside the r^2), so that at the converged h the symmetric rows of the
// gradient and force passes can be taken from them.

template<bool Periodic, bool Mixed>
__global__ void __launch_bounds__(kThreads)
newton_rows_kernel(const int4* __restrict__ items, int cap, const uint32_t* __restrict__ layout,
                   const uint32_t* __restrict__ jOffset, const uint32_t* __restrict__ jcount,
                   const int* __restrict__ jlist, const double4* __restrict__ xyzh, const DevBox* __restrict__ box,
                   const double* __restrict__ listH, void* __restrict__ rowsR2, int* __restrict__ nblCount,
                   double* __restrict__ rowH, DevScalars* __restrict__ ds, int* __restrict__ rowsJ)
{
    using R2 = typename std::conditional<Mixed, float, double>::type;   // FP32 rows in the mixed form
    R2* nblR2 = static_cast<R2*>(rowsR2);
    __shared__ __align__(16) unsigned char sScr[kWarpsPerBlock][kRowsScratch];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double lx = 0, ly = 0, lz = 0;
    if (Periodic) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }
    // lists that outgrew their storage in a graph-run loop are incomplete: the solve is
    // redone on the host loop, so nothing reads them
    if (ds->err & kErrListFull) return;
    // the index rows are written when the solve asks for them (a flag, so that a graph
    // captured with the buffer serves solves that do and solves that do not)
    if (!ds->rowsJOn) rowsJ = nullptr;
    const int nHeavy = ds->itemsHeavy, nItems = nHeavy + ds->itemsLight;
    const double wide2 = kRadK2 * (kRowMargin * kRowMargin);
    for (;;)
    {
        const int w = next_item(ds, nHeavy, nItems, cap);
        if (w < 0) break;
        const Item d = decode_item(items[w], layout);
        const int slot = group_slot(d.m0, d.m1, d.nAct, d.grp, d.G, lane);
        const bool mine = slot >= 0;
        const uint32_t i = d.g0 + uint32_t(mine ? slot : 0);
        if (w < nHeavy)
        {
            // a cut group's leaf streams far more than a row holds: it keeps the group path
            if (mine) nblCount[i] = kNbl + 1;
            continue;
        }
        const double4 pi = xyzh[i];
        const double hinv2 = 1.0 / (pi.w * pi.w);
        const double rs = kRadKernel * kRowMargin * pi.w;
        const double rmax = warp_max(mine ? rs : 0.0);
        const GroupBox bx = group_box(mine, pi.x, pi.y, pi.z, rs, rmax);
        int rowLen = 0;
        rows_group<1, Periodic>(sScr[wib], mine, d.ng, make_double4(pi.x, pi.y, pi.z, hinv2), rs, bx, lx, ly, lz,
                   jOffset[d.leaf], jcount[d.leaf], jlist, LayoutRanges{layout}, xyzh,
                   [&](const double4& pj) { return in_gather_box<Periodic>(pj, bx, lx, ly, lz); },
                   [](const double4&) { return 0.0; },
                   [&](const double4& g, const double4& pj, int) {   // r^2 within the wide support
                       double dx = g.x - pj.x, dy = g.y - pj.y, dz = g.z - pj.z;
                       nearest_image<Periodic>(dx, dy, dz, lx, ly, lz);
                       const double r2 = pair_r2(dx, dy, dz);
                       return RowEntry<R2>{r2 * g.w < wide2, R2(r2)};
                   },
                   mine ? row_flat(nblR2, uint32_t(i)) : nullptr, rowLen,
                   mine && rowsJ ? row_flat(rowsJ, uint32_t(i)) : nullptr);
        if (mine)
        {
            nblCount[i] = rowLen;
            rowH[i] = fmin(kRowMargin * pi.w, listH[d.leaf]) * (1.0 - 1e-12);
        }
    }
}

// One Newton iteration for the particles whose rows are complete for their h: one lane
// per particle over its row (ascending j), the exact test and the sums in the row's
// order -- the group path's pairs and order, so the plain results agree with it bit for
// bit; mixed: the mixed pair arithmetic on FP64 separations rounded to FP32, Kahan sums.
template<bool Periodic, bool Mixed>
__global__ void __launch_bounds__(kThreads)
density_row_kernel(const int* __restrict__ rowItems, const void* __restrict__ rowsR2, const int* __restrict__ nblCount,
                   double4* __restrict__ xyzh, double* __restrict__ rho, double* __restrict__ gradh,
                   int* __restrict__ converged, double pmass, double tolh, double hfact,
                   const DevBox* __restrict__ box, const double* __restrict__ listH,
                   const int* __restrict__ particleLeaf, int* __restrict__ leafNext, int* __restrict__ nextLeaves,
                   DevScalars* __restrict__ ds)
{
    const int n = ds->rowParticles;
    const int lane = threadIdx.x & 31;
    unsigned long long pairs = 0;
    for (int t0 = blockIdx.x * blockDim.x; t0 < n; t0 += gridDim.x * blockDim.x)
    {
        const int t = t0 + threadIdx.x;
        bool stillActive = false;
        int leaf = 0;
        if (t < n)
        {
            const int i = rowItems[t];
            const double4 pi = xyzh[i];
            const double hi = pi.w;
            const double hinv2 = 1.0 / (hi * hi);
            const float hinv2f = float(hinv2);
            const int cnt = nblCount[i];
            using R2 = typename std::conditional<Mixed, float, double>::type;
            const R2* row = row_flat(static_cast<const R2*>(rowsR2), uint32_t(i));
            double sr = 0.0, sg = 0.0;
            KahanF kr, kg;
            unsigned int gp = 0;
            auto pair = [&](R2 r2) {
                const double q2 = double(r2) * hinv2;
                if (!(q2 < kRadK2)) return;
                ++gp;
                if constexpr (!Mixed)
                {
                    const double q = sqrt(q2);
                    double wk, dwk;
                    sph_kernel(q2, q, wk, dwk);
                    sr += wk;
                    sg += -q * dwk - 3.0 * wk;
                }
                else
                {
                    const float q2f = float(r2) * hinv2f;
                    const float q = sqrt_q(q2f);
                    float wk, dwk;
                    sph_kernel_f(q2f, q, wk, dwk);
                    kr.add(wk);
                    kg.add(fmaf(-q, dwk, -3.0f * wk));
                }
            };
            for_flat_row(row, cnt, pair);
            if constexpr (Mixed) { sr = kr.value(); sg = kg.value(); }
            pairs += gp;
            double ro, go, ho;
            int conv;
            stillActive = newton_step(sr, sg, hi, pmass, hfact, tolh, ro, go, ho, conv);
            rho[i] = ro;
            gradh[i] = go;
            reinterpret_cast<double*>(xyzh + i)[3] = ho;
            converged[i] = conv;
            leaf = particleLeaf[i];
            if (stillActive && ho > listH[leaf]) ds->listStale = 1;
        }
        const uint32_t still = __ballot_sync(0xffffffffu, stillActive);
        if (still && lane == 0) atomicAdd(&ds->unconverged, __popc(still));
        if (stillActive && atomicExch(&leafNext[leaf], 1) == 0) nextLeaves[atomicAdd(&ds->nextActive, 1)] = leaf;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if (lane == 0) atomicAdd(&ds->pairs[0], pairs);
}

} // namespace

// The three Newton kernels share one signature per kind whatever the form.
using NrKernelFn = decltype(&density_nr_kernel<false, false, false>);
using RowsKernelFn = decltype(&newton_rows_kernel<false, false>);
using RowKernelFn = decltype(&density_row_kernel<false, false>);

// The mixed form's kernels, compiled in density_mixed.cu.
NrKernelFn mixed_density_nr_kernel(bool periodic, bool staged);
RowsKernelFn mixed_newton_rows_kernel(bool periodic);
RowKernelFn mixed_density_row_kernel(bool periodic);

} // namespace cosmo
