/*
 * density.cu -- the Newton-Raphson smoothing-length / density solve and the
 * post-convergence gradient sweep (the reference's src/density_base.cu:237-334, 511-1015).
 *
 * One warp per i-leaf.  The leaf's unconverged particles are packed onto the lanes
 * (ballot + __fns), every lane walks the leaf's j-leaf list in ascending order, so each
 * particle's sums run over j in ascending Hilbert index -- the oracle's order -- and the
 * FP64 results agree with it bit for bit.  Compaction is on the device: a warp whose leaf
 * still holds an unconverged particle appends the leaf to the next iteration's list.
 */
#include <algorithm>

#include "pairstream.cuh"
#include "state.hpp"

namespace cosmo {

namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kThreads = 32 * kWarpsPerBlock;

constexpr int kRec = 256;                       // pair records per warp
constexpr double kListMargin = 1.15;            // gather-radius widening of the Newton lists

// Zero the per-iteration counters of the Newton work queue and the leaf re-queue flags.
__global__ void begin_iteration_kernel(DevScalars* __restrict__ ds, int* __restrict__ leafNext, int nL)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0)
    {
        ds->nextActive = 0;
        ds->unconverged = 0;
        ds->listStale = 0;
        ds->workCounter[0] = 0;
        ds->itemsHeavy = 0;
        ds->itemsLight = 0;
    }
    for (int l = t; l < nL; l += gridDim.x * blockDim.x) leafNext[l] = 0;
}

// Work items of one Newton iteration: every group of a leaf's 64-slot window of
// unconverged particles is one item (leaf, window << 16 | group << 8 | groups, the two
// halves of the window's active mask).  Groups hold up to 32 particles; a leaf whose
// gather list streams more than kSplitStream particles is cut into smaller groups, about
// kSplitWork / stream particles each, so that no single warp carries the iteration's
// tail.  Cut items are queued from the front of the buffer and run first, whole groups
// from the back.  The items of a window hold at most its active particles, so cap = the
// particle count always suffices.
constexpr uint32_t kSplitStream = 4096;
constexpr uint32_t kSplitWork = 32u * 4096u;

__global__ void plan_items_kernel(const int* __restrict__ leaves, int nActive, const uint32_t* __restrict__ layout,
                                  const int* __restrict__ converged, const uint32_t* __restrict__ jstream,
                                  int4* __restrict__ items, int cap, DevScalars* __restrict__ ds)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nWarps = (gridDim.x * blockDim.x) >> 5;
    for (int w = warp; w < nActive; w += nWarps)
    {
        const int leaf = leaves[w];
        const uint32_t p0 = layout[leaf], p1 = layout[leaf + 1];
        const uint32_t S = jstream[leaf];
        const int gsize = S <= kSplitStream ? 32 : max(1, int(kSplitWork / S));
        for (uint32_t g = p0; g < p1; g += 64)
        {
            const uint32_t a0 = g + lane, a1 = g + 32 + lane;
            const uint32_t m0 = __ballot_sync(0xffffffffu, a0 < p1 && converged[a0] == 0);
            const uint32_t m1 = __ballot_sync(0xffffffffu, a1 < p1 && converged[a1] == 0);
            const int nAct = __popc(m0) + __popc(m1);
            if (nAct == 0) continue;
            const int whole = (nAct + 31) >> 5;
            const int G = max(whole, (nAct + gsize - 1) / gsize);
            const bool split = G > whole;
            int base = 0;
            if (lane == 0) base = atomicAdd(split ? &ds->itemsHeavy : &ds->itemsLight, G);
            base = __shfl_sync(0xffffffffu, base, 0);
            const int wnd = int((g - p0) >> 6);
            for (int k = lane; k < G; k += 32)
            {
                const int idx = split ? base + k : cap - 1 - (base + k);
                if (idx >= 0 && idx < cap) items[idx] = make_int4(leaf, (wnd << 16) | (k << 8) | G, int(m0), int(m1));
            }
        }
    }
}

// One Newton iteration over the work items, taken dynamically (a persistent grid).
//
// A warp owns one group of a leaf.  Candidates stream through the group filter into the
// ring (stream_pairs); every batch of up to 32 is then tested with j on the lanes: for each
// group particle in turn, all lanes apply the exact FP64 test q^2 = r^2/h_i^2 < R^2 to their
// candidate, and the accepted pairs are appended, particle-major, to the warp's record
// buffer -- so each particle's records are contiguous and in ascending j.  The records are
// then evaluated with one pair per lane (W, -q dW/dq - 3W), and each particle's owner lane
// adds its own records in order.  Every lane works in all three phases whatever the
// group's size or spatial spread, and each particle's sums still run over j in ascending
// Hilbert index, the oracle's order, so the results agree with it bit for bit.
template<bool Periodic>
__global__ void __launch_bounds__(kThreads, 6)
density_nr_kernel(const int4* __restrict__ items, int cap, const uint32_t* __restrict__ layout,
                  const uint32_t* __restrict__ jOffset, const uint32_t* __restrict__ jcount,
                  const int* __restrict__ jlist, double4* __restrict__ xyzh, double* __restrict__ rho,
                  double* __restrict__ gradh, int* __restrict__ converged, double pmass, double tolh,
                  double hfact, const DevBox* __restrict__ box, const double* __restrict__ listH,
                  int* __restrict__ leafNext, int* __restrict__ nextLeaves, DevScalars* __restrict__ ds)
{
    __shared__ double4 sRing[kWarpsPerBlock][kRing];
    __shared__ double4 sGrp[kWarpsPerBlock][32];
    __shared__ double sRecA[kWarpsPerBlock][kRec];
    __shared__ double sRecB[kWarpsPerBlock][kRec];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    double lx = 0, ly = 0, lz = 0;
    if (Periodic) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }
    const int nHeavy = ds->itemsHeavy, nItems = nHeavy + ds->itemsLight;
    unsigned long long pairs = 0, cand = 0;
    double* recA = sRecA[wib];
    double* recB = sRecB[wib];

    for (;;)
    {
        int w = 0;
        if (lane == 0) w = atomicAdd(&ds->workCounter[0], 1);
        w = __shfl_sync(0xffffffffu, w, 0);
        if (w >= nItems) break;
        const int4 it = items[w < nHeavy ? w : cap - 1 - (w - nHeavy)];
        const int leaf = it.x;
        const int wnd = it.y >> 16, grp = (it.y >> 8) & 255, G = it.y & 255;
        const uint32_t m0 = uint32_t(it.z), m1 = uint32_t(it.w);
        const int nAct = __popc(m0) + __popc(m1);
        const int ng = (grp + 1) * nAct / G - grp * nAct / G;
        const uint32_t g0 = layout[leaf] + 64u * uint32_t(wnd);
        const int slot = group_slot(m0, m1, nAct, grp, G, lane);
        const bool mine = slot >= 0;
        const uint32_t i = g0 + uint32_t(mine ? slot : 0);
        const double4 pi = xyzh[i];
        const double hi = pi.w;
        const double hinv2 = 1.0 / (hi * hi);
        const double rs = kRadKernel * hi;
        const double rmax = warp_max(mine ? rs : 0.0);
        const GroupBox bx = group_box(mine, pi.x, pi.y, pi.z, rs, rmax);
        if (mine) sGrp[wib][lane] = make_double4(pi.x, pi.y, pi.z, hinv2);
        __syncwarp();
        double rhoi = 0.0, gradhi = 0.0;
        unsigned int gp = 0, gc = 0;
        const uint32_t jb = jOffset[leaf], nj = jcount[leaf];
        stream_pairs<false, false>(
            sRing[wib], nullptr, nullptr, bx.cx, bx.cy, bx.cz, jb, nj, jlist, layout, xyzh,
            [&](const double4& pj) { return in_gather_box<Periodic>(pj, bx, lx, ly, lz); },
            [&](const double4* ring, const float4*, const int*, int head, int count) {
                gc += count;
                const double4 pj = ring[(head + (lane < count ? lane : 0)) & (kRing - 1)];
                int nrec = 0, segStart = 0, segCount = 0;
                auto flush = [&]() {
                    __syncwarp();
                    for (int r = lane; r < nrec; r += 32)
                    {
                        const double q2 = recA[r];
                        const double q = sqrt(q2);
                        double wk, dwk;
                        sph_kernel(q2, q, wk, dwk);
                        recA[r] = wk;
                        recB[r] = -q * dwk - 3.0 * wk;
                    }
                    __syncwarp();
                    for (int t = 0; t < segCount; ++t)
                    {
                        rhoi += recA[segStart + t];
                        gradhi += recB[segStart + t];
                    }
                    gp += segCount;
                    segCount = 0;
                    nrec = 0;
                    __syncwarp();
                };
                // four group particles per step: independent FP64 chains for the scheduler
                for (int i0 = 0; i0 < ng; i0 += 4)
                {
                    if (nrec + 4 * 32 > kRec) flush();
                    double q2u[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                    {
                        const double4 g = sGrp[wib][min(i0 + u, 31)];
                        double dx = g.x - pj.x, dy = g.y - pj.y, dz = g.z - pj.z;
                        nearest_image<Periodic>(dx, dy, dz, lx, ly, lz);
                        q2u[u] = pair_r2(dx, dy, dz) * g.w;
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                    {
                        const bool acc = lane < count && i0 + u < ng && q2u[u] < kRadK2;
                        const uint32_t m = __ballot_sync(0xffffffffu, acc);
                        const int c = __popc(m);
                        if (acc) recA[nrec + __popc(m & lt)] = q2u[u];
                        if (lane == i0 + u) { segStart = nrec; segCount = c; }
                        nrec += c;
                    }
                }
                if (nrec > 0) flush();
            });
        bool stillActive = false;
        if (mine)
        {
            pairs += gp;
            cand += gc;
            // Newton-Raphson step, src/density_base.cu:294-333
            const double hi1 = 1.0 / hi;
            const double hi31 = hi1 * hi1 * hi1;
            const double hi41 = hi31 * hi1;
            const double rho_i = rhoi * kCnormk * pmass * hi31;
            const double grad_i = gradhi * kCnormk * pmass * hi41;
            if (!(rho_i > 0.0))
            {
                rho[i] = 0.0;
                gradh[i] = 0.0;
                converged[i] = 0;
                stillActive = true;
            }
            else
            {
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
                rho[i] = rho_i;
                gradh[i] = grad_i;
                reinterpret_cast<double*>(xyzh + i)[3] = hnew;
                const int conv = (fabs((hnew - hi) / hi) < tolh) ? 1 : 0;
                converged[i] = conv;
                stillActive = !conv;
                if (!conv && hnew > listH[leaf]) ds->listStale = 1;
            }
        }
        const uint32_t still = __ballot_sync(0xffffffffu, stillActive);
        if (still && lane == 0)
        {
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

// Cullen & Dehnen xi limiter from the velocity gradient (src/density_base.cu:511-527):
// components rounded to float as phantom stores them.
__device__ inline double xi_limiter(const double g[9])
{
    const double dvxdx = (float)g[0], dvxdy = (float)g[1], dvxdz = (float)g[2];
    const double dvydx = (float)g[3], dvydy = (float)g[4], dvydz = (float)g[5];
    const double dvzdx = (float)g[6], dvzdy = (float)g[7], dvzdz = (float)g[8];
    const double divv = dvxdx + dvydy + dvzdz;
    const double cx = dvzdy - dvydz;
    const double cy = dvxdz - dvzdx;
    const double cz = dvydx - dvxdy;
    const double mdiv = fmax(-divv, 0.0);
    const double fac = mdiv * mdiv;
    const double trS = cx * cx + cy * cy + cz * cz;
    return (fac + trS > 2.220446049250313e-16) ? fac / (fac + trS) : 1.0;
}

// Post-convergence sweep (src/density_base.cu:529-714): rho, gradh at the converged h,
// div v, the xi limiter and d(div v)/dt, for every live particle.
template<bool Periodic>
__global__ void __launch_bounds__(kThreads)
gradient_kernel(int nL, const uint32_t* __restrict__ layout, const uint32_t* __restrict__ jOffset,
                const uint32_t* __restrict__ jcount, const int* __restrict__ jlist,
                const double4* __restrict__ xyzh, const double4* __restrict__ vel4,
                const double4* __restrict__ acc4, double* __restrict__ rho, double* __restrict__ gradh,
                double* __restrict__ divv, double* __restrict__ xiOut, double* __restrict__ ddivvdt,
                double pmass, const DevBox* __restrict__ box, DevScalars* __restrict__ ds)
{
    __shared__ double4 sRing[kWarpsPerBlock][kRing];
    __shared__ float4 sRingF[kWarpsPerBlock][kRing];
    __shared__ int sIdx[kWarpsPerBlock][kRing];
    const int wib = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int warpGlobal = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nWarps = (gridDim.x * blockDim.x) >> 5;
    double lx = 0, ly = 0, lz = 0;
    if (Periodic) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }
    unsigned long long pairs = 0;
    const double pm = pmass;
    for (int leaf = warpGlobal; leaf < nL; leaf += nWarps)
    {
        const uint32_t p0 = layout[leaf], p1 = layout[leaf + 1];
        const uint32_t jb = jOffset[leaf], nj = jcount[leaf];
        for (uint32_t g = p0; g < p1; g += 64)
        {
            const uint32_t m0 = __ballot_sync(0xffffffffu, g + lane < p1);
            const uint32_t m1 = __ballot_sync(0xffffffffu, g + 32 + lane < p1);
            const int nAct = __popc(m0) + __popc(m1);
            const int G = (nAct + 31) >> 5;
            for (int grp = 0; grp < G; ++grp)
            {
            const int slot = group_slot(m0, m1, nAct, grp, G, lane);
            const bool mine = slot >= 0;
            const uint32_t i = g + uint32_t(mine ? slot : 0);
            const double4 pi = xyzh[i];
            const double4 vi = vel4[i];
            const double4 ai = acc4[i];
            const double hi = pi.w;
            const double hinv2 = 1.0 / (hi * hi);
            const double rs = kRadKernel * hi;
            const double rmax = warp_max(mine ? rs : 0.0);
            const GroupBox bx = group_box(mine, pi.x, pi.y, pi.z, rs, rmax);
            double rhoi = 0.0, gradhi = 0.0, divs = 0.0;
            double dv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, da[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            double rxx = 0, rxy = 0, rxz = 0, ryy = 0, ryz = 0, rzz = 0;
            unsigned int gp = 0;
            const float xf = float(pi.x - bx.cx), yf = float(pi.y - bx.cy), zf = float(pi.z - bx.cz);
            const double rm = rs + fp32_margin(bx, Periodic ? fmax(lx, fmax(ly, lz)) : 0.0);
            const float tf = __double2float_ru(rm * rm * (1.0 + 1e-6));
            const float Lx = float(lx), Ly = float(ly), Lz = float(lz);
            stream_pairs(
                sRing[wib], sRingF[wib], sIdx[wib], bx.cx, bx.cy, bx.cz, jb, nj, jlist, layout, xyzh,
                [&](const double4& pj) { return in_gather_box<Periodic>(pj, bx, lx, ly, lz); },
                [&](const double4* ring, const float4* ringf, const int* ringIdx, int head, int count) {
                  two_pass(ring, ringf, ringIdx, head, count, mine,
                  [&](const float4& pf) { return r2_f32<Periodic>(xf, yf, zf, pf, Lx, Ly, Lz) <= tf; },
                  [&](const double4& pj, const float4&, int j) {
                    double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
                    nearest_image<Periodic>(dx, dy, dz, lx, ly, lz);
                    const double r2 = pair_r2(dx, dy, dz);
                    const double q2 = r2 * hinv2;
                    if (!(q2 < kRadK2)) return;
                    ++gp;
                    const double q = sqrt(q2);
                    double wk, dwk;
                    sph_kernel(q2, q, wk, dwk);
                    rhoi += wk;
                    gradhi += -q * dwk - 3.0 * wk;
                    const double rij = sqrt(r2);
                    const double rij1 = 1.0 / (rij + 2.220446049250313e-16);
                    const double rg = rij1 * dwk;
                    const double rx = dx * rg * pm, ry = dy * rg * pm, rz = dz * rg * pm;
                    const double4 vj = ldg4(vel4 + j);
                    const double dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
                    divs += dvx * rx + dvy * ry + dvz * rz;
                    dv[0] += dvx * rx; dv[1] += dvx * ry; dv[2] += dvx * rz;
                    dv[3] += dvy * rx; dv[4] += dvy * ry; dv[5] += dvy * rz;
                    dv[6] += dvz * rx; dv[7] += dvz * ry; dv[8] += dvz * rz;
                    const double4 aj = ldg4(acc4 + j);
                    const double dax = ai.x - aj.x, day = ai.y - aj.y, daz = ai.z - aj.z;
                    da[0] += dax * rx; da[1] += dax * ry; da[2] += dax * rz;
                    da[3] += day * rx; da[4] += day * ry; da[5] += day * rz;
                    da[6] += daz * rx; da[7] += daz * ry; da[8] += daz * rz;
                    rxx -= dx * rx; rxy -= dx * ry; rxz -= dx * rz;
                    ryy -= dy * ry; ryz -= dy * rz; rzz -= dz * rz;
                  });
                });
            if (!mine) continue;
            pairs += gp;
            const double hi1 = 1.0 / hi;
            const double hi31 = hi1 * hi1 * hi1;
            const double hi41 = hi31 * hi1;
            const double rho_i = rhoi * kCnormk * pm * hi31;
            const double grad_i = gradhi * kCnormk * pm * hi41;
            rho[i] = rho_i;
            gradh[i] = grad_i;
            if (!(rho_i > 0.0))
            {
                divv[i] = 0.0; ddivvdt[i] = 0.0; xiOut[i] = 1.0;
                continue;
            }
            const double omega = 1.0 + (hi / (3.0 * rho_i)) * grad_i;
            const double omega_inv = (omega > 0.0) ? (1.0 / omega) : 1.0;
            const double term = kCnormk * omega_inv * hi41 / rho_i;
            const double denom = rxx * ryy * rzz + 2.0 * rxy * rxz * ryz - rxx * ryz * ryz - ryy * rxz * rxz
                                 - rzz * rxy * rxy;
            const double rm0 = ryy * rzz - ryz * ryz;
            const double rm1 = rxz * ryz - rzz * rxy;
            const double rm2 = rxy * ryz - rxz * ryy;
            const double rm3 = rzz * rxx - rxz * rxz;
            const double rm4 = rxy * rxz - rxx * ryz;
            const double rm5 = rxx * ryy - rxy * rxy;
            divv[i] = -divs * term;
            double gm[9], div_a;
            if (fabs(denom) > 2.2250738585072014e-308)
            {
                const double dd = 1.0 / denom;
#pragma unroll
                for (int r = 0; r < 3; ++r)
                {
                    const double sx = dv[3 * r], sy = dv[3 * r + 1], sz = dv[3 * r + 2];
                    gm[3 * r]     = -(sx * rm0 + sy * rm1 + sz * rm2) * dd;
                    gm[3 * r + 1] = -(sx * rm1 + sy * rm3 + sz * rm4) * dd;
                    gm[3 * r + 2] = -(sx * rm2 + sy * rm4 + sz * rm5) * dd;
                }
                double diag = 0.0;
#pragma unroll
                for (int r = 0; r < 3; ++r)
                {
                    const double sx = da[3 * r], sy = da[3 * r + 1], sz = da[3 * r + 2];
                    const double gx = (sx * rm0 + sy * rm1 + sz * rm2) * dd;
                    const double gy = (sx * rm1 + sy * rm3 + sz * rm4) * dd;
                    const double gz = (sx * rm2 + sy * rm4 + sz * rm5) * dd;
                    diag += (r == 0) ? gx : ((r == 1) ? gy : gz);
                }
                div_a = -diag;
            }
            else
            {
#pragma unroll
                for (int c = 0; c < 9; ++c) gm[c] = -dv[c] * term;
                div_a = -term * (da[0] + da[4] + da[8]);
            }
            xiOut[i] = xi_limiter(gm);
            ddivvdt[i] = div_a - (gm[0] * gm[0] + gm[4] * gm[4] + gm[8] * gm[8]
                                  + 2.0 * (gm[1] * gm[3] + gm[2] * gm[6] + gm[5] * gm[7]));
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if (lane == 0) atomicAdd(&ds->pairs[1], pairs);
}

// Dead particles (h <= 0) sit after nAlive: div v = d(div v)/dt = 0, xi = 1.
__global__ void gradient_dead_kernel(int nAlive, int n, double* __restrict__ divv, double* __restrict__ xiOut,
                                     double* __restrict__ ddivvdt)
{
    const long i = nAlive + long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    divv[i] = 0.0; ddivvdt[i] = 0.0; xiOut[i] = 1.0;
}

__global__ void hmax_live_kernel(const double4* __restrict__ xyzh, int nAlive, double* __restrict__ part)
{
    double m = 0.0;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nAlive; i += long(gridDim.x) * blockDim.x)
        m = fmax(m, xyzh[i].w);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ double s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        for (int w = 1; w < int(blockDim.x >> 5); ++w) m = fmax(m, s[w]);
        part[blockIdx.x] = m;
    }
}

int grid_for(const State& s, int work)
{
    const int maxBlocks = s.numSMs * 8;
    return std::max(1, std::min(maxBlocks, iceil(work, kWarpsPerBlock)));
}

// A persistent grid: as many blocks of the kernel as fit on the device at once.
template<class K>
int persistent_grid(const State& s, K kernel)
{
    int perSM = 0;
    COSMO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, kThreads, 0));
    return std::max(1, perSM) * s.numSMs;
}

} // namespace

DensResult solve_density(State& s, int n, double pmass, const double* periodicBox, double tolh, double hfact,
                         int maxIter, bool withGradients)
{
    DensResult res{0, 0, 0};
    if (!(hfact > 0.0)) hfact = kHfactDefault;
    s.ngas = n;
    s.pmass = pmass;
    s.hfact = hfact;
    s.periodic = periodicBox ? 1 : 0;
    if (periodicBox) std::copy(periodicBox, periodicBox + 6, s.boxHost);
    s.activePerIter.clear();
    s.t = Timings{};
    ev_reset(s);
    DevScalars* ds = s.dscal.get();
    COSMO_CUDA(cudaMemsetAsync(s.rho.get(), 0, size_t(n) * 8, s.st));
    COSMO_CUDA(cudaMemsetAsync(s.gradh.get(), 0, size_t(n) * 8, s.st));
    COSMO_CUDA(cudaMemsetAsync(s.converged.get(), 0, size_t(n) * 4, s.st));
    COSMO_CUDA(cudaMemsetAsync(&ds->pairs[0], 0, sizeof(ds->pairs), s.st));

    build_tree(s, periodicBox, withGradients);
    s.orderFor = n;
    const int nL = s.nLeaves;
    s.activeA.resize(nL, s.st);
    s.activeB.resize(nL, s.st);
    s.leafNext.resize(nL, s.st);
    const int itemCap = std::max(s.nAlive, 1);
    s.items.resize(itemCap, s.st);
    COSMO_CUDA(cudaMemcpyAsync(s.activeA.get(), s.allLeaves.get(), size_t(nL) * 4, cudaMemcpyDeviceToDevice, s.st));
    int nActiveLeaves = nL;
    long long nActiveParticles = s.nAlive;

    // The gather lists are built with a widened radius and reused while every active h
    // stays inside it: a superset list in ascending leaf order offers the same accepted
    // pairs in the same order, so the sums do not change.  hmaxLeaf is still refreshed
    // for the active leaves every iteration, as the reference does, so the exact lists of
    // the last iteration can be rebuilt afterwards.
    bool listsValid = false, listsWidened = false;
    cudaEvent_t e3 = ev(s);
    for (int iter = 0; iter < maxIter; ++iter)
    {
        cudaEvent_t j0 = ev(s);
        hmax_leaves(s, s.activeA.get(), nActiveLeaves);
        if (!listsValid)
        {
            build_lists(s, false, kListMargin);
            listsValid = listsWidened = true;
        }
        cudaEvent_t j1 = ev(s);
        if (s.precision == 1)
        {
            COSMO_CUDA(cudaMemsetAsync(&ds->nextActive, 0, 3 * sizeof(int), s.st));
            launch_density_mixed(s, nActiveLeaves, pmass, tolh, hfact);
        }
        else
        {
            begin_iteration_kernel<<<std::min(iceil(nL, 256), 4 * s.numSMs), 256, 0, s.st>>>(ds, s.leafNext.get(),
                                                                                            nL);
            COSMO_LAUNCHED();
            plan_items_kernel<<<grid_for(s, nActiveLeaves), kThreads, 0, s.st>>>(
                s.activeA.get(), nActiveLeaves, s.layout.get(), s.converged.get(), s.jstream.get(), s.items.get(),
                itemCap, ds);
            COSMO_LAUNCHED();
            auto nr = s.periodic ? density_nr_kernel<true> : density_nr_kernel<false>;
            nr<<<persistent_grid(s, nr), kThreads, 0, s.st>>>(
                s.items.get(), itemCap, s.layout.get(), s.jOffset.get(), s.jcount.get(), s.jlist.get(), s.xyzh.get(),
                s.rho.get(), s.gradh.get(), s.converged.get(), pmass, tolh, hfact, s.box.get(), s.listH.get(),
                s.leafNext.get(), s.activeB.get(), ds);
            COSMO_LAUNCHED();
        }
        cudaEvent_t j2 = ev(s);
        read_scalars(s);
        s.t.jbuild += elapsed_s(j0, j1);
        s.t.nrkern += elapsed_s(j1, j2);
        s.activePerIter.push_back(nActiveParticles);
        s.itersRun = iter + 1;
        nActiveLeaves = s.hscal->nextActive;
        nActiveParticles = s.hscal->unconverged;
        if (s.hscal->listStale) listsValid = false;
        std::swap(s.activeA, s.activeB);
        if (nActiveParticles == 0) break;
    }
    (void)e3;
    if (listsWidened && !withGradients)
    {
        cudaEvent_t j0 = ev(s);
        build_lists(s, false);
        cudaEvent_t j1 = ev(s);
        COSMO_CUDA(cudaEventSynchronize(j1));
        s.t.jbuild += elapsed_s(j0, j1);
    }
    check_dev_err(s, "solveDensH");
    res.itersRun = s.itersRun;
    res.unconverged = int(nActiveParticles);
    if (nActiveParticles > 0)
    {
        res.status = 1;
        return res;
    }
    if (s.periodic && s.nAlive > 0)
    {
        const int nb = std::min(iceil(s.nAlive, 256), 2 * s.numSMs);
        s.redTmp.resize(std::max<size_t>(s.redTmp.n, nb), s.st, false);
        hmax_live_kernel<<<nb, 256, 0, s.st>>>(s.xyzh.get(), s.nAlive, s.redTmp.get());
        COSMO_LAUNCHED();
        std::vector<double> part(nb);
        COSMO_CUDA(cudaMemcpyAsync(part.data(), s.redTmp.get(), nb * 8, cudaMemcpyDeviceToHost, s.st));
        COSMO_CUDA(cudaStreamSynchronize(s.st));
        double hm = 0.0;
        for (double v : part) hm = std::max(hm, v);
        const double lmin = std::min({periodicBox[1] - periodicBox[0], periodicBox[3] - periodicBox[2],
                                      periodicBox[5] - periodicBox[4]});
        if (kRadKernel * hm >= 0.5 * lmin)
        {
            res.status = 2;
            return res;
        }
    }
    if (withGradients)
    {
        cudaEvent_t g0 = ev(s);
        hmax_leaves(s, s.allLeaves.get(), nL);
        build_lists(s, false);
        cudaEvent_t g1 = ev(s);
        const int grid = grid_for(s, nL);
        if (s.precision == 1)
            launch_gradient_mixed(s, pmass);
        else if (s.periodic)
            gradient_kernel<true><<<grid, kThreads, 0, s.st>>>(
                nL, s.layout.get(), s.jOffset.get(), s.jcount.get(), s.jlist.get(), s.xyzh.get(), s.vel4.get(),
                s.acc4.get(), s.rho.get(), s.gradh.get(), s.divv.get(), s.xi.get(), s.ddivvdt.get(), pmass,
                s.box.get(), ds);
        else
            gradient_kernel<false><<<grid, kThreads, 0, s.st>>>(
                nL, s.layout.get(), s.jOffset.get(), s.jcount.get(), s.jlist.get(), s.xyzh.get(), s.vel4.get(),
                s.acc4.get(), s.rho.get(), s.gradh.get(), s.divv.get(), s.xi.get(), s.ddivvdt.get(), pmass,
                s.box.get(), ds);
        COSMO_LAUNCHED();
        if (n > s.nAlive)
        {
            gradient_dead_kernel<<<iceil(n - s.nAlive, 256), 256, 0, s.st>>>(s.nAlive, n, s.divv.get(), s.xi.get(),
                                                                             s.ddivvdt.get());
            COSMO_LAUNCHED();
        }
        cudaEvent_t g2 = ev(s);
        read_scalars(s);
        s.t.gjbuild += elapsed_s(g0, g1);
        s.t.gradkern += elapsed_s(g1, g2);
    }
    check_dev_err(s, "solveDensH");
    ++s.token;
    return res;
}

} // namespace cosmo
