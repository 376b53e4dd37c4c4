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
#include <type_traits>

#include "newton_kernels.cuh"

namespace cosmo {

namespace {

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

// The sums of the post-convergence sweep for one particle (src/density_base.cu:529-714),
// added pair by pair in ascending j, and the finish: rho, gradh at the converged h, div v,
// the xi limiter and d(div v)/dt.
struct GradSums
{
    double rhoi = 0.0, gradhi = 0.0, divs = 0.0;
    double dv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, da[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double rxx = 0, rxy = 0, rxz = 0, ryy = 0, ryz = 0, rzz = 0;
    unsigned int gp = 0;

    // One pair: separation (dx, dy, dz) at the nearest image, r^2 and q^2 = r^2 / h_i^2.
    __device__ __forceinline__ void add(double dx, double dy, double dz, double r2, double q2, const double4& vi,
                                        const double4& ai, const double4& vj, const double4& aj, double pm)
    {
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
        const double dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
        divs += dvx * rx + dvy * ry + dvz * rz;
        dv[0] += dvx * rx; dv[1] += dvx * ry; dv[2] += dvx * rz;
        dv[3] += dvy * rx; dv[4] += dvy * ry; dv[5] += dvy * rz;
        dv[6] += dvz * rx; dv[7] += dvz * ry; dv[8] += dvz * rz;
        const double dax = ai.x - aj.x, day = ai.y - aj.y, daz = ai.z - aj.z;
        da[0] += dax * rx; da[1] += dax * ry; da[2] += dax * rz;
        da[3] += day * rx; da[4] += day * ry; da[5] += day * rz;
        da[6] += daz * rx; da[7] += daz * ry; da[8] += daz * rz;
        rxx -= dx * rx; rxy -= dx * ry; rxz -= dx * rz;
        ryy -= dy * ry; ryz -= dy * rz; rzz -= dz * rz;
    }

    __device__ __forceinline__ void finish(uint32_t i, double hi, double pm, double* __restrict__ rho,
                                           double* __restrict__ gradh, double* __restrict__ divv,
                                           double* __restrict__ xiOut, double* __restrict__ ddivvdt) const
    {
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
            return;
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
};

// Post-convergence sweep over the symmetric rows: one lane per live particle over its row
// (at the converged h a superset of the gather pairs, ascending), the sweep's exact test
// and the sums in the row's order -- the same pairs and order as the group sweep, so the
// results agree with it bit for bit.  Overflowed rows are left to gradient_kernel.
template<bool Periodic>
__global__ void __launch_bounds__(kThreads)
gradient_row_kernel(int nAlive, const int* __restrict__ nbl, const int* __restrict__ nblCount,
                    const double4* __restrict__ xyzh, const double4* __restrict__ vel4,
                    const double4* __restrict__ acc4, double* __restrict__ rho, double* __restrict__ gradh,
                    double* __restrict__ divv, double* __restrict__ xiOut, double* __restrict__ ddivvdt,
                    double pmass, const DevBox* __restrict__ box, DevScalars* __restrict__ ds)
{
    double lx = 0, ly = 0, lz = 0;
    if (Periodic) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }
    unsigned long long pairs = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nAlive; i += gridDim.x * blockDim.x)
    {
        const int cnt = nblCount[i];
        if (unsigned(cnt) > unsigned(kNbl)) continue;
        const double4 pi = xyzh[i];
        const double4 vi = vel4[i];
        const double4 ai = acc4[i];
        const double hi = pi.w;
        const double hinv2 = 1.0 / (hi * hi);
        const int* row = row_of(nbl, uint32_t(i));
        GradSums g;
        auto pair = [&](int j) {
            const double4 pj = ldg4(xyzh + j);
            double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            nearest_image<Periodic>(dx, dy, dz, lx, ly, lz);
            const double r2 = pair_r2(dx, dy, dz);
            const double q2 = r2 * hinv2;
            if (!(q2 < kRadK2)) return;
            g.add(dx, dy, dz, r2, q2, vi, ai, ldg4(vel4 + j), ldg4(acc4 + j), pmass);
        };
        for_row(row, cnt, pair);
        pairs += g.gp;
        g.finish(uint32_t(i), hi, pmass, rho, gradh, divv, xiOut, ddivvdt);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&ds->pairs[1], pairs);
}

// Post-convergence sweep over the group path (src/density_base.cu:529-714) for the
// particles whose rows overflowed (nblCount > kNbl), or for all live ones when nblCount is
// null: rho, gradh at the converged h, div v, the xi limiter and d(div v)/dt.
template<bool Periodic>
__global__ void __launch_bounds__(kThreads)
gradient_kernel(int nL, const uint32_t* __restrict__ layout, const uint32_t* __restrict__ jOffset,
                const uint32_t* __restrict__ jcount, const int* __restrict__ jlist,
                const double4* __restrict__ xyzh, const double4* __restrict__ vel4,
                const double4* __restrict__ acc4, double* __restrict__ rho, double* __restrict__ gradh,
                double* __restrict__ divv, double* __restrict__ xiOut, double* __restrict__ ddivvdt,
                double pmass, const DevBox* __restrict__ box, const int* __restrict__ nblCount,
                DevScalars* __restrict__ ds)
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
    if (nblCount != nullptr && ds->rowOverflow == 0) return;   // every row complete: nothing to do
    auto wanted = [&](uint32_t a) { return nblCount == nullptr || unsigned(nblCount[a]) > unsigned(kNbl); };
    for (int leaf = warpGlobal; leaf < nL; leaf += nWarps)
    {
        const uint32_t p0 = layout[leaf], p1 = layout[leaf + 1];
        const uint32_t jb = jOffset[leaf], nj = jcount[leaf];
        for (uint32_t g = p0; g < p1; g += 64)
        {
            const uint32_t m0 = __ballot_sync(0xffffffffu, g + lane < p1 && wanted(g + lane));
            const uint32_t m1 = __ballot_sync(0xffffffffu, g + 32 + lane < p1 && wanted(g + 32 + lane));
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
            GradSums gs;
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
                    gs.add(dx, dy, dz, r2, q2, vi, ai, ldg4(vel4 + j), ldg4(acc4 + j), pm);
                  });
                });
            if (!mine) continue;
            pairs += gs.gp;
            gs.finish(i, hi, pm, rho, gradh, divv, xiOut, ddivvdt);
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

// Rows from the Newton rows: whether each live particle's row covers its converged h
// with the force test's slack to spare (written this solve, not overflowed, and
// h (1 + 1e-9) <= rowH, the h it is complete for, cleared at the start of the solve).
// flag = 1 if it does; a leaf with particles that do not is listed, and they are counted.
__global__ void row_cover_kernel(int nL, const uint32_t* __restrict__ layout, const double4* __restrict__ xyzh,
                                 const int* __restrict__ nblCount, const double* __restrict__ rowH,
                                 const uint32_t* __restrict__ jstream, uint32_t streamCut, int* __restrict__ flag,
                                 int* __restrict__ leaves, double* __restrict__ hs, DevScalars* __restrict__ ds)
{
    const int lane = threadIdx.x & 31;
    const int nWarps = (gridDim.x * blockDim.x) >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        // the counters of the passes that follow (nothing else touches them here)
        ds->extraCount = 0;
        ds->mergeOverflow = 0;
        ds->rowOverflow = 0;
    }
    for (int leaf = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; leaf < nL; leaf += nWarps)
    {
        const uint32_t p0 = layout[leaf], p1 = layout[leaf + 1];
        int miss = 0;
        for (uint32_t a = p0 + lane; a < p1; a += 32)
        {
            const double h = xyzh[a].w;
            const bool ok = unsigned(nblCount[a]) <= unsigned(kNbl) && h * (1.0 + 1e-9) <= rowH[a];
            flag[a] = ok ? 1 : 0;
            hs[a] = h;
            miss += ok ? 0 : 1;
        }
        miss = __reduce_add_sync(0xffffffffu, miss);
        if (lane == 0 && miss > 0)
        {
            atomicAdd(&ds->coverNeed, miss);
            // a leaf whose stream the work queue cuts keeps the group path: no row for it
            if (jstream[leaf] > streamCut) atomicAdd(&ds->coverCut, 1);
            leaves[atomicAdd(&ds->coverLeaves, 1)] = leaf;
        }
    }
}

// The symmetric rows from the Newton rows, for every live particle whose row covers its
// converged h: the j of its Newton row (flat, ascending, r^2 beside each -- the same
// double as the force pass's dr^2) that the force pass takes,
// dr^2 < R^2 max(h_i^2, h_j^2) (1 + 1e-10) -- sym_rows_kernel's test -- written in the
// same order into the interleaved rows of the gradient and force passes (hs: h in the
// sorted order, 8 bytes a particle).  A pair the force pass takes because of this
// particle's support (dr^2 < R^2 h_i^2 (1 + 1e-10)) is in j's Newton row too unless dr^2
// reaches the radius j's row covers (R rowH, with 1e-9 to spare; only a pair beyond j's
// own support can); such a pair is appended as (j << 32 | i), for i to be merged into
// j's row.  The mixed form's rows hold that double rounded to float (within 2^-24 of
// it): where it lies within 1e-6 of a bound the test uses, dr^2 is taken again from the
// positions, so every test decides as on the double and the rows are the same.
template<class T, bool Periodic>
__global__ void __launch_bounds__(kThreads)
sym_from_rows_kernel(int nAlive, const int* __restrict__ rowsJ, const T* __restrict__ rowsR2,
                     int* __restrict__ nblCount, const double* __restrict__ hs, const double* __restrict__ rowH,
                     const double4* __restrict__ xyzh, const DevBox* __restrict__ box, int* __restrict__ nbl,
                     unsigned long long* __restrict__ extras, int extraCap, int* __restrict__ extraCnt,
                     DevScalars* __restrict__ ds)
{
    constexpr bool kExact = std::is_same<T, double>::value;
    using R4 = typename std::conditional<kExact, double4, float4>::type;
    double lx = 0, ly = 0, lz = 0;
    if (Periodic && !kExact) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nAlive; i += gridDim.x * blockDim.x)
    {
        extraCnt[i] = 0;
        const int cnt = nblCount[i];
        const double hi = hs[i];
        const double bi = kRadK2 * (hi * hi) * (1.0 + 1e-10);
        const int4* inJ = reinterpret_cast<const int4*>(row_flat(rowsJ, uint32_t(i)));
        const R4* inR = reinterpret_cast<const R4*>(row_flat(rowsR2, uint32_t(i)));
        int* out = row_of(nbl, uint32_t(i));
        int w = 0;
        auto entry = [&](int j, double dr2, double hj) {
            bool exact = kExact;
            auto near = [&](double bound) { return fabs(dr2 - bound) <= 1e-6 * bound; };
            auto retake = [&]() {
                if (exact) return;
                const double4 pa = xyzh[i], pb = ldg4(xyzh + j);
                double dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
                nearest_image<Periodic>(dx, dy, dz, lx, ly, lz);
                dr2 = pair_r2(dx, dy, dz);
                exact = true;
            };
            const double bj = kRadK2 * (hj * hj) * (1.0 + 1e-10);
            const double own = kRadK2 * (hj * hj);
            if (!exact && (near(fmax(bi, bj)) || near(bi) || near(own))) retake();
            if (!(dr2 >= fmax(bi, bj))) out[size_t(w++) * kRowStride] = j;
            if (dr2 < bi && !(dr2 < own))
            {
                const double ch = __ldg(rowH + j);
                const double cover = kRadK2 * (ch * ch) * (1.0 - 1e-9);
                if (!exact && near(cover)) retake();
                if (!(dr2 < cover))
                {
                    const int k = atomicAdd(&ds->extraCount, 1);
                    if (k < extraCap) extras[k] = (static_cast<unsigned long long>(j) << 32) | uint32_t(i);
                }
            }
        };
        // groups of four entries in a two-stage pipeline: while a group is tested, the next
        // group's h and the one after's j and r^2 are in flight (a row's groups lie within
        // its kNbl entries; slots past the count read this particle's own h)
        const int nq = (cnt + 3) >> 2;
        const int me = i;
        auto ldj = [&](int q) { return q < nq ? __ldg(inJ + q) : make_int4(me, me, me, me); };
        auto ldr = [&](int q) {
            R4 z{};
            if constexpr (kExact) return q < nq ? ldg4(inR + q) : z;
            else return q < nq ? __ldg(inR + q) : z;
        };
        auto ldh = [&](int q, const int4& v) {
            const int left = cnt - 4 * q;
            return make_double4(__ldg(hs + (left > 0 ? v.x : me)), __ldg(hs + (left > 1 ? v.y : me)),
                                __ldg(hs + (left > 2 ? v.z : me)), __ldg(hs + (left > 3 ? v.w : me)));
        };
        int4 v0 = ldj(0), v1 = ldj(1);
        R4 r0 = ldr(0), r1 = ldr(1);
        double4 h0 = ldh(0, v0);
        for (int q = 0; q < nq; ++q)
        {
            const double4 h1 = ldh(q + 1, v1);
            const int4 v2 = ldj(q + 2);
            const R4 r2 = ldr(q + 2);
            const int left = cnt - 4 * q;
            entry(v0.x, double(r0.x), h0.x);
            if (left > 1) entry(v0.y, double(r0.y), h0.y);
            if (left > 2) entry(v0.z, double(r0.z), h0.z);
            if (left > 3) entry(v0.w, double(r0.w), h0.w);
            v0 = v1; r0 = r1; h0 = h1;
            v1 = v2; r1 = r2;
        }
        nblCount[i] = w;
    }
}

// The extras of each row owner (their number read on the device, at most cap of them):
// counted, then placed at the owner's offset.
__global__ void extras_count_kernel(const unsigned long long* __restrict__ extras, int cap,
                                    const DevScalars* __restrict__ ds, int* __restrict__ cnt)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < min(ds->extraCount, cap)) atomicAdd(&cnt[int(extras[k] >> 32)], 1);
}

__global__ void extras_place_kernel(const unsigned long long* __restrict__ extras, int cap,
                                    const DevScalars* __restrict__ ds, const uint32_t* __restrict__ off,
                                    int* __restrict__ cnt, int* __restrict__ bucket)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= min(ds->extraCount, cap)) return;
    const int t = int(extras[k] >> 32);
    bucket[off[t] + uint32_t(atomicSub(&cnt[t], 1) - 1)] = int(uint32_t(extras[k]));
}

// Each row owner merges its extras into its row: sorted, those the row already holds
// dropped, the rest merged in from the back so the row stays ascending.  A row that would
// exceed kNbl sets mergeOverflow (the symmetric rows are then built instead).
__global__ void extras_merge_kernel(int nA, const uint32_t* __restrict__ off, int* __restrict__ bucket,
                                    int* __restrict__ nbl, int* __restrict__ nblCount, DevScalars* __restrict__ ds)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nA) return;
    const uint32_t b0 = off[t], e = off[t + 1] - b0;
    if (e == 0) return;
    const int cnt = nblCount[t];
    if (cnt + int(e) > 2 * kNbl)
    {
        ds->mergeOverflow = 1;
        return;
    }
    int* ex = bucket + b0;
    for (uint32_t a = 1; a < e; ++a)
    {
        const int v = ex[a];
        uint32_t k = a;
        for (; k > 0 && ex[k - 1] > v; --k) ex[k] = ex[k - 1];
        ex[k] = v;
    }
    int* row = row_of(nbl, uint32_t(t));
    auto at = [&](int k) -> int& { return row[size_t(k) * kRowStride]; };
    uint32_t u = 0;
    for (uint32_t a = 0; a < e; ++a)
    {
        const int v = ex[a];
        int lo = 0, hi = cnt;
        while (lo < hi)
        {
            const int mid = (lo + hi) >> 1;
            if (at(mid) < v) lo = mid + 1;
            else hi = mid;
        }
        if (!(lo < cnt && at(lo) == v)) ex[u++] = v;
    }
    if (u == 0) return;
    if (cnt + int(u) > kNbl)
    {
        ds->mergeOverflow = 1;
        return;
    }
    int r = cnt - 1, x = int(u) - 1, w = cnt + int(u) - 1;
    while (x >= 0)
    {
        if (r >= 0 && at(r) > ex[x]) at(w--) = at(r--);
        else at(w--) = ex[x--];
    }
    nblCount[t] = cnt + int(u);
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

// Converged flags of the fixed particles (the caller's mask through the sort order).
__global__ void freeze_kernel(const int* __restrict__ order, const int* __restrict__ frozen, int nAlive,
                              int* __restrict__ converged, DevScalars* __restrict__ ds)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const bool f = k < nAlive && frozen[order[k]] != 0;
    if (k < nAlive) converged[k] = f ? 1 : 0;
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(&ds->frozenAlive, __popc(m));
}

// ---------------------------------------------------------- the Newton loop as a graph
__global__ void newton_loop_init_kernel(NewtonLoop* L, int nLeaves, int numNodes, int nAlive, int maxIter)
{
    *L = NewtonLoop{};
    L->nLeaves = nLeaves;
    L->numNodes = numNodes;
    L->nActiveLeaves = nLeaves;
    L->nActiveParticles = nAlive;
    L->maxIter = maxIter;
}

// First node of an iteration: the list-rebuild and row-build decisions the last
// iteration's epilogue recorded become the conditions of this iteration's two branches.
__global__ void newton_decide_kernel(const NewtonLoop* L, cudaGraphConditionalHandle hList,
                                     cudaGraphConditionalHandle hRows)
{
    cudaGraphSetConditional(hList, L->rebuildNext ? 1u : 0u);
    cudaGraphSetConditional(hRows, L->rowsNext ? 1u : 0u);
}

__global__ void newton_count_kernel(NewtonLoop* L, int rows)
{
    if (rows)
    {
        L->rowsReady = 1;
        ++L->rowBuilds;
    }
    else ++L->rebuilds;
}

// The next active leaves become the active ones (the host loop swaps the two buffers).
__global__ void newton_copy_active_kernel(const int* __restrict__ src, int* __restrict__ dst,
                                          const DevScalars* __restrict__ ds, int cap)
{
    const int n = min(ds->nextActive, cap);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) dst[t] = src[t];
}

// Last node of an iteration: what the host loop read back after it -- the counts, the
// stale-list flag, the settling particles -- decides the next iteration on the device.
__global__ void newton_epilogue_kernel(NewtonLoop* L, const DevScalars* ds, const uint32_t* jOffset,
                                       cudaGraphConditionalHandle hMore)
{
    const int it = L->iter;
    if (it < kLoopIters)
    {
        L->activePerIter[it] = L->nActiveParticles;
        L->listEntries[it] = jOffset[L->nLeaves];
    }
    if (it == 0) L->settling0 = ds->settling;
    const int active = ds->unconverged;
    L->nActiveLeaves = ds->nextActive;
    L->nActiveParticles = active;
    L->iter = it + 1;
    const int more = (active > 0 && it + 1 < L->maxIter && ds->err == 0) ? 1 : 0;
    L->rebuildNext = (more && ds->listStale) ? 1 : 0;
    L->rowsNext = (more && !L->rowsReady && 5ll * ds->settling >= 4ll * active) ? 1 : 0;
    cudaGraphSetConditional(hMore, unsigned(more));
}

// Bytes of the values a captured loop depends on.
struct KeyBytes
{
    std::vector<unsigned char> b;
    template<class T>
    void add(const T& v)
    {
        const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
        b.insert(b.end(), p, p + sizeof(T));
    }
};

} // namespace

// The Newton loop of one solve as one graph launch: a while node whose body is one
// iteration -- the conditions of its two branches, hmax of the active leaves, [the
// incremental list rebuild], [the Newton rows], the work items, the Newton kernel, the
// row kernel, the next active leaves and the epilogue that decides the next iteration.
// Same kernels, same order, same decisions as the host loop, so the same results; the
// first lists are built before it (their total sizes the storage of the rebuilds).  The
// graph reads the tree's counts on the device and is launched over the capacities of the
// buffers, so it depends only on the buffers, the options and the solve's scalars: it is
// captured and instantiated once and launched again by every later solve with the same
// ones (a time-stepping caller's trees change; its buffers, grown to the largest tree,
// do not).  Returns false, having changed nothing the caller keeps, when the graph cannot
// be built or a rebuild outgrew the storage: the caller then solves again on the host loop.
enum class LoopGraph { Ran, Deferred, Failed };

static LoopGraph newton_loop_graph(State& s, double pmass, double tolh, double hfact, int maxIter, FixedSplit cut,
                                   int spreadG, long long& nActiveParticles, int* rowsJ)
{
    DevScalars* ds = s.dscal.get();
    const int nL = s.nLeaves;
    const bool mx = s.precision == 1;
    cudaEvent_t j0 = ev(s);
    hmax_leaves(s, s.activeA.get(), nL);
    build_lists(s, false, kListMargin, false, true, cut.work);
    // list storage of the rebuilds: grown to twice the first lists (never shrunk, so the
    // graph's buffers stay put), or a set share of them for the fallback's test
    size_t listStore;
    if (s.graphListStorePct > 0)
    {
        listStore = size_t(s.listTotal) * size_t(s.graphListStorePct) / 100;
        s.jlist.resize(std::max<size_t>(listStore, s.jlist.n), s.st, true);
    }
    else
    {
        const size_t want = 2 * size_t(s.listTotal) + 65536;
        if (s.jlist.cap < want) s.jlist.resize(want, s.st, true);
        listStore = s.jlist.cap;
    }
    if (s.jlistPrev.cap < s.jlist.cap) s.jlistPrev.resize(s.jlist.cap, s.st);
    if (s.jOffsetPrev.cap < s.jOffset.cap) s.jOffsetPrev.resize(s.jOffset.cap, s.st);
    s.walked.resize(nL, s.st);
    s.nloop.resize(1, s.st);
    NewtonLoop* L = s.nloop.get();
    newton_loop_init_kernel<<<1, 1, 0, s.st>>>(L, nL, s.numNodes, int(nActiveParticles), maxIter);
    COSMO_LAUNCHED();
    cudaEvent_t j1 = ev(s);

    // launch extents: the buffers' capacities (every buffer was sized for this tree)
    size_t lc = std::min<size_t>({s.activeA.cap, s.activeB.cap, s.leafNext.cap, s.jcount.cap, s.jstream.cap,
                                  s.listH.cap, s.hmaxLeaf.cap, s.walked.cap, s.leafToInternal.cap,
                                  s.walkScratch.cap / size_t(kWalkScratch)});
    lc = std::min<size_t>({lc, s.jOffset.cap - 1, s.jOffsetPrev.cap - 1, s.layout.cap - 1});
    const int leafCap = int(std::min<size_t>(lc, size_t(1) << 30));
    const size_t ic = std::min<size_t>({s.items.cap, s.rowItems.cap, s.nblCount.cap, s.nblH.cap,
                                        s.nblR2.cap / size_t(kNbl)});
    const int itemCap = int(std::min<size_t>(ic, size_t(1) << 30));
    scan_reserve(s, leafCap);

    RowsKernelFn nrows = mx ? mixed_newton_rows_kernel(s.periodic)
                            : (s.periodic ? newton_rows_kernel<true, false> : newton_rows_kernel<false, false>);
    NrKernelFn nr = mx ? mixed_density_nr_kernel(s.periodic, s.staging)
                  : s.staging ? (s.periodic ? density_nr_kernel<true, false, true> : density_nr_kernel<false, false, true>)
                              : (s.periodic ? density_nr_kernel<true, false, false> : density_nr_kernel<false, false, false>);
    RowKernelFn rk = mx ? mixed_density_row_kernel(s.periodic)
                        : (s.periodic ? density_row_kernel<true, false> : density_row_kernel<false, false>);
    const int gridRows = persistent_grid(s, nrows, kThreads), gridNr = persistent_grid(s, nr, kThreads);
    const int gridRow = std::max(1, std::min(iceil(itemCap, kThreads), 8 * s.numSMs));
    const int bgrid = std::min(iceil(leafCap, 256), 4 * s.numSMs);
    const int pgrid = grid_for(s, leafCap);
    const RowSplit rows{s.nblCount.get(), s.nblH.get(), kNbl, s.rowItems.get()};
    const PreorderTree tree{s.preCenter.get(), s.preHalf.get(), s.preSkip.get(), s.preLeaf.get(), 0, 0, &L->numNodes};
    const long long waitNs = wait_limit_ns();
    const int* dims = &L->nLeaves;

    KeyBytes key;
    for (const void* q : {(const void*)L, (const void*)ds, (const void*)s.activeA.get(), (const void*)s.activeB.get(),
                          (const void*)s.leafNext.get(), (const void*)s.items.get(), (const void*)s.rowItems.get(),
                          (const void*)s.nblR2.get(), (const void*)s.nblCount.get(), (const void*)s.nblH.get(),
                          (const void*)s.layout.get(), (const void*)s.converged.get(), (const void*)s.jstream.get(),
                          (const void*)s.xyzh.get(), (const void*)s.rho.get(), (const void*)s.gradh.get(),
                          (const void*)s.box.get(), (const void*)s.listH.get(), (const void*)s.preCenter.get(),
                          (const void*)s.preHalf.get(), (const void*)s.preSkip.get(), (const void*)s.preLeaf.get(),
                          (const void*)s.leafToInternal.get(), (const void*)s.centers.get(), (const void*)s.sizes.get(),
                          (const void*)s.jOffset.get(), (const void*)s.jcount.get(), (const void*)s.jlist.get(),
                          (const void*)s.jlistPrev.get(), (const void*)s.jOffsetPrev.get(), (const void*)s.walked.get(),
                          (const void*)s.walkScratch.get(), (const void*)s.hmaxLeaf.get(), (const void*)s.hmaxPre.get(),
                          (const void*)s.particleLeaf.get(), (const void*)s.scanTmp.get(), (const void*)nrows,
                          (const void*)nr, (const void*)rk, (const void*)rowsJ})
        key.add(q);
    for (long long v : {(long long)leafCap, (long long)itemCap, (long long)gridRows, (long long)gridNr,
                        (long long)gridRow, (long long)bgrid, (long long)pgrid, (long long)s.periodic,
                        (long long)spreadG, (long long)cut.stream, (long long)cut.work, (long long)listStore, waitNs,
                        (long long)s.numSMs})
        key.add(v);
    for (double v : {pmass, tolh, hfact}) key.add(v);

    s.loopKeyLast = key.b;
    if (!s.loopGraphExec || key.b != s.loopGraphKey)
    {
        // a graph is built for parameters met a second time in a row (a stepping caller's
        // solves, whose buffers have stopped growing); a one-off solve -- another set, a
        // new particle mass, a buffer that grew -- runs on the host loop, with the first
        // lists already built, instead of paying a capture and an instantiation
        if (key.b != s.loopKeyPending)
        {
            s.loopKeyPending = key.b;
            return LoopGraph::Deferred;
        }
        if (s.loopGraphExec) COSMO_CUDA(cudaGraphExecDestroy(s.loopGraphExec));
        if (s.loopGraphDef) COSMO_CUDA(cudaGraphDestroy(s.loopGraphDef));
        s.loopGraphExec = nullptr;
        s.loopGraphDef = nullptr;
        s.loopGraphKey.clear();
        s.listStore = listStore;
        const unsigned long long launches0 = g_launches.load();
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ex = nullptr;
        bool built = false;
        unsigned long long kMain = 0, kList = 0, kRows = 0;
        do
        {
            if (cudaGraphCreate(&g, 0) != cudaSuccess) break;
            cudaGraphConditionalHandle hMore, hList, hRows;
            if (cudaGraphConditionalHandleCreate(&hMore, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) break;
            cudaGraphNodeParams wp = {};
            wp.type = cudaGraphNodeTypeConditional;
            wp.conditional.handle = hMore;
            wp.conditional.type = cudaGraphCondTypeWhile;
            wp.conditional.size = 1;
            cudaGraphNode_t wnode;
            if (cudaGraphAddNode(&wnode, g, nullptr, 0, &wp) != cudaSuccess) break;
            cudaGraph_t body = wp.conditional.phGraph_out[0];
            if (cudaGraphConditionalHandleCreate(&hList, body, 0, 0) != cudaSuccess) break;
            if (cudaGraphConditionalHandleCreate(&hRows, body, 0, 0) != cudaSuccess) break;

            // the branch conditions and hmax of the active leaves
            unsigned long long c0 = g_launches.load();
            if (cudaStreamBeginCaptureToGraph(s.st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) !=
                cudaSuccess)
                break;
            newton_decide_kernel<<<1, 1, 0, s.st>>>(L, hList, hRows);
            COSMO_LAUNCHED();
            hmax_leaves(s, s.activeA.get(), leafCap, &L->nActiveLeaves);
            cudaStreamCaptureStatus cs;
            const cudaGraphNode_t* deps = nullptr;
            size_t nd = 0;
            const bool infoOk = cudaStreamGetCaptureInfo(s.st, &cs, nullptr, nullptr, &deps, &nd) == cudaSuccess;
            std::vector<cudaGraphNode_t> sink(deps, deps + (infoOk ? nd : 0));
            if (cudaStreamEndCapture(s.st, &body) != cudaSuccess || !infoOk) break;
            kMain += g_launches.load() - c0;

            // [the incremental list rebuild]
            cudaGraphNodeParams lp = {};
            lp.type = cudaGraphNodeTypeConditional;
            lp.conditional.handle = hList;
            lp.conditional.type = cudaGraphCondTypeIf;
            lp.conditional.size = 1;
            cudaGraphNode_t lnode;
            if (cudaGraphAddNode(&lnode, body, sink.data(), sink.size(), &lp) != cudaSuccess) break;
            cudaGraph_t lbody = lp.conditional.phGraph_out[0];
            c0 = g_launches.load();
            if (cudaStreamBeginCaptureToGraph(s.st, lbody, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) !=
                cudaSuccess)
                break;
            build_lists_device(s, kListMargin, true, cut.work, dims, leafCap);
            newton_count_kernel<<<1, 1, 0, s.st>>>(L, 0);
            COSMO_LAUNCHED();
            if (cudaStreamEndCapture(s.st, &lbody) != cudaSuccess) break;
            kList = g_launches.load() - c0;

            // [the Newton rows of the still-active particles at their current h]
            cudaGraphNodeParams rp = {};
            rp.type = cudaGraphNodeTypeConditional;
            rp.conditional.handle = hRows;
            rp.conditional.type = cudaGraphCondTypeIf;
            rp.conditional.size = 1;
            cudaGraphNode_t rnode;
            if (cudaGraphAddNode(&rnode, body, &lnode, 1, &rp) != cudaSuccess) break;
            cudaGraph_t rbody = rp.conditional.phGraph_out[0];
            c0 = g_launches.load();
            if (cudaStreamBeginCaptureToGraph(s.st, rbody, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) !=
                cudaSuccess)
                break;
            begin_iteration_kernel<<<bgrid, 256, 0, s.st>>>(ds, s.leafNext.get(), leafCap, dims);
            COSMO_LAUNCHED();
            plan_items_count_kernel<<<pgrid, kThreads, 0, s.st>>>(
                s.activeA.get(), &L->nActiveLeaves, nullptr, s.layout.get(), s.converged.get(), s.jstream.get(),
                s.xyzh.get(), s.items.get(), itemCap, ds, RowSplit{nullptr, nullptr, 0, nullptr}, cut, spreadG);
            COSMO_LAUNCHED();
            nrows<<<gridRows, kThreads, 0, s.st>>>(s.items.get(), itemCap, s.layout.get(), s.jOffset.get(),
                                                   s.jcount.get(), s.jlist.get(), s.xyzh.get(), s.box.get(),
                                                   s.listH.get(), s.nblR2.get(), s.nblCount.get(), s.nblH.get(), ds,
                                                   rowsJ);
            COSMO_LAUNCHED();
            newton_count_kernel<<<1, 1, 0, s.st>>>(L, 1);
            COSMO_LAUNCHED();
            if (cudaStreamEndCapture(s.st, &rbody) != cudaSuccess) break;
            kRows = g_launches.load() - c0;

            // the iteration proper
            c0 = g_launches.load();
            if (cudaStreamBeginCaptureToGraph(s.st, body, &rnode, nullptr, 1, cudaStreamCaptureModeRelaxed) !=
                cudaSuccess)
                break;
            begin_iteration_kernel<<<bgrid, 256, 0, s.st>>>(ds, s.leafNext.get(), leafCap, dims);
            COSMO_LAUNCHED();
            plan_items_count_kernel<<<pgrid, kThreads, 0, s.st>>>(
                s.activeA.get(), &L->nActiveLeaves, &L->rowsReady, s.layout.get(), s.converged.get(),
                s.jstream.get(), s.xyzh.get(), s.items.get(), itemCap, ds, rows, cut, spreadG);
            COSMO_LAUNCHED();
            nr<<<gridNr, kThreads, 0, s.st>>>(s.items.get(), itemCap, s.layout.get(), s.jOffset.get(), s.jcount.get(),
                                              s.jlist.get(), s.xyzh.get(), s.rho.get(), s.gradh.get(),
                                              s.converged.get(), pmass, tolh, hfact, s.box.get(), s.listH.get(),
                                              s.leafNext.get(), s.activeB.get(), tree, s.leafToInternal.get(),
                                              s.centers.get(), s.sizes.get(), ds, waitNs);
            COSMO_LAUNCHED();
            rk<<<gridRow, kThreads, 0, s.st>>>(s.rowItems.get(), s.nblR2.get(), s.nblCount.get(), s.xyzh.get(),
                                              s.rho.get(), s.gradh.get(), s.converged.get(), pmass, tolh, hfact,
                                              s.box.get(), s.listH.get(), s.particleLeaf.get(), s.leafNext.get(),
                                              s.activeB.get(), ds);
            COSMO_LAUNCHED();
            newton_copy_active_kernel<<<bgrid, 256, 0, s.st>>>(s.activeB.get(), s.activeA.get(), ds, leafCap);
            COSMO_LAUNCHED();
            newton_epilogue_kernel<<<1, 1, 0, s.st>>>(L, ds, s.jOffset.get(), hMore);
            COSMO_LAUNCHED();
            if (cudaStreamEndCapture(s.st, &body) != cudaSuccess) break;
            kMain += g_launches.load() - c0;
            if (cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) break;
            built = true;
        } while (false);
        s.listStore = 0;
        // what was captured did not run: the launches counted are those the graph executes
        g_launches -= g_launches.load() - launches0;
        if (!built)
        {
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            if (cudaStreamIsCapturing(s.st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
            {
                cudaGraph_t junk = nullptr;
                cudaStreamEndCapture(s.st, &junk);
                if (junk) cudaGraphDestroy(junk);
            }
            if (ex) cudaGraphExecDestroy(ex);
            if (g) cudaGraphDestroy(g);
            (void)cudaGetLastError();
            return LoopGraph::Failed;
        }
        s.loopGraphDef = g;
        s.loopGraphExec = ex;
        s.loopGraphKey = key.b;
        s.loopKernels[0] = kMain;
        s.loopKernels[1] = kList;
        s.loopKernels[2] = kRows;
        ++s.loopGraphBuilds;
    }
    COSMO_CUDA(cudaGraphLaunch(s.loopGraphExec, s.st));
    cudaEvent_t j2 = ev(s);
    NewtonLoop h;
    uint32_t total = 0;
    COSMO_CUDA(cudaMemcpyAsync(&total, s.jOffset.get() + nL, sizeof(uint32_t), cudaMemcpyDeviceToHost, s.st));
    COSMO_CUDA(cudaMemcpyAsync(&h, L, sizeof(NewtonLoop), cudaMemcpyDeviceToHost, s.st));
    read_scalars(s);
    if (s.hscal->err & kErrListFull) return LoopGraph::Failed;
    g_launches += h.iter * s.loopKernels[0] + h.rebuilds * s.loopKernels[1] + h.rowBuilds * s.loopKernels[2];
    s.listTotal = total;
    s.lastLoopRebuilds = h.rebuilds;
    s.lastLoopRowBuilds = h.rowBuilds;
    s.loopListEntries.assign(h.listEntries, h.listEntries + std::min(h.iter, kLoopIters));
    s.itersRun = h.iter;
    s.settling0 = h.settling0;
    s.activePerIter.assign(h.activePerIter, h.activePerIter + std::min(h.iter, kLoopIters));
    nActiveParticles = h.nActiveParticles;
    s.t.jbuild += elapsed_s(j0, j1);
    s.t.nrkern += elapsed_s(j1, j2);
    return LoopGraph::Ran;
}

constexpr int kSymRowsSkip = 8;   // solves that write no index rows after one that could not use them

// After a converged solve whose Newton rows wrote their j: whether every live particle's
// row covers its converged h.  The particles whose rows do not (those that converged
// before the rows were built, or outgrew them) get rows now, at their converged h, from
// the same lists; false if some still do not (a leaf that streams too much, a row that
// overflows) or too many lack one, and the symmetric rows are built instead.
static bool cover_rows(State& s, int itemCap, FixedSplit cut, int spreadG)
{
    DevScalars* ds = s.dscal.get();
    const int nL = s.nLeaves;
    s.coverFlag.resize(itemCap, s.st);
    s.coverLeaves.resize(nL, s.st);
    s.hs.resize(itemCap, s.st);
    for (int pass = 0; pass < 2; ++pass)
    {
        COSMO_CUDA(cudaMemsetAsync(&ds->coverNeed, 0, 3 * sizeof(int), s.st));   // need, leaves, cut
        row_cover_kernel<<<grid_for(s, nL), kThreads, 0, s.st>>>(
            nL, s.layout.get(), s.xyzh.get(), s.nblCount.get(), s.nblH.get(), s.jstream.get(), cut.stream,
            s.coverFlag.get(), s.coverLeaves.get(), s.hs.get(), ds);
        COSMO_LAUNCHED();
        read_scalars(s);
        const int need = s.hscal->coverNeed;
        if (need == 0) return true;
        if (pass == 1 || need > s.nAlive / 4 || s.hscal->coverCut > 0) return false;
        begin_iteration_kernel<<<std::min(iceil(nL, 256), 4 * s.numSMs), 256, 0, s.st>>>(ds, s.leafNext.get(), nL);
        COSMO_LAUNCHED();
        plan_items_count_kernel<<<grid_for(s, nL), kThreads, 0, s.st>>>(
            s.coverLeaves.get(), &ds->coverLeaves, nullptr, s.layout.get(), s.coverFlag.get(), s.jstream.get(),
            s.xyzh.get(), s.items.get(), itemCap, ds, RowSplit{nullptr, nullptr, 0, nullptr}, cut, spreadG);
        COSMO_LAUNCHED();
        RowsKernelFn nrows = s.precision == 1
                                 ? mixed_newton_rows_kernel(s.periodic)
                                 : (s.periodic ? newton_rows_kernel<true, false> : newton_rows_kernel<false, false>);
        nrows<<<persistent_grid(s, nrows, kThreads), kThreads, 0, s.st>>>(
            s.items.get(), itemCap, s.layout.get(), s.jOffset.get(), s.jcount.get(), s.jlist.get(), s.xyzh.get(),
            s.box.get(), s.listH.get(), s.nblR2.get(), s.nblCount.get(), s.nblH.get(), ds, s.nblJ.get());
        COSMO_LAUNCHED();
    }
    return false;
}

// The symmetric rows from the covering Newton rows (sym_from_rows_kernel), then the
// pairs other particles' supports add, merged into their rows -- all on the device, the
// extras' number read there.  Whether they all fitted is known from extraCount (at most
// extraCap) and mergeOverflow once the stream has been read.
static void sym_rows_from_newton(State& s, int extraCap)
{
    DevScalars* ds = s.dscal.get();
    const int nA = s.nAlive;
    s.extras.resize(extraCap, s.st);
    s.extraCnt.resize(nA, s.st);
    s.extraOff.resize(size_t(nA) + 1, s.st);
    s.extraBucket.resize(extraCap, s.st);
    // extraCount, mergeOverflow and rowOverflow were zeroed by the coverage check; each
    // particle's extras count by the compaction
    const int grid = std::max(1, std::min(iceil(nA, kThreads), 16 * s.numSMs));
    auto compact = [&](auto kern, const auto* rows) {
        kern<<<grid, kThreads, 0, s.st>>>(nA, s.nblJ.get(), rows, s.nblCount.get(), s.hs.get(), s.nblH.get(),
                                          s.xyzh.get(), s.box.get(), s.nbl.get(), s.extras.get(), extraCap,
                                          s.extraCnt.get(), ds);
    };
    // the mixed form's Newton rows hold FP32 r^2 in the same buffer
    const float* rowsF = reinterpret_cast<const float*>(s.nblR2.get());
    if (s.precision == 1)
    {
        if (s.periodic) compact(sym_from_rows_kernel<float, true>, rowsF);
        else compact(sym_from_rows_kernel<float, false>, rowsF);
    }
    else compact(sym_from_rows_kernel<double, false>, s.nblR2.get());
    COSMO_LAUNCHED();
    extras_count_kernel<<<iceil(extraCap, 256), 256, 0, s.st>>>(s.extras.get(), extraCap, ds, s.extraCnt.get());
    COSMO_LAUNCHED();
    scan_exclusive(s, reinterpret_cast<const uint32_t*>(s.extraCnt.get()), s.extraOff.get(), nA, false);
    extras_place_kernel<<<iceil(extraCap, 256), 256, 0, s.st>>>(s.extras.get(), extraCap, ds, s.extraOff.get(),
                                                               s.extraCnt.get(), s.extraBucket.get());
    COSMO_LAUNCHED();
    extras_merge_kernel<<<iceil(nA, 256), 256, 0, s.st>>>(nA, s.extraOff.get(), s.extraBucket.get(), s.nbl.get(),
                                                         s.nblCount.get(), ds);
    COSMO_LAUNCHED();
}

DensResult solve_density(State& s, int n, double pmass, const double* periodicBox, double tolh, double hfact,
                         int maxIter, bool withGradients, bool allowGraph)
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
    // The Newton rows also write their j when the gradient and force passes may run over
    // them: a solve with gradients whose particles all start active (with fixed particles,
    // leaves that never walk would hold no list this solve).  After a solve
    // whose rows did not all cover (a workload with leaves the work queue cuts, say), the
    // next few solves do not write them.
    const bool tryRows = s.symRowsSkip == 0;
    if (s.symRowsSkip > 0) --s.symRowsSkip;
    const bool writeJ = withGradients && s.symFromRows && s.frozenFor != n && tryRows;

    // the tree; its particle gather also zeroes rho, gradh, the convergence flags, the
    // Newton rows' h (0: no row this solve) and the pair counters
    build_tree(s, periodicBox, withGradients, writeJ);
    s.orderFor = n;
    const int nL = s.nLeaves;
    s.activeA.resize(nL, s.st);
    s.activeB.resize(nL, s.st);
    s.leafNext.resize(nL, s.st);
    const int itemCap = std::max(s.nAlive, 1);
    s.items.resize(itemCap, s.st);
    s.rowItems.resize(itemCap, s.st);
    s.nblR2.resize(size_t(itemCap) * kNbl, s.st);
    s.nblCount.resize(itemCap, s.st);
    s.nblH.resize(itemCap, s.st);
    // the index rows' buffer is passed whenever the form has one (the Newton-loop graph
    // keeps one key); the gather set the device switch from writeJ
    int* rowsJ = nullptr;
    if (s.precision == 0 || s.precision == 1)
    {
        s.nblJ.resize(size_t(itemCap) * kNbl, s.st);
        s.nbl.resize(row_buffer_entries(size_t(itemCap)), s.st);
        rowsJ = s.nblJ.get();
    }
    s.rowsFromNewton = false;
    s.hmaxNodeDone = true;
    s.listsLoose = false;

    // the host loop swaps the two active-leaf buffers every iteration: put them back in
    // one order, so that a graph captured with them serves the next solve too
    if (s.activeA.get() > s.activeB.get()) std::swap(s.activeA, s.activeB);
    COSMO_CUDA(cudaMemcpyAsync(s.activeA.get(), s.allLeaves.get(), size_t(nL) * 4, cudaMemcpyDeviceToDevice, s.st));
    int nActiveLeaves = nL;
    long long nActiveParticles = s.nAlive;
    if (s.frozenFor == n && s.nAlive > 0)
    {
        // the caller's fixed particles start converged: neighbours only
        COSMO_CUDA(cudaMemsetAsync(&ds->frozenAlive, 0, sizeof(int), s.st));
        freeze_kernel<<<iceil(s.nAlive, 256), 256, 0, s.st>>>(s.orderA.get(), s.frozen.get(), s.nAlive,
                                                             s.converged.get(), ds);
        COSMO_LAUNCHED();
        read_scalars(s);
        nActiveParticles = s.nAlive - s.hscal->frozenAlive;
    }

    // The gather lists are built with a widened radius and reused while every active h
    // stays inside it: a superset list in ascending leaf order offers the same accepted
    // pairs in the same order, so the sums do not change.  When an h outgrows its leaf's
    // list, only the leaves whose hmax left their radius walk again.  hmaxLeaf is still refreshed
    // for the active leaves every iteration, as the reference does, so the exact lists of
    // the last iteration can be rebuilt afterwards.
    FixedSplit cut;
    if (s.splitStream > 0) cut.stream = s.splitStream;
    if (s.splitWork > 0) cut.work = s.splitWork;
    const int spreadG = s.spreadGroups > 0 ? s.spreadGroups : kSpreadGroups;
    bool listsValid = false, listsWidened = false, rowsReady = false;
    long long settlingPrev = 0;
    bool graphRan = false;
    if (allowGraph && s.newtonGraph && maxIter <= kLoopIters && nActiveParticles > 0)
    {
        const LoopGraph lg =
            newton_loop_graph(s, pmass, tolh, hfact, maxIter, cut, spreadG, nActiveParticles, rowsJ);
        graphRan = lg == LoopGraph::Ran;
        listsWidened = graphRan;
        // deferred: the first lists are built and valid for the host loop's first iteration
        if (lg == LoopGraph::Deferred) listsValid = listsWidened = true;
        if (lg == LoopGraph::Failed && (s.hscal->err & kErrListFull))
        {
            // a list rebuild outgrew the storage the first lists sized: solve again from
            // the caller's arrays with the host loop, which sizes every build
            COSMO_CUDA(cudaMemsetAsync(&ds->err, 0, sizeof(int), s.st));
            s.hscal->err = 0;
            return solve_density(s, n, pmass, periodicBox, tolh, hfact, maxIter, withGradients, false);
        }
    }
    s.lastLoopGraph = graphRan ? 1 : 0;
    cudaEvent_t e3 = ev(s);
    for (int iter = 0; iter < maxIter && !graphRan; ++iter)
    {
        cudaEvent_t j0 = ev(s);
        hmax_leaves(s, s.activeA.get(), nActiveLeaves);
        if (!listsValid)
        {
            // widened, rounded lists; after the first build only outgrown leaves walk
            build_lists(s, false, kListMargin, listsWidened, true, cut.work);
            listsValid = listsWidened = true;
        }
        cudaEvent_t j1 = ev(s);
        {
            const int bgrid = std::min(iceil(nL, 256), 4 * s.numSMs);
            if (!rowsReady && iter >= 1 && nActiveParticles > 0 && 5 * settlingPrev >= 4 * nActiveParticles)
            {
                // rows of the still-active particles at their h after the last update
                begin_iteration_kernel<<<bgrid, 256, 0, s.st>>>(ds, s.leafNext.get(), nL);
                COSMO_LAUNCHED();
                plan_items_kernel<<<grid_for(s, nActiveLeaves), kThreads, 0, s.st>>>(
                    s.activeA.get(), nActiveLeaves, s.layout.get(), s.converged.get(), s.jstream.get(),
                    s.xyzh.get(), s.items.get(), itemCap, ds, RowSplit{nullptr, nullptr, 0, nullptr}, cut, spreadG);
                COSMO_LAUNCHED();
                RowsKernelFn nrows = s.precision == 1
                                         ? mixed_newton_rows_kernel(s.periodic)
                                         : (s.periodic ? newton_rows_kernel<true, false> : newton_rows_kernel<false, false>);
                nrows<<<persistent_grid(s, nrows, kThreads), kThreads, 0, s.st>>>(
                    s.items.get(), itemCap, s.layout.get(), s.jOffset.get(), s.jcount.get(), s.jlist.get(),
                    s.xyzh.get(), s.box.get(), s.listH.get(), s.nblR2.get(), s.nblCount.get(), s.nblH.get(), ds,
                    rowsJ);
                COSMO_LAUNCHED();
                rowsReady = true;
            }
            begin_iteration_kernel<<<bgrid, 256, 0, s.st>>>(ds, s.leafNext.get(), nL);
            COSMO_LAUNCHED();
            plan_items_kernel<<<grid_for(s, nActiveLeaves), kThreads, 0, s.st>>>(
                s.activeA.get(), nActiveLeaves, s.layout.get(), s.converged.get(), s.jstream.get(), s.xyzh.get(),
                s.items.get(), itemCap, ds,
                rowsReady ? RowSplit{s.nblCount.get(), s.nblH.get(), kNbl, s.rowItems.get()}
                          : RowSplit{nullptr, nullptr, 0, nullptr},
                cut, spreadG);
            COSMO_LAUNCHED();
            const bool mx = s.precision == 1;
            NrKernelFn nr = mx ? mixed_density_nr_kernel(s.periodic, s.staging)
                          : s.staging ? (s.periodic ? density_nr_kernel<true, false, true>
                                                    : density_nr_kernel<false, false, true>)
                                      : (s.periodic ? density_nr_kernel<true, false, false>
                                                    : density_nr_kernel<false, false, false>);
            nr<<<persistent_grid(s, nr, kThreads), kThreads, 0, s.st>>>(
                s.items.get(), itemCap, s.layout.get(), s.jOffset.get(), s.jcount.get(), s.jlist.get(), s.xyzh.get(),
                s.rho.get(), s.gradh.get(), s.converged.get(), pmass, tolh, hfact, s.box.get(), s.listH.get(),
                s.leafNext.get(), s.activeB.get(),
                PreorderTree{s.preCenter.get(), s.preHalf.get(), s.preSkip.get(), s.preLeaf.get(), 0, s.numNodes},
                s.leafToInternal.get(), s.centers.get(), s.sizes.get(), ds, wait_limit_ns());
            COSMO_LAUNCHED();
            if (rowsReady)
            {
                RowKernelFn rk = mx ? mixed_density_row_kernel(s.periodic)
                                    : (s.periodic ? density_row_kernel<true, false> : density_row_kernel<false, false>);
                rk<<<std::max(1, std::min(iceil(int(nActiveParticles), kThreads), 8 * s.numSMs)), kThreads, 0,
                     s.st>>>(s.rowItems.get(), s.nblR2.get(), s.nblCount.get(), s.xyzh.get(), s.rho.get(),
                             s.gradh.get(), s.converged.get(), pmass, tolh, hfact, s.box.get(), s.listH.get(),
                             s.particleLeaf.get(), s.leafNext.get(), s.activeB.get(), ds);
                COSMO_LAUNCHED();
            }
        }
        cudaEvent_t j2 = ev(s);
        read_scalars(s);
        s.t.jbuild += elapsed_s(j0, j1);
        s.t.nrkern += elapsed_s(j1, j2);
        s.activePerIter.push_back(nActiveParticles);
        s.itersRun = iter + 1;
        nActiveLeaves = s.hscal->nextActive;
        nActiveParticles = s.hscal->unconverged;
        settlingPrev = s.hscal->settling;
        if (iter == 0) s.settling0 = settlingPrev;
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
    check_dev_err(s, "solveDensH", listsWidened && !withGradients);
    tree_timings(s);
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
    bool symBuilt = false, fromRows = false;
    if (withGradients)
    {
        // hmax of every leaf at the converged h; then the symmetric rows of the gradient
        // and force passes (at the converged h they hold every pair of the gather sweep
        // too): taken from the Newton rows when every live particle's row covers its
        // converged h, otherwise built from the symmetric lists
        cudaEvent_t g0 = ev(s);
        hmax_leaves(s, s.allLeaves.get(), nL);
        const bool rowsBuilt = graphRan ? s.lastLoopRowBuilds > 0 : rowsReady;
        fromRows = writeJ && s.nAlive > 0 && rowsBuilt && cover_rows(s, itemCap, cut, spreadG);
        const int extraCap = s.symExtraCap > 0 ? std::min(s.symExtraCap, itemCap) : itemCap;
        if (fromRows)
            sym_rows_from_newton(s, extraCap);
        else
        {
            build_symmetric(s);
            symBuilt = true;
        }
        cudaEvent_t g1 = ev(s);
        const int grid = grid_for(s, nL);
        if (s.precision == 1)
            launch_gradient_mixed(s, pmass);
        else
        {
            auto gr = s.periodic ? gradient_row_kernel<true> : gradient_row_kernel<false>;
            gr<<<std::max(1, std::min(iceil(s.nAlive, kThreads), 8 * s.numSMs)), kThreads, 0, s.st>>>(
                s.nAlive, s.nbl.get(), s.nblCount.get(), s.xyzh.get(), s.vel4.get(), s.acc4.get(), s.rho.get(),
                s.gradh.get(), s.divv.get(), s.xi.get(), s.ddivvdt.get(), pmass, s.box.get(), ds);
            COSMO_LAUNCHED();
            // the group sweep of the rows that overflowed (none: it returns at once)
            auto gk = s.periodic ? gradient_kernel<true> : gradient_kernel<false>;
            gk<<<grid, kThreads, 0, s.st>>>(nL, s.layout.get(), s.jOffset.get(), s.jcount.get(), s.jlist.get(),
                                            s.xyzh.get(), s.vel4.get(), s.acc4.get(), s.rho.get(), s.gradh.get(),
                                            s.divv.get(), s.xi.get(), s.ddivvdt.get(), pmass, s.box.get(),
                                            s.nblCount.get(), ds);
            COSMO_LAUNCHED();
        }
        if (n > s.nAlive)
        {
            gradient_dead_kernel<<<iceil(n - s.nAlive, 256), 256, 0, s.st>>>(s.nAlive, n, s.divv.get(), s.xi.get(),
                                                                             s.ddivvdt.get());
            COSMO_LAUNCHED();
        }
        cudaEvent_t g2 = ev(s);
        read_scalars(s);
        // the rows serve the force pass if every extra was kept and merged
        if (fromRows) s.rowsFromNewton = s.hscal->extraCount <= extraCap && s.hscal->mergeOverflow == 0;
        if (writeJ && !s.rowsFromNewton) s.symRowsSkip = kSymRowsSkip;
        s.t.gjbuild += elapsed_s(g0, g1);
        s.t.gradkern += elapsed_s(g1, g2);
    }
    check_dev_err(s, "solveDensH", false);
    ++s.token;
    s.forceSinceSolve = false;
    if (symBuilt) s.jlistToken = s.rowsToken = s.token;
    if (s.rowsFromNewton)
    {
        s.rowsToken = s.token;
        s.hmaxNodeDone = false;
    }
    // the lists held are the Newton loop's widened gather lists
    s.listsLoose = withGradients && !symBuilt && listsWidened;
    return res;
}

} // namespace cosmo
