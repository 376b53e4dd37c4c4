/*
 * mixed.cu -- the mixed-precision form of the three pair kernels.
 *
 * Pair interactions run in FP32: coordinates relative to the i-group's box centre (a
 * sub-box of the i-leaf, so relative coordinates are small and keep FP32's precision),
 * W and dW/dq in FP32, and each lane's sums in FP32 with Kahan compensation, combined in
 * FP64 (sum - compensation).  FP64 is kept for the Hilbert keys and the tree (shared with
 * the plain form), velocity differences, the Newton-Raphson h update and convergence
 * test, Omega, the gradient-sweep finish (R-matrix, xi, d(div v)/dt) and the per-particle
 * force factors.  The neighbour sets, the grouping and the j-stream are the plain form's
 * (pairstream.cuh); only the arithmetic of each pair changes.  Accuracy against the FP64
 * form is measured, not assumed (tests/test_mixed_gpu.py, bench.py --precision mixed).
 */
#include <algorithm>

#include "pairstream.cuh"
#include "rows.cuh"
#include "state.hpp"

namespace cosmo {

namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kThreads = 32 * kWarpsPerBlock;

// q = sqrt(q2) for the FP32 path (q2 >= 0); exact 0 for the self pair.
__device__ __forceinline__ float sqrt_f(float q2) { return q2 > 0.0f ? q2 * rsqrtf(q2) : 0.0f; }

// The Newton iteration's mixed form is density_nr_kernel<Periodic, true> (density.cu,
// densengine.cuh); the gradient sweep and the force pass follow.

__device__ inline double xi_limiter_m(const double g[9])
{
    const double dvxdx = (float)g[0], dvxdy = (float)g[1], dvxdz = (float)g[2];
    const double dvydx = (float)g[3], dvydy = (float)g[4], dvydz = (float)g[5];
    const double dvzdx = (float)g[6], dvzdy = (float)g[7], dvzdz = (float)g[8];
    const double divv = dvxdx + dvydy + dvzdz;
    const double cx = dvzdy - dvydz, cy = dvxdz - dvzdx, cz = dvydx - dvxdy;
    const double mdiv = fmax(-divv, 0.0);
    const double fac = mdiv * mdiv;
    const double trS = cx * cx + cy * cy + cz * cz;
    return (fac + trS > 2.220446049250313e-16) ? fac / (fac + trS) : 1.0;
}

// The mixed form's sums of the post-convergence sweep for one particle: FP32 pair terms,
// rho, d(rho)/dh and div v with Kahan compensation, the 24 velocity- and acceleration-
// gradient and R-matrix sums as plain FP32 sums (the compensation of 24 more sums held
// the kernel at 128 registers, four blocks per SM, on a pass that waits on its gathers);
// all combined in FP64 for the FP64 finish of the plain form (src/density_base.cu:
// 635-713).  Their error against the FP64 form is measured with the rest.
struct SumF
{
    float s = 0.0f;
    __device__ __forceinline__ void add(float x) { s += x; }
    __device__ __forceinline__ double value() const { return double(s); }
};

struct GradSumsF
{
    KahanF srho, sgh, sdiv;
    SumF sdv[9], sda[9], sr[6];
    unsigned int gp = 0;

    // One pair: FP32 separation (dx, dy, dz) at the nearest image, r^2 and q^2.
    __device__ __forceinline__ void add(float dx, float dy, float dz, float r2, float q2, const double4& vi,
                                        const double4& ai, const double4& vj, const double4& aj, float pmf)
    {
        const float q = sqrt_f(q2);
        float wk, dwk;
        sph_kernel_f(q2, q, wk, dwk);
        srho.add(wk);
        sgh.add(fmaf(-q, dwk, -3.0f * wk));
        ++gp;
        const float rij1 = r2 > 0.0f ? rsqrtf(r2) : 0.0f;
        const float rg = rij1 * dwk * pmf;
        const float rx = dx * rg, ry = dy * rg, rz = dz * rg;
        const float dvx = float(vi.x - vj.x), dvy = float(vi.y - vj.y), dvz = float(vi.z - vj.z);
        sdiv.add(fmaf(dvz, rz, fmaf(dvy, ry, dvx * rx)));
        sdv[0].add(dvx * rx); sdv[1].add(dvx * ry); sdv[2].add(dvx * rz);
        sdv[3].add(dvy * rx); sdv[4].add(dvy * ry); sdv[5].add(dvy * rz);
        sdv[6].add(dvz * rx); sdv[7].add(dvz * ry); sdv[8].add(dvz * rz);
        const float dax = float(ai.x - aj.x), day = float(ai.y - aj.y), daz = float(ai.z - aj.z);
        sda[0].add(dax * rx); sda[1].add(dax * ry); sda[2].add(dax * rz);
        sda[3].add(day * rx); sda[4].add(day * ry); sda[5].add(day * rz);
        sda[6].add(daz * rx); sda[7].add(daz * ry); sda[8].add(daz * rz);
        sr[0].add(-dx * rx); sr[1].add(-dx * ry); sr[2].add(-dx * rz);
        sr[3].add(-dy * ry); sr[4].add(-dy * rz); sr[5].add(-dz * rz);
    }

    __device__ __forceinline__ void finish(uint32_t i, double hi, double pmass, double* __restrict__ rho,
                                           double* __restrict__ gradh, double* __restrict__ divv,
                                           double* __restrict__ xiOut, double* __restrict__ ddivvdt) const
    {
        double dv[9], da[9];
        for (int c = 0; c < 9; ++c) { dv[c] = sdv[c].value(); da[c] = sda[c].value(); }
        const double rxx = sr[0].value(), rxy = sr[1].value(), rxz = sr[2].value();
        const double ryy = sr[3].value(), ryz = sr[4].value(), rzz = sr[5].value();
        const double hi1 = 1.0 / hi;
        const double hi31 = hi1 * hi1 * hi1;
        const double hi41 = hi31 * hi1;
        const double rho_i = srho.value() * kCnormk * pmass * hi31;
        const double grad_i = sgh.value() * kCnormk * pmass * hi41;
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
        const double rm0 = ryy * rzz - ryz * ryz, rm1 = rxz * ryz - rzz * rxy, rm2 = rxy * ryz - rxz * ryy;
        const double rm3 = rzz * rxx - rxz * rxz, rm4 = rxy * rxz - rxx * ryz, rm5 = rxx * ryy - rxy * rxy;
        divv[i] = -sdiv.value() * term;
        double gm[9], div_a;
        if (fabs(denom) > 2.2250738585072014e-308)
        {
            const double dd = 1.0 / denom;
            for (int r = 0; r < 3; ++r)
            {
                const double sx = dv[3 * r], sy = dv[3 * r + 1], sz = dv[3 * r + 2];
                gm[3 * r]     = -(sx * rm0 + sy * rm1 + sz * rm2) * dd;
                gm[3 * r + 1] = -(sx * rm1 + sy * rm3 + sz * rm4) * dd;
                gm[3 * r + 2] = -(sx * rm2 + sy * rm4 + sz * rm5) * dd;
            }
            double diag = 0.0;
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
            for (int c = 0; c < 9; ++c) gm[c] = -dv[c] * term;
            div_a = -term * (da[0] + da[4] + da[8]);
        }
        xiOut[i] = xi_limiter_m(gm);
        ddivvdt[i] = div_a - (gm[0] * gm[0] + gm[4] * gm[4] + gm[8] * gm[8]
                              + 2.0 * (gm[1] * gm[3] + gm[2] * gm[6] + gm[5] * gm[7]));
    }
};

// Mixed sweep over the group path for the particles whose rows overflowed.
template<bool Periodic>
__global__ void __launch_bounds__(kThreads)
gradient_mixed_kernel(int nL, const uint32_t* __restrict__ layout, const uint32_t* __restrict__ jOffset,
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
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int warpGlobal = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nWarps = (gridDim.x * blockDim.x) >> 5;
    double lx = 0, ly = 0, lz = 0;
    if (Periodic) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }
    const float Lx = float(lx), Ly = float(ly), Lz = float(lz);
    const float pmf = float(pmass);
    unsigned long long pairs = 0;
    auto wanted = [&](uint32_t a) { return nblCount == nullptr || !row_ok(nblCount, a); };
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
                const double rs = kRadKernel * hi;
                const double rmax = warp_max(mine ? rs : 0.0);
                const GroupBox bx = group_box(mine, pi.x, pi.y, pi.z, rs, rmax);
                const float xf = float(pi.x - bx.cx), yf = float(pi.y - bx.cy), zf = float(pi.z - bx.cz);
                const float hinv2f = float(1.0 / (hi * hi));
                GradSumsF gs;
                stream_pairs(
                    sRing[wib], sRingF[wib], sIdx[wib], bx.cx, bx.cy, bx.cz, jb, nj, jlist, layout, xyzh,
                    [&](const double4& pj) { return in_gather_box<Periodic>(pj, bx, lx, ly, lz); },
                    [&](const double4* ring, const float4* ringf, const int* ringIdx, int head, int count) {
                        two_pass(ring, ringf, ringIdx, head, count, mine,
                                 [&](const float4& pf) {
                                     return r2_f32<Periodic>(xf, yf, zf, pf, Lx, Ly, Lz) * hinv2f < float(kRadK2);
                                 },
                                 [&](const double4&, const float4& pf, int j) {
                                     float dx = xf - pf.x, dy = yf - pf.y, dz = zf - pf.z;
                                     if (Periodic)
                                     {
                                         if (fabsf(dx) > 0.5f * Lx) dx -= copysignf(Lx, dx);
                                         if (fabsf(dy) > 0.5f * Ly) dy -= copysignf(Ly, dy);
                                         if (fabsf(dz) > 0.5f * Lz) dz -= copysignf(Lz, dz);
                                     }
                                     const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                                     gs.add(dx, dy, dz, r2, r2 * hinv2f, vi, ai, ldg4(vel4 + j), ldg4(acc4 + j),
                                            pmf);
                                 });
                    });
                if (!mine) continue;
                pairs += gs.gp;
                gs.finish(i, hi, pmass, rho, gradh, divv, xiOut, ddivvdt);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if (lane == 0) atomicAdd(&ds->pairs[1], pairs);
}

// Mixed sweep over the symmetric rows: one lane per particle, the gather pairs selected
// by the FP64 test; the separation is formed in FP64 at the nearest image and rounded to
// FP32, the pair terms are the group path's.
template<bool Periodic>
__global__ void __launch_bounds__(kThreads, 6)
gradient_row_mixed_kernel(int nAlive, const int* __restrict__ nbl, const int* __restrict__ nblCount,
                          const double4* __restrict__ xyzh, const double4* __restrict__ vel4,
                          const double4* __restrict__ acc4, double* __restrict__ rho, double* __restrict__ gradh,
                          double* __restrict__ divv, double* __restrict__ xiOut, double* __restrict__ ddivvdt,
                          double pmass, const DevBox* __restrict__ box, DevScalars* __restrict__ ds)
{
    double lx = 0, ly = 0, lz = 0;
    if (Periodic) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }
    const float pmf = float(pmass);
    unsigned long long pairs = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nAlive; i += gridDim.x * blockDim.x)
    {
        if (!row_ok(nblCount, uint32_t(i))) continue;
        const int cnt = nblCount[i];
        const double4 pi = xyzh[i];
        const double4 vi = vel4[i];
        const double4 ai = acc4[i];
        const float hinv2f = float(1.0 / (pi.w * pi.w));
        const int* row = row_of(nbl, uint32_t(i));
        GradSumsF gs;
        const double hinv2 = 1.0 / (pi.w * pi.w);
        auto pair = [&](int j) {
            const double4 pj = ldg4(xyzh + j);
            double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            nearest_image<Periodic>(dx, dy, dz, lx, ly, lz);
            if (!(pair_r2(dx, dy, dz) * hinv2 < kRadK2)) return;   // the gather pairs of the row
            const float fx = float(dx), fy = float(dy), fz = float(dz);
            const float r2 = fmaf(fz, fz, fmaf(fy, fy, fx * fx));
            gs.add(fx, fy, fz, r2, r2 * hinv2f, vi, ai, ldg4(vel4 + j), ldg4(acc4 + j), pmf);
        };
        for_row(row, cnt, pair);
        pairs += gs.gp;
        gs.finish(uint32_t(i), pi.w, pmass, rho, gradh, divv, xiOut, ddivvdt);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&ds->pairs[1], pairs);
}

// FP32 copies of the per-particle force factors (the FP64 ones are formed by the plain
// prep kernel first, with the reference's expressions).
__global__ void force_prep_f32_kernel(const double4* __restrict__ prepA, const double4* __restrict__ prepB,
                                      const double4* __restrict__ thermo4, int n, float4* __restrict__ prepAf,
                                      float4* __restrict__ prepBf, float4* __restrict__ thermof)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 a = prepA[i], b = prepB[i], t = thermo4[i];
    prepAf[i] = make_float4(float(a.x), float(a.y), float(a.z), float(a.w));
    prepBf[i] = make_float4(float(b.x), float(b.y), float(b.z), float(b.w));
    thermof[i] = make_float4(float(t.x), float(t.y), float(t.z), float(t.w));
}

// The mixed form's force sums of one particle: FP32 pair arithmetic on FP32 factors, Kahan
// sums combined in FP64.
struct ForceAccF
{
    double4 p, v;
    float hif, pro2i, vwavei, alphai, eni, hsqinvi, hinvi, rhoi, rho1i, grkfaci, pri, autermi, divfac;
    KahanF sfx, sfy, sfz, sf4, sdiv;
    float vsm = 0.0f;
    unsigned int gp = 0;

    __device__ __forceinline__ void load(uint32_t i, const double4* __restrict__ xyzh,
                                         const double4* __restrict__ vel4, const float4* __restrict__ thermof,
                                         const float4* __restrict__ prepAf, const float4* __restrict__ prepBf)
    {
        p = xyzh[i]; v = vel4[i];
        const float4 ti = thermof[i], ai = prepAf[i], bi = prepBf[i];
        hif = float(p.w);
        pro2i = ti.x; vwavei = ti.y; alphai = ti.z; eni = ti.w;
        hsqinvi = ai.x; hinvi = ai.y; rhoi = ai.z; rho1i = ai.w;
        grkfaci = bi.x; pri = bi.y; autermi = bi.z; divfac = bi.w;
    }

    // One pair with j at FP32 separation (dx, dy, dz), dr2 > 0, h_j = hj.
    template<bool Disc>
    __device__ __forceinline__ void add(float dx, float dy, float dz, float dr2, float hj, int j,
                                        const double4* __restrict__ vel4, const float4* __restrict__ thermof,
                                        const float4* __restrict__ prepAf, const float4* __restrict__ prepBf,
                                        float pm, float bt, int pdv, int shock)
    {
        const float R2 = float(kRadK2);
        const float4 aj = __ldg(prepAf + j);
        const float qi2 = dr2 * hsqinvi, qj2 = dr2 * aj.x;
        const float rij1 = rsqrtf(dr2);
        const float dr = dr2 * rij1;
        const float rx = dx * rij1, ry = dy * rij1, rz = dz * rij1;
        const double4 vj = ldg4(vel4 + j);
        const float dvx = float(v.x - vj.x), dvy = float(v.y - vj.y), dvz = float(v.z - vj.z);
        const float projv = fmaf(dvz, rz, fmaf(dvy, ry, dvx * rx));
        const float4 tj = __ldg(thermof + j);
        const float4 bj = __ldg(prepBf + j);
        const float rhoj = aj.z, rho1j = aj.w, pro2j = tj.x;
        const float vwavej = tj.y, alphaj = tj.z, enj = tj.w;
        const float prj = bj.y, autermj = bj.z;
        const float vsigi = fmaxf(fmaf(-bt, projv, vwavei), 0.0f);
        const float vsigavi = fmaxf(fmaf(-bt, projv, alphai * vwavei), 0.0f);
        const float vsigj = fmaxf(fmaf(-bt, projv, vwavej), 0.0f);
        const float vsigavj = fmaxf(fmaf(-bt, projv, alphaj * vwavej), 0.0f);
        const float pvs = fmaxf(vsigi, vsigj);
        float qr2i = 0.0f, qr2j = 0.0f;
        const float denij = eni - enj;
        const float vsigu = sqrtf(fabsf(pri - prj) * (2.0f / (rhoi + rhoj)));
        if (Disc)
        {
            const float hori = hif * rij1, horj = hj * rij1;
            if (projv < 0.0f)
            {
                qr2i = -0.5f * rho1i * fmaf(-bt, projv, alphai * vwavei) * hori * projv;
                qr2j = -0.5f * rho1j * fmaf(-bt, projv, alphaj * vwavej) * horj * projv;
            }
            else
            {
                qr2i = -0.5f * rho1i * alphai * vwavei * hori * projv;
                qr2j = -0.5f * rho1j * alphaj * vwavej * horj * projv;
            }
        }
        else if (projv < 0.0f)
        {
            qr2i = -0.5f * rho1i * vsigavi * projv;
            qr2j = -0.5f * rho1j * vsigavj * projv;
        }
        bool took = false;
        if (qi2 < R2)
        {
            took = true;
            vsm = fmaxf(vsm, pvs);
            float wk, dwk;
            sph_kernel_f(qi2, dr * hinvi, wk, dwk);
            sdiv.add(pm * dwk * projv);
            const float gki = dwk * grkfaci;
            const float gpi = pm * (pro2i + qr2i) * gki;
            sfx.add(-gpi * rx); sfy.add(-gpi * ry); sfz.add(-gpi * rz);
            const float pdvi = pm * pro2i * projv * gki;
            const float dissi = Disc ? -0.5f * pm * rho1i * alphai * vwavei * (hif * rij1) * projv * projv * gki
                                     : pm * qr2i * projv * gki;
            const float condi = vsigu * denij * autermi * gki;
            if (pdv) sf4.add(pdvi);
            if (shock) sf4.add(dissi);
            sf4.add(condi);
        }
        if (qj2 < R2)
        {
            took = true;
            vsm = fmaxf(vsm, pvs);
            float wk, dwk;
            sph_kernel_f(qj2, dr * aj.y, wk, dwk);
            const float gkj = dwk * bj.x;
            const float gpj = pm * (pro2j + qr2j) * gkj;
            sfx.add(-gpj * rx); sfy.add(-gpj * ry); sfz.add(-gpj * rz);
            sf4.add(vsigu * denij * autermj * gkj);
        }
        if (took) ++gp;
    }

    __device__ __forceinline__ void store(uint32_t i, double* __restrict__ fx, double* __restrict__ fy,
                                          double* __restrict__ fz, double* __restrict__ f4,
                                          double* __restrict__ vsigmax, double* __restrict__ divvF) const
    {
        fx[i] = sfx.value();
        fy[i] = sfy.value();
        fz[i] = sfz.value();
        f4[i] = sf4.value();
        vsigmax[i] = double(vsm);
        divvF[i] = -sdiv.value() * double(divfac);
    }
};

// Mixed force pass over the group path for the particles whose rows overflowed.
template<bool Periodic, bool Disc>
__global__ void __launch_bounds__(kThreads)
force_mixed_kernel(int nL, const uint32_t* __restrict__ layout, const uint32_t* __restrict__ jOffset,
                   const uint32_t* __restrict__ jcount, const int* __restrict__ jlist,
                   const double4* __restrict__ xyzh, const double4* __restrict__ vel4,
                   const float4* __restrict__ thermof, const float4* __restrict__ prepAf,
                   const float4* __restrict__ prepBf, double* __restrict__ fx, double* __restrict__ fy,
                   double* __restrict__ fz, double* __restrict__ f4, double* __restrict__ vsigmax,
                   double* __restrict__ divvF, double pmass, double beta, int pdv, int shock,
                   const DevBox* __restrict__ box, const int* __restrict__ nblCount, DevScalars* __restrict__ ds)
{
    __shared__ double4 sRing[kWarpsPerBlock][kRing];
    __shared__ float4 sRingF[kWarpsPerBlock][kRing];
    __shared__ int sIdx[kWarpsPerBlock][kRing];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int warpGlobal = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nWarps = (gridDim.x * blockDim.x) >> 5;
    double lx = 0, ly = 0, lz = 0;
    if (Periodic) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }
    const float Lx = float(lx), Ly = float(ly), Lz = float(lz);
    const float pm = float(pmass), bt = float(beta);
    const float R2 = float(kRadK2);
    unsigned long long pairs = 0;
    auto wanted = [&](uint32_t a) { return nblCount == nullptr || !row_ok(nblCount, a); };
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
                ForceAccF A;
                A.load(i, xyzh, vel4, thermof, prepAf, prepBf);
                const double hi = A.p.w;
                const double rg = kRadKernel * warp_max(mine ? hi : 0.0);
                const GroupBox bx = group_box(mine, A.p.x, A.p.y, A.p.z, 0.0, rg);
                const float xf = float(A.p.x - bx.cx), yf = float(A.p.y - bx.cy), zf = float(A.p.z - bx.cz);
                stream_pairs(
                    sRing[wib], sRingF[wib], sIdx[wib], bx.cx, bx.cy, bx.cz, jb, nj, jlist, layout, xyzh,
                    [&](const double4& pj) { return in_sym_box<Periodic>(pj, bx, rg, lx, ly, lz); },
                    [&](const double4* ring, const float4* ringf, const int* ringIdx, int head, int count) {
                        two_pass(ring, ringf, ringIdx, head, count, mine,
                                 [&](const float4& pf) {
                                     const float r2 = r2_f32<Periodic>(xf, yf, zf, pf, Lx, Ly, Lz);
                                     const float hm = fmaxf(A.hif, pf.w);
                                     return r2 > 0.0f && r2 < R2 * hm * hm;
                                 },
                                 [&](const double4&, const float4& pf, int j) {
                                     float dx = xf - pf.x, dy = yf - pf.y, dz = zf - pf.z;
                                     if (Periodic)
                                     {
                                         if (fabsf(dx) > 0.5f * Lx) dx -= copysignf(Lx, dx);
                                         if (fabsf(dy) > 0.5f * Ly) dy -= copysignf(Ly, dy);
                                         if (fabsf(dz) > 0.5f * Lz) dz -= copysignf(Lz, dz);
                                     }
                                     const float dr2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                                     A.add<Disc>(dx, dy, dz, dr2, pf.w, j, vel4, thermof, prepAf, prepBf, pm, bt,
                                                 pdv, shock);
                                 });
                    });
                if (!mine) continue;
                pairs += A.gp;
                A.store(i, fx, fy, fz, f4, vsigmax, divvF);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if (lane == 0) atomicAdd(&ds->pairs[2], pairs);
}

// Mixed force pass over the symmetric rows: one lane per particle; the separation is
// formed in FP64 at the nearest image and rounded to FP32.
template<bool Periodic, bool Disc>
__global__ void __launch_bounds__(kThreads)
force_row_mixed_kernel(int nAlive, const int* __restrict__ nbl, const int* __restrict__ nblCount,
                       const double4* __restrict__ xyzh, const double4* __restrict__ vel4,
                       const float4* __restrict__ thermof, const float4* __restrict__ prepAf,
                       const float4* __restrict__ prepBf, double* __restrict__ fx, double* __restrict__ fy,
                       double* __restrict__ fz, double* __restrict__ f4, double* __restrict__ vsigmax,
                       double* __restrict__ divvF, double pmass, double beta, int pdv, int shock,
                       const DevBox* __restrict__ box, DevScalars* __restrict__ ds)
{
    double lx = 0, ly = 0, lz = 0;
    if (Periodic) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }
    const float pm = float(pmass), bt = float(beta);
    unsigned long long pairs = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nAlive; i += gridDim.x * blockDim.x)
    {
        if (!row_ok(nblCount, uint32_t(i))) continue;
        const int cnt = nblCount[i];
        ForceAccF A;
        A.load(uint32_t(i), xyzh, vel4, thermof, prepAf, prepBf);
        const int* row = row_of(nbl, uint32_t(i));
        auto pair = [&](int j) {
            const double4 pj = ldg4(xyzh + j);
            double dx = A.p.x - pj.x, dy = A.p.y - pj.y, dz = A.p.z - pj.z;
            nearest_image<Periodic>(dx, dy, dz, lx, ly, lz);
            const float fx = float(dx), fy = float(dy), fz = float(dz);
            const float dr2 = fmaf(fz, fz, fmaf(fy, fy, fx * fx));
            if (dr2 > 0.0f)
                A.add<Disc>(fx, fy, fz, dr2, float(pj.w), j, vel4, thermof, prepAf, prepBf, pm, bt, pdv, shock);
        };
        for_row(row, cnt, pair);
        pairs += A.gp;
        A.store(uint32_t(i), fx, fy, fz, f4, vsigmax, divvF);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&ds->pairs[2], pairs);
}

int grid_for(const State& s, int work)
{
    return std::max(1, std::min(s.numSMs * 8, iceil(work, kWarpsPerBlock)));
}

} // namespace

void launch_gradient_mixed(State& s, double pmass)
{
    const int nL = s.nLeaves;
    const int grid = grid_for(s, nL);
    auto rows = [&](auto kern) {
        kern<<<std::max(1, std::min(iceil(s.nAlive, kThreads), 8 * s.numSMs)), kThreads, 0, s.st>>>(
            s.nAlive, s.nbl.get(), s.nblCount.get(), s.xyzh.get(), s.vel4.get(), s.acc4.get(), s.rho.get(),
            s.gradh.get(), s.divv.get(), s.xi.get(), s.ddivvdt.get(), pmass, s.box.get(), s.dscal.get());
    };
    auto go = [&](auto kern) {
        kern<<<grid, kThreads, 0, s.st>>>(nL, s.layout.get(), s.jOffset.get(), s.jcount.get(), s.jlist.get(),
                                          s.xyzh.get(), s.vel4.get(), s.acc4.get(), s.rho.get(), s.gradh.get(),
                                          s.divv.get(), s.xi.get(), s.ddivvdt.get(), pmass, s.box.get(),
                                          s.nblCount.get(), s.dscal.get());
    };
    if (s.periodic) { rows(gradient_row_mixed_kernel<true>); go(gradient_mixed_kernel<true>); }
    else { rows(gradient_row_mixed_kernel<false>); go(gradient_mixed_kernel<false>); }
    COSMO_LAUNCHED();
    COSMO_LAUNCHED();
}

void launch_force_mixed(State& s, double pmass, double beta, bool disc, bool pdv, bool shock)
{
    const int n = s.ngas, nL = s.nLeaves;
    s.prepAf.resize(n, s.st);
    s.prepBf.resize(n, s.st);
    s.thermof.resize(n, s.st);
    force_prep_f32_kernel<<<iceil(n, 256), 256, 0, s.st>>>(s.prepA.get(), s.prepB.get(), s.thermo4.get(), n,
                                                           s.prepAf.get(), s.prepBf.get(), s.thermof.get());
    COSMO_LAUNCHED();
    const int grid = grid_for(s, nL);
    auto rows = [&](auto kern) {
        kern<<<std::max(1, std::min(iceil(s.nAlive, kThreads), 8 * s.numSMs)), kThreads, 0, s.st>>>(
            s.nAlive, s.nbl.get(), s.nblCount.get(), s.xyzh.get(), s.vel4.get(), s.thermof.get(), s.prepAf.get(),
            s.prepBf.get(), s.fx.get(), s.fy.get(), s.fz.get(), s.f4.get(), s.vsigmax.get(), s.divvF.get(), pmass,
            beta, pdv ? 1 : 0, shock ? 1 : 0, s.box.get(), s.dscal.get());
    };
    auto go = [&](auto kern) {
        kern<<<grid, kThreads, 0, s.st>>>(nL, s.layout.get(), s.jOffset.get(), s.jcount.get(), s.jlist.get(),
                                          s.xyzh.get(), s.vel4.get(), s.thermof.get(), s.prepAf.get(),
                                          s.prepBf.get(), s.fx.get(), s.fy.get(), s.fz.get(), s.f4.get(),
                                          s.vsigmax.get(), s.divvF.get(), pmass, beta, pdv ? 1 : 0, shock ? 1 : 0,
                                          s.box.get(), s.nblCount.get(), s.dscal.get());
    };
    if (s.periodic)
    {
        if (disc) { rows(force_row_mixed_kernel<true, true>); go(force_mixed_kernel<true, true>); }
        else { rows(force_row_mixed_kernel<true, false>); go(force_mixed_kernel<true, false>); }
    }
    else
    {
        if (disc) { rows(force_row_mixed_kernel<false, true>); go(force_mixed_kernel<false, true>); }
        else { rows(force_row_mixed_kernel<false, false>); go(force_mixed_kernel<false, false>); }
    }
    COSMO_LAUNCHED();
    COSMO_LAUNCHED();
}

} // namespace cosmo
