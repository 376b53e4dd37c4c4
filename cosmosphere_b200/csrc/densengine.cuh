/*
 * densengine.cuh -- the density sums of one warp group over its leaf's gather list, shared
 * by the single-set Newton kernel and the batched forest kernel, plain FP64 or mixed.
 *
 * Candidates pass the group box filter into the warp's ring (stream_ranges).  Each batch
 * of up to 32 is then tested with j on the lanes: for each group particle in turn, every
 * lane tests its candidate, and the accepted pairs are appended, particle-major, to the
 * warp's record buffer -- so each particle's records are contiguous and in ascending j.
 * The records are evaluated with one pair per lane (W and -q dW/dq - 3W), and each
 * particle's owner lane adds its own records in order.  All lanes work in every phase
 * whatever the group's size or spatial spread.
 *
 *   plain  the exact FP64 test q^2 = r^2 / h_i^2 < R^2 (src/density_base.cu:270-283) and
 *          FP64 sums in ascending j: bit for bit the oracle's.
 * The periodic form with zero periods behaves, bit for bit, as the open form (the batched
 * kernel runs open and periodic sets through the one periodic instance).
 *
 *   mixed  coordinates relative to the group box centre (at the nearest periodic image
 *          of that centre when the box is small enough for it to be every pair's nearest
 *          image), the test and W, dW in FP32, two group particles per packed f32x2
 *          instruction; the owner's sums are FP32 with Kahan compensation, combined in
 *          FP64.
 */
#pragma once

#include "pairstream.cuh"

namespace cosmo {

constexpr int kRec = 256;   // pair records per warp

// Per-warp shared scratch of density_group: the ring, the group's particles, the pair
// records, and at kBoxAt the group's rounded box (read by the filter from shared memory
// rather than held in registers through the stream).
template<bool Mixed>
struct DensScratch
{
    static constexpr int kBoxAt = Mixed ? (kRing * 16 + 4 * 32 * 4 + 2 * kRec * 4)
                                        : (kRing * 32 + 32 * 32 + 2 * kRec * 8);
    static constexpr int kBytes = kBoxAt + 64;
};

// q = sqrt(q2) in FP32 (q2 >= 0); exact 0 for the self pair.
__device__ __forceinline__ float sqrt_q(float q2) { return q2 > 0.0f ? q2 * rsqrtf(q2) : 0.0f; }

// Sums over the gather list of one group: the lanes [0, ng) own the group's particles
// (pi, with mine set); rhoi and gradhi receive the un-normalised sums (W and
// -q dW/dq - 3W over accepted j), gp the accepted pairs and gc the candidates offered.
template<bool Periodic, bool Mixed, bool Staged = false, bool Round = true, class Ranges>
__device__ __forceinline__ void density_group(unsigned char* scr, bool mine, int ng, const double4& pi, double lx,
                                              double ly, double lz, const GroupSource<Ranges>& src, double& rhoi,
                                              double& gradhi, unsigned int& gp, unsigned int& gc)
{
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const double hi = pi.w;
    const double hinv2 = 1.0 / (hi * hi);
    const double rs = kRadKernel * hi;
    const double rmax = warp_max(mine ? rs : 0.0);
    const GroupBox bx = group_box(mine, pi.x, pi.y, pi.z, rs, rmax);
    // Round: candidates, and the cells of a cut group's tree scan, are taken within the
    // largest support of the members' own bounding box (a rounded box: a single particle's
    // is its sphere), with the box's slack (1e-9 of the support, 1e-13 of |c|) on the
    // radius, far above the rounding of the exact test, so no accepted pair is lost.
    // Otherwise within the box of the search spheres (the batched kernel: its sets' h do
    // not scatter, and its registers are tighter).
    RoundBox* rbp = Round ? reinterpret_cast<RoundBox*>(scr + DensScratch<Mixed>::kBoxAt) : nullptr;
    if constexpr (Round)
    {
        const GroupBox pb = group_box(mine, pi.x, pi.y, pi.z, 0.0, rmax);
        if (lane == 0)
            *rbp = RoundBox{pb.cx, pb.cy, pb.cz, pb.ex, pb.ey, pb.ez,
                            rmax + 1e-9 * rmax + 1e-13 * (fabs(pb.cx) + fabs(pb.cy) + fabs(pb.cz)) + 1e-300};
        __syncwarp();
    }
    auto gather = [&](const double4& pj) {
        if constexpr (Round) return in_round_box<Periodic>(pj, *rbp, lx, ly, lz);
        else return in_gather_box<Periodic>(pj, bx, lx, ly, lz);
    };
    gp = 0;
    gc = 0;
    if constexpr (!Mixed)
    {
        double4* ring = reinterpret_cast<double4*>(scr);
        double4* grp = ring + kRing;
        double* recA = reinterpret_cast<double*>(grp + 32);
        double* recB = recA + kRec;
        if (mine) grp[lane] = make_double4(pi.x, pi.y, pi.z, hinv2);
        __syncwarp();
        double sr = 0.0, sg = 0.0;
        src.template stream<true, false, false, Periodic, Staged>(
            ring, nullptr, nullptr, bx, 0.0, 0.0, 0.0, lx, ly, lz, gather,
            [&](const double4* rg, const float4*, const int*, int head, int count) {
                gc += count;
                const double4 pj = rg[(head + (lane < count ? lane : 0)) & (kRing - 1)];
                if (ng == 1)
                {
                    // a single particle (a cut group): every lane evaluates its own pair, the
                    // accepted values are packed into the record buffers in lane (= j) order,
                    // and the sums add them in that order from broadcast shared-memory loads
                    // -- one add per accepted pair, as in the oracle's loop, so the chain is
                    // bound by the add latency alone
                    const double4 g = grp[0];
                    double dx = g.x - pj.x, dy = g.y - pj.y, dz = g.z - pj.z;
                    nearest_image<Periodic>(dx, dy, dz, lx, ly, lz);
                    const double q2 = pair_r2(dx, dy, dz) * g.w;
                    const bool acc = lane < count && q2 < kRadK2;
                    double wv = 0.0, tv = 0.0;
                    if (acc)
                    {
                        const double q = sqrt(q2);
                        double wk, dwk;
                        sph_kernel(q2, q, wk, dwk);
                        wv = wk;
                        tv = -q * dwk - 3.0 * wk;
                    }
                    const uint32_t am = __ballot_sync(0xffffffffu, acc);
                    const int c = __popc(am);
                    gp += c;
                    if (acc)
                    {
                        recA[__popc(am & lt)] = wv;
                        recB[__popc(am & lt)] = tv;
                    }
                    __syncwarp();
                    for (int t = 0; t < c; ++t)
                    {
                        sr += recA[t];
                        sg += recB[t];
                    }
                    __syncwarp();
                    return;
                }
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
                        sr += recA[segStart + t];
                        sg += recB[segStart + t];
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
                        const double4 g = grp[min(i0 + u, 31)];
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
            },
            rbp);
        rhoi = sr;
        gradhi = sg;
    }
    else
    {
        float4* ringf = reinterpret_cast<float4*>(scr);
        float* gx = reinterpret_cast<float*>(ringf + kRing);
        float* gy = gx + 32;
        float* gz = gy + 32;
        float* gh = gz + 32;
        float* recQ = gh + 32;
        float* recG = recQ + kRec;
        // relative coordinates at the centre's nearest image are every accepted pair's
        // nearest image when the box (search spheres included) spans under half a period
        const bool shifted = !Periodic || lx == 0.0 || (bx.ex < 0.5 * lx && bx.ey < 0.5 * ly && bx.ez < 0.5 * lz);
        const double sx = shifted && Periodic ? lx : 0.0, sy = shifted && Periodic ? ly : 0.0;
        const double sz = shifted && Periodic ? lz : 0.0;
        gx[lane] = mine ? float(pi.x - bx.cx) : 0.0f;
        gy[lane] = mine ? float(pi.y - bx.cy) : 0.0f;
        gz[lane] = mine ? float(pi.z - bx.cz) : 0.0f;
        gh[lane] = mine ? float(hinv2) : 0.0f;
        __syncwarp();
        const float Lx = float(lx), Ly = float(ly), Lz = float(lz);
        KahanF kr, kg, lr, lg;
        src.template stream<false, true, false, Periodic, Staged>(
            nullptr, ringf, nullptr, bx, sx, sy, sz, lx, ly, lz, gather,
            [&](const double4*, const float4* rf, const int*, int head, int count) {
                gc += count;
                const float4 pf = rf[(head + (lane < count ? lane : 0)) & (kRing - 1)];
                if (ng == 1)
                {
                    // a single particle (a cut group): every lane keeps its own compensated
                    // partial sums, combined in FP64 after the stream
                    float dx = gx[0] - pf.x, dy = gy[0] - pf.y, dz = gz[0] - pf.z;
                    if (Periodic && !shifted)
                    {
                        dx = axis_df<true>(gx[0], pf.x, Lx);
                        dy = axis_df<true>(gy[0], pf.y, Ly);
                        dz = axis_df<true>(gz[0], pf.z, Lz);
                    }
                    const float q2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx)) * gh[0];
                    const bool acc = lane < count && q2 < float(kRadK2);
                    if (acc)
                    {
                        const float q = sqrt_q(q2);
                        float wk, dwk;
                        sph_kernel_f(q2, q, wk, dwk);
                        lr.add(wk);
                        lg.add(fmaf(-q, dwk, -3.0f * wk));
                    }
                    gp += __popc(__ballot_sync(0xffffffffu, acc));
                    return;
                }
                int nrec = 0, segStart = 0, segCount = 0;
                auto flush = [&]() {
                    __syncwarp();
                    for (int r = lane; r < nrec; r += 32)
                    {
                        const float q2 = recQ[r];
                        const float q = sqrt_q(q2);
                        float wk, dwk;
                        sph_kernel_f(q2, q, wk, dwk);
                        recQ[r] = wk;
                        recG[r] = fmaf(-q, dwk, -3.0f * wk);
                    }
                    __syncwarp();
                    for (int t = 0; t < segCount; ++t)
                    {
                        kr.add(recQ[segStart + t]);
                        kg.add(recG[segStart + t]);
                    }
                    gp += segCount;
                    segCount = 0;
                    nrec = 0;
                    __syncwarp();
                };
                const float2 nx = make_float2(-pf.x, -pf.x), ny = make_float2(-pf.y, -pf.y);
                const float2 nz = make_float2(-pf.z, -pf.z);
                for (int i0 = 0; i0 < ng; i0 += 4)
                {
                    if (nrec + 4 * 32 > kRec) flush();
                    float q2u[4];
                    if (!Periodic || shifted)
                    {
#pragma unroll
                        for (int h = 0; h < 2; ++h)
                        {
                            const int k = i0 + 2 * h;
                            const float2 dx = __fadd2_rn(*reinterpret_cast<const float2*>(gx + k), nx);
                            const float2 dy = __fadd2_rn(*reinterpret_cast<const float2*>(gy + k), ny);
                            const float2 dz = __fadd2_rn(*reinterpret_cast<const float2*>(gz + k), nz);
                            float2 r2 = __fmul2_rn(dx, dx);
                            r2 = __ffma2_rn(dy, dy, r2);
                            r2 = __ffma2_rn(dz, dz, r2);
                            const float2 q2 = __fmul2_rn(r2, *reinterpret_cast<const float2*>(gh + k));
                            q2u[2 * h] = q2.x;
                            q2u[2 * h + 1] = q2.y;
                        }
                    }
                    else
                    {
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                        {
                            const int k = i0 + u;
                            const float dx = axis_df<true>(gx[k], pf.x, Lx);
                            const float dy = axis_df<true>(gy[k], pf.y, Ly);
                            const float dz = axis_df<true>(gz[k], pf.z, Lz);
                            q2u[u] = fmaf(dz, dz, fmaf(dy, dy, dx * dx)) * gh[k];
                        }
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                    {
                        const bool acc = lane < count && i0 + u < ng && q2u[u] < float(kRadK2);
                        const uint32_t m = __ballot_sync(0xffffffffu, acc);
                        const int c = __popc(m);
                        if (acc) recQ[nrec + __popc(m & lt)] = q2u[u];
                        if (lane == i0 + u) { segStart = nrec; segCount = c; }
                        nrec += c;
                    }
                }
                if (nrec > 0) flush();
            },
            rbp);
        rhoi = kr.value();
        gradhi = kg.value();
        if (ng == 1)
        {
            double a = lr.value(), b = lg.value();
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
            {
                a += __shfl_xor_sync(0xffffffffu, a, o);
                b += __shfl_xor_sync(0xffffffffu, b, o);
            }
            rhoi = a;
            gradhi = b;
        }
    }
}

} // namespace cosmo
