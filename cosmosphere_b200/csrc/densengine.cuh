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
 *   plain  a conservative FP32 prefilter decides which (particle, candidate) pairs are
 *          recorded: coordinates relative to the group box centre, two group particles
 *          per packed f32x2 instruction, against fp32_bound2(R h_i, eps), where eps
 *          bounds the FP32 distance error (fp32_margin) -- it can pass a pair the exact
 *          test rejects, never the reverse.  The records are then evaluated one pair per
 *          lane with the exact FP64 test q^2 = r^2 / h_i^2 < R^2 (src/density_base.cu:
 *          270-283) on the FP64 positions, and the owner adds the exact-accepted ones in
 *          ascending j: the accepted pairs and their order are the oracle's, bit for bit.
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

// Per-warp shared scratch of density_group.
template<bool Mixed>
struct DensScratch
{
    static constexpr int kBytes = (Mixed ? (kRing * 16 + 4 * 32 * 4 + 2 * kRec * 4)
                                         : (kRing * 32 + 32 * 32 + 4 * 32 * 4 + 2 * kRec * 8 + kRec * 4)) +
                                  2 * 8 * 16;   // sub-group boxes
};

// Sub-group boxes.  A group whose smoothing lengths spread widely (largest over smallest
// above kSubSpread) has a box much larger than most of its particles' search spheres -- one
// wide particle sets it.  Such a group gets one box per four consecutive particles (their
// search spheres, widened by eps), and a batch of candidates none of which lies inside a
// sub-group's box skips that sub-group's tests: a candidate outside the box of particle i's
// search sphere can pass neither the prefilter nor the exact test for i.  Offsets are FP32
// from the group box centre (c, e: 8 centres and half extents per warp).
constexpr double kSubSpread = 1.3;

__device__ __forceinline__ bool sub_boxes(float4* sc, float4* se, bool mine, int ng, double hi, double rs,
                                          double ox, double oy, double oz, double eps)
{
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    const double hmin = warp_min(mine ? hi : inf), hmax = warp_max(mine ? hi : 0.0);
    if (!(ng > 4 && hmax > kSubSpread * hmin)) return false;
    const int lane = threadIdx.x & 31;
    double lx = mine ? ox - rs : inf, hx = mine ? ox + rs : -inf;
    double ly = mine ? oy - rs : inf, hy = mine ? oy + rs : -inf;
    double lz = mine ? oz - rs : inf, hz = mine ? oz + rs : -inf;
#pragma unroll
    for (int o = 1; o < 4; o <<= 1)
    {
        lx = fmin(lx, __shfl_xor_sync(0xffffffffu, lx, o)); hx = fmax(hx, __shfl_xor_sync(0xffffffffu, hx, o));
        ly = fmin(ly, __shfl_xor_sync(0xffffffffu, ly, o)); hy = fmax(hy, __shfl_xor_sync(0xffffffffu, hy, o));
        lz = fmin(lz, __shfl_xor_sync(0xffffffffu, lz, o)); hz = fmax(hz, __shfl_xor_sync(0xffffffffu, hz, o));
    }
    if ((lane & 3) == 0 && lane < ng)
    {
        sc[lane >> 2] = make_float4(float(0.5 * (lx + hx)), float(0.5 * (ly + hy)), float(0.5 * (lz + hz)), 0.0f);
        se[lane >> 2] = make_float4(__double2float_ru(0.5 * (hx - lx) + eps), __double2float_ru(0.5 * (hy - ly) + eps),
                                    __double2float_ru(0.5 * (hz - lz) + eps), 0.0f);
    }
    __syncwarp();
    return true;
}

// The sub-groups whose boxes hold a lane's candidate (px, py, pz), OR-ed over the batch.
template<bool Periodic>
__device__ __forceinline__ uint32_t sub_need(const float4* sc, const float4* se, int ng, bool valid, float px,
                                             float py, float pz, float Lx, float Ly, float Lz)
{
    uint32_t m = 0;
    if (valid)
    {
        const int nsub = (ng + 3) >> 2;
        for (int s = 0; s < nsub; ++s)
        {
            const float4 c = sc[s], e = se[s];
            if (axis_df<Periodic>(px, c.x, Lx) <= e.x && axis_df<Periodic>(py, c.y, Ly) <= e.y &&
                axis_df<Periodic>(pz, c.z, Lz) <= e.z)
                m |= 1u << s;
        }
    }
    return __reduce_or_sync(0xffffffffu, m);
}

// q = sqrt(q2) in FP32 (q2 >= 0); exact 0 for the self pair.
__device__ __forceinline__ float sqrt_q(float q2) { return q2 > 0.0f ? q2 * rsqrtf(q2) : 0.0f; }

// Sums over the gather list of one group: the lanes [0, ng) own the group's particles
// (pi, with mine set); rhoi and gradhi receive the un-normalised sums (W and
// -q dW/dq - 3W over accepted j), gp the accepted pairs and gc the candidates offered.
template<bool Periodic, bool Mixed, class Ranges>
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
    gp = 0;
    gc = 0;
    if constexpr (!Mixed)
    {
        double4* ring = reinterpret_cast<double4*>(scr);
        double4* grp = ring + kRing;
        float* gfx = reinterpret_cast<float*>(grp + 32);   // FP32 offsets from the box centre
        float* gfy = gfx + 32;
        float* gfz = gfy + 32;
        float* gfT = gfz + 32;                              // prefilter bound on r^2
        double* recA = reinterpret_cast<double*>(gfT + 32);
        double* recB = recA + kRec;
        int* recI = reinterpret_cast<int*>(recB + kRec);    // (group particle << 8) | ring slot
        float4* subC = reinterpret_cast<float4*>(recI + kRec);
        float4* subE = subC + 8;
        const double period = Periodic ? fmax(lx, fmax(ly, lz)) : 0.0;
        const double eps = fp32_margin(bx, period);
        const bool useSub = sub_boxes(subC, subE, mine, ng, hi, rs, pi.x - bx.cx, pi.y - bx.cy, pi.z - bx.cz, eps);
        if (mine)
        {
            grp[lane] = make_double4(pi.x, pi.y, pi.z, hinv2);
            gfx[lane] = float(pi.x - bx.cx);
            gfy[lane] = float(pi.y - bx.cy);
            gfz[lane] = float(pi.z - bx.cz);
            gfT[lane] = fp32_bound2(rs, eps);
        }
        else
        {
            gfx[lane] = 0.0f;
            gfy[lane] = 0.0f;
            gfz[lane] = 0.0f;
            gfT[lane] = -1.0f;
        }
        __syncwarp();
        const float Lx = float(lx), Ly = float(ly), Lz = float(lz);
        double sr = 0.0, sg = 0.0;
        src.template stream<true, false, false, Periodic>(
            ring, nullptr, nullptr, bx, 0.0, 0.0, 0.0, lx, ly, lz,
            [&](const double4& pj) { return in_gather_box<Periodic>(pj, bx, lx, ly, lz); },
            [&](const double4* rg, const float4*, const int*, int head, int count) {
                gc += count;
                const int mySlot = (head + (lane < count ? lane : 0)) & (kRing - 1);
                const double4 pj = rg[mySlot];
                if (ng == 1)
                {
                    // a single particle (a cut group): every lane evaluates its own pair and
                    // the sums take the accepted lanes in order through shuffles -- the
                    // serial chain is one add per accepted pair, as in the oracle's loop
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
                    uint32_t am = __ballot_sync(0xffffffffu, acc);
                    gp += __popc(am);
                    while (am)
                    {
                        const int k = __ffs(am) - 1;
                        am &= am - 1;
                        sr += __shfl_sync(0xffffffffu, wv, k);
                        sg += __shfl_sync(0xffffffffu, tv, k);
                    }
                    return;
                }
                // the candidate's FP32 offset from the box centre, at its nearest image
                const float px = float(image_offset(pj.x, bx.cx, lx)), py = float(image_offset(pj.y, bx.cy, ly));
                const float pz = float(image_offset(pj.z, bx.cz, lz));
                int nrec = 0, segStart = 0, segCount = 0;
                auto flush = [&]() {
                    __syncwarp();
                    // the exact FP64 test and the pair terms, one record per lane
                    for (int r = lane; r < nrec; r += 32)
                    {
                        const int code = recI[r];
                        const double4 g = grp[code >> 8];
                        const double4 q = ring[code & 0xff];
                        double dx = g.x - q.x, dy = g.y - q.y, dz = g.z - q.z;
                        nearest_image<Periodic>(dx, dy, dz, lx, ly, lz);
                        const double q2 = pair_r2(dx, dy, dz) * g.w;
                        double wv = -1.0, tv = 0.0;   // W >= 0 for an accepted pair
                        if (q2 < kRadK2)
                        {
                            const double qq = sqrt(q2);
                            double wk, dwk;
                            sph_kernel(q2, qq, wk, dwk);
                            wv = wk;
                            tv = -qq * dwk - 3.0 * wk;
                        }
                        recA[r] = wv;
                        recB[r] = tv;
                    }
                    __syncwarp();
                    for (int t = 0; t < segCount; ++t)
                    {
                        const double a = recA[segStart + t];
                        if (a >= 0.0)
                        {
                            sr += a;
                            sg += recB[segStart + t];
                            ++gp;
                        }
                    }
                    segCount = 0;
                    nrec = 0;
                    __syncwarp();
                };
                const float2 nx = make_float2(-px, -px), ny = make_float2(-py, -py), nz = make_float2(-pz, -pz);
                uint32_t need = 0xffffffffu;
                if (useSub)
                    need = (Periodic && Lx != 0.0f)
                               ? sub_need<true>(subC, subE, ng, lane < count, px, py, pz, Lx, Ly, Lz)
                               : sub_need<false>(subC, subE, ng, lane < count, px, py, pz, Lx, Ly, Lz);
                // four group particles per step, two per packed FP32 instruction
                for (int i0 = 0; i0 < ng; i0 += 4)
                {
                    if (!((need >> (i0 >> 2)) & 1u)) continue;   // no candidate of the batch in its box
                    if (nrec + 4 * 32 > kRec) flush();
                    float r2u[4];
                    if (!Periodic || Lx == 0.0f)   // zero periods (an open set) fold nothing
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
                        const bool acc = lane < count && i0 + u < ng && r2u[u] < gfT[i0 + u];
                        const uint32_t m = __ballot_sync(0xffffffffu, acc);
                        const int c = __popc(m);
                        if (acc) recI[nrec + __popc(m & lt)] = ((i0 + u) << 8) | mySlot;
                        if (lane == i0 + u) { segStart = nrec; segCount = c; }
                        nrec += c;
                    }
                }
                if (nrec > 0) flush();
            });
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
        float4* subC = reinterpret_cast<float4*>(recG + kRec);
        float4* subE = subC + 8;
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
        const bool useSub = sub_boxes(subC, subE, mine, ng, hi, rs, pi.x - bx.cx, pi.y - bx.cy, pi.z - bx.cz,
                                      fp32_margin(bx, Periodic ? fmax(lx, fmax(ly, lz)) : 0.0));
        KahanF kr, kg, lr, lg;
        src.template stream<false, true, false, Periodic>(
            nullptr, ringf, nullptr, bx, sx, sy, sz, lx, ly, lz,
            [&](const double4& pj) { return in_gather_box<Periodic>(pj, bx, lx, ly, lz); },
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
                uint32_t need = 0xffffffffu;
                if (useSub)
                    need = (Periodic && !shifted)
                               ? sub_need<true>(subC, subE, ng, lane < count, pf.x, pf.y, pf.z, Lx, Ly, Lz)
                               : sub_need<false>(subC, subE, ng, lane < count, pf.x, pf.y, pf.z, Lx, Ly, Lz);
                for (int i0 = 0; i0 < ng; i0 += 4)
                {
                    if (!((need >> (i0 >> 2)) & 1u)) continue;   // no candidate of the batch in its box
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
            });
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
