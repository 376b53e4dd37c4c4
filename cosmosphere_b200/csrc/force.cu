/*
 * force.cu -- the SPH force pass over the symmetric j-leaf lists: per-particle factors
 * (src/force.cu:92-137), pressure + artificial-viscosity accelerations, du/dt, vsigmax
 * and div v (src/force.cu:145-383), and the list rebuild with its hmax upsweep
 * (src/force.cu:19-88).  One warp per i-leaf; j runs in ascending Hilbert index, as the
 * oracle's, so the plain FP64 results agree with it bit for bit.
 */
#include <algorithm>

#include "pairstream.cuh"
#include "rows.cuh"
#include "state.hpp"
#include "workitems.cuh"

namespace cosmo {

namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kThreads = 32 * kWarpsPerBlock;

// The per-particle factors.  grkfac (prepB.x) is also written to the unused fourth
// component of vel4, so that a pair reads the j side's velocity and grkfac in one 32-byte
// record; the pair derives the j side's pr and auterm from prepA and thermo4 with the
// prep's own operations, so those are the same bits as prepB.y and prepB.z.
__global__ void force_prep_kernel(const double4* __restrict__ xyzh, const double* __restrict__ gradh,
                                  const double4* __restrict__ thermo4, int n, double pmass, double alphau,
                                  double hfact, double4* __restrict__ prepA, double4* __restrict__ prepB,
                                  double4* __restrict__ vel4, DevScalars* __restrict__ ds)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i == 0) ds->pairs[2] = 0;   // the force pass's pair counter
    if (i >= n) return;
    const double hi = xyzh[i].w;
    if (!(hi > 0.0))
    {
        prepA[i] = make_double4(0, 0, 0, 0);
        prepB[i] = make_double4(0, 0, 0, 0);
        vel4[i].w = 0.0;
        return;
    }
    const double hsq = 1.0 / (hi * hi);
    const double h4 = hsq * hsq;
    const double hfoh = hfact / hi;
    const double rho = pmass * hfoh * hfoh * hfoh;
    const double dhdrho = -hi / (3.0 * rho);
    const double omega = 1.0 - dhdrho * gradh[i];
    const double oinv = (omega > 0.0) ? (1 / omega) : 1.0;
    const double pro2 = thermo4[i].x;
    prepA[i] = make_double4(hsq, 1.0 / hi, rho, 1.0 / rho);
    const double grkfac = h4 * kCnormk * oinv;
    prepB[i] = make_double4(grkfac, pro2 * rho * rho, 0.5 * pmass * (1.0 / rho) * alphau,
                            kCnormk * oinv * h4 / rho);
    vel4[i].w = grkfac;
}

// The i-side quantities of one particle and its force sums.
struct ForceAcc
{
    double4 p, v, t, a, b;      // xyzh, vel4, thermo4, prepA, prepB of i
    double itx = 0, ity = 0, itz = 0, jtx = 0, jty = 0, jtz = 0;
    double f4s = 0.0, vsm = 0.0, divs = 0.0;
    unsigned int gp = 0;

    __device__ __forceinline__ void load(uint32_t i, const double4* __restrict__ xyzh,
                                         const double4* __restrict__ vel4, const double4* __restrict__ thermo4,
                                         const double4* __restrict__ prepA, const double4* __restrict__ prepB)
    {
        p = xyzh[i]; v = vel4[i]; t = thermo4[i]; a = prepA[i]; b = prepB[i];
    }

    // One pair with j (src/force.cu:232-383): the exact tests dr^2 > 0 and
    // dr^2 < R^2 max(h_i^2, h_j^2)(1 + 1e-10), then the i-side and j-side terms.  The j
    // side is four 32-byte records (xyzh, prepA, vel4 with grkfac, thermo4).
    template<bool Periodic, bool Disc>
    __device__ __forceinline__ void add(const double4& pj, int j, const double4* __restrict__ vel4,
                                        const double4* __restrict__ thermo4, const double4* __restrict__ prepA,
                                        double lx, double ly, double lz, double pm, double alphau, double beta,
                                        int pdv, int shock)
    {
        double dx = p.x - pj.x, dy = p.y - pj.y, dz = p.z - pj.z;
        nearest_image<Periodic>(dx, dy, dz, lx, ly, lz);
        const double dr2 = pair_r2(dx, dy, dz);
        if (!(dr2 > 0.0)) return;
        const double hi = p.w, hj = pj.w;
        if (dr2 >= kRadK2 * fmax(hi * hi, hj * hj) * (1.0 + 1e-10)) return;
        const double pro2i = t.x, vwavei = t.y, alphai = t.z, eni = t.w;
        const double hsqinvi = a.x, hinvi = a.y, rhoi = a.z, rho1i = a.w;
        const double grkfaci = b.x, pri = b.y, autermi = b.z;
        const double4 aj = ldg4(prepA + j);
        const double qi2 = dr2 * hsqinvi;
        const double qj2 = dr2 * aj.x;
        const double dr = sqrt(dr2);
        const double rij1 = 1.0 / dr;
        const double rx = dx * rij1, ry = dy * rij1, rz = dz * rij1;
        const double4 vj = ldg4(vel4 + j);
        const double dvx = v.x - vj.x, dvy = v.y - vj.y, dvz = v.z - vj.z;
        const double projv = dvx * rx + dvy * ry + dvz * rz;
        const double4 tj = ldg4(thermo4 + j);
        const double rhoj = aj.z, rho1j = aj.w, pro2j = tj.x;
        const double vwavej = tj.y, alphaj = tj.z, enj = tj.w;
        // the prep's pro2 * rho * rho and 0.5 * pmass * (1 / rho) * alphau, operation for
        // operation
        const double prj = pro2j * rhoj * rhoj, autermj = 0.5 * pm * rho1j * alphau;
        const double vsigi = fmax(vwavei - beta * projv, 0.0);
        const double vsigavi = fmax(alphai * vwavei - beta * projv, 0.0);
        const double vsigj = fmax(vwavej - beta * projv, 0.0);
        const double vsigavj = fmax(alphaj * vwavej - beta * projv, 0.0);
        const double pvs = fmax(vsigi, vsigj);
        double qr2i = 0.0, qr2j = 0.0;
        const double denij = eni - enj;
        const double vsigu = sqrt(fabs(pri - prj) * (2.0 / (rhoi + rhoj)));
        if (Disc)
        {
            const double hori = hi * rij1, horj = hj * rij1;
            if (projv < 0.0)
            {
                qr2i = -0.5 * rho1i * (alphai * vwavei - beta * projv) * hori * projv;
                qr2j = -0.5 * rho1j * (alphaj * vwavej - beta * projv) * horj * projv;
            }
            else
            {
                qr2i = -0.5 * rho1i * alphai * vwavei * hori * projv;
                qr2j = -0.5 * rho1j * alphaj * vwavej * horj * projv;
            }
        }
        else if (projv < 0.0)
        {
            qr2i = -0.5 * rho1i * vsigavi * projv;
            qr2j = -0.5 * rho1j * vsigavj * projv;
        }
        bool took = false;
        if (qi2 < kRadK2)
        {
            took = true;
            vsm = fmax(vsm, pvs);
            double wk, dwk;
            const double q = dr * hinvi;
            sph_kernel(qi2, q, wk, dwk);
            divs += pm * dwk * projv;
            const double gki = dwk * grkfaci;
            const double gpi = pm * (pro2i + qr2i) * gki;
            itx += -gpi * rx; ity += -gpi * ry; itz += -gpi * rz;
            const double pdvi = pm * pro2i * projv * gki;
            const double dissi = Disc ? -0.5 * pm * rho1i * alphai * vwavei * (hi * rij1) * projv * projv * gki
                                      : pm * qr2i * projv * gki;
            const double condi = vsigu * denij * autermi * gki;
            if (pdv) f4s += pdvi;
            if (shock) f4s += dissi;
            f4s += condi;
        }
        if (qj2 < kRadK2)
        {
            took = true;
            vsm = fmax(vsm, pvs);
            double wk, dwk;
            const double q = dr * aj.y;
            sph_kernel(qj2, q, wk, dwk);
            const double gkj = dwk * vj.w;
            const double gpj = pm * (pro2j + qr2j) * gkj;
            jtx -= gpj * rx; jty -= gpj * ry; jtz -= gpj * rz;
            f4s += vsigu * denij * autermj * gkj;
        }
        if (took) ++gp;
    }

    __device__ __forceinline__ void store(uint32_t i, double* __restrict__ fx, double* __restrict__ fy,
                                          double* __restrict__ fz, double* __restrict__ f4,
                                          double* __restrict__ vsigmax, double* __restrict__ divvF) const
    {
        fx[i] = itx + jtx;
        fy[i] = ity + jty;
        fz[i] = itz + jtz;
        f4[i] = f4s;
        vsigmax[i] = vsm;
        divvF[i] = -divs * b.w;
    }
};

// Force pass over the group path (one warp per i-leaf, the symmetric list streamed in
// ascending j) for the particles whose rows overflowed (nblCount > kNbl), or for all when
// nblCount is null.
template<bool Periodic, bool Disc>
__global__ void __launch_bounds__(kThreads)
force_kernel(int nL, const uint32_t* __restrict__ layout, const uint32_t* __restrict__ jOffset,
             const uint32_t* __restrict__ jcount, const int* __restrict__ jlist, const double4* __restrict__ xyzh,
             const double4* __restrict__ vel4, const double4* __restrict__ thermo4,
             const double4* __restrict__ prepA, const double4* __restrict__ prepB, double* __restrict__ fx,
             double* __restrict__ fy, double* __restrict__ fz, double* __restrict__ f4,
             double* __restrict__ vsigmax, double* __restrict__ divvF, double pmass, double alphau, double beta,
             int pdv, int shock, const DevBox* __restrict__ box, const int* __restrict__ nblCount,
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
            ForceAcc A;
            A.load(i, xyzh, vel4, thermo4, prepA, prepB);
            const double hi = A.p.w;
            const double rg = kRadKernel * warp_max(mine ? hi : 0.0);
            const GroupBox bx = group_box(mine, A.p.x, A.p.y, A.p.z, 0.0, rg);
            // float prefilter: r_f^2 <= (R max(h_i, h_j) (1 + 1e-5) + margin)^2; the exact
            // tests run in the accept pass
            const float xf = float(A.p.x - bx.cx), yf = float(A.p.y - bx.cy), zf = float(A.p.z - bx.cz);
            const float mf = __double2float_ru(fp32_margin(bx, Periodic ? fmax(lx, fmax(ly, lz)) : 0.0) +
                                               1e-6 * rg);
            const float hif = float(hi);
            const float Lx = float(lx), Ly = float(ly), Lz = float(lz);
            stream_pairs(
                sRing[wib], sRingF[wib], sIdx[wib], bx.cx, bx.cy, bx.cz, jb, nj, jlist, layout, xyzh,
                [&](const double4& pj) { return in_sym_box<Periodic>(pj, bx, rg, lx, ly, lz); },
                [&](const double4* ring, const float4* ringf, const int* ringIdx, int head, int count) {
                  two_pass(ring, ringf, ringIdx, head, count, mine,
                  [&](const float4& pf) {
                    const float r = fmaf(float(kRadKernel) * 1.00001f, fmaxf(hif, pf.w), mf);
                    return r2_f32<Periodic>(xf, yf, zf, pf, Lx, Ly, Lz) <= r * r;
                  },
                  [&](const double4& pj, const float4&, int j) {
                    A.add<Periodic, Disc>(pj, j, vel4, thermo4, prepA, lx, ly, lz, pm, alphau, beta, pdv, shock);
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

// Symmetric rows: every live particle's j with dr^2 < R^2 max(h_i^2, h_j^2)(1 + 1e-10),
// ascending -- the force pass's pairs (which also need dr^2 > 0, tested where the row is
// used) and, at the converged h, every pair of the gather sweep (i itself included).
template<bool Periodic>
__global__ void __launch_bounds__(kThreads)
sym_rows_kernel(const int4* __restrict__ items, int cap, const uint32_t* __restrict__ layout,
                const uint32_t* __restrict__ jOffset, const uint32_t* __restrict__ jcount,
                const int* __restrict__ jlist, const double4* __restrict__ xyzh, const DevBox* __restrict__ box,
                int* __restrict__ nbl, int* __restrict__ nblCount, DevScalars* __restrict__ ds, int prefilter)
{
    __shared__ __align__(16) unsigned char sScr[kWarpsPerBlock][kRowsScratch];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double lx = 0, ly = 0, lz = 0;
    if (Periodic) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }
    const int nHeavy = ds->itemsHeavy, nItems = nHeavy + ds->itemsLight;
    for (;;)
    {
        const int w = next_item(ds, nHeavy, nItems, cap);
        if (w < 0) break;
        const Item d = decode_item(items[w], layout);
        const int slot = group_slot(d.m0, d.m1, d.nAct, d.grp, d.G, lane);
        const bool mine = slot >= 0;
        const uint32_t i = d.g0 + uint32_t(mine ? slot : 0);
        const double4 pi = xyzh[i];
        const double rg = kRadKernel * warp_max(mine ? pi.w : 0.0);
        const GroupBox bx = group_box(mine, pi.x, pi.y, pi.z, 0.0, rg);
        int rowLen = 0;
        // the force pass's test dr^2 < R^2 max(h_i^2, h_j^2)(1 + 1e-10), with each side's
        // bound formed once: rounding is monotone, so the bound of the larger h is the
        // larger bound and max(bound_i, bound_j) is the same double as the test's own
        auto bound = [](double h) { return kRadK2 * (h * h) * (1.0 + 1e-10); };
        // prefilter distances: R h (1 + 1e-10) bounds sqrt(bound(h)) for either side
        auto filt = [&](const double4& pj) { return in_sym_box<Periodic>(pj, bx, rg, lx, ly, lz); };
        auto candB = [](const double4& pj) { return kRadKernel * pj.w * (1.0 + 1e-10); };
        auto exact = [&](const double4& g, const double4& pj, int j) {
            double dx = g.x - pj.x, dy = g.y - pj.y, dz = g.z - pj.z;
            nearest_image<Periodic>(dx, dy, dz, lx, ly, lz);
            const double dr2 = pair_r2(dx, dy, dz);
            return RowEntry<int>{!(dr2 >= fmax(g.w, bound(pj.w))), j};
        };
        int* myRow = mine ? row_of(nbl, uint32_t(i)) : nullptr;
        const double4 gi = make_double4(pi.x, pi.y, pi.z, bound(pi.w));
        const double Bi = kRadKernel * pi.w * (1.0 + 1e-10);
        if (prefilter)
            rows_group<kRowStride, Periodic, true>(sScr[wib], mine, d.ng, gi, Bi, bx, lx, ly, lz, jOffset[d.leaf],
                                                   jcount[d.leaf], jlist, LayoutRanges{layout}, xyzh, filt, candB,
                                                   exact, myRow, rowLen);
        else
            rows_group<kRowStride, Periodic, false>(sScr[wib], mine, d.ng, gi, Bi, bx, lx, ly, lz, jOffset[d.leaf],
                                                    jcount[d.leaf], jlist, LayoutRanges{layout}, xyzh, filt, candB,
                                                    exact, myRow, rowLen);
        if (mine) nblCount[i] = rowLen;
        if (mine && rowLen > kNbl) ds->rowOverflow = 1;
    }
}

// Force pass over the rows: one lane per live particle, its row's pairs in ascending j --
// the group pass's pairs and order, so the results agree with it bit for bit.
template<bool Periodic, bool Disc>
__global__ void __launch_bounds__(kThreads)
force_row_kernel(int nAlive, const int* __restrict__ nbl, const int* __restrict__ nblCount,
                 const double4* __restrict__ xyzh, const double4* __restrict__ vel4,
                 const double4* __restrict__ thermo4, const double4* __restrict__ prepA,
                 const double4* __restrict__ prepB, double* __restrict__ fx, double* __restrict__ fy,
                 double* __restrict__ fz, double* __restrict__ f4, double* __restrict__ vsigmax,
                 double* __restrict__ divvF, double pmass, double alphau, double beta, int pdv, int shock,
                 const DevBox* __restrict__ box, DevScalars* __restrict__ ds)
{
    double lx = 0, ly = 0, lz = 0;
    if (Periodic) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }
    unsigned long long pairs = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nAlive; i += gridDim.x * blockDim.x)
    {
        if (!row_ok(nblCount, uint32_t(i))) continue;
        const int cnt = nblCount[i];
        ForceAcc A;
        A.load(uint32_t(i), xyzh, vel4, thermo4, prepA, prepB);
        const int* row = row_of(nbl, uint32_t(i));
        auto pair = [&](int j) {
            A.add<Periodic, Disc>(ldg4(xyzh + j), j, vel4, thermo4, prepA, lx, ly, lz, pmass, alphau, beta,
                                  pdv, shock);
        };
        for_row(row, cnt, pair);
        pairs += A.gp;
        A.store(uint32_t(i), fx, fy, fz, f4, vsigmax, divvF);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&ds->pairs[2], pairs);
}

// Dead particles: no force (src/force.cu:191-200).
__global__ void force_dead_kernel(int nAlive, int n, double* fx, double* fy, double* fz, double* f4,
                                  double* vsigmax, double* divvF)
{
    const long i = nAlive + long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    fx[i] = 0.0; fy[i] = 0.0; fz[i] = 0.0; f4[i] = 0.0; vsigmax[i] = 0.0; divvF[i] = 0.0;
}

} // namespace

void build_symmetric(State& s)
{
    DevScalars* ds = s.dscal.get();
    const int nL = s.nLeaves;
    hmax_upsweep(s);
    build_lists(s, true);
    if (nL <= 0) return;
    const int grid = std::max(1, std::min(s.numSMs * 8, iceil(nL, kWarpsPerBlock)));
    const int nA = std::max(s.nAlive, 1);
    s.items.resize(nA, s.st);
    s.nbl.resize(row_buffer_entries(size_t(nA)), s.st);
    s.nblCount.resize(nA, s.st);
    begin_iteration_kernel<<<1, 32, 0, s.st>>>(ds, nullptr, 0);
    COSMO_LAUNCHED();
    COSMO_CUDA(cudaMemsetAsync(&ds->rowOverflow, 0, sizeof(int), s.st));
    plan_items_kernel<<<grid, kThreads, 0, s.st>>>(nullptr, nL, s.layout.get(), nullptr, s.jstream.get(),
                                                    s.xyzh.get(), s.items.get(), nA, ds);
    COSMO_LAUNCHED();
    auto rows = s.periodic ? sym_rows_kernel<true> : sym_rows_kernel<false>;
    rows<<<persistent_grid(s, rows, kThreads), kThreads, 0, s.st>>>(
        s.items.get(), nA, s.layout.get(), s.jOffset.get(), s.jcount.get(), s.jlist.get(), s.xyzh.get(),
        s.box.get(), s.nbl.get(), s.nblCount.get(), ds, s.symPrefilter);
    COSMO_LAUNCHED();
}

void compute_forces(State& s, double pmass, double beta, double alphau, bool disc, bool pdv, bool shock)
{
    const int n = s.ngas;
    DevScalars* ds = s.dscal.get();
    cudaEvent_t e0 = ev(s);
    s.forceSinceSolve = true;
    // The symmetric lists and rows are cached per tree (src/force.cu:19-24); the density
    // solve's gradient sweep has normally built the rows already (from the Newton rows, or
    // with the symmetric lists).
    const bool rowsReady = s.rowsToken == s.token && (s.rowsFromNewton || (s.jlistToken == s.token && s.listsSym));
    if (!rowsReady)
    {
        build_symmetric(s);
        s.jlistToken = s.rowsToken = s.token;
        s.rowsFromNewton = false;
        s.hmaxNodeDone = true;
        cudaEvent_t e2 = ev(s);
        COSMO_CUDA(cudaStreamSynchronize(s.st));
        s.t.fjbuild += elapsed_s(e0, e2);
    }
    cudaEvent_t p0 = ev(s);
    force_prep_kernel<<<iceil(n, 256), 256, 0, s.st>>>(s.xyzh.get(), s.gradh.get(), s.thermo4.get(), n, pmass,
                                                       alphau, s.hfact, s.prepA.get(), s.prepB.get(),
                                                       s.vel4.get(), ds);
    COSMO_LAUNCHED();
    cudaEvent_t p1 = ev(s);
    const int nL = s.nLeaves;
    const int grid = std::max(1, std::min(s.numSMs * 8, iceil(nL, kWarpsPerBlock)));
    auto launch = [&](auto kern) {
        kern<<<grid, kThreads, 0, s.st>>>(nL, s.layout.get(), s.jOffset.get(), s.jcount.get(), s.jlist.get(),
                                          s.xyzh.get(), s.vel4.get(), s.thermo4.get(), s.prepA.get(),
                                          s.prepB.get(), s.fx.get(), s.fy.get(), s.fz.get(), s.f4.get(),
                                          s.vsigmax.get(), s.divvF.get(), pmass, alphau, beta, pdv ? 1 : 0,
                                          shock ? 1 : 0, s.box.get(), s.nblCount.get(), ds);
    };
    auto launchRows = [&](auto kern) {
        kern<<<std::max(1, std::min(iceil(s.nAlive, kThreads), 8 * s.numSMs)), kThreads, 0, s.st>>>(
            s.nAlive, s.nbl.get(), s.nblCount.get(), s.xyzh.get(), s.vel4.get(), s.thermo4.get(), s.prepA.get(),
            s.prepB.get(), s.fx.get(), s.fy.get(), s.fz.get(), s.f4.get(), s.vsigmax.get(), s.divvF.get(), pmass,
            alphau, beta, pdv ? 1 : 0, shock ? 1 : 0, s.box.get(), ds);
    };
    // one lane per particle over its symmetric row; the group pass covers only the rows
    // that overflowed
    if (s.precision == 1)
        launch_force_mixed(s, pmass, beta, disc, pdv, shock);
    else if (nL > 0)
    {
        if (s.periodic) { if (disc) launchRows(force_row_kernel<true, true>); else launchRows(force_row_kernel<true, false>); }
        else { if (disc) launchRows(force_row_kernel<false, true>); else launchRows(force_row_kernel<false, false>); }
        COSMO_LAUNCHED();
        if (!s.rowsFromNewton)
        {
            // the group pass of the rows that overflowed (none: it returns at once); rows
            // from the Newton rows never overflow
            if (s.periodic) { if (disc) launch(force_kernel<true, true>); else launch(force_kernel<true, false>); }
            else { if (disc) launch(force_kernel<false, true>); else launch(force_kernel<false, false>); }
            COSMO_LAUNCHED();
        }
    }
    if (n > s.nAlive)
    {
        force_dead_kernel<<<iceil(n - s.nAlive, 256), 256, 0, s.st>>>(s.nAlive, n, s.fx.get(), s.fy.get(),
                                                                      s.fz.get(), s.f4.get(), s.vsigmax.get(),
                                                                      s.divvF.get());
        COSMO_LAUNCHED();
    }
    cudaEvent_t p2 = ev(s);
    read_scalars(s);
    s.t.prep += elapsed_s(p0, p1);
    s.t.fkern += elapsed_s(p1, p2);
    check_dev_err(s, "force_gpu_c", false);
}

} // namespace cosmo
