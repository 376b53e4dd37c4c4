/*
 * c_api.cu -- the drop-in C-ABI (declared in include/cosmosphere.h) and the state
 * plumbing behind it: sizing, the slot table, host <-> device transfers through the
 * Hilbert ordering, pinning, the compute entry points, and their stderr statistics.
 *
 * Semantics follow the reference's src/arrays_c_api.cu, src/dens_c_api.cu,
 * src/force_c_api.cu, src/pin_c_api.cu and src/gpu_state.cu: one process-wide state on
 * one device, every call synchronous with respect to the host, errors abort with a
 * "FATAL:" line.  Test and harness hooks are exported with the cosmo_x_ prefix.
 */
#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "state.hpp"
#include "tma.cuh"
#include "../../include/cosmosphere.h"
#include "../../include/cosmo_density.hpp"

namespace cosmo {

std::atomic<unsigned long long> g_launches{0};
std::atomic<long long> g_deviceBytes{0};

cudaMemPool_t device_pool()
{
    static std::mutex m;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    COSMO_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) fatal("device_pool: device ordinal out of range");
    std::lock_guard<std::mutex> lk(m);
    if (!pools[dev])
    {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        COSMO_CUDA(cudaMemPoolCreate(&pools[dev], &props));
        uint64_t keep = UINT64_MAX;   // freed blocks stay cached for the next state
        COSMO_CUDA(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep));
    }
    return pools[dev];
}

namespace {

// Page-locked scalar blocks of released states, reused by new ones: freeing page-locked
// memory waits for the whole device, which would stall every other state's work.
std::mutex g_pinnedMutex;
std::vector<std::pair<DevScalars*, int*>> g_pinnedFree;

}

// FP64 throughput probe: independent FMA chains per thread, no memory traffic.
__global__ void fp64_peak_kernel(double* out, int iters, double a, double b)
{
    double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-3, x2 = x0 + 2e-3, x3 = x0 + 3e-3;
    double x4 = x0 + 4e-3, x5 = x0 + 5e-3, x6 = x0 + 6e-3, x7 = x0 + 7e-3;
    for (int k = 0; k < iters; ++k)
    {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    const double r = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (r == 12345.0) out[0] = r;   // keeps the chains live
}

void fatal(const char* fmt, ...)
{
    std::fprintf(stderr, "FATAL: ");
    va_list ap;
    va_start(ap, fmt);
    std::vfprintf(stderr, fmt, ap);
    va_end(ap);
    std::fprintf(stderr, "\n");
    std::fflush(stderr);
    std::abort();
}

// Deliberately leaked (src/gpu_state.cu:1-19): no device memory is released during
// static teardown, after the CUDA runtime may have unloaded.
State& state()
{
    static State* s = new State();
    return *s;
}

void ensure_init(State& s)
{
    if (s.st) return;
    COSMO_CUDA(cudaGetDevice(&s.device));
    COSMO_CUDA(cudaDeviceGetAttribute(&s.numSMs, cudaDevAttrMultiProcessorCount, s.device));
    COSMO_CUDA(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
    s.dscal.resize(1, s.st);
    {
        std::lock_guard<std::mutex> lk(g_pinnedMutex);
        if (!g_pinnedFree.empty())
        {
            s.hscal = g_pinnedFree.back().first;
            s.hsmall = g_pinnedFree.back().second;
            g_pinnedFree.pop_back();
        }
    }
    if (!s.hscal)
    {
        COSMO_CUDA(cudaMallocHost(&s.hscal, sizeof(DevScalars)));
        COSMO_CUDA(cudaMallocHost(&s.hsmall, 64 * sizeof(int)));
    }
    std::memset(s.hscal, 0, sizeof(DevScalars));
    s.box.resize(1, s.st);
    if (const char* e = std::getenv("COSMO_MAX_ITER")) s.maxIter = std::max(1, std::atoi(e));
    if (const char* e = std::getenv("COSMO_PRECISION")) s.precision = (std::string(e) == "mixed") ? 1 : 0;
    if (const char* e = std::getenv("COSMO_STAGING")) s.staging = std::atoi(e) != 0;
    if (const char* e = std::getenv("COSMO_SYM_PREFILTER")) s.symPrefilter = std::atoi(e) != 0;
    if (const char* e = std::getenv("COSMO_NEWTON_GRAPH")) s.newtonGraph = std::atoi(e) != 0;
    if (const char* e = std::getenv("COSMO_SYM_FROM_ROWS")) s.symFromRows = std::atoi(e) != 0;
    if (const char* e = std::getenv("COSMO_SPREAD_GROUPS")) s.spreadGroups = std::max(0, std::min(32, std::atoi(e)));
}

size_t state_device_bytes(const State& s)
{
    size_t b = 0;
    auto add = [&](const auto& buf) { b += buf.cap * sizeof(*buf.p); };
    for (auto* d : {&s.ux, &s.uy, &s.uz, &s.uh, &s.uvx, &s.uvy, &s.uvz, &s.uax, &s.uay, &s.uaz, &s.rho, &s.gradh,
                    &s.divv, &s.xi, &s.ddivvdt, &s.fx, &s.fy, &s.fz, &s.f4, &s.vsigmax, &s.divvF, &s.xfer, &s.centers,
                    &s.sizes, &s.hmaxLeaf, &s.hmaxNode, &s.hmaxPre, &s.redTmp, &s.listH, &s.nblH, &s.nblR2, &s.hs})
        add(*d);
    for (auto* d : {&s.xyzh, &s.vel4, &s.acc4, &s.thermo4, &s.prepA, &s.prepB, &s.preCenter, &s.preHalf}) add(*d);
    for (auto* d : {&s.prepAf, &s.prepBf, &s.thermof}) add(*d);
    for (auto* d : {&s.keysA, &s.keysB, &s.csTree, &s.csTree2, &s.prePrefix, &s.bfsPrefix, &s.nodeKeysTmp}) add(*d);
    for (auto* d : {&s.orderA, &s.orderB, &s.particleLeaf, &s.converged, &s.preLeaf, &s.preSkip, &s.bfsToPre,
                    &s.preToBfs, &s.childOffsets, &s.internalToLeaf, &s.levelRange, &s.leafToInternal, &s.jlist,
                    &s.activeA, &s.activeB, &s.allLeaves, &s.nodeValsTmp, &s.leafNext, &s.nbl, &s.nblCount,
                    &s.rowItems, &s.jlistPrev, &s.walked, &s.walkScratch, &s.coverFlag, &s.coverLeaves, &s.extraCnt,
                    &s.extraBucket, &s.nblJ})
        add(*d);
    add(s.items);
    add(s.extras);
    add(s.extraOff);
    for (auto* d : {&s.counts, &s.ops, &s.opsScan, &s.layout, &s.startBounds, &s.nodeCount, &s.leafPreStart, &s.jcount,
                    &s.jstream, &s.jOffset, &s.scanTmp, &s.sortHist, &s.sortBase, &s.sortLookback, &s.jOffsetPrev})
        add(*d);
    add(s.box);
    add(s.dscal);
    return b;
}

void release_state(State& s)
{
    if (!s.st) return;
    COSMO_CUDA(cudaStreamSynchronize(s.st));
    for (auto* b : {&s.ux, &s.uy, &s.uz, &s.uh, &s.uvx, &s.uvy, &s.uvz, &s.uax, &s.uay, &s.uaz, &s.rho, &s.gradh,
                    &s.divv, &s.xi, &s.ddivvdt, &s.fx, &s.fy, &s.fz, &s.f4, &s.vsigmax, &s.divvF, &s.xfer, &s.centers,
                    &s.sizes, &s.hmaxLeaf, &s.hmaxNode, &s.hmaxPre, &s.redTmp, &s.listH, &s.nblH, &s.nblR2, &s.hs})
        b->release(s.st);
    for (auto* b : {&s.xyzh, &s.vel4, &s.acc4, &s.thermo4, &s.prepA, &s.prepB, &s.preCenter, &s.preHalf}) b->release(s.st);
    for (auto* b : {&s.prepAf, &s.prepBf, &s.thermof}) b->release(s.st);
    for (auto* b : {&s.keysA, &s.keysB, &s.csTree, &s.csTree2, &s.prePrefix, &s.bfsPrefix, &s.nodeKeysTmp}) b->release(s.st);
    for (auto* b : {&s.orderA, &s.orderB, &s.particleLeaf, &s.converged, &s.preLeaf, &s.preSkip, &s.bfsToPre,
                    &s.preToBfs, &s.childOffsets, &s.internalToLeaf, &s.levelRange, &s.leafToInternal, &s.jlist,
                    &s.activeA, &s.activeB, &s.allLeaves, &s.nodeValsTmp, &s.leafNext, &s.nbl, &s.nblCount,
                    &s.rowItems, &s.jlistPrev, &s.walked, &s.walkScratch, &s.coverFlag, &s.coverLeaves, &s.extraCnt,
                    &s.extraBucket, &s.nblJ})
        b->release(s.st);
    s.items.release(s.st);
    s.extras.release(s.st);
    s.extraOff.release(s.st);
    for (auto* b : {&s.counts, &s.ops, &s.opsScan, &s.layout, &s.startBounds, &s.nodeCount, &s.leafPreStart, &s.jcount,
                    &s.jstream, &s.jOffset, &s.scanTmp, &s.sortHist, &s.sortBase, &s.sortLookback, &s.jOffsetPrev})
        b->release(s.st);
    s.box.release(s.st);
    s.dscal.release(s.st);
    s.nloop.release(s.st);
    if (s.loopGraphExec) COSMO_CUDA(cudaGraphExecDestroy(s.loopGraphExec));
    if (s.loopGraphDef) COSMO_CUDA(cudaGraphDestroy(s.loopGraphDef));
    s.loopGraphExec = nullptr;
    s.loopGraphDef = nullptr;
    s.loopGraphKey.clear();
    s.loopKeyPending.clear();
    for (auto& e : s.evPool) COSMO_CUDA(cudaEventDestroy(e));
    s.evPool.clear();
    if (s.hscal)
    {
        std::lock_guard<std::mutex> lk(g_pinnedMutex);
        g_pinnedFree.emplace_back(s.hscal, s.hsmall);
    }
    s.hscal = nullptr;
    s.hsmall = nullptr;
    COSMO_CUDA(cudaStreamDestroy(s.st));
    s.st = nullptr;
    s.sizedFor = 0;
    s.orderFor = 0;
}

// src/gpu_state.cu:21-46: every particle-length array, sized once per count.
void size_particle_arrays(State& s, int n)
{
    ensure_init(s);
    if (s.sizedFor == n) return;
    for (auto* b : {&s.ux, &s.uy, &s.uz, &s.uh, &s.uvx, &s.uvy, &s.uvz, &s.uax, &s.uay, &s.uaz, &s.rho, &s.gradh,
                    &s.divv, &s.xi, &s.ddivvdt, &s.fx, &s.fy, &s.fz, &s.f4, &s.vsigmax, &s.divvF})
        b->resize(n, s.st);
    for (auto* b : {&s.xyzh, &s.vel4, &s.acc4, &s.thermo4, &s.prepA, &s.prepB}) b->resize(n, s.st);
    s.xfer.resize(size_t(6) * n, s.st);
    s.keysA.resize(n, s.st);
    s.keysB.resize(n, s.st);
    for (auto* b : {&s.orderA, &s.orderB, &s.particleLeaf, &s.converged}) b->resize(n, s.st);
    COSMO_CUDA(cudaStreamSynchronize(s.st));
    s.sizedFor = n;
}

void read_scalars(State& s)
{
    COSMO_CUDA(cudaMemcpyAsync(s.hscal, s.dscal.get(), sizeof(DevScalars), cudaMemcpyDeviceToHost, s.st));
    COSMO_CUDA(cudaStreamSynchronize(s.st));
}

void check_dev_err(State& s, const char* where, bool reread)
{
    if (reread) read_scalars(s);
    const int e = s.hscal->err;
    if (e)
        fatal("%s: device error 0x%x (%s%s%s%s)", where, e, (e & kErrSortSpin) ? "sort look-back timeout " : "",
              (e & kErrListCap) ? "j-list capacity " : "", (e & kErrStageWait) ? "staging wait timeout " : "",
              (e & kErrFlagWait) ? "flag wait timeout" : "");
}

// Limit of every bounded device wait (sort look-back, staging barriers), nanoseconds.
static std::atomic<long long> g_waitLimitNs{1000000000ll};
long long wait_limit_ns() { return g_waitLimitNs.load(); }

// Test-only waits that can never be satisfied, through the same bounded-wait code as the
// library's own: kind 0 polls a flag no block sets (as the sort's look-back polls its
// predecessor's), kind 1 waits on an mbarrier armed for 32 bytes of bulk copy that is never
// issued (as a staging wait does).  Each gives up after limitNs and raises its bit.
__global__ void wait_test_kernel(int kind, const int* flag, int* err, long long limitNs)
{
    __shared__ __align__(8) uint64_t bar;
    if (kind == 0)
    {
        if (threadIdx.x != 0) return;
        WaitClock clk;
        while (*reinterpret_cast<const volatile int*>(flag) == 0)
            if (clk.over(limitNs)) { atomicOr(err, int(kErrFlagWait)); return; }
        return;
    }
    if (threadIdx.x == 0)
    {
        mbar_init(&bar, 1);
        fence_mbar_init();
        mbar_arrive_expect_tx(&bar, 32u);
    }
    __syncwarp();
    const bool got = mbar_wait_bounded(&bar, 0u, limitNs);
    if (!__all_sync(0xffffffffu, got) && threadIdx.x == 0) atomicOr(err, int(kErrStageWait));
}

// Each state records its phase timings with its own pool of events (the served form runs
// several states from several host threads); elapsed times are read right after the
// synchronisations that follow them, so a ring of 1024 is never overrun.
constexpr int kEvPool = 1024;

cudaEvent_t ev(State& s)
{
    if (s.evPool.empty())
    {
        s.evPool.resize(kEvPool);
        for (auto& e : s.evPool) COSMO_CUDA(cudaEventCreate(&e));
    }
    cudaEvent_t e = s.evPool[s.evNext];
    s.evNext = (s.evNext + 1) % kEvPool;
    COSMO_CUDA(cudaEventRecord(e, s.st));
    return e;
}

void ev_reset(State& s) { s.evNext = 0; }

double elapsed_s(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.0f;
    COSMO_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms * 1e-3;
}

// ------------------------------------------------------------------ slots
struct Comp
{
    double* base;   // Hilbert-order device array
    int stride;     // in doubles
    double* caller; // caller-order upload target, or nullptr
};

static int slot_components(State& s, int slot, Comp* c)
{
    auto d4 = [](DBuf<double4>& b, int off) { return reinterpret_cast<double*>(b.get()) + off; };
    switch (slot)
    {
        case COSMO_POS:
            c[0] = {d4(s.xyzh, 0), 4, s.ux.get()};
            c[1] = {d4(s.xyzh, 1), 4, s.uy.get()};
            c[2] = {d4(s.xyzh, 2), 4, s.uz.get()};
            return 3;
        case COSMO_HSML: c[0] = {d4(s.xyzh, 3), 4, s.uh.get()}; return 1;
        case COSMO_VEL:
            c[0] = {d4(s.vel4, 0), 4, s.uvx.get()};
            c[1] = {d4(s.vel4, 1), 4, s.uvy.get()};
            c[2] = {d4(s.vel4, 2), 4, s.uvz.get()};
            return 3;
        case COSMO_ACCEL:
            c[0] = {d4(s.acc4, 0), 4, s.uax.get()};
            c[1] = {d4(s.acc4, 1), 4, s.uay.get()};
            c[2] = {d4(s.acc4, 2), 4, s.uaz.get()};
            return 3;
        case COSMO_DENS_OUT:
            c[0] = {s.rho.get(), 1, nullptr};
            c[1] = {s.gradh.get(), 1, nullptr};
            return 2;
        case COSMO_GRAD_OUT:
            c[0] = {s.divv.get(), 1, nullptr};
            c[1] = {s.xi.get(), 1, nullptr};
            c[2] = {s.ddivvdt.get(), 1, nullptr};
            return 3;
        case COSMO_THERMO:
            for (int k = 0; k < 4; ++k) c[k] = {d4(s.thermo4, k), 4, nullptr};
            return 4;
        case COSMO_FORCE_OUT:
            c[0] = {s.fx.get(), 1, nullptr};
            c[1] = {s.fy.get(), 1, nullptr};
            c[2] = {s.fz.get(), 1, nullptr};
            c[3] = {s.f4.get(), 1, nullptr};
            c[4] = {s.vsigmax.get(), 1, nullptr};
            c[5] = {s.divvF.get(), 1, nullptr};
            return 6;
        default: return 0;
    }
}

static int slot_ncomp_static(int slot)
{
    switch (slot)
    {
        case COSMO_POS: return 3;
        case COSMO_HSML: return 1;
        case COSMO_VEL: return 3;
        case COSMO_ACCEL: return 3;
        case COSMO_DENS_OUT: return 2;
        case COSMO_GRAD_OUT: return 3;
        case COSMO_THERMO: return 4;
        case COSMO_FORCE_OUT: return 6;
        default: return 0;
    }
}

struct CompSet
{
    double* base[6];
    int stride[6];
};

// dst component c at sorted k  <-  xfer[c*n + order[k]]   (cosmo_upload_sorted)
__global__ void gather_slot_kernel(CompSet cs, int nc, const int* __restrict__ order, int n,
                                   const double* __restrict__ xfer)
{
    const long k = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int src = order[k];
    for (int c = 0; c < nc; ++c) cs.base[c][size_t(k) * cs.stride[c]] = xfer[size_t(c) * n + src];
}

// xfer[c*n + order[k]]  <-  src component c at sorted k   (cosmo_download)
__global__ void scatter_slot_kernel(CompSet cs, int nc, const int* __restrict__ order, int n,
                                    double* __restrict__ xfer)
{
    const long k = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int dst = order[k];
    for (int c = 0; c < nc; ++c) xfer[size_t(c) * n + dst] = cs.base[c][size_t(k) * cs.stride[c]];
}

// dst component c at k  <-  xfer[c*n + k]   (raw upload of a result slot, no permutation)
__global__ void copy_slot_kernel(CompSet cs, int nc, int n, const double* __restrict__ xfer)
{
    const long k = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    for (int c = 0; c < nc; ++c) cs.base[c][size_t(k) * cs.stride[c]] = xfer[size_t(c) * n + k];
}

static void check_sized(State& s, int slot, int n, const char* what, Comp* comps, int& nc)
{
    if (s.sizedFor != n)
        fatal("%s(slot=%d) with n=%d but the device arrays are sized for %d", what, slot, n, s.sizedFor);
    nc = slot_components(s, slot, comps);
    if (nc == 0) fatal("%s called for slot %d, which has no arrays", what, slot);
}

static void require_order(State& s, int slot, int n, const char* what)
{
    if (s.orderFor != n)
        fatal("%s(slot=%d) with no ordering: a density solve must have run first", what, slot);
}

struct XferTimer
{
    State& s;
    double& sink;
    cudaEvent_t a;
    XferTimer(State& st, double& k) : s(st), sink(k) { a = ev(s); }
    ~XferTimer()
    {
        cudaEvent_t b = ev(s);
        COSMO_CUDA(cudaEventSynchronize(b));
        sink += elapsed_s(a, b);
    }
};

static void upload_slot(int slot, const double* host, int n, bool sorted, const char* what)
{
    State& s = state();
    if (n <= 0) return;
    Comp comps[6];
    int nc = 0;
    check_sized(s, slot, n, what, comps, nc);
    if (sorted) require_order(s, slot, n, what);
    XferTimer timer(s, s.uploadSeconds);
    const size_t bytes = size_t(n) * sizeof(double);
    if (!sorted && comps[0].caller)
    {
        for (int c = 0; c < nc; ++c)
            COSMO_CUDA(cudaMemcpyAsync(comps[c].caller, host + size_t(c) * n, bytes, cudaMemcpyHostToDevice, s.st));
        return;
    }
    COSMO_CUDA(cudaMemcpyAsync(s.xfer.get(), host, bytes * nc, cudaMemcpyHostToDevice, s.st));
    CompSet cs{};
    for (int c = 0; c < nc; ++c) { cs.base[c] = comps[c].base; cs.stride[c] = comps[c].stride; }
    if (sorted) gather_slot_kernel<<<iceil(n, 256), 256, 0, s.st>>>(cs, nc, s.orderA.get(), n, s.xfer.get());
    else copy_slot_kernel<<<iceil(n, 256), 256, 0, s.st>>>(cs, nc, n, s.xfer.get());
    COSMO_LAUNCHED();
}

// ------------------------------------------------------------------ stats lines
static bool env_on(const char* k) { return std::getenv(k) != nullptr; }

// Host high-water mark (VmHWM, kB) of this process, as the reference's COSMO_MEM line
// reports it (src/dens_c_api.cu:84-92); 0 where /proc is unavailable.
static long host_peak_kb()
{
    long kb = 0;
    if (FILE* fp = std::fopen("/proc/self/status", "r"))
    {
        char line[256];
        while (std::fgets(line, sizeof line, fp))
            if (std::strncmp(line, "VmHWM:", 6) == 0)
            {
                std::sscanf(line + 6, "%ld", &kb);
                break;
            }
        std::fclose(fp);
    }
    return kb;
}


// The three stderr lines, formatted from their values in the order the reference prints
// them: COSMO_STATS (src/dens_c_api.cu:113-122), COSMO_FORCE (src/force_c_api.cu:74-79)
// and COSMO_MEM (src/dens_c_api.cu:95-97).  Operators grep these key=value fields, so
// the keys, their order and the number formats are the reference's.
// v: n leaves iters vecin upload bbox keysort tree nodes jbuild nrkern gjbuild gradkern
//    download gpusum solve unaccounted total (ms)
static int format_dens_stats(char* buf, size_t len, const double* v)
{
    return std::snprintf(buf, len,
                         "COSMO_STATS n=%d leaves=%d iters=%d | vecin=%.2f upload=%.2f bbox=%.2f keysort=%.2f "
                         "tree=%.2f nodes=%.2f jbuild=%.2f nrkern=%.2f gjbuild=%.2f gradkern=%.2f download=%.2f | "
                         "gpusum=%.2f solve=%.2f unaccounted=%.2f total=%.2f\n",
                         int(v[0]), int(v[1]), int(v[2]), v[3], v[4], v[5], v[6], v[7], v[8], v[9], v[10], v[11],
                         v[12], v[13], v[14], v[15], v[16], v[17]);
}
// v: n leaves upsweep jbuild upload prep kernel download gpusum wall unaccounted (ms)
static int format_force_stats(char* buf, size_t len, const double* v)
{
    return std::snprintf(buf, len,
                         "COSMO_FORCE n=%d leaves=%d | upsweep=%.2f jbuild=%.2f upload=%.2f prep=%.2f kernel=%.2f "
                         "download=%.2f | gpusum=%.2f wall=%.2f unaccounted=%.2f\n",
                         int(v[0]), int(v[1]), v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9], v[10]);
}
// v: n device_used_GB total_GB bytes_per_particle host_peak_GB
static int format_mem_line(char* buf, size_t len, const double* v)
{
    return std::snprintf(buf, len,
                         "COSMO_MEM n=%d device_used=%.2f GB of %.2f GB (%.0f bytes/particle) host_peak=%.2f GB\n",
                         int(v[0]), v[1], v[2], v[3], v[4]);
}

static void print_line(int (*fmt)(char*, size_t, const double*), const double* v)
{
    char buf[512];
    fmt(buf, sizeof buf, v);
    std::fputs(buf, stderr);
}

} // namespace cosmo

using namespace cosmo;

// ====================================================================== the C-ABI
extern "C" {

void cosmo_arrays_init(int n)
{
    if (n <= 0) return;
    size_particle_arrays(state(), n);
}

int cosmo_slot_ncomp(int slot) { return slot_ncomp_static(slot); }

void cosmo_upload(int slot, const double* host, int n) { upload_slot(slot, host, n, false, "cosmo_upload"); }

void cosmo_upload_sorted(int slot, const double* host, int n)
{
    upload_slot(slot, host, n, true, "cosmo_upload_sorted");
}

void cosmo_download(int slot, double* host, int n)
{
    State& s = state();
    if (n <= 0) return;
    Comp comps[6];
    int nc = 0;
    check_sized(s, slot, n, "cosmo_download", comps, nc);
    require_order(s, slot, n, "cosmo_download");
    XferTimer timer(s, s.downloadSeconds);
    CompSet cs{};
    for (int c = 0; c < nc; ++c) { cs.base[c] = comps[c].base; cs.stride[c] = comps[c].stride; }
    scatter_slot_kernel<<<iceil(n, 256), 256, 0, s.st>>>(cs, nc, s.orderA.get(), n, s.xfer.get());
    COSMO_LAUNCHED();
    COSMO_CUDA(cudaMemcpyAsync(host, s.xfer.get(), size_t(n) * nc * sizeof(double), cudaMemcpyDeviceToHost, s.st));
}

void cosmo_pin_host(void* ptr, size_t nbytes)
{
    if (ptr == nullptr || nbytes == 0) return;
    if (cudaHostRegister(ptr, nbytes, cudaHostRegisterDefault) != cudaSuccess) (void)cudaGetLastError();
}

void cosmo_unpin_host(void* ptr)
{
    if (ptr == nullptr) return;
    if (cudaHostUnregister(ptr) != cudaSuccess) (void)cudaGetLastError();
}

double cosmo_kernel_radius(void) { return kRadKernel; }

void densityiterate_gpu_c(int n, double pmass, int periodic, const double* box, double tolh, double hfact)
{
    State& s = state();
    if (s.sizedFor != n)
        fatal("%s called with n=%d but the device arrays are sized for %d "
              "(cosmo_arrays_init not called, or called with a different count)",
              "densityiterate_gpu_c", n, s.sizedFor);
    if (n <= 0) return;
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    // vecin= is the host time between entry and the start of the solve, as the reference
    // reports it (src/dens_c_api.cu:73-76); with the transfers outside the call it is ~0.
    const auto tv = clk::now();
    const DensResult r = solve_density(s, n, pmass, periodic ? box : nullptr, tolh, hfact, s.maxIter, true);
    const auto t1 = clk::now();
    if (r.status == 1)
        fatal("solveDensH: unconverged=%d jlist_trunc=%d stack_drops=%d (iters=%d)", r.unconverged, 0, 0,
              r.itersRun);
    if (r.status == 2)
        fatal("solveDensH: kernel support %gh reaches half the periodic box; too few particles for this box",
              kRadKernel);
    static bool memReported = false;
    if (!memReported && env_on("COSMO_MEM"))
    {
        memReported = true;
        size_t fr = 0, tot = 0;
        COSMO_CUDA(cudaMemGetInfo(&fr, &tot));
        const double v[5] = {double(n), (tot - fr) / 1e9, tot / 1e9, double(tot - fr) / n, host_peak_kb() / 1e6};
        print_line(format_mem_line, v);
    }
    static const bool stats = env_on("COSMO_DENS_STATS");
    if (stats)
    {
        const Timings& t = s.t;
        const double gpu = 1e3 * (t.bbox + t.keysSort + t.tree + t.nodes + t.jbuild + t.nrkern + t.gjbuild + t.gradkern);
        auto ms = [](clk::time_point a, clk::time_point b) {
            return std::chrono::duration<double, std::milli>(b - a).count();
        };
        const double solve = ms(tv, t1);
        const double v[18] = {double(n), double(s.nLeaves), double(s.itersRun), ms(t0, tv), 1e3 * s.uploadSeconds,
                              1e3 * t.bbox, 1e3 * t.keysSort, 1e3 * t.tree, 1e3 * t.nodes, 1e3 * t.jbuild,
                              1e3 * t.nrkern, 1e3 * t.gjbuild, 1e3 * t.gradkern, 1e3 * s.downloadSeconds, gpu,
                              solve, solve - gpu, ms(t0, t1)};
        print_line(format_dens_stats, v);
    }
    s.uploadSeconds = 0.0;
    s.downloadSeconds = 0.0;
}

void force_gpu_c(int n, double pmass, double beta, double alphau, int disc_viscosity, int pdv_heating,
                 int shock_heating)
{
    State& s = state();
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    if (s.sizedFor != n)
        fatal("%s called with n=%d but the device arrays are sized for %d "
              "(cosmo_arrays_init not called, or called with a different count)",
              "force_gpu_c", n, s.sizedFor);
    if (!(s.ngas == n && s.token != 0))
        fatal("force_gpu_c called with no GPU density solve for this particle set (n=%d state.ngas=%d token=%llu)",
              n, s.ngas, (unsigned long long)s.token);
    s.t.upsweep = s.t.fjbuild = s.t.prep = s.t.fkern = 0.0;
    compute_forces(s, pmass, beta, alphau, disc_viscosity != 0, pdv_heating > 0, shock_heating > 0);
    static const bool stats = env_on("COSMO_DENS_STATS");
    if (stats)
    {
        const double wall = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
        const Timings& t = s.t;
        // upload= and download= are the transfers inside the call (src/force_c_api.cu:74-79):
        // the caller moves THERMO, VEL and FORCE_OUT with cosmo_upload_sorted / cosmo_download,
        // so the force pass itself moves nothing and both are 0.
        const double upload = 0.0, download = 0.0;
        const double gpu = 1e3 * (t.upsweep + t.fjbuild + t.prep + t.fkern) + upload + download;
        const double v[11] = {double(s.ngas), double(s.nLeaves), 1e3 * t.upsweep, 1e3 * t.fjbuild, upload,
                              1e3 * t.prep, 1e3 * t.fkern, download, gpu, wall, wall - gpu};
        print_line(format_force_stats, v);
    }
}

// Select the arithmetic of the pair kernels for the following solves and force passes.
void cosmo_set_precision(int mode)
{
    State& s = state();
    ensure_init(s);
    s.precision = (mode == 1) ? 1 : 0;
}

int cosmo_get_precision(void)
{
    State& s = state();
    ensure_init(s);
    return s.precision;
}

// ---------------------------------------------------------------- harness hooks
void cosmo_x_set_max_iter(int m) { state().maxIter = std::max(1, m); }

void cosmo_x_set_device(int dev) { COSMO_CUDA(cudaSetDevice(dev)); }

static cudaEvent_t g_marks[16];
static bool g_marksInit = false;

void cosmo_x_mark(int id)
{
    State& s = state();
    ensure_init(s);
    if (!g_marksInit)
    {
        for (auto& e : g_marks) COSMO_CUDA(cudaEventCreate(&e));
        g_marksInit = true;
    }
    COSMO_CUDA(cudaEventRecord(g_marks[id & 15], s.st));
}

double cosmo_x_mark_elapsed(int a, int b)
{
    COSMO_CUDA(cudaEventSynchronize(g_marks[b & 15]));
    float ms = 0.0f;
    COSMO_CUDA(cudaEventElapsedTime(&ms, g_marks[a & 15], g_marks[b & 15]));
    return ms * 1e-3;
}

unsigned long long cosmo_x_launches(void) { return g_launches.load(); }

// Measured FP64 FMA throughput of this GPU in TFLOP/s (2 flops per FMA).
double cosmo_x_fp64_peak(void)
{
    State& s = state();
    ensure_init(s);
    double* out = nullptr;
    COSMO_CUDA(cudaMalloc(&out, sizeof(double)));
    const int threads = 256, blocks = s.numSMs * 8, iters = 1 << 14;
    fp64_peak_kernel<<<blocks, threads, 0, s.st>>>(out, iters, 0.999999, 1e-7);
    COSMO_LAUNCHED();
    cudaEvent_t a = ev(s);
    fp64_peak_kernel<<<blocks, threads, 0, s.st>>>(out, iters, 0.999999, 1e-7);
    COSMO_LAUNCHED();
    cudaEvent_t b = ev(s);
    COSMO_CUDA(cudaEventSynchronize(b));
    const double t = elapsed_s(a, b);
    COSMO_CUDA(cudaFree(out));
    return 2.0 * 8.0 * double(iters) * threads * blocks / t / 1e12;
}

// Density solve that reports instead of aborting: 0 ok, 1 unconverged, 2 periodic support.
int cosmo_x_density(int n, double pmass, int periodic, const double* box, double tolh, double hfact, int maxIter,
                    int withGradients)
{
    State& s = state();
    if (s.sizedFor != n || n <= 0) return -1;
    const DensResult r = solve_density(s, n, pmass, periodic ? box : nullptr, tolh, hfact,
                                       maxIter > 0 ? maxIter : s.maxIter, withGradients != 0);
    return r.status;
}

void cosmo_x_sync(void)
{
    State& s = state();
    if (s.st) COSMO_CUDA(cudaStreamSynchronize(s.st));
}

int cosmo_x_set_option(const char* name, int value)
{
    State& s = state();
    ensure_init(s);
    const std::string k(name ? name : "");
    if (k == "staging") { s.staging = value != 0; return 0; }
    if (k == "sym_prefilter") { s.symPrefilter = value != 0; return 0; }
    if (k == "newton_graph") { s.newtonGraph = value != 0; return 0; }
    if (k == "sym_extra_cap")
    {
        if (value < 0) return -1;
        s.symExtraCap = value;
        s.symRowsSkip = 0;
        return 0;
    }
    if (k == "sym_from_rows")
    {
        s.symFromRows = value != 0;
        s.symRowsSkip = 0;
        return 0;
    }
    if (k == "graph_list_store")
    {
        if (value < 0) return -1;
        s.graphListStorePct = value;
        return 0;
    }
    if (k == "spread_groups")
    {
        if (value < 0 || value > 32) return -1;
        s.spreadGroups = value;
        return 0;
    }
    if (k == "split_stream" || k == "split_work")
    {
        if (value < 0) return -1;
        (k == "split_stream" ? s.splitStream : s.splitWork) = uint32_t(value);
        return 0;
    }
    return -1;
}

void cosmo_x_set_key_extent(const double* ext6)
{
    State& s = state();
    s.keyExtentSet = ext6 != nullptr;
    if (ext6) std::copy(ext6, ext6 + 6, s.keyExtent);
}

int cosmo_x_set_frozen(const int* mask, int n)
{
    State& s = state();
    ensure_init(s);
    if (mask == nullptr || n <= 0)
    {
        s.frozenFor = 0;
        return 0;
    }
    s.frozen.resize(size_t(n), s.st);
    COSMO_CUDA(cudaMemcpyAsync(s.frozen.get(), mask, size_t(n) * sizeof(int), cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaStreamSynchronize(s.st));
    s.frozenFor = n;
    return 0;
}

int cosmo_x_refresh_h(void)
{
    State& s = state();
    if (!s.st || s.nLeaves <= 0 || s.orderFor != s.ngas) return -1;
    hmax_leaves(s, s.allLeaves.get(), s.nLeaves);
    s.jlistToken = s.rowsToken = 0;
    COSMO_CUDA(cudaStreamSynchronize(s.st));
    return 0;
}

void cosmo_x_set_wait_limit(long long ns)
{
    g_waitLimitNs.store(ns > 0 ? ns : 1000000000ll);
}

long long cosmo_x_get_wait_limit(void) { return wait_limit_ns(); }

int cosmo_x_wait_test(int kind, int fatal_on_error)
{
    if (kind != 0 && kind != 1) return -1;
    State& s = state();
    ensure_init(s);
    DBuf<int> flag;
    flag.resize(1, s.st);
    COSMO_CUDA(cudaMemsetAsync(flag.get(), 0, sizeof(int), s.st));
    COSMO_CUDA(cudaMemsetAsync(&s.dscal.get()->err, 0, sizeof(int), s.st));
    wait_test_kernel<<<1, 32, 0, s.st>>>(kind, flag.get(), &s.dscal.get()->err, wait_limit_ns());
    COSMO_LAUNCHED();
    if (fatal_on_error) check_dev_err(s, "cosmo_x_wait_test");
    read_scalars(s);
    const int e = s.hscal->err;
    COSMO_CUDA(cudaMemsetAsync(&s.dscal.get()->err, 0, sizeof(int), s.st));
    flag.release(s.st);
    COSMO_CUDA(cudaStreamSynchronize(s.st));
    return e;
}

// Format one of the stderr statistics lines from given values (0 COSMO_STATS, 1
// COSMO_FORCE, 2 COSMO_MEM), exactly as the entry points print it; no device work.
int cosmo_x_stats_line(int which, const double* values, char* buf, int len)
{
    if (!values || !buf || len <= 0) return -1;
    switch (which)
    {
    case 0: return format_dens_stats(buf, size_t(len), values);
    case 1: return format_force_stats(buf, size_t(len), values);
    case 2: return format_mem_line(buf, size_t(len), values);
    default: return -1;
    }
}

double cosmo_x_scalar(const char* name)
{
    State& s = state();
    const std::string k(name);
    if (k == "nAlive") return s.nAlive;
    if (k == "nLeaves") return s.nLeaves;
    if (k == "numNodes") return s.numNodes;
    if (k == "itersRun") return s.itersRun;
    if (k == "token") return double(s.token);
    if (k == "hfact") return s.hfact;
    if (k == "maxIter") return s.maxIter;
    if (k == "settling0") return double(s.settling0);
    if (k == "loopGraph") return double(s.lastLoopGraph);
    if (k == "hmaxSeen" && s.hscal)
    {
        read_scalars(s);
        const unsigned long long b = s.hscal->hmaxSeen;
        double v;
        std::memcpy(&v, &b, sizeof v);
        return v;
    }
    if (k == "loopRebuilds") return double(s.lastLoopRebuilds);
    if (k == "loopGraphBuilds") return double(s.loopGraphBuilds);
    if (k == "loopGraphUpdates") return double(s.loopGraphUpdates);
    if (k == "loopRowBuilds") return double(s.lastLoopRowBuilds);
    if (k == "rowsFromNewton") return s.rowsFromNewton ? 1.0 : 0.0;
    if (k == "listTotal") return double(s.listTotal);
    if (s.hscal)
    {
        read_scalars(s);
        if (k == "pairsDensity") return double(s.hscal->pairs[0]);
        if (k == "extraCount") return double(s.hscal->extraCount);
        if (k == "coverNeed") return double(s.hscal->coverNeed);
        if (k == "pairsGrad") return double(s.hscal->pairs[1]);
        if (k == "pairsForce") return double(s.hscal->pairs[2]);
        if (k == "rowOverflow") return double(s.hscal->rowOverflow);
        if (k == "candDensity") return double(s.hscal->pairs[3]);
        if (k == "unconverged") return s.hscal->unconverged;
    }
    const Timings& t = s.t;
    if (k == "t_bbox") return t.bbox;
    if (k == "t_keysort") return t.keysSort;
    if (k == "t_tree") return t.tree;
    if (k == "t_nodes") return t.nodes;
    if (k == "t_jbuild") return t.jbuild;
    if (k == "t_nrkern") return t.nrkern;
    if (k == "t_gjbuild") return t.gjbuild;
    if (k == "t_gradkern") return t.gradkern;
    if (k == "t_upsweep") return t.upsweep;
    if (k == "t_fjbuild") return t.fjbuild;
    if (k == "t_prep") return t.prep;
    if (k == "t_fkern") return t.fkern;
    return NAN;
}

// Copy a named device array to the host.  Returns the element count (or -1 if unknown);
// *dtype: 0 f64, 1 i32, 2 u32, 3 u64, 4 i64.  out == nullptr only queries.
long cosmo_x_array(const char* name, void* out, int* dtype)
{
    State& s = state();
    const std::string k(name);
    auto put = [&](const void* dev, size_t cnt, size_t es, int code, size_t stride = 1, size_t off = 0) -> long {
        if (dtype) *dtype = code;
        if (out && cnt)
        {
            if (stride == 1)
                COSMO_CUDA(cudaMemcpyAsync(out, static_cast<const char*>(dev) + off * es, cnt * es,
                                           cudaMemcpyDeviceToHost, s.st));
            else
                COSMO_CUDA(cudaMemcpy2DAsync(out, es, static_cast<const char*>(dev) + off * es, stride * es, es, cnt,
                                             cudaMemcpyDeviceToHost, s.st));
            COSMO_CUDA(cudaStreamSynchronize(s.st));
        }
        return long(cnt);
    };
    const size_t n = size_t(s.ngas), nL = size_t(s.nLeaves), nN = size_t(s.numNodes);
    if (k == "x") return put(s.xyzh.get(), n, 8, 0, 4, 0);
    if (k == "y") return put(s.xyzh.get(), n, 8, 0, 4, 1);
    if (k == "z") return put(s.xyzh.get(), n, 8, 0, 4, 2);
    if (k == "h") return put(s.xyzh.get(), n, 8, 0, 4, 3);
    if (k == "vx") return put(s.vel4.get(), n, 8, 0, 4, 0);
    if (k == "vy") return put(s.vel4.get(), n, 8, 0, 4, 1);
    if (k == "vz") return put(s.vel4.get(), n, 8, 0, 4, 2);
    if (k == "rho") return put(s.rho.get(), n, 8, 0);
    if (k == "gradh") return put(s.gradh.get(), n, 8, 0);
    if (k == "divv") return put(s.divv.get(), n, 8, 0);
    if (k == "xi") return put(s.xi.get(), n, 8, 0);
    if (k == "ddivvdt") return put(s.ddivvdt.get(), n, 8, 0);
    if (k == "fx") return put(s.fx.get(), n, 8, 0);
    if (k == "fy") return put(s.fy.get(), n, 8, 0);
    if (k == "fz") return put(s.fz.get(), n, 8, 0);
    if (k == "f4") return put(s.f4.get(), n, 8, 0);
    if (k == "vsigmax") return put(s.vsigmax.get(), n, 8, 0);
    if (k == "divvF") return put(s.divvF.get(), n, 8, 0);
    if (k == "converged") return put(s.converged.get(), n, 4, 1);
    if (k == "keys") return put(s.keysA.get(), n, 8, 3);
    if (k == "order") return put(s.orderA.get(), n, 4, 1);
    if (k == "particleLeaf") return put(s.particleLeaf.get(), size_t(s.nAlive), 4, 1);
    if (k == "csTree") return put(s.csTree.get(), nL + 1, 8, 3);
    if (k == "counts") return put(s.counts.get(), nL, 4, 2);
    if (k == "layout") return put(s.layout.get(), nL + 1, 4, 2);
    if (k == "prefixes") return put(s.bfsPrefix.get(), nN, 8, 3);
    if (k == "childOffsets") return put(s.childOffsets.get(), nN, 4, 1);
    if (k == "internalToLeaf") return put(s.internalToLeaf.get(), nN, 4, 1);
    if (k == "levelRange") return put(s.levelRange.get(), kMaxLevel + 2, 4, 1);
    if (k == "leafToInternal") return put(s.leafToInternal.get(), nL, 4, 1);
    if (k == "centers") return put(s.centers.get(), 3 * nN, 8, 0);
    if (k == "sizes") return put(s.sizes.get(), 3 * nN, 8, 0);
    if (k == "hmax_leaf") return put(s.hmaxLeaf.get(), nL, 8, 0);
    // hmax per node is the force pass's upsweep; when the force pass ran over rows made
    // from the Newton rows it was not needed, and is made when asked for
    if ((k == "hmax_node" || ((k == "jcount" || k == "jOffset" || k == "jlist") && s.forceSinceSolve)) &&
        !s.hmaxNodeDone && nL > 0)
    {
        hmax_upsweep(s);
        s.hmaxNodeDone = true;
        COSMO_CUDA(cudaStreamSynchronize(s.st));
    }
    if (k == "hmax_node") return put(s.hmaxNode.get(), nN, 8, 0);
    // the reference's state holds the gather lists after a density solve and the
    // symmetric ones after a force pass.  This library builds the symmetric ones with the
    // gradient sweep, or none (rows from the Newton rows), and ends a solve with the
    // Newton loop's widened lists: each view is rebuilt (exactly) when asked for
    if ((k == "jcount" || k == "jOffset" || k == "jlist") && nL > 0)
    {
        const bool gatherView = !s.forceSinceSolve && (s.listsSym || s.listsLoose);
        const bool symView = s.forceSinceSolve && !s.listsSym;
        if (gatherView || symView)
        {
            build_lists(s, symView);
            s.listsLoose = false;
            s.jlistToken = symView ? s.token : 0;
            COSMO_CUDA(cudaStreamSynchronize(s.st));
        }
    }
    if (k == "jcount") return put(s.jcount.get(), nL, 4, 2);
    if (k == "jOffset") return put(s.jOffset.get(), nL + 1, 4, 2);
    if (k == "jlist")
    {
        uint32_t tot = 0;
        if (nL)
        {
            COSMO_CUDA(cudaMemcpy(&tot, s.jOffset.get() + nL, 4, cudaMemcpyDeviceToHost));
        }
        return put(s.jlist.get(), tot, 4, 1);
    }
    if (k == "loopKey")
    {
        // the parameters the last solve's Newton-loop graph was keyed on, as 8-byte words
        const size_t w = (s.loopKeyLast.size() + 7) / 8;
        if (dtype) *dtype = 4;
        if (out)
        {
            std::memset(out, 0, w * 8);
            std::memcpy(out, s.loopKeyLast.data(), s.loopKeyLast.size());
        }
        return long(w);
    }
    if (k == "loopListEntries")
    {
        if (dtype) *dtype = 4;
        if (out) std::memcpy(out, s.loopListEntries.data(), s.loopListEntries.size() * 8);
        return long(s.loopListEntries.size());
    }
    if (k == "activePerIter")
    {
        if (dtype) *dtype = 4;
        if (out) std::memcpy(out, s.activePerIter.data(), s.activePerIter.size() * 8);
        return long(s.activePerIter.size());
    }
    if (dtype) *dtype = -1;
    return -1;
}

} // extern "C"

// ---------------------------------------------------------------- C++ entry point
// The reference's own C++ API (include/density.hpp:85-91), used by its standalone driver.
// Both kernel modes run this library's warp-per-leaf Newton kernel.
DensTimings solveDensH(int n, double pmass, KernelMode mode, bool withGradients, const double* periodicBox,
                       double tolh, double hfact)
{
    State& s = state();
    if (s.sizedFor != n)
        fatal("solveDensH called with n=%d but the device arrays are sized for %d", n, s.sizedFor);
    DensTimings t{};
    t.kernelMode = mode;
    t.nParticles = n;
    if (n <= 0) return t;
    const DensResult r = solve_density(s, n, pmass, periodicBox, tolh, hfact, s.maxIter, withGradients);
    if (r.status == 1)
        fatal("solveDensH: unconverged=%d jlist_trunc=%d stack_drops=%d (iters=%d)", r.unconverged, 0, 0,
              r.itersRun);
    if (r.status == 2) fatal("solveDensH: kernel support reaches half the periodic box");
    t.upload = s.uploadSeconds;
    s.uploadSeconds = 0.0;
    t.bboxAndSetup = s.t.bbox;
    t.keysAndSort = s.t.keysSort;
    t.treeBuild = s.t.tree;
    t.nodeCenters = s.t.nodes;
    t.jleafBuild = s.t.jbuild;
    t.densKernel = s.t.nrkern;
    t.gradJleafBuild = s.t.gjbuild;
    t.gradKernel = s.t.gradkern;
    t.download = s.downloadSeconds;
    s.downloadSeconds = 0.0;
    t.itersRun = r.itersRun;
    t.nLeavesOut = s.nLeaves;
    return t;
}
