/*
 * serve.cu -- the served form: a request loop with continuous batching over the same
 * density + force pipeline.
 *
 *   slots      a fixed number of worker threads, each running one request at a time on
 *              the CUDA stream of that request's particle set, so requests overlap on
 *              the device; a queued request is taken as soon as a slot is free and, for a
 *              new set, as soon as the HBM budget has room for it.
 *   resident   a solved set stays on the device (positions, velocities, h, thermo, tree
 *              storage) until released or evicted; a continuing request advances its
 *              positions on the device (x += v dt) and starts Newton-Raphson from the
 *              previous converged h, so only the re-sort, the tree and a few Newton
 *              iterations are paid again.
 *   budget     new sets are admitted while the library's device bytes plus the reserved
 *              estimates of admitted-but-not-yet-sized requests fit the budget; idle
 *              resident sets with no queued continuation are evicted least-recently-used
 *              first to make room; a request that cannot fit even beside only the memory
 *              held outside the server (measured at start) is rejected, not queued.
 * Each request's result depends only on its own set: it is the same alone and in a mix.
 */
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "state.hpp"
#include "../../include/cosmosphere.h"

namespace cosmo {

namespace {

struct DevBox3
{
    double lo[3], hi[3];
};

// Drift x += v dt; in a periodic box a coordinate that leaves [lo, hi) is wrapped back
// by one box length.
__device__ __forceinline__ double drift(double x, double v, double dt, int periodic, double lo, double hi)
{
    double y = x + v * dt;
    if (periodic)
    {
        if (y >= hi) y = y - (hi - lo);
        else if (y < lo) y = y + (hi - lo);
    }
    return y;
}

__global__ void advance_kernel(double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
                               const double* __restrict__ vx, const double* __restrict__ vy,
                               const double* __restrict__ vz, int n, double dt, int periodic, DevBox3 box)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] = drift(x[i], vx[i], dt, periodic, box.lo[0], box.hi[0]);
    y[i] = drift(y[i], vy[i], dt, periodic, box.lo[1], box.hi[1]);
    z[i] = drift(z[i], vz[i], dt, periodic, box.lo[2], box.hi[2]);
}

// Previous converged h (Hilbert order) back to the caller's order: the warm start.
__global__ void warm_h_kernel(const int* __restrict__ order, int n, const double4* __restrict__ xyzh,
                              double* __restrict__ uh)
{
    const long k = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < n) uh[order[k]] = xyzh[k].w;
}

// thermo4[k] = caller-order thermo of the particle at sorted position k
__global__ void gather_thermo_kernel(const int* __restrict__ order, int n, const double* __restrict__ ut,
                                     double4* __restrict__ thermo4)
{
    const long k = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = order[k];
    thermo4[k] = make_double4(ut[i], ut[size_t(n) + i], ut[2 * size_t(n) + i], ut[3 * size_t(n) + i]);
}

// Results back to the caller's order: h, rho, gradh, divv, xi, ddivvdt, fx..divvF.
__global__ void scatter_results_kernel(const int* __restrict__ order, int n, const double4* __restrict__ xyzh,
                                       const double* __restrict__ rho, const double* __restrict__ gradh,
                                       const double* __restrict__ divv, const double* __restrict__ xi,
                                       const double* __restrict__ ddivvdt, const double* __restrict__ fx,
                                       const double* __restrict__ fy, const double* __restrict__ fz,
                                       const double* __restrict__ f4, const double* __restrict__ vs,
                                       const double* __restrict__ dv, double* __restrict__ out)
{
    const long k = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t o = size_t(order[k]), N = size_t(n);
    out[o] = xyzh[k].w;
    out[N + o] = rho[k];
    out[2 * N + o] = gradh[k];
    out[3 * N + o] = divv[k];
    out[4 * N + o] = xi[k];
    out[5 * N + o] = ddivvdt[k];
    out[6 * N + o] = fx[k];
    out[7 * N + o] = fy[k];
    out[8 * N + o] = fz[k];
    out[9 * N + o] = f4[k];
    out[10 * N + o] = vs[k];
    out[11 * N + o] = dv[k];
}

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Device bytes a new set of n particles is charged at admission, until its real footprint
// is known: ≈ 1 KB of particle arrays, FP32 copies, tree and lists, plus the neighbour
// rows -- 4 bytes (symmetric, j) and 8 bytes (Newton, r^2) per row entry, 128 entries
// per particle for the cubic kernel and 256 for the quintic one.
constexpr long long kBytesPerParticle = 1024 + 12 * (kQuintic ? 256 : 128);
constexpr long long kBytesFixed = 1ll << 20;

struct Request
{
    long id = 0, setId = 0;
    bool isNew = true, keep = true;
    int n = 0, periodic = 0;
    double pmass = 0, tolh = 1e-4, hfact = -1, beta = 2, alphau = 0, dt = 0;
    double box[6] = {0, 0, 0, 0, 0, 0};
    std::vector<double> pos, h, vel, thermo;    // host copies taken at submission
    std::vector<double> out;                    // 12 n results, caller order
    double tSubmit = 0, tStart = 0, tDone = 0;
    long long updates = 0;
    int status = 0;                             // 0 pending, 1 done, -1 rejected, -2 unconverged
    int itersRun = 0;
    int slot = -1;
    int pendingConts = 0;                       // continuations submitted before admission
};

struct ResidentSet
{
    long id = 0;
    std::unique_ptr<State> st;
    DBuf<double> uthermo;                       // caller-order thermo, 4 n
    int n = 0, periodic = 0;
    double pmass = 0, tolh = 1e-4, hfact = -1, beta = 2, alphau = 0;
    double box[6] = {0, 0, 0, 0, 0, 0};
    bool busy = false;
    int queued = 0;                             // continuations waiting for it
    double lastUse = 0;
    long long bytes = 0;                        // device bytes it holds once solved
};

struct Server
{
    std::mutex m;
    std::condition_variable cvWork, cvDone;
    std::deque<Request*> queue;
    std::map<long, std::unique_ptr<Request>> reqs;
    std::map<long, std::unique_ptr<ResidentSet>> sets;
    std::vector<std::thread> workers;
    bool running = false, stopping = false;
    int device = 0, precision = 0, slots = 0;
    long nextId = 1;
    long long budget = 0, reserved = 0;
    long long baseBytes = 0;                    // device bytes held outside the server at start
    int inflight = 0, maxInflight = 0, completed = 0, rejected = 0, evicted = 0;
};

Server& server()
{
    static Server* s = new Server();   // deliberately leaked, as the other states
    return *s;
}

long long estimate_bytes(int n) { return kBytesFixed + kBytesPerParticle * (long long)n; }

// Choose the next runnable request (caller holds the lock).  Continuations need their
// set idle; new sets need budget room, made by evicting idle resident sets that no queued
// request refers to, least recently used first.  Returns the request and fills `evict`
// with the states to release outside the lock.
Request* pick(Server& S, std::vector<std::unique_ptr<ResidentSet>>& evict)
{
    for (auto it = S.queue.begin(); it != S.queue.end(); ++it)
    {
        Request* r = *it;
        if (!r->isNew)
        {
            auto si = S.sets.find(r->setId);
            if (si == S.sets.end())
            {
                auto oi = S.reqs.find(r->setId);
                if (oi != S.reqs.end() && oi->second->status == 0) continue;   // set not admitted yet
                r->status = -1;   // its set was released, rejected or failed
                S.queue.erase(it);
                S.cvDone.notify_all();
                return pick(S, evict);
            }
            if (si->second->busy) continue;
            si->second->busy = true;
            si->second->queued -= 1;
            S.queue.erase(it);
            return r;
        }
        const long long need = estimate_bytes(r->n);
        // never admissible, even with every resident set evicted: reject now instead of
        // leaving it queued forever
        if (S.baseBytes + need > S.budget)
        {
            r->status = -1;
            S.rejected += 1;
            S.queue.erase(it);
            S.cvDone.notify_all();
            return pick(S, evict);
        }
        long long used = g_deviceBytes.load() + S.reserved;
        if (used + need > S.budget)
        {
            std::vector<ResidentSet*> idle;
            for (auto& kv : S.sets)
                if (!kv.second->busy && kv.second->queued == 0) idle.push_back(kv.second.get());
            std::sort(idle.begin(), idle.end(), [](ResidentSet* a, ResidentSet* b) { return a->lastUse < b->lastUse; });
            for (ResidentSet* rs : idle)
            {
                if (used + need <= S.budget) break;
                used -= rs->bytes;
                auto node = S.sets.find(rs->id);
                evict.push_back(std::move(node->second));
                S.sets.erase(node);
                S.evicted += 1;
            }
            if (used + need > S.budget) continue;   // wait for memory; later requests may fit
        }
        S.reserved += need;
        auto rs = std::make_unique<ResidentSet>();
        rs->id = r->id;
        rs->st = std::make_unique<State>();
        rs->n = r->n;
        rs->periodic = r->periodic;
        rs->pmass = r->pmass;
        rs->tolh = r->tolh;
        rs->hfact = r->hfact;
        rs->beta = r->beta;
        rs->alphau = r->alphau;
        std::copy(r->box, r->box + 6, rs->box);
        rs->busy = true;
        rs->queued = r->pendingConts;
        S.sets[r->id] = std::move(rs);
        S.queue.erase(it);
        return r;
    }
    return nullptr;
}

int run_request(Server& S, Request* r, ResidentSet* rs)
{
    State& st = *rs->st;
    const int n = r->n;
    const size_t bytes = size_t(n) * sizeof(double);
    if (r->isNew)
    {
        ensure_init(st);
        st.precision = S.precision;
        size_particle_arrays(st, n);
        rs->uthermo.resize(size_t(4) * n, st.st);
        COSMO_CUDA(cudaMemcpyAsync(st.ux.get(), r->pos.data(), bytes, cudaMemcpyHostToDevice, st.st));
        COSMO_CUDA(cudaMemcpyAsync(st.uy.get(), r->pos.data() + n, bytes, cudaMemcpyHostToDevice, st.st));
        COSMO_CUDA(cudaMemcpyAsync(st.uz.get(), r->pos.data() + 2 * size_t(n), bytes, cudaMemcpyHostToDevice, st.st));
        COSMO_CUDA(cudaMemcpyAsync(st.uh.get(), r->h.data(), bytes, cudaMemcpyHostToDevice, st.st));
        if (!r->vel.empty())
        {
            COSMO_CUDA(cudaMemcpyAsync(st.uvx.get(), r->vel.data(), bytes, cudaMemcpyHostToDevice, st.st));
            COSMO_CUDA(cudaMemcpyAsync(st.uvy.get(), r->vel.data() + n, bytes, cudaMemcpyHostToDevice, st.st));
            COSMO_CUDA(cudaMemcpyAsync(st.uvz.get(), r->vel.data() + 2 * size_t(n), bytes, cudaMemcpyHostToDevice,
                                       st.st));
        }
    }
    else
    {
        const DevBox3 b3 = {{rs->box[0], rs->box[2], rs->box[4]}, {rs->box[1], rs->box[3], rs->box[5]}};
        advance_kernel<<<iceil(n, 256), 256, 0, st.st>>>(st.ux.get(), st.uy.get(), st.uz.get(), st.uvx.get(),
                                                         st.uvy.get(), st.uvz.get(), n, r->dt, rs->periodic, b3);
        COSMO_LAUNCHED();
        warm_h_kernel<<<iceil(n, 256), 256, 0, st.st>>>(st.orderA.get(), n, st.xyzh.get(), st.uh.get());
        COSMO_LAUNCHED();
    }
    if (!r->thermo.empty())
        COSMO_CUDA(cudaMemcpyAsync(rs->uthermo.get(), r->thermo.data(), 4 * bytes, cudaMemcpyHostToDevice, st.st));
    const DensResult d = solve_density(st, n, rs->pmass, rs->periodic ? rs->box : nullptr, rs->tolh, rs->hfact, 100,
                                       true);
    r->itersRun = d.itersRun;
    if (d.status != 0) return -2;
    gather_thermo_kernel<<<iceil(n, 256), 256, 0, st.st>>>(st.orderA.get(), n, rs->uthermo.get(), st.thermo4.get());
    COSMO_LAUNCHED();
    compute_forces(st, rs->pmass, rs->beta, rs->alphau, false, true, true);
    r->out.resize(size_t(12) * n);
    st.xfer.resize(size_t(12) * n, st.st);
    scatter_results_kernel<<<iceil(n, 256), 256, 0, st.st>>>(
        st.orderA.get(), n, st.xyzh.get(), st.rho.get(), st.gradh.get(), st.divv.get(), st.xi.get(),
        st.ddivvdt.get(), st.fx.get(), st.fy.get(), st.fz.get(), st.f4.get(), st.vsigmax.get(), st.divvF.get(),
        st.xfer.get());
    COSMO_LAUNCHED();
    COSMO_CUDA(cudaMemcpyAsync(r->out.data(), st.xfer.get(), 12 * bytes, cudaMemcpyDeviceToHost, st.st));
    COSMO_CUDA(cudaStreamSynchronize(st.st));
    long long u = st.nAlive;
    for (long long a : st.activePerIter) u += a;
    r->updates = u;
    return 1;
}

void worker(Server& S, int slot)
{
    COSMO_CUDA(cudaSetDevice(S.device));
    for (;;)
    {
        Request* r = nullptr;
        ResidentSet* rs = nullptr;
        std::vector<std::unique_ptr<ResidentSet>> evict;
        {
            std::unique_lock<std::mutex> lk(S.m);
            S.cvWork.wait(lk, [&] {
                if (S.stopping) return true;
                std::vector<std::unique_ptr<ResidentSet>> ev2;
                r = pick(S, ev2);
                for (auto& e : ev2) evict.push_back(std::move(e));
                return r != nullptr;
            });
            if (!r) return;
            rs = S.sets[r->isNew ? r->id : r->setId].get();
            r->slot = slot;
            r->tStart = now_s();
            S.inflight += 1;
            S.maxInflight = std::max(S.maxInflight, S.inflight);
        }
        for (auto& e : evict) release_state(*e->st), e->uthermo.release();
        evict.clear();
        const int status = run_request(S, r, rs);
        std::unique_ptr<ResidentSet> drop;
        {
            std::lock_guard<std::mutex> lk(S.m);
            r->tDone = now_s();
            r->status = status;
            if (r->isNew) S.reserved -= estimate_bytes(r->n);
            S.inflight -= 1;
            S.completed += 1;
            rs->busy = false;
            rs->lastUse = r->tDone;
            rs->bytes = (long long)(state_device_bytes(*rs->st) + rs->uthermo.cap * sizeof(double));
            const long sid = r->isNew ? r->id : r->setId;
            if ((!r->keep && rs->queued == 0) || r->status != 1)
            {
                auto node = S.sets.find(sid);
                drop = std::move(node->second);
                S.sets.erase(node);
            }
            r->pos.clear(); r->pos.shrink_to_fit();
            r->h.clear(); r->h.shrink_to_fit();
            r->vel.clear(); r->vel.shrink_to_fit();
            r->thermo.clear(); r->thermo.shrink_to_fit();
        }
        if (drop)
        {
            release_state(*drop->st);
            drop->uthermo.release();
        }
        S.cvDone.notify_all();
        S.cvWork.notify_all();
    }
}

} // namespace
} // namespace cosmo

using namespace cosmo;

extern "C" {

int cosmo_serve_start(int slots, double hbm_budget_gb)
{
    Server& S = server();
    std::lock_guard<std::mutex> lk(S.m);
    if (S.running || slots < 1) return -1;
    COSMO_CUDA(cudaGetDevice(&S.device));
    S.precision = cosmo_get_precision();
    S.slots = slots;
    S.budget = (long long)(hbm_budget_gb * 1e9);
    S.baseBytes = g_deviceBytes.load();
    S.stopping = false;
    S.running = true;
    S.reserved = 0;
    S.inflight = S.maxInflight = S.completed = S.rejected = S.evicted = 0;
    for (int k = 0; k < slots; ++k) S.workers.emplace_back(worker, std::ref(S), k);
    return 0;
}

long cosmo_serve_submit(int n, double pmass, int periodic, const double* box6, double tolh, double hfact,
                        const double* pos3, const double* h, const double* vel3, const double* thermo4, double beta,
                        double alphau, int keep_resident)
{
    Server& S = server();
    if (n < 1 || pos3 == nullptr || h == nullptr || thermo4 == nullptr) return -1;
    auto r = std::make_unique<Request>();
    r->isNew = true;
    r->keep = keep_resident != 0;
    r->n = n;
    r->pmass = pmass;
    r->periodic = periodic;
    if (periodic && box6) std::copy(box6, box6 + 6, r->box);
    r->tolh = tolh;
    r->hfact = hfact;
    r->beta = beta;
    r->alphau = alphau;
    r->pos.assign(pos3, pos3 + 3 * size_t(n));
    r->h.assign(h, h + n);
    if (vel3) r->vel.assign(vel3, vel3 + 3 * size_t(n));
    else r->vel.assign(3 * size_t(n), 0.0);
    r->thermo.assign(thermo4, thermo4 + 4 * size_t(n));
    std::lock_guard<std::mutex> lk(S.m);
    if (!S.running) return -1;
    r->id = S.nextId++;
    r->setId = r->id;
    r->tSubmit = now_s();
    Request* raw = r.get();
    S.reqs[r->id] = std::move(r);
    S.queue.push_back(raw);
    S.cvWork.notify_one();
    return raw->id;
}

long cosmo_serve_continue(long set_id, double dt, const double* thermo4, int keep_resident)
{
    Server& S = server();
    std::lock_guard<std::mutex> lk(S.m);
    if (!S.running) return -1;
    // the set is resident, or its first request is still waiting for admission
    auto si = S.sets.find(set_id);
    Request* origin = nullptr;
    if (si == S.sets.end())
    {
        auto oi = S.reqs.find(set_id);
        if (oi == S.reqs.end() || !oi->second->isNew || oi->second->status != 0 || !oi->second->keep) return -1;
        if (std::find(S.queue.begin(), S.queue.end(), oi->second.get()) == S.queue.end()) return -1;
        origin = oi->second.get();
    }
    auto r = std::make_unique<Request>();
    r->isNew = false;
    r->keep = keep_resident != 0;
    r->setId = set_id;
    r->n = origin ? origin->n : si->second->n;
    r->dt = dt;
    if (thermo4) r->thermo.assign(thermo4, thermo4 + 4 * size_t(r->n));
    r->id = S.nextId++;
    r->tSubmit = now_s();
    if (origin) origin->pendingConts += 1;
    else si->second->queued += 1;
    Request* raw = r.get();
    S.reqs[r->id] = std::move(r);
    S.queue.push_back(raw);
    S.cvWork.notify_all();
    return raw->id;
}

// Wait for a request; copy its results (caller order) into whichever outputs are given:
// h (n), dens (rho, gradh: 2n), grad (divv, xi, ddivvdt: 3n), force (fx, fy, fz, du/dt,
// vsigmax, divv: 6n).  Returns 1 done, -1 rejected, -2 unconverged.
int cosmo_serve_wait(long request_id, double* h, double* dens, double* grad, double* force)
{
    Server& S = server();
    std::unique_lock<std::mutex> lk(S.m);
    auto it = S.reqs.find(request_id);
    if (it == S.reqs.end()) return -1;
    Request* r = it->second.get();
    S.cvDone.wait(lk, [&] { return r->status != 0; });
    if (r->status == 1 && !r->out.empty())
    {
        const size_t N = size_t(r->n);
        if (h) std::memcpy(h, r->out.data(), N * 8);
        if (dens) std::memcpy(dens, r->out.data() + N, 2 * N * 8);
        if (grad) std::memcpy(grad, r->out.data() + 3 * N, 3 * N * 8);
        if (force) std::memcpy(force, r->out.data() + 6 * N, 6 * N * 8);
        r->out.clear();
        r->out.shrink_to_fit();
    }
    return r->status;
}

double cosmo_serve_request_stat(long request_id, const char* name)
{
    Server& S = server();
    std::lock_guard<std::mutex> lk(S.m);
    auto it = S.reqs.find(request_id);
    if (it == S.reqs.end()) return NAN;
    const Request* r = it->second.get();
    const std::string k(name);
    if (k == "latency") return r->tDone - r->tSubmit;
    if (k == "queue") return r->tStart - r->tSubmit;
    if (k == "service") return r->tDone - r->tStart;
    if (k == "submit") return r->tSubmit;
    if (k == "start") return r->tStart;
    if (k == "done") return r->tDone;
    if (k == "updates") return double(r->updates);
    if (k == "iters") return r->itersRun;
    if (k == "slot") return r->slot;
    if (k == "n") return r->n;
    if (k == "status") return r->status;
    return NAN;
}

int cosmo_serve_release(long set_id)
{
    Server& S = server();
    std::unique_ptr<ResidentSet> drop;
    {
        std::lock_guard<std::mutex> lk(S.m);
        auto si = S.sets.find(set_id);
        if (si == S.sets.end() || si->second->busy || si->second->queued) return -1;
        drop = std::move(si->second);
        S.sets.erase(si);
    }
    release_state(*drop->st);
    drop->uthermo.release();
    S.cvWork.notify_all();
    return 0;
}

double cosmo_serve_stat(const char* name)
{
    Server& S = server();
    std::lock_guard<std::mutex> lk(S.m);
    const std::string k(name);
    if (k == "device_bytes") return double(g_deviceBytes.load());
    if (k == "bytes_per_particle") return double(kBytesPerParticle);
    if (k == "bytes_fixed") return double(kBytesFixed);
    if (k == "budget") return double(S.budget);
    if (k == "resident_sets") return double(S.sets.size());
    if (k == "max_inflight") return S.maxInflight;
    if (k == "completed") return S.completed;
    if (k == "rejected") return S.rejected;
    if (k == "evicted") return S.evicted;
    if (k == "queued") return double(S.queue.size());
    if (k == "slots") return S.slots;
    return NAN;
}

int cosmo_serve_stop(void)
{
    Server& S = server();
    {
        std::lock_guard<std::mutex> lk(S.m);
        if (!S.running) return -1;
        S.stopping = true;
    }
    S.cvWork.notify_all();
    for (auto& t : S.workers) t.join();
    std::vector<std::unique_ptr<ResidentSet>> drop;
    {
        std::lock_guard<std::mutex> lk(S.m);
        S.workers.clear();
        for (auto& kv : S.sets) drop.push_back(std::move(kv.second));
        S.sets.clear();
        S.queue.clear();
        S.reqs.clear();
        S.running = false;
    }
    for (auto& d : drop)
    {
        release_state(*d->st);
        d->uthermo.release();
    }
    return 0;
}

} // extern "C"
