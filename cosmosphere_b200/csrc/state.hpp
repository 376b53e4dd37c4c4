/*
 * state.hpp -- the persistent device state behind the C-ABI: the B200 counterpart of the
 * reference's GpuState (include/gpu_state.hpp:36-123).
 *
 * Layout in HBM (all Hilbert-ordered arrays are indexed by sorted position k):
 *   caller order   ux uy uz uh | uvx uvy uvz | uax uay uaz    upload targets (f64 SoA)
 *   Hilbert order  xyzh   double4 (x, y, z, h)                 32-byte records: bulk-copied
 *                                                              into shared memory by the
 *                                                              Newton kernels, read as two
 *                                                              128-bit loads elsewhere
 *                  vel4   double4 (vx, vy, vz, 0), acc4 likewise
 *                  thermo4 double4 (pro2, cs, alpha, u)
 *                  prepA  double4 (1/h^2, 1/h, rho(h), 1/rho)   force per-particle factors
 *                  prepB  double4 (grkfac, P, auterm, divfac)
 *                  rho gradh divv xi ddivvdt, fx fy fz f4 vsigmax divvF   f64 SoA
 *   tree           cornerstone leaf array, linked octree (BFS), pre-order walk arrays,
 *                  CSR j-leaf lists
 * Buffers grow and are never freed: like the reference's state, it is deliberately
 * leaked so no CUDA call runs during static teardown.
 */
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "common.cuh"

namespace cosmo {

// Device bytes currently held by every state of the library (admission control of the
// served form charges requests against it).
extern std::atomic<long long> g_deviceBytes;

// The library's stream-ordered memory pool on the current device (created on first use,
// release threshold unlimited): buffers are taken and returned in stream order, so growing
// or dropping one state's buffers never synchronises the device under other states' work.
cudaMemPool_t device_pool();

template<class T>
struct DBuf
{
    T*     p   = nullptr;
    size_t n   = 0;
    size_t cap = 0;

    // Return the buffer to the pool after the work already queued on st.
    void release(cudaStream_t st = nullptr)
    {
        if (p)
        {
            COSMO_CUDA(cudaFreeAsync(p, st));
            g_deviceBytes -= (long long)(cap * sizeof(T));
        }
        p = nullptr;
        n = cap = 0;
    }

    // Grow to hold c elements, in st's order.  Contents are kept only when keep is set;
    // new memory is zeroed, as the reference's thrust::device_vector value-initialises.
    void resize(size_t c, cudaStream_t st, bool keep = false)
    {
        if (c > cap)
        {
            void* q = nullptr;
            const size_t newCap = c + c / 8 + 16;
            COSMO_CUDA(cudaMallocFromPoolAsync(&q, newCap * sizeof(T), device_pool(), st));
            g_deviceBytes += (long long)(newCap * sizeof(T));
            COSMO_CUDA(cudaMemsetAsync(q, 0, newCap * sizeof(T), st));
            if (keep && p && n) COSMO_CUDA(cudaMemcpyAsync(q, p, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
            if (p)
            {
                COSMO_CUDA(cudaFreeAsync(p, st));
                g_deviceBytes -= (long long)(cap * sizeof(T));
            }
            p = static_cast<T*>(q);
            cap = newCap;
        }
        n = c;
    }
    T* get() const { return p; }
};

// Device-side scalars, one block, so a solve reads its counters with one copy.
struct DevScalars
{
    int nAlive;
    int err;                     // DevErr bits
    int nextActive;              // active-leaf appends of the current NR iteration
    int unconverged;             // particles left unconverged by the current iteration
    int listStale;               // an updated h outgrew the gather radius its leaf's list has
    int pad0;
    int workCounter[4];          // dynamic work distribution for persistent kernels
    unsigned long long pairs[4]; // accepted pairs: density, gradient, force, candidates
    unsigned int sortTiles[16];  // onesweep tile tickets, one per digit pass
    int itemsHeavy, itemsLight;  // Newton work items of the current iteration (split, whole)
    int rowParticles;            // particles of the current iteration on their neighbour rows
    int settling;                // unconverged particles whose h moved by less than kSettle
    int rowOverflow;             // some symmetric row overflowed (its particle takes the group path)
    int frozenAlive;             // live particles a solve keeps fixed (neighbours only)
    unsigned long long hmaxSeen; // bits of the largest h any leaf had at the start of an iteration
    int coverNeed;               // live particles whose Newton row does not cover their converged h
    int coverLeaves;             // leaves holding such particles
    int coverCut;                // those of them in leaves the work queue cuts (no row for them)
    int extraCount;              // pairs a Newton row may miss from the other side (appended)
    int mergeOverflow;           // a row with its extras would exceed kNbl
    int rowsJOn;                 // the Newton row builder writes the index rows (nonzero)
    int leafStart;               // leaves of the grid the leaf tree's refinement starts from
    int leafDone;                // that grid is the leaf tree (no node of it holds more than kBucket)
};

// The single-set Newton loop run as a graph: what the host loop kept in host variables
// (active counts, the iteration, the list and row decisions) lives here on the device.
constexpr int kLoopIters = 128;
struct NewtonLoop
{
    int nLeaves, numNodes;       // the tree's counts (the graph reads them, so it serves any tree)
    int nActiveLeaves, nActiveParticles, iter, maxIter;
    int rebuildNext, rowsNext, rowsReady, rebuilds;
    int rowBuilds, pad0;
    long long settling0;
    long long activePerIter[kLoopIters];
    unsigned int listEntries[kLoopIters];   // gather-list entries each iteration ran on
};

struct Timings
{
    double bbox = 0, keysSort = 0, tree = 0, nodes = 0, jbuild = 0, nrkern = 0, gjbuild = 0,
           gradkern = 0, upsweep = 0, fjbuild = 0, prep = 0, fkern = 0;
};

struct State
{
    cudaStream_t st = nullptr;
    int device = -1;
    int numSMs = 148;

    int sizedFor = 0;      // particle count the arrays were sized for (cosmo_arrays_init)
    int orderFor = 0;      // particle count the current Hilbert ordering belongs to
    int ngas = 0, nAlive = 0, nLeaves = 0, numNodes = 0;
    double pmass = 0.0, hfact = 0.0;
    int periodic = 0;
    double boxHost[6] = {0, 0, 0, 0, 0, 0};
    uint64_t token = 0, jlistToken = 0, rowsToken = 0;
    bool listsSym = false;                      // the lists held are the symmetric ones
    bool listsLoose = false;                    // the lists held are the Newton loop's widened ones
    bool forceSinceSolve = false;               // a force pass ran on the current tree
    // The symmetric rows of the current tree come from the Newton rows (their j, with the
    // pairs another particle's support adds merged in): the symmetric lists and hmax per
    // node were not built, and are built only if asked for (hmaxNodeDone once done).
    bool rowsFromNewton = false, hmaxNodeDone = true;
    int itersRun = 0, maxIter = 100;
    long long settling0 = 0;                    // settling particles after the first Newton update
    int precision = 0;     // 0 plain FP64 (the drop-in form), 1 mixed FP32/FP64
    // Kernel variants (results are the same either way): staging = 1 stages the Newton
    // kernels' j-stream into shared memory by bulk copies (cp.async.bulk + mbarrier)
    // instead of loading it directly (COSMO_STAGING); symPrefilter = 1 runs the symmetric
    // row builder's tests through the FP32 prefilter (COSMO_SYM_PREFILTER).
    int staging = 0;
    int symPrefilter = 0;
    // The Newton work queue's leaf cut (0 = the built-in figures): a leaf whose gather
    // list streams more than splitStream particles is cut into groups of about
    // splitWork / stream particles (cosmo_x_set_option "split_stream", "split_work").
    uint32_t splitStream = 0, splitWork = 0;
    // h-ordered groups a window whose h spreads is cut into, at least (0 = built-in 1;
    // cosmo_x_set_option "spread_groups")
    int spreadGroups = 0;
    // 1: the Newton loop runs as one graph launch (a while node over the iterations, the
    // list rebuilds and the row build as conditional nodes: no host read per iteration);
    // 0: one host round trip per iteration (cosmo_x_set_option "newton_graph",
    // COSMO_NEWTON_GRAPH).  The results are the same either way.
    int newtonGraph = 1;
    // 1: the gradient and force passes run over the Newton rows' j when every live
    // particle's row covers its converged h (the symmetric lists and rows are not built);
    // 0: the symmetric lists and rows are built after every solve (cosmo_x_set_option
    // "sym_from_rows", COSMO_SYM_FROM_ROWS).  The results are the same either way.
    int symFromRows = 1;
    int symRowsSkip = 0;   // solves left that do not try it (after one that could not)
    // pairs the other side's supports may add that the rows' merge holds (0: one per live
    // particle); a smaller figure sends the force pass back to the list-built rows when
    // more are found (cosmo_x_set_option "sym_extra_cap", a test of that fallback)
    int symExtraCap = 0;
    // list storage of the graph loop's rebuilds as a percentage of the first lists' total
    // (0: the built-in, twice the total plus 65536 entries); a figure under 100 makes a
    // rebuild outgrow it, so the fallback to the host loop can be exercised
    // (cosmo_x_set_option "graph_list_store")
    int graphListStorePct = 0;
    size_t listStore = 0;   // list entries a fill may write (0: all jlist holds)
    // Open boundaries: the particle extents the bounding box is made from, when the caller
    // gives them (a rank of a decomposed set uses the whole set's, so its keys and order
    // are the whole set's); otherwise the extents of the particles uploaded.
    // Particles a solve takes as neighbours only (caller order, 1 = fixed): they start
    // converged, so the Newton loop never updates them (a rank's halo particles).
    DBuf<int> frozen;
    int frozenFor = 0;   // the particle count the mask was given for (0: none)
    bool keyExtentSet = false;
    double keyExtent[6] = {0, 0, 0, 0, 0, 0};   // xmin, xmax, ymin, ymax, zmin, zmax
    int lastLoopGraph = 0;  // the last solve's Newton loop ran as a graph (1) or on the host (0)
    // The graph-run loop's instantiated graph, kept while the parameters it was captured
    // with (the key: buffers, counts, scalars, launch shapes) stay the same; a solve with
    // other parameters captures again and updates it in place.
    cudaGraph_t loopGraphDef = nullptr;
    cudaGraphExec_t loopGraphExec = nullptr;
    std::vector<unsigned char> loopGraphKey;
    std::vector<unsigned char> loopKeyPending;   // parameters met once, not yet built for
    std::vector<unsigned char> loopKeyLast;      // the last solve's parameters (a diagnostic)
    unsigned long long loopKernels[3] = {0, 0, 0};   // kernels of the body, the list branch, the rows branch
    int loopGraphBuilds = 0, loopGraphUpdates = 0;
    int lastLoopRebuilds = 0, lastLoopRowBuilds = 0;   // its list rebuilds and row builds
    std::vector<long long> loopListEntries;              // its gather-list entries per iteration
    std::vector<long long> activePerIter;
    cudaEvent_t treeEv[5] = {};   // the last tree build's stage marks (read after the next sync)
    double uploadSeconds = 0.0, downloadSeconds = 0.0;
    Timings t;

    // caller-order upload targets
    DBuf<double> ux, uy, uz, uh, uvx, uvy, uvz, uax, uay, uaz;
    // Hilbert-order particle data
    DBuf<double4> xyzh, vel4, acc4, thermo4, prepA, prepB;
    DBuf<float4> prepAf, prepBf, thermof;       // FP32 force factors (mixed form)
    DBuf<double> rho, gradh, divv, xi, ddivvdt, fx, fy, fz, f4, vsigmax, divvF;
    DBuf<double> xfer;                          // 6n: one slot's worth of host traffic
    DBuf<uint64_t> keysA, keysB;
    DBuf<int> orderA, orderB, particleLeaf, converged;

    // tree
    DBuf<DevBox> box;
    DBuf<uint64_t> csTree, csTree2;
    DBuf<uint32_t> counts, ops, opsScan, layout;
    DBuf<uint32_t> startBounds;                 // where each level-4 cell starts in the sorted keys
    DBuf<uint64_t> prePrefix, bfsPrefix;
    DBuf<uint32_t> nodeCount, leafPreStart;
    DBuf<int> preLeaf, preSkip, bfsToPre, preToBfs;
    DBuf<int> childOffsets, internalToLeaf, levelRange, leafToInternal;
    DBuf<double> centers, sizes;                // 3 per BFS node
    DBuf<double4> preCenter, preHalf;           // pre-order copies for the walk
    DBuf<double> hmaxLeaf, hmaxNode, hmaxPre;
    DBuf<uint32_t> jcount, jOffset;
    DBuf<uint32_t> jstream;                     // particles in each leaf's gather list
    DBuf<double> listH;                         // h each leaf's gather list covers
    DBuf<int> jlist;
    DBuf<uint32_t> jOffsetPrev;                 // an incremental rebuild's copy of the lists it replaces
    DBuf<int> jlistPrev, walked;
    DBuf<int> walkScratch;                      // the count pass's copy of each list it walks
    uint32_t listTotal = 0;                     // entries of the current lists
    DBuf<int4> items;                           // Newton work items (leaf, window|group|G, m0, m1)
    DBuf<int> nbl;                              // symmetric rows (j), kNbl entries per particle
    DBuf<double> nblR2;                         // Newton rows (r^2), kNbl entries per particle
    DBuf<int> nblCount;                         // entries of each row (> kNbl: overflowed)
    DBuf<double> nblH;                          // largest h a Newton row stays complete for
    DBuf<int> rowItems;                         // particles of a Newton iteration on their rows
    DBuf<int> nblJ;                             // the Newton rows' j (flat, beside nblR2)
    DBuf<double> hs;                            // h in the sorted order (rows from the Newton rows)
    DBuf<int> coverFlag, coverLeaves;           // rows to complete after a solve: particle flags, leaves
    DBuf<unsigned long long> extras;            // (row owner << 32 | j) a row must gain
    DBuf<int> extraCnt;                         // extras per particle
    DBuf<uint32_t> extraOff;                    // their offsets (exclusive scan)
    DBuf<int> extraBucket;                      // the extras' j, grouped by owner
    DBuf<int> leafNext;                         // leaf already queued for the next iteration
    DBuf<int> activeA, activeB, allLeaves;

    // scratch
    DBuf<uint32_t> scanTmp, sortHist, sortBase, sortLookback;
    DBuf<uint64_t> nodeKeysTmp;
    DBuf<int> nodeValsTmp;
    DBuf<double> redTmp;
    DBuf<DevScalars> dscal;
    DBuf<NewtonLoop> nloop;                     // the graph-run Newton loop's state
    DevScalars* hscal = nullptr;                // pinned host mirror
    int* hsmall = nullptr;                      // pinned scratch for small reads (64 ints)
    std::vector<cudaEvent_t> evPool;            // timing events of this state's stream
    int evNext = 0;
};

State& state();
void ensure_init(State& s);
void release_state(State& s);        // free every device and pinned buffer and the stream
size_t state_device_bytes(const State& s);
void size_particle_arrays(State& s, int n);

// tree.cu
void build_tree(State& s, const double* periodicBox, bool alsoSortVA, bool rowsJOn = false);
void tree_timings(State& s);   // the last tree build's stage times, once its marks have passed
// hmax of the leaves [0, nLeavesActive) of leaves, or of the first *countPtr of them when
// countPtr is given (a count on the device; nLeavesActive then bounds it).
void hmax_leaves(State& s, const int* leaves, int nLeavesActive, const int* countPtr = nullptr);
// Gather (symmetric = false) or symmetric j-leaf lists for all leaves.  margin > 1 widens
// the gather radius to R * hmax * margin, so the lists stay valid while h grows by up to
// that factor; listH records the h each leaf's list covers.
void build_lists(State& s, bool symmetric, double margin = 1.0, bool incremental = false, bool rounded = false,
                 uint32_t streamCap = 0);
// The same incremental gather-list rebuild with no host read (for a captured Newton
// loop): the fill stays inside the storage jlist already holds, kErrListFull otherwise.
// jOffsetPrev, jlistPrev (as large as jlist), walked and the walk scratch must be sized.
// The leaf and node counts are read on the device (dims[0], dims[1]); leafCap bounds the
// leaf count and sizes the launches, so the same sequence serves any tree up to it.
void build_lists_device(State& s, double margin, bool rounded, uint32_t streamCap, const int* dims, int leafCap);
// The symmetric lists and the symmetric neighbour rows of the current tree and h (the
// force pass's pairs; every gather pair of the converged h is among them).
void build_symmetric(State& s);
void hmax_upsweep(State& s);
void radix_sort_u64(State& s, uint64_t* kA, uint64_t* kB, int* vA, int* vB, int n, bool iotaValues);
uint32_t scan_exclusive(State& s, const uint32_t* in, uint32_t* out, int n, bool readTotal);
// The same with the element count on the device (*nPtr <= nCap); the total goes to out[*nPtr].
void scan_exclusive_dev(State& s, const uint32_t* in, uint32_t* out, int nCap, const int* nPtr);
void scan_reserve(State& s, int nCap);   // size the scan scratch for up to nCap elements

// density.cu
struct DensResult { int itersRun; int unconverged; int status; };
// allowGraph = false keeps the Newton loop on the host (the graph loop's fallback).
DensResult solve_density(State& s, int n, double pmass, const double* periodicBox, double tolh,
                         double hfact, int maxIter, bool withGradients, bool allowGraph = true);

// mixed.cu
void launch_gradient_mixed(State& s, double pmass);
void launch_force_mixed(State& s, double pmass, double beta, bool disc, bool pdv, bool shock);

// force.cu
void compute_forces(State& s, double pmass, double beta, double alphau, bool disc, bool pdv,
                    bool shock);

// timing helpers
struct EventPair
{
    cudaEvent_t a = nullptr, b = nullptr;
};
double elapsed_s(cudaEvent_t a, cudaEvent_t b);
cudaEvent_t ev(State& s);            // record an event on the state's stream (pooled)
void ev_reset(State& s);

void read_scalars(State& s);         // dscal -> hscal, synchronising the stream
// FATAL if the device raised an error bit; reread = false when the scalars were just read
// (nothing has run since)
void check_dev_err(State& s, const char* where, bool reread = true);

} // namespace cosmo
