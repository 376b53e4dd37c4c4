/*
 * sph_oracle.cpp -- CPU FP64 restatement of cosmoSPHere's density / smoothing-length /
 * force path.  TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA library and the
 * timed CPU baseline.  Nothing in the product links or calls this.
 *
 * Parity status
 *   pinned    the M4/M6 kernel functions and constants: checked bit-for-bit against the
 *             reference's include/kernel.hpp compiled here (oracle/ref_pin, tests/golden);
 *   pinned    the lattice and jiggle generators (harness input): checked against the
 *             reference's src/main.cu compiled here against a capture stub;
 *   UNPINNED  Hilbert keys, the leaf tree, the linked octree, node geometry and the
 *             j-leaf lists.  The reference takes them from Cornerstone (exafmm
 *             cornerstone-octree, no version pinned: Makefile:24, README.md:21-28), which is
 *             absent, and the reference has no tests or fixtures for them.  They are
 *             restated here from published algorithms: J. Skilling, "Programming the
 *             Hilbert curve", AIP Conf. Proc. 707 (2004) for the curve, and the
 *             split-until-bucket cornerstone leaf array of Keller et al., PASC 2023.
 *   physics   density / Newton-Raphson, gradient sweep, force prep and force follow the
 *             reference's own source line by line (cited per function).  Expression
 *             trees are kept as the reference writes them, compiled with
 *             -ffp-contract=off; the one deliberate fusion is r^2 = fma(dz,dz,fma(dy,dy,
 *             dx*dx)) in every pair loop, which the CUDA library forms the same way.
 *
 * j-leaf lists are emitted in ascending leaf (= Hilbert key) order, not the LIFO order
 * of the reference's stack walk (include/tree.cuh:324-345): the SET of j-leaves per
 * i-leaf is the reference's; pair sums therefore run over j in ascending sorted index.
 */

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <vector>

#include <omp.h>

namespace orc {

constexpr int      kMaxLevel = 21;                 // 21 bits per axis, 63-bit keys
constexpr uint64_t kKeyEnd   = 1ull << 63;         // one past the last live key
constexpr uint64_t kDeadKey  = ~0ull;              // parks h <= 0 at the end (tree.cuh:104)
constexpr unsigned kBucket   = 64;                 // BUCKET_SIZE, include/tree.cuh:53

// ------------------------------------------------------------------------------------
// SPH kernel (include/kernel.hpp:35-99).  Values are unnormalised, as the reference's.
// ------------------------------------------------------------------------------------
struct KernelDef
{
    int    quintic;
    double radkernel, radk2, cnormk, hfact_default;
};

inline KernelDef kernel_def(int quintic)
{
    const double pi = 3.141592653589793;
    if (quintic) return {1, 3.0, 9.0, 1.0 / (120.0 * pi), 1.0};
    return {0, 2.0, 4.0, 1.0 / pi, 1.2};
}

// M4 cubic, include/kernel.hpp:35-47
inline void cubic_kernel(double q, double& w, double& dw)
{
    const double a  = (2.0 - q > 0.0) ? (2.0 - q) : 0.0;
    const double b  = (1.0 - q > 0.0) ? (1.0 - q) : 0.0;
    const double a2 = a * a, a3 = a2 * a;
    const double b2 = b * b, b3 = b2 * b;
    w  = 0.25 * (a3 - 4.0 * b3);
    dw = 0.25 * (-3.0 * a2 + 12.0 * b2);
}

// M6 quintic, include/kernel.hpp:53-78
inline void quintic_kernel(double q2, double q, double& w, double& dw)
{
    if (q < 1.0)
    {
        const double q4 = q2 * q2;
        w  = -10.0 * q4 * q + 30.0 * q4 - 60.0 * q2 + 66.0;
        dw = q * (-50.0 * q2 * q + 120.0 * q2 - 120.0);
    }
    else if (q < 2.0)
    {
        const double a = q - 3.0, b = q - 2.0;
        const double a2 = a * a, b2 = b * b;
        w  = -(a2 * a2 * a) + 6.0 * (b2 * b2 * b);
        dw = -5.0 * (a2 * a2) + 30.0 * (b2 * b2);
    }
    else if (q < 3.0)
    {
        const double a = q - 3.0, a2 = a * a;
        w  = -(a2 * a2 * a);
        dw = -5.0 * (a2 * a2);
    }
    else { w = 0.0; dw = 0.0; }
}

inline void kern(const KernelDef& K, double q2, double q, double& w, double& dw)
{
    if (K.quintic) quintic_kernel(q2, q, w, dw);
    else           cubic_kernel(q, w, dw);
}

// ------------------------------------------------------------------------------------
// Hilbert curve (Skilling 2004): axes -> transposed index -> interleaved 3*bits key.
// Every aligned cube of side 2^s cells is one contiguous key range of length 8^s, so a
// key prefix names an octree node, as Cornerstone's hilbert3D does for the reference
// (include/tree.cuh:104).  The orientation is Skilling's, not Cornerstone's.
// ------------------------------------------------------------------------------------
inline uint64_t hilbert_encode(uint32_t ix, uint32_t iy, uint32_t iz, int bits = kMaxLevel)
{
    uint32_t X[3] = {ix, iy, iz};
    const uint32_t top = 1u << (bits - 1);
    for (uint32_t Q = top; Q > 1; Q >>= 1)
    {
        const uint32_t P = Q - 1;
        for (int i = 0; i < 3; ++i)
        {
            if (X[i] & Q) X[0] ^= P;
            else
            {
                const uint32_t t = (X[0] ^ X[i]) & P;
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    X[1] ^= X[0];
    X[2] ^= X[1];
    uint32_t t = 0;
    for (uint32_t Q = top; Q > 1; Q >>= 1)
        if (X[2] & Q) t ^= Q - 1;
    X[0] ^= t; X[1] ^= t; X[2] ^= t;

    uint64_t key = 0;
    for (int b = bits - 1; b >= 0; --b)
        key = (key << 3) | (uint64_t((X[0] >> b) & 1u) << 2) | (uint64_t((X[1] >> b) & 1u) << 1)
                         | uint64_t((X[2] >> b) & 1u);
    return key;
}

inline void hilbert_decode(uint64_t key, uint32_t out[3], int bits = kMaxLevel)
{
    uint32_t X[3] = {0, 0, 0};
    for (int b = bits - 1; b >= 0; --b)
    {
        const uint32_t o = uint32_t(key >> (3 * b)) & 7u;
        X[0] |= ((o >> 2) & 1u) << b;
        X[1] |= ((o >> 1) & 1u) << b;
        X[2] |= (o & 1u) << b;
    }
    const uint32_t N = 2u << (bits - 1);
    uint32_t t = X[2] >> 1;
    X[2] ^= X[1];
    X[1] ^= X[0];
    X[0] ^= t;
    for (uint32_t Q = 2; Q != N; Q <<= 1)
    {
        const uint32_t P = Q - 1;
        for (int i = 2; i >= 0; --i)
        {
            if (X[i] & Q) X[0] ^= P;
            else
            {
                const uint32_t s = (X[0] ^ X[i]) & P;
                X[0] ^= s;
                X[i] ^= s;
            }
        }
    }
    out[0] = X[0]; out[1] = X[1]; out[2] = X[2];
}

// Quantise one coordinate to 21 bits inside [lo, lo + len).
inline uint32_t quantise(double x, double lo, double scale)
{
    const double v = (x - lo) * scale;
    if (!(v >= 0.0)) return 0u;
    if (v >= 2097151.0) return 2097151u;
    return uint32_t(std::floor(v));
}

struct Box
{
    double lo[3], hi[3];
    bool periodic;
    double len(int d) const { return hi[d] - lo[d]; }
};

// Level of a cornerstone node from its key range length (8^(21-L)).
inline int level_of_range(uint64_t len)
{
    return kMaxLevel - __builtin_ctzll(len) / 3;
}
inline uint64_t node_range(int level) { return 1ull << (3 * (kMaxLevel - level)); }

// Placeholder-bit prefix: level-major, key-minor order when sorted.
inline uint64_t encode_prefix(uint64_t start, int level)
{
    return (start >> (3 * (kMaxLevel - level))) | (1ull << (3 * level));
}
inline int prefix_level(uint64_t p) { return (63 - __builtin_clzll(p)) / 3; }
inline uint64_t prefix_start(uint64_t p)
{
    const int L = prefix_level(p);
    return (p ^ (1ull << (3 * L))) << (3 * (kMaxLevel - L));
}

// ------------------------------------------------------------------------------------
// The state: everything the reference keeps in GpuState (include/gpu_state.hpp:36-123),
// in Hilbert order.
// ------------------------------------------------------------------------------------
struct State
{
    KernelDef K;
    int n = 0, nAlive = 0, nLeaves = 0, numNodes = 0;
    double pmass = 0.0, hfact = 0.0;
    Box box{};
    int itersRun = 0, unconverged = 0;
    std::vector<int64_t> activePerIter;

    std::vector<double> x, y, z, h, vx, vy, vz, ax, ay, az;      // sorted
    std::vector<double> rho, gradh, divv, xi, ddivvdt;
    std::vector<int32_t> converged;
    std::vector<uint64_t> keys;                                 // sorted keys
    std::vector<int32_t> order;                                 // sorted -> caller index

    std::vector<uint64_t> csTree;                               // nLeaves + 1
    std::vector<uint32_t> counts, layout;                       // nLeaves, nLeaves + 1
    std::vector<uint64_t> prefixes;                             // numNodes, BFS order
    std::vector<int32_t> childOffsets, internalToLeaf, levelRange, leafToInternal;
    std::vector<double> centers, sizes;                         // 3 per node
    std::vector<int32_t> particleLeaf;
    std::vector<double> hmax_leaf, hmax_node;
    std::vector<int32_t> jcount, jOffset, jlist;
    int64_t pairsDensity = 0, pairsGrad = 0, pairsForce = 0;    // accepted pair counts
    int64_t candDensity = 0;

    // force
    std::vector<double> pro2, cs, alpha, u;
    std::vector<double> fx, fy, fz, f4, vsigmax, divvF;
    int forceListBuilt = 0;
};

// ---------------------------------------------------------------- tree build
// src/tree.cu:47-72: bounding box.
static Box make_box(const State& s, const double* x, const double* y, const double* z, int n,
                    const double* periodicBox)
{
    Box b{};
    if (periodicBox)
    {
        for (int d = 0; d < 3; ++d) { b.lo[d] = periodicBox[2 * d]; b.hi[d] = periodicBox[2 * d + 1]; }
        b.periodic = true;
        return b;
    }
    double mn[3] = {x[0], y[0], z[0]}, mx[3] = {x[0], y[0], z[0]};
    const double* c[3] = {x, y, z};
    for (int d = 0; d < 3; ++d)
        for (int i = 0; i < n; ++i) { mn[d] = std::min(mn[d], c[d][i]); mx[d] = std::max(mx[d], c[d][i]); }
    const double span = std::max({mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]}) * 1.00001;
    const double half = 0.5 * span;
    for (int d = 0; d < 3; ++d)
    {
        const double ctr = 0.5 * (mn[d] + mx[d]);
        b.lo[d] = ctr - half;
        b.hi[d] = ctr + half;
    }
    b.periodic = false;
    (void)s;
    return b;
}

static uint64_t key_of(double x, double y, double z, double h, const Box& b)
{
    if (!(h > 0.0)) return kDeadKey;
    const double sx = 2097152.0 / b.len(0), sy = 2097152.0 / b.len(1), sz = 2097152.0 / b.len(2);
    return hilbert_encode(quantise(x, b.lo[0], sx), quantise(y, b.lo[1], sy), quantise(z, b.lo[2], sz));
}

// Leaf array: start from the root and split every node holding more than the bucket,
// until none does (src/tree.cu:126-136, from a fresh single-root seed every call).
static void build_leaf_tree(State& s)
{
    const uint64_t* kb = s.keys.data();
    const uint64_t* ke = kb + s.nAlive;
    std::vector<uint64_t> tree = {0, kKeyEnd};
    std::vector<uint32_t> cnt;
    for (;;)
    {
        const size_t nl = tree.size() - 1;
        cnt.assign(nl, 0);
        for (size_t i = 0; i < nl; ++i)
            cnt[i] = uint32_t(std::lower_bound(kb, ke, tree[i + 1]) - std::lower_bound(kb, ke, tree[i]));
        std::vector<uint64_t> next;
        next.reserve(tree.size() * 2);
        bool split = false;
        for (size_t i = 0; i < nl; ++i)
        {
            const uint64_t len = tree[i + 1] - tree[i];
            const int L = level_of_range(len);
            if (cnt[i] > kBucket && L < kMaxLevel)
            {
                const uint64_t child = len >> 3;
                for (int o = 0; o < 8; ++o) next.push_back(tree[i] + o * child);
                split = true;
            }
            else next.push_back(tree[i]);
        }
        next.push_back(kKeyEnd);
        if (!split) break;
        tree.swap(next);
    }
    s.csTree = tree;
    s.counts = cnt;
    s.nLeaves = int(tree.size() - 1);
    s.layout.assign(s.nLeaves + 1, 0);
    for (int i = 0; i < s.nLeaves; ++i) s.layout[i + 1] = s.layout[i] + s.counts[i];
}

// Fully linked octree in BFS (level-major) order, as Cornerstone's OctreeData
// (src/tree.cu:138-153): prefixes, childOffsets (0 = leaf), internalToLeaf, levelRange.
static void build_linked_tree(State& s)
{
    std::vector<uint64_t> nodes;
    for (int i = 0; i < s.nLeaves; ++i)
    {
        const uint64_t k = s.csTree[i];
        const int L = level_of_range(s.csTree[i + 1] - k);
        int L0 = 0;
        if (k != 0) L0 = std::max(0, kMaxLevel - __builtin_ctzll(k) / 3);
        for (int a = L0; a < L; ++a) nodes.push_back(encode_prefix(k, a));
        nodes.push_back(encode_prefix(k, L));
    }
    std::sort(nodes.begin(), nodes.end());
    s.prefixes = nodes;
    s.numNodes = int(nodes.size());
    s.childOffsets.assign(s.numNodes, 0);
    s.internalToLeaf.assign(s.numNodes, -1);
    s.levelRange.assign(kMaxLevel + 2, 0);
    std::vector<int> perLevel(kMaxLevel + 1, 0);
    for (int i = 0; i < s.numNodes; ++i)
    {
        const uint64_t p = nodes[i];
        const int L = prefix_level(p);
        perLevel[L]++;
        const uint64_t start = prefix_start(p);
        const uint64_t leafPos =
            std::lower_bound(s.csTree.begin(), s.csTree.end() - 1, start) - s.csTree.begin();
        const bool isLeaf = leafPos < (uint64_t)s.nLeaves && s.csTree[leafPos] == start &&
                            s.csTree[leafPos + 1] - start == node_range(L);
        if (isLeaf) s.internalToLeaf[i] = int32_t(leafPos);
        else
            s.childOffsets[i] =
                int32_t(std::lower_bound(nodes.begin(), nodes.end(), p << 3) - nodes.begin());
    }
    for (int L = 0; L <= kMaxLevel; ++L) s.levelRange[L + 1] = s.levelRange[L] + perLevel[L];

    // Node geometry (include/tree.cuh:110-125): centre and half-size from the prefix.
    s.centers.assign(3 * s.numNodes, 0.0);
    s.sizes.assign(3 * s.numNodes, 0.0);
    for (int i = 0; i < s.numNodes; ++i)
    {
        const uint64_t p = nodes[i];
        const int L = prefix_level(p);
        uint32_t ic[3];
        hilbert_decode(prefix_start(p), ic);
        const uint32_t side = 1u << (kMaxLevel - L);
        const double sd = double(side);
        for (int d = 0; d < 3; ++d)
        {
            const double unit = s.box.len(d) / 2097152.0;
            const double corner = double(ic[d] & ~(side - 1u));
            s.centers[3 * i + d] = s.box.lo[d] + (corner + 0.5 * sd) * unit;
            s.sizes[3 * i + d]   = 0.5 * sd * unit;
        }
    }
    // include/tree.cuh:151-174: leaf -> node and particle -> leaf maps
    s.leafToInternal.assign(s.nLeaves, -1);
    for (int i = 0; i < s.numNodes; ++i)
        if (s.childOffsets[i] == 0) s.leafToInternal[s.internalToLeaf[i]] = i;
    s.particleLeaf.assign(s.n, -1);
    for (int l = 0; l < s.nLeaves; ++l)
        for (uint32_t j = s.layout[l]; j < s.layout[l + 1]; ++j) s.particleLeaf[j] = l;
}

// ---------------------------------------------------------------- neighbour walk
// include/tree.cuh:228-252, nodeInRange<Symmetric, Periodic>.
static inline bool node_in_range(const State& s, bool symmetric, const double* ic, const double* isz,
                                 const double* ihalf, double radHi, int node)
{
    const double* a = symmetric ? isz : ihalf;
    double d[3];
    for (int k = 0; k < 3; ++k)
    {
        double dd = std::fabs(ic[k] - s.centers[3 * node + k]);
        if (s.box.periodic) dd = std::min(dd, s.box.len(k) - dd);
        const double g = dd - a[k] - s.sizes[3 * node + k];
        d[k] = (g > 0.0) ? g : 0.0;
    }
    const double n2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (symmetric)
    {
        const double rs = std::fmax(radHi, s.K.radkernel * s.hmax_node[node]);
        return n2 <= rs * rs;
    }
    return n2 <= 0.0;
}

// One i-leaf's list, in ascending leaf order (pre-order walk over key-ordered children).
static void walk_leaf(const State& s, bool symmetric, int iLeaf, std::vector<int32_t>& out)
{
    out.clear();
    const int iNode = s.leafToInternal[iLeaf];
    const double* ic = &s.centers[3 * iNode];
    const double* isz = &s.sizes[3 * iNode];
    double hmax = s.hmax_leaf[iLeaf];
    if (!std::isfinite(hmax) || hmax <= 0.0) hmax = 0.0;
    const double radHi = s.K.radkernel * hmax;
    const double ihalf[3] = {isz[0] + radHi, isz[1] + radHi, isz[2] + radHi};
    // explicit stack, children pushed in reverse so they pop in key order
    std::vector<int32_t> stack;
    stack.push_back(0);
    while (!stack.empty())
    {
        const int node = stack.back();
        stack.pop_back();
        if (!node_in_range(s, symmetric, ic, isz, ihalf, radHi, node)) continue;
        if (s.childOffsets[node] == 0) { out.push_back(s.internalToLeaf[node]); continue; }
        for (int o = 7; o >= 0; --o) stack.push_back(s.childOffsets[node] + o);
    }
}

// include/tree.cuh:360-389: CSR lists of ALL leaves.
static void build_lists(State& s, bool symmetric)
{
    const int nL = s.nLeaves;
    std::vector<std::vector<int32_t>> rows(nL);
#pragma omp parallel
    {
        std::vector<int32_t> tmp;
#pragma omp for schedule(dynamic, 64)
        for (int l = 0; l < nL; ++l)
        {
            walk_leaf(s, symmetric, l, tmp);
            rows[l] = tmp;
        }
    }
    s.jcount.assign(nL, 0);
    s.jOffset.assign(nL + 1, 0);
    for (int l = 0; l < nL; ++l)
    {
        s.jcount[l] = int32_t(rows[l].size());
        s.jOffset[l + 1] = s.jOffset[l] + s.jcount[l];
    }
    s.jlist.assign(std::max(s.jOffset[nL], 1), 0);
    for (int l = 0; l < nL; ++l)
        std::copy(rows[l].begin(), rows[l].end(), s.jlist.begin() + s.jOffset[l]);
}

// include/tree.cuh:177-191
static void hmax_leaves(State& s, const std::vector<int32_t>& leaves)
{
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < leaves.size(); ++k)
    {
        const int l = leaves[k];
        double hm = 0.0;
        for (uint32_t j = s.layout[l]; j < s.layout[l + 1]; ++j)
            if (std::isfinite(s.h[j])) hm = std::fmax(hm, s.h[j]);
        s.hmax_leaf[l] = hm;
    }
}

// include/tree.cuh:196-217, deepest level first (src/force.cu:50-60).
static void hmax_upsweep(State& s)
{
    s.hmax_node.assign(s.numNodes, 0.0);
    for (int L = kMaxLevel; L >= 0; --L)
        for (int i = s.levelRange[L]; i < s.levelRange[L + 1]; ++i)
        {
            const int c = s.childOffsets[i];
            if (c == 0)
            {
                const double hm = s.hmax_leaf[s.internalToLeaf[i]];
                s.hmax_node[i] = (std::isfinite(hm) && hm > 0.0) ? hm : 0.0;
                continue;
            }
            double m = 0.0;
            for (int o = 0; o < 8; ++o) m = std::fmax(m, s.hmax_node[c + o]);
            s.hmax_node[i] = m;
        }
}

// include/tree.cuh:75-84
static inline void nearest_image(const Box& b, double& dx, double& dy, double& dz)
{
    if (!b.periodic) return;
    const double lx = b.len(0), ly = b.len(1), lz = b.len(2);
    if (std::fabs(dx) > 0.5 * lx) dx = dx - lx * std::copysign(1.0, dx);
    if (std::fabs(dy) > 0.5 * ly) dy = dy - ly * std::copysign(1.0, dy);
    if (std::fabs(dz) > 0.5 * lz) dz = dz - lz * std::copysign(1.0, dz);
}

static inline double r2_of(double dx, double dy, double dz)
{
    return std::fma(dz, dz, std::fma(dy, dy, dx * dx));
}

// ---------------------------------------------------------------- density NR
// src/density_base.cu:237-334, one Newton step of one active particle.
static void density_step(State& s, int i, double tolh, int64_t& pairs, int64_t& cand)
{
    const KernelDef& K = s.K;
    const double xi = s.x[i], yi = s.y[i], zi = s.z[i];
    const double hi = s.h[i];
    const double hi_sq_inv = 1.0 / (hi * hi);
    double rhoi = 0.0, gradhi = 0.0;
    const int iLeaf = s.particleLeaf[i];
    const int jBase = s.jOffset[iLeaf], nj = s.jcount[iLeaf];
    for (int jl = 0; jl < nj; ++jl)
    {
        const int jLeaf = s.jlist[jBase + jl];
        for (uint32_t j = s.layout[jLeaf]; j < s.layout[jLeaf + 1]; ++j)
        {
            double dx = xi - s.x[j], dy = yi - s.y[j], dz = zi - s.z[j];
            nearest_image(s.box, dx, dy, dz);
            const double q2 = r2_of(dx, dy, dz) * hi_sq_inv;
            ++cand;
            if (q2 < K.radk2)
            {
                const double q = std::sqrt(q2);
                double w, dw;
                kern(K, q2, q, w, dw);
                rhoi += w;
                gradhi += -q * dw - 3.0 * w;
                ++pairs;
            }
        }
    }
    const double hi_old = hi;
    const double hi1 = 1.0 / hi;
    const double hi31 = hi1 * hi1 * hi1;
    const double hi41 = hi31 * hi1;
    const double rho_i = rhoi * K.cnormk * s.pmass * hi31;
    const double grad_i = gradhi * K.cnormk * s.pmass * hi41;
    if (!(rho_i > 0.0))
    {
        s.rho[i] = 0.0; s.gradh[i] = 0.0; s.converged[i] = 0;
        return;
    }
    const double hf = s.hfact;
    const double rhoh_i = s.pmass * (hf * hi1) * (hf * hi1) * (hf * hi1);
    const double funci = rhoh_i - rho_i;
    const double dhdrhoi = -hi / (3.0 * rhoh_i);
    const double omegai = 1.0 - dhdrhoi * grad_i;
    const double safe_omega = (omegai > 0.0) ? omegai : std::fabs(omegai + 1e-300);
    const double hnew_raw = hi - funci * dhdrhoi / safe_omega;
    double hnew;
    if (hnew_raw > 1.2 * hi) hnew = 1.2 * hi;
    else if (hnew_raw < 0.8 * hi) hnew = 0.8 * hi;
    else hnew = hnew_raw;
    s.rho[i] = rho_i;
    s.gradh[i] = grad_i;
    s.h[i] = hnew;
    s.converged[i] = (std::fabs((hnew - hi) / hi_old) < tolh) ? 1 : 0;
}

// src/density_base.cu:511-527
static double xi_limiter(const double g[9])
{
    const double dvxdx = (float)g[0], dvxdy = (float)g[1], dvxdz = (float)g[2];
    const double dvydx = (float)g[3], dvydy = (float)g[4], dvydz = (float)g[5];
    const double dvzdx = (float)g[6], dvzdy = (float)g[7], dvzdz = (float)g[8];
    const double divv = dvxdx + dvydy + dvzdz;
    const double cx = dvzdy - dvydz;
    const double cy = dvxdz - dvzdx;
    const double cz = dvydx - dvxdy;
    const double mdiv = std::fmax(-divv, 0.0);
    const double fac = mdiv * mdiv;
    const double trS = cx * cx + cy * cy + cz * cz;
    return (fac + trS > 2.220446049250313e-16) ? fac / (fac + trS) : 1.0;
}

// src/density_base.cu:529-714, one particle of the post-convergence sweep.
static void gradient_step(State& s, int i, int64_t& pairs)
{
    const KernelDef& K = s.K;
    if (!(s.h[i] > 0.0))
    {
        s.divv[i] = 0.0; s.ddivvdt[i] = 0.0; s.xi[i] = 1.0;
        return;
    }
    const double pm = s.pmass;
    const double xi = s.x[i], yi = s.y[i], zi = s.z[i];
    const double vxi = s.vx[i], vyi = s.vy[i], vzi = s.vz[i];
    const double axi = s.ax[i], ayi = s.ay[i], azi = s.az[i];
    const double hi = s.h[i];
    const double hi_sq_inv = 1.0 / (hi * hi);
    double rhoi = 0.0, gradhi = 0.0, divs = 0.0;
    double dv[9] = {0}, da[9] = {0};
    double rxx = 0, rxy = 0, rxz = 0, ryy = 0, ryz = 0, rzz = 0;
    const int iLeaf = s.particleLeaf[i];
    const int jBase = s.jOffset[iLeaf], nj = s.jcount[iLeaf];
    for (int jl = 0; jl < nj; ++jl)
    {
        const int jLeaf = s.jlist[jBase + jl];
        for (uint32_t j = s.layout[jLeaf]; j < s.layout[jLeaf + 1]; ++j)
        {
            double dx = xi - s.x[j], dy = yi - s.y[j], dz = zi - s.z[j];
            nearest_image(s.box, dx, dy, dz);
            const double r2 = r2_of(dx, dy, dz);
            const double q2 = r2 * hi_sq_inv;
            if (q2 >= K.radk2) continue;
            ++pairs;
            const double q = std::sqrt(q2);
            double w, dw;
            kern(K, q2, q, w, dw);
            rhoi += w;
            gradhi += -q * dw - 3.0 * w;
            const double rij = std::sqrt(r2);
            const double rij1 = 1.0 / (rij + 2.220446049250313e-16);
            const double rg = rij1 * dw;
            const double rx = dx * rg * pm, ry = dy * rg * pm, rz = dz * rg * pm;
            const double dvx = vxi - s.vx[j], dvy = vyi - s.vy[j], dvz = vzi - s.vz[j];
            divs += dvx * rx + dvy * ry + dvz * rz;
            dv[0] += dvx * rx; dv[1] += dvx * ry; dv[2] += dvx * rz;
            dv[3] += dvy * rx; dv[4] += dvy * ry; dv[5] += dvy * rz;
            dv[6] += dvz * rx; dv[7] += dvz * ry; dv[8] += dvz * rz;
            const double dax = axi - s.ax[j], day = ayi - s.ay[j], daz = azi - s.az[j];
            da[0] += dax * rx; da[1] += dax * ry; da[2] += dax * rz;
            da[3] += day * rx; da[4] += day * ry; da[5] += day * rz;
            da[6] += daz * rx; da[7] += daz * ry; da[8] += daz * rz;
            rxx -= dx * rx; rxy -= dx * ry; rxz -= dx * rz;
            ryy -= dy * ry; ryz -= dy * rz; rzz -= dz * rz;
        }
    }
    const double hi1 = 1.0 / hi;
    const double hi31 = hi1 * hi1 * hi1;
    const double hi41 = hi31 * hi1;
    const double rho_i = rhoi * K.cnormk * pm * hi31;
    const double grad_i = gradhi * K.cnormk * pm * hi41;
    s.rho[i] = rho_i;
    s.gradh[i] = grad_i;
    if (!(rho_i > 0.0))
    {
        s.divv[i] = 0.0; s.ddivvdt[i] = 0.0; s.xi[i] = 1.0;
        return;
    }
    const double omega = 1.0 + (hi / (3.0 * rho_i)) * grad_i;
    const double omega_inv = (omega > 0.0) ? (1.0 / omega) : 1.0;
    const double term = K.cnormk * omega_inv * hi41 / rho_i;
    const double denom = rxx * ryy * rzz + 2.0 * rxy * rxz * ryz - rxx * ryz * ryz - ryy * rxz * rxz
                         - rzz * rxy * rxy;
    const double rm0 = ryy * rzz - ryz * ryz;
    const double rm1 = rxz * ryz - rzz * rxy;
    const double rm2 = rxy * ryz - rxz * ryy;
    const double rm3 = rzz * rxx - rxz * rxz;
    const double rm4 = rxy * rxz - rxx * ryz;
    const double rm5 = rxx * ryy - rxy * rxy;
    s.divv[i] = -divs * term;
    double g[9], div_a;
    if (std::fabs(denom) > 2.2250738585072014e-308)
    {
        const double dd = 1.0 / denom;
        for (int r = 0; r < 3; ++r)
        {
            const double sx = dv[3 * r], sy = dv[3 * r + 1], sz = dv[3 * r + 2];
            g[3 * r]     = -(sx * rm0 + sy * rm1 + sz * rm2) * dd;
            g[3 * r + 1] = -(sx * rm1 + sy * rm3 + sz * rm4) * dd;
            g[3 * r + 2] = -(sx * rm2 + sy * rm4 + sz * rm5) * dd;
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
        for (int c = 0; c < 9; ++c) g[c] = -dv[c] * term;
        div_a = -term * (da[0] + da[4] + da[8]);
    }
    s.xi[i] = xi_limiter(g);
    s.ddivvdt[i] = div_a - (g[0] * g[0] + g[4] * g[4] + g[8] * g[8]
                            + 2.0 * (g[1] * g[3] + g[2] * g[6] + g[5] * g[7]));
}

template<class T>
static void gather(std::vector<T>& v, const std::vector<int32_t>& order)
{
    std::vector<T> t(v.size());
    for (size_t k = 0; k < order.size(); ++k) t[k] = v[order[k]];
    v.swap(t);
}

// src/density_base.cu:720-1015 (solveDensH, FLAT_PARTICLE).  Returns 0, or
// 1 = unconverged / list overflow, 2 = periodic support reaches half the box.
static int density_solve(State& s, int n, double pmass, const double* periodicBox, double tolh,
                         double hfact, int maxIter, int withGradients, const double* x,
                         const double* y, const double* z, const double* h, const double* v3,
                         const double* a3)
{
    s.n = n;
    s.pmass = pmass;
    s.hfact = (hfact > 0.0) ? hfact : s.K.hfact_default;
    s.x.assign(x, x + n); s.y.assign(y, y + n); s.z.assign(z, z + n); s.h.assign(h, h + n);
    auto load3 = [&](const double* p, std::vector<double>& a, std::vector<double>& b,
                     std::vector<double>& c) {
        if (p) { a.assign(p, p + n); b.assign(p + n, p + 2 * n); c.assign(p + 2 * n, p + 3 * n); }
        else { a.assign(n, 0.0); b.assign(n, 0.0); c.assign(n, 0.0); }
    };
    load3(v3, s.vx, s.vy, s.vz);
    load3(a3, s.ax, s.ay, s.az);
    s.rho.assign(n, 0.0); s.gradh.assign(n, 0.0); s.converged.assign(n, 0);
    s.divv.assign(n, 0.0); s.xi.assign(n, 0.0); s.ddivvdt.assign(n, 0.0);
    s.activePerIter.clear();
    s.pairsDensity = s.pairsGrad = s.candDensity = 0;
    s.forceListBuilt = 0;

    // buildTree, src/tree.cu:28-200
    s.box = make_box(s, x, y, z, n, periodicBox);
    std::vector<uint64_t> keys(n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) keys[i] = key_of(x[i], y[i], z[i], h[i], s.box);
    s.order.resize(n);
    std::iota(s.order.begin(), s.order.end(), 0);
    std::stable_sort(s.order.begin(), s.order.end(),
                     [&](int a, int b) { return keys[a] < keys[b]; });
    s.keys.resize(n);
    for (int k = 0; k < n; ++k) s.keys[k] = keys[s.order[k]];
    s.nAlive = int(std::lower_bound(s.keys.begin(), s.keys.end(), kDeadKey) - s.keys.begin());
    for (auto* v : {&s.x, &s.y, &s.z, &s.h}) gather(*v, s.order);
    if (withGradients)
        for (auto* v : {&s.vx, &s.vy, &s.vz, &s.ax, &s.ay, &s.az}) gather(*v, s.order);
    build_leaf_tree(s);
    build_linked_tree(s);
    s.hmax_leaf.assign(s.nLeaves, 0.0);

    std::vector<int32_t> active(s.nAlive), activeLeaves(s.nLeaves);
    std::iota(active.begin(), active.end(), 0);
    std::iota(activeLeaves.begin(), activeLeaves.end(), 0);
    s.itersRun = 0;
    for (int iter = 0; iter < maxIter; ++iter)
    {
        hmax_leaves(s, activeLeaves);
        build_lists(s, false);
        s.activePerIter.push_back((int64_t)active.size());
        int64_t pairs = 0, cand = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : pairs, cand)
        for (size_t k = 0; k < active.size(); ++k) density_step(s, active[k], tolh, pairs, cand);
        s.pairsDensity += pairs;
        s.candDensity += cand;
        s.itersRun = iter + 1;
        std::vector<int32_t> next;
        for (int i : active)
            if (!s.converged[i]) next.push_back(i);
        active.swap(next);
        if (active.empty()) break;
        std::vector<int32_t> lv;
        for (int i : active) lv.push_back(s.particleLeaf[i]);
        std::sort(lv.begin(), lv.end());
        lv.erase(std::unique(lv.begin(), lv.end()), lv.end());
        activeLeaves.swap(lv);
    }
    s.unconverged = int(active.size());
    if (!active.empty()) return 1;
    if (s.box.periodic && s.nAlive > 0)
    {
        double hm = 0.0;
        for (int i = 0; i < s.nAlive; ++i) hm = std::max(hm, s.h[i]);
        const double lmin = std::min({s.box.len(0), s.box.len(1), s.box.len(2)});
        if (s.K.radkernel * hm >= 0.5 * lmin) return 2;
    }
    if (withGradients)
    {
        std::vector<int32_t> all(s.nLeaves);
        std::iota(all.begin(), all.end(), 0);
        hmax_leaves(s, all);
        build_lists(s, false);
        int64_t pairs = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : pairs)
        for (int i = 0; i < n; ++i) gradient_step(s, i, pairs);
        s.pairsGrad = pairs;
    }
    return 0;
}

// ---------------------------------------------------------------- force
// src/force.cu:92-137 (prep) and :145-383 (pair loop), for one particle.
struct Prep { double hsqinv, hinv, rhoh, rho1, grkfac, pres, auterm, divfac; };

static Prep force_prep(const State& s, int i, double alphau)
{
    Prep p{};
    const double hi = s.h[i];
    if (!(hi > 0.0)) return p;
    const double hsq = 1.0 / (hi * hi);
    const double h4 = hsq * hsq;
    const double hfoh = s.hfact / hi;
    const double rho = s.pmass * hfoh * hfoh * hfoh;
    const double dhdrho = -hi / (3.0 * rho);
    const double omega = 1.0 - dhdrho * s.gradh[i];
    const double oinv = (omega > 0.0) ? (1 / omega) : 1.0;
    p.hsqinv = hsq;
    p.hinv = 1.0 / hi;
    p.rhoh = rho;
    p.rho1 = 1.0 / rho;
    p.grkfac = h4 * s.K.cnormk * oinv;
    p.pres = s.pro2[i] * rho * rho;
    p.auterm = 0.5 * s.pmass * (1.0 / rho) * alphau;
    p.divfac = s.K.cnormk * oinv * h4 / rho;
    return p;
}

static void force_step(State& s, const std::vector<Prep>& P, int i, double beta, bool disc,
                       bool pdv, bool shock, int64_t& pairs)
{
    const KernelDef& K = s.K;
    const double hi = s.h[i];
    if (!(hi > 0.0))
    {
        s.fx[i] = s.fy[i] = s.fz[i] = s.f4[i] = s.vsigmax[i] = s.divvF[i] = 0.0;
        return;
    }
    const double pm = s.pmass;
    const double xi = s.x[i], yi = s.y[i], zi = s.z[i];
    const Prep& pi = P[i];
    const double pro2i = s.pro2[i], vwavei = s.cs[i], alphai = s.alpha[i], eni = s.u[i];
    double itx = 0, ity = 0, itz = 0, jtx = 0, jty = 0, jtz = 0;
    double f4s = 0.0, vsm = 0.0, divs = 0.0;
    const int iLeaf = s.particleLeaf[i];
    const int jBase = s.jOffset[iLeaf], nj = s.jcount[iLeaf];
    for (int jl = 0; jl < nj; ++jl)
    {
        const int jLeaf = s.jlist[jBase + jl];
        for (uint32_t j = s.layout[jLeaf]; j < s.layout[jLeaf + 1]; ++j)
        {
            double dx = xi - s.x[j], dy = yi - s.y[j], dz = zi - s.z[j];
            nearest_image(s.box, dx, dy, dz);
            const double dr2 = r2_of(dx, dy, dz);
            if (!(dr2 > 0.0)) continue;
            const double hj = s.h[j];
            {
                const double rmax2 = K.radk2 * std::fmax(hi * hi, hj * hj) * (1.0 + 1e-10);
                if (dr2 >= rmax2) continue;
            }
            const Prep& pj = P[j];
            const double qi2 = dr2 * pi.hsqinv;
            const double qj2 = dr2 * pj.hsqinv;
            const double dr = std::sqrt(dr2);
            const double rij1 = 1.0 / dr;
            const double rx = dx * rij1, ry = dy * rij1, rz = dz * rij1;
            const double dvx = s.vx[i] - s.vx[j], dvy = s.vy[i] - s.vy[j], dvz = s.vz[i] - s.vz[j];
            const double projv = dvx * rx + dvy * ry + dvz * rz;
            const double rhoj = pj.rhoh, rho1j = pj.rho1, pro2j = s.pro2[j];
            const double vwavej = s.cs[j], alphaj = s.alpha[j], enj = s.u[j];
            const double prj = pj.pres, autermj = pj.auterm;
            const double vsigi = std::fmax(vwavei - beta * projv, 0.0);
            const double vsigavi = std::fmax(alphai * vwavei - beta * projv, 0.0);
            const double vsigj = std::fmax(vwavej - beta * projv, 0.0);
            const double vsigavj = std::fmax(alphaj * vwavej - beta * projv, 0.0);
            const double pvs = std::fmax(vsigi, vsigj);
            double qr2i = 0.0, qr2j = 0.0;
            const double denij = eni - enj;
            const double vsigu = std::sqrt(std::fabs(pi.pres - prj) * (2.0 / (pi.rhoh + rhoj)));
            if (disc)
            {
                const double hori = hi * rij1, horj = hj * rij1;
                if (projv < 0.0)
                {
                    qr2i = -0.5 * pi.rho1 * (alphai * vwavei - beta * projv) * hori * projv;
                    qr2j = -0.5 * rho1j * (alphaj * vwavej - beta * projv) * horj * projv;
                }
                else
                {
                    qr2i = -0.5 * pi.rho1 * alphai * vwavei * hori * projv;
                    qr2j = -0.5 * rho1j * alphaj * vwavej * horj * projv;
                }
            }
            else if (projv < 0.0)
            {
                qr2i = -0.5 * pi.rho1 * vsigavi * projv;
                qr2j = -0.5 * rho1j * vsigavj * projv;
            }
            bool took = false;
            if (qi2 < K.radk2)
            {
                took = true;
                vsm = std::fmax(vsm, pvs);
                double w, dw;
                const double q = dr * pi.hinv;
                kern(K, qi2, q, w, dw);
                divs += pm * dw * projv;
                const double gki = dw * pi.grkfac;
                const double gpi = pm * (pro2i + qr2i) * gki;
                itx += -gpi * rx; ity += -gpi * ry; itz += -gpi * rz;
                const double pdvi = pm * pro2i * projv * gki;
                const double dissi = disc
                    ? -0.5 * pm * pi.rho1 * alphai * vwavei * (hi * rij1) * projv * projv * gki
                    : pm * qr2i * projv * gki;
                const double condi = vsigu * denij * pi.auterm * gki;
                if (pdv) f4s += pdvi;
                if (shock) f4s += dissi;
                f4s += condi;
            }
            if (qj2 < K.radk2)
            {
                took = true;
                vsm = std::fmax(vsm, pvs);
                double w, dw;
                const double q = dr * pj.hinv;
                kern(K, qj2, q, w, dw);
                const double gkj = dw * pj.grkfac;
                const double gpj = pm * (pro2j + qr2j) * gkj;
                jtx -= gpj * rx; jty -= gpj * ry; jtz -= gpj * rz;
                f4s += vsigu * denij * autermj * gkj;
            }
            if (took) ++pairs;
        }
    }
    s.fx[i] = itx + jtx;
    s.fy[i] = ity + jty;
    s.fz[i] = itz + jtz;
    s.f4[i] = f4s;
    s.vsigmax[i] = vsm;
    s.divvF[i] = -divs * pi.divfac;
}

// src/force.cu:385-455 (computeForces, with buildForceJLeafList :19-88).  thermo4 and
// vel3 are in the caller's order (component-major), gathered as cosmo_upload_sorted does;
// vel3 == nullptr keeps the velocities the density solve sorted.
static int force_pass(State& s, double beta, double alphau, int disc, int pdv, int shock,
                      const double* thermo4, const double* vel3)
{
    const int n = s.n;
    auto g = [&](const double* src, std::vector<double>& dst) {
        dst.resize(n);
        for (int k = 0; k < n; ++k) dst[k] = src[s.order[k]];
    };
    g(thermo4, s.pro2); g(thermo4 + n, s.cs); g(thermo4 + 2 * size_t(n), s.alpha);
    g(thermo4 + 3 * size_t(n), s.u);
    if (vel3) { g(vel3, s.vx); g(vel3 + n, s.vy); g(vel3 + 2 * size_t(n), s.vz); }
    if (!s.forceListBuilt)
    {
        hmax_upsweep(s);
        build_lists(s, true);
        s.forceListBuilt = 1;
    }
    std::vector<Prep> P(n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) P[i] = force_prep(s, i, alphau);
    for (auto* v : {&s.fx, &s.fy, &s.fz, &s.f4, &s.vsigmax, &s.divvF}) v->assign(n, 0.0);
    int64_t pairs = 0;
    const bool pd = pdv > 0, sh = shock > 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : pairs)
    for (int i = 0; i < n; ++i) force_step(s, P, i, beta, disc != 0, pd, sh, pairs);
    s.pairsForce = pairs;
    return 0;
}

} // namespace orc

// ====================================================================================
// C interface for the Python test harness (ctypes).
// ====================================================================================
using orc::State;

extern "C" {

State* orc_create(int quintic)
{
    State* s = new State();
    s->K = orc::kernel_def(quintic);
    return s;
}

void orc_destroy(State* s) { delete s; }

void orc_set_threads(int t)
{
    if (t > 0) omp_set_num_threads(t);
}

int orc_max_threads(void) { return omp_get_max_threads(); }

int orc_density(State* s, int n, double pmass, int periodic, const double* box6, double tolh,
                double hfact, int maxIter, int withGradients, const double* x, const double* y,
                const double* z, const double* h, const double* v3, const double* a3)
{
    if (n <= 0) return 0;
    return orc::density_solve(*s, n, pmass, periodic ? box6 : nullptr, tolh, hfact, maxIter,
                              withGradients, x, y, z, h, v3, a3);
}

int orc_force(State* s, double beta, double alphau, int disc, int pdv, int shock,
              const double* thermo4, const double* vel3)
{
    if (s->n <= 0) return 0;
    return orc::force_pass(*s, beta, alphau, disc, pdv, shock, thermo4, vel3);
}

// Scalar results: name -> value.
double orc_scalar(State* s, const char* name)
{
    const std::string k(name);
    if (k == "n") return s->n;
    if (k == "nAlive") return s->nAlive;
    if (k == "nLeaves") return s->nLeaves;
    if (k == "numNodes") return s->numNodes;
    if (k == "itersRun") return s->itersRun;
    if (k == "unconverged") return s->unconverged;
    if (k == "pairsDensity") return double(s->pairsDensity);
    if (k == "candDensity") return double(s->candDensity);
    if (k == "pairsGrad") return double(s->pairsGrad);
    if (k == "pairsForce") return double(s->pairsForce);
    if (k == "hfact") return s->hfact;
    for (int d = 0; d < 3; ++d)
    {
        if (k == std::string("boxlo") + char('0' + d)) return s->box.lo[d];
        if (k == std::string("boxhi") + char('0' + d)) return s->box.hi[d];
    }
    return NAN;
}

// Array results: returns the element count and copies into out when out != nullptr.
// dtype codes: 0 f64, 1 i32, 2 u32, 3 u64, 4 i64.
long orc_array(State* s, const char* name, void* out, int* dtype)
{
    const std::string k(name);
    auto put = [&](const void* p, size_t cnt, size_t es, int code) -> long {
        if (dtype) *dtype = code;
        if (out && cnt) std::memcpy(out, p, cnt * es);
        return long(cnt);
    };
#define ORC_F64(nm) if (k == #nm) return put(s->nm.data(), s->nm.size(), 8, 0);
#define ORC_I32(nm) if (k == #nm) return put(s->nm.data(), s->nm.size(), 4, 1);
#define ORC_U32(nm) if (k == #nm) return put(s->nm.data(), s->nm.size(), 4, 2);
#define ORC_U64(nm) if (k == #nm) return put(s->nm.data(), s->nm.size(), 8, 3);
    ORC_F64(x) ORC_F64(y) ORC_F64(z) ORC_F64(h) ORC_F64(vx) ORC_F64(vy) ORC_F64(vz)
    ORC_F64(rho) ORC_F64(gradh) ORC_F64(divv) ORC_F64(xi) ORC_F64(ddivvdt)
    ORC_F64(centers) ORC_F64(sizes) ORC_F64(hmax_leaf) ORC_F64(hmax_node)
    ORC_F64(fx) ORC_F64(fy) ORC_F64(fz) ORC_F64(f4) ORC_F64(vsigmax) ORC_F64(divvF)
    ORC_I32(order) ORC_I32(childOffsets) ORC_I32(internalToLeaf) ORC_I32(levelRange)
    ORC_I32(leafToInternal) ORC_I32(particleLeaf) ORC_I32(jcount) ORC_I32(jOffset)
    ORC_I32(jlist) ORC_I32(converged)
    ORC_U32(counts) ORC_U32(layout)
    ORC_U64(keys) ORC_U64(csTree) ORC_U64(prefixes)
#undef ORC_F64
#undef ORC_I32
#undef ORC_U32
#undef ORC_U64
    if (k == "activePerIter")
        return put(s->activePerIter.data(), s->activePerIter.size(), 8, 4);
    if (dtype) *dtype = -1;
    return -1;
}

// Building blocks, for the harness's property tests.
uint64_t orc_hilbert_encode(uint32_t ix, uint32_t iy, uint32_t iz, int bits)
{
    return orc::hilbert_encode(ix, iy, iz, bits);
}

void orc_hilbert_decode(uint64_t key, int bits, uint32_t* out3) { orc::hilbert_decode(key, out3, bits); }

void orc_kernel_eval(int quintic, int n, const double* q, double* w, double* dw)
{
    const orc::KernelDef K = orc::kernel_def(quintic);
    for (int i = 0; i < n; ++i) orc::kern(K, q[i] * q[i], q[i], w[i], dw[i]);
}

void orc_kernel_consts(int quintic, double* out4)
{
    const orc::KernelDef K = orc::kernel_def(quintic);
    out4[0] = K.radkernel; out4[1] = K.radk2; out4[2] = K.cnormk; out4[3] = K.hfact_default;
}

} // extern "C"
