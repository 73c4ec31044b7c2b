// tree.cu -- sm_100a octree build of the TSR volumetric core.
//
// Reproduces Tree::Tree() (Scene/Tree/Tree.cpp:26-37): Nodes (containment,
// sampling nodes, 2:1 balancing, block-DFS relayout, sample reorder;
// Nodes.cpp:186-636), Leaves (scopes, node->leaf links, face-neighbour CSR;
// Leaves.cpp:22-180) and DualCells (Schaefer-Warren enumeration;
// DualCells.cpp:49-357).  Paths are relative to
// SurfaceReconstruction/SurfaceReconstruction/ of the reference.
//
// All topology predicates run in FP64 with explicit round-to-nearest
// arithmetic (common.cuh), so every node the reference creates is created
// here and nothing else.  Node storage indices during the build follow
// allocation order; the relayout at the end maps them onto the reference's
// block-DFS numbering, which depends only on topology.
#include <cooperative_groups.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "handles.h"

namespace cg = cooperative_groups;

namespace tsr {
namespace {

constexpr unsigned BLK = 256;

// ------------------------------------------------------------------ storage
struct NodeStore {
    DBuf<uint32_t> children, parents, cc, cnt;
    DBuf<uint8_t> depth;
    DBuf<D3> nmin;
    uint32_t count = 0, cap = 0;
    cudaStream_t st = nullptr;

    template <class T>
    void grow_one(DBuf<T> &b, uint32_t newcap) {
        DBuf<T> nb(newcap, st);
        if (count) TSR_CUDA(cudaMemcpyAsync(nb.p, b.p, (size_t)count * sizeof(T), cudaMemcpyDeviceToDevice, st));
        b = std::move(nb);
    }
    void ensure(uint64_t need) {
        if (need >= (uint64_t)INVALID - 8) fail(TSR_ERR_OVERFLOW_U32, "node count exceeds 2^32 - 2 (Nodes.cpp:399-407)");
        if (need <= cap) return;
        uint64_t nc = std::max<uint64_t>(need, (uint64_t)cap + cap / 2 + 1024);
        if (nc >= INVALID) nc = INVALID - 1;
        uint32_t newcap = (uint32_t)nc;
        grow_one(children, newcap); grow_one(parents, newcap); grow_one(cc, newcap); grow_one(cnt, newcap);
        grow_one(depth, newcap); grow_one(nmin, newcap);
        cap = newcap;
    }
};

struct NV {   // device view of the node store
    uint32_t *children, *parents, *cc, *cnt;
    uint8_t *depth;
    D3 *nmin;
};

inline NV view(NodeStore &s) { return NV{s.children.p, s.parents.p, s.cc.p, s.cnt.p, s.depth.p, s.nmin.p}; }

struct Root {
    D3 mn;
    double size;
};

// Initializes the 8 children of `node` in block `base`.
__device__ inline void make_children(const NV &v, uint32_t node, uint32_t base, double child_size, uint32_t key) {
    D3 mn = v.nmin[node];
    uint8_t d = v.depth[node] + 1;
    for (uint32_t c = 0; c < 8; ++c) {
        uint32_t i = base + c;
        v.children[i] = INVALID;
        v.parents[i] = node;
        v.cc[i] = 0;
        v.cnt[i] = 0;
        v.depth[i] = d;
        v.nmin[i] = child_coords(mn, child_size, c);
    }
    v.cc[node] = key;
    v.children[node] = base;
}

// ------------------------------------------------------------ root scope
__global__ void k_bounds(uint32_t n, const D3 *pos, const double *scale, double h_svo, double *part) {
    __shared__ double sm[6][BLK];
    double lo[3] = {REAL_MAX, REAL_MAX, REAL_MAX}, hi[3] = {-REAL_MAX, -REAL_MAX, -REAL_MAX};
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        D3 p = pos[s];
        double r = dadd(dmul(scale[s], h_svo), EPS);   // Samples.cpp:442-449
        double a[3] = {p.x, p.y, p.z};
        for (int j = 0; j < 3; ++j) {
            double l = dsub(a[j], r), h = dadd(a[j], r);
            lo[j] = l < lo[j] ? l : lo[j];
            hi[j] = h > hi[j] ? h : hi[j];
        }
    }
    for (int j = 0; j < 3; ++j) { sm[j][threadIdx.x] = lo[j]; sm[3 + j][threadIdx.x] = hi[j]; }
    __syncthreads();
    for (unsigned o = BLK / 2; o; o >>= 1) {
        if (threadIdx.x < o)
            for (int j = 0; j < 3; ++j) {
                double a = sm[j][threadIdx.x + o], b = sm[3 + j][threadIdx.x + o];
                if (a < sm[j][threadIdx.x]) sm[j][threadIdx.x] = a;
                if (b > sm[3 + j][threadIdx.x]) sm[3 + j][threadIdx.x] = b;
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int j = 0; j < 6; ++j) part[blockIdx.x * 6 + j] = sm[j][0];
}

// ------------------------------------------------------------- containment
// One level of Nodes::createNodesForContainment/findContainer
// (Nodes.cpp:222-269): samples whose node is small enough stop there,
// the others request children for their node.
__global__ void k_contain_mark(uint32_t n, const double *scale, double h_svo, double size_l, uint32_t *cur,
                               uint32_t *container, uint32_t *need, uint32_t *cnt) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || container[s] != INVALID) return;
    double r = dmul(scale[s], h_svo);
    uint32_t node = cur[s];
    if (size_l <= r) {
        container[s] = node;
        atomicAdd(&cnt[node], 1u);
        return;
    }
    need[node] = 1;
}

__global__ void k_contain_alloc(uint32_t lo, uint32_t hi, const uint32_t *need, const uint32_t *rank, NV v,
                                uint32_t base, double child_size) {
    uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hi || !need[i]) return;
    make_children(v, i, base + 8 * rank[i - lo], child_size, 0);
}

__global__ void k_contain_step(uint32_t n, const D3 *pos, double child_size, uint32_t *cur,
                               const uint32_t *container, NV v) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || container[s] != INVALID) return;
    uint32_t node = cur[s];
    D3 mn = v.nmin[node];
    D3 p = pos[s];
    D3 c{dadd(mn.x, child_size), dadd(mn.y, child_size), dadd(mn.z, child_size)};
    uint32_t d = 0;   // Nodes.cpp:32-44 on p - centre
    if (dsub(p.x, c.x) >= 0.0) d |= 1u;
    if (dsub(p.y, c.y) >= 0.0) d |= 2u;
    if (dsub(p.z, c.z) >= 0.0) d |= 4u;
    cur[s] = v.children[node] + d;
}

// ---------------------------------------------------------------- sampling
struct SampleRef {
    D3 p, n;
    double r;
    bool positive;
};

__device__ inline SampleRef sample_side(uint32_t key, const D3 *pos, const D3 *nrm, const double *scale, double h_svo) {
    uint32_t s = (key - 1) >> 1;
    SampleRef q;
    q.p = pos[s];
    q.n = nrm[s];
    q.r = dmul(scale[s], h_svo);
    q.positive = ((key - 1) & 1u) == 0;
    return q;
}

// Nodes.cpp:471-488
__device__ inline bool fitting_center(const D3 &node_min, double child_size, const SampleRef &q) {
    D3 c{dadd(node_min.x, child_size), dadd(node_min.y, child_size), dadd(node_min.z, child_size)};
    double d2 = d3len2(d3sub(c, q.p));
    if (d2 > dmul(q.r, q.r)) return false;
    bool on_pos = plane_distance(q.p, q.n, c) > 0.0;
    return on_pos == q.positive;
}

// Nodes.cpp:490-517
__device__ inline bool intersect_side(const D3 &mn, double size, const SampleRef &q) {
    bool all_wrong = true;
    for (uint32_t i = 0; i < 8; ++i) {
        D3 corner = child_coords(mn, size, i);
        bool in_pos = plane_distance(q.p, q.n, corner) > 0.0;
        if (in_pos == q.positive) { all_wrong = false; break; }
    }
    if (all_wrong) return false;
    D3 mx{dadd(mn.x, size), dadd(mn.y, size), dadd(mn.z, size)};
    return aabb_sphere(mn, mx, q.p, q.r);
}

// Leaf test of the tree as the sample side `key` saw it: children created by
// a side with a key >= `key` do not exist yet for it.
__device__ inline bool leaf_v(const NV &v, uint32_t n, uint32_t key) {
    return v.children[n] == INVALID || v.cc[n] >= key;
}

// Reliability of a leaf (Nodes.cpp:440-451).
__device__ inline bool leaf_reliable(const D3 &mn, double size, const SampleRef &q) {
    double cs = dmul(size, 0.5);
    if (!fitting_center(mn, cs, q)) return false;
    double g = dmul(cs, 0.5);
    for (uint32_t i = 0; i < 8; ++i)
        if (fitting_center(child_coords(mn, cs, i), g, q)) return true;
    return false;
}

// Deepest node of the versioned tree whose box contains the side's sphere
// (radius r around the sample) with a margin: every node outside its subtree
// is then disjoint from the sphere by at least the margin, so the exact tests
// of the reference reject all of them, and the descent's best child along
// the path is always the one containing the sphere.  Both searches can start
// there and give the reference's results.  The margin, 1e-12 of the largest
// coordinate magnitude plus the root size, dwarfs the FP64 rounding of the
// corner recurrence and of the tests.
__device__ inline uint32_t sphere_start_v(const NV &v, const Root &root, uint32_t key, const SampleRef &q,
                                          double margin) {
    uint32_t node = 0;
    D3 mn = root.mn;
    uint32_t d = 0;
    const double lo[3] = {q.p.x - q.r, q.p.y - q.r, q.p.z - q.r};
    const double hi[3] = {q.p.x + q.r, q.p.y + q.r, q.p.z + q.r};
    while (!leaf_v(v, node, key) && d < MAX_TREE_DEPTH) {
        double cs = size_at(root.size, d + 1);
        const double c3[3] = {dadd(mn.x, cs), dadd(mn.y, cs), dadd(mn.z, cs)};
        uint32_t digit = 0;
        for (int a = 0; a < 3; ++a) {
            if (hi[a] < c3[a] - margin) continue;
            if (lo[a] > c3[a] + margin) { digit |= 1u << a; continue; }
            return node;
        }
        node = v.children[node] + digit;
        mn = child_coords(mn, cs, digit);
        ++d;
    }
    return node;
}

// Nodes::findReliableSamplingNode (Nodes.cpp:433-469) over the versioned
// tree, from `start` (the root, or a node that contains the side's sphere,
// see sphere_start_v); calls on_read(leaf) for every leaf it rejects.
// Returns the reliable leaf or INVALID.  The order is the reference's
// depth-first order (children 0..7, each subtree before the next sibling),
// which decides the returned leaf.
template <class OnRead>
__device__ uint32_t find_reliable_v(const NV &v, const Root &root, uint32_t start, uint32_t key,
                                    const SampleRef &q, OnRead on_read, int *err) {
    if (leaf_v(v, start, key)) {
        D3 smn = start ? v.nmin[start] : root.mn;
        double ssz = start ? size_at(root.size, v.depth[start]) : root.size;
        if (leaf_reliable(smn, ssz, q)) return start;
        on_read(start);
        return INVALID;
    }
    // The node being scanned lives in registers (its children block, corner,
    // depth and next child); children's corners come from the build's own
    // recurrence (child_coords, exact), so a child costs a load only when it
    // meets the side.  Stack entries are (node, next child); resuming reloads
    // the node's block, corner and depth.
    uint64_t st[MAX_TREE_DEPTH];
    int sp = 0;
    uint32_t cur = start, c0 = v.children[start], next = 0, d = v.depth[start];
    D3 pmn = start ? v.nmin[start] : root.mn;
    double cs = size_at(root.size, d + 1);
    while (true) {
        if (next == 8) {
            if (sp == 0) return INVALID;
            uint64_t e = st[--sp];
            cur = (uint32_t)e;
            next = (uint32_t)(e >> 32);
            c0 = v.children[cur];
            d = v.depth[cur];
            pmn = cur ? v.nmin[cur] : root.mn;
            cs = size_at(root.size, d + 1);
            continue;
        }
        uint32_t c = next++;
        D3 cmn = child_coords(pmn, cs, c);
        if (!intersect_side(cmn, cs, q)) continue;
        uint32_t idx = c0 + c;
        uint32_t ch = v.children[idx];
        if (ch == INVALID || v.cc[idx] >= key) {   // leaf_v
            if (leaf_reliable(cmn, cs, q)) return idx;
            on_read(idx);
            continue;
        }
        if (next < 8) {   // nothing to resume after the last child
            if (sp >= MAX_TREE_DEPTH) { *err = 1; return INVALID; }
            st[sp++] = (uint64_t)cur | ((uint64_t)next << 32);
        }
        cur = idx;
        c0 = ch;
        pmn = cmn;
        ++d;
        cs = dmul(cs, 0.5);
        next = 0;
    }
}

// Child with the largest overlap with the sampling segment (Nodes.cpp:300-331).
__device__ inline uint32_t best_child(const D3 &mn, double size, const D3 &p, const D3 &endp) {
    double cs = dmul(size, 0.5);
    double score = -REAL_MAX;
    uint32_t best = INVALID;
    for (uint32_t c = 0; c < 8; ++c) {
        D3 bmin = child_coords(mn, cs, c);
        D3 bmax{dadd(bmin.x, cs), dadd(bmin.y, cs), dadd(bmin.z, cs)};
        double t0, t1;
        if (!segment_aabb(t0, t1, p, endp, bmin, bmax)) continue;
        double ov = dsub(t1, t0);
        if (ov <= score) continue;
        score = ov;
        best = c;
        if (ov >= dsub(1.0, EPS)) break;
    }
    return best;
}

__device__ inline D3 segment_end(const SampleRef &q) {
    double r = q.positive ? q.r : -q.r;
    return D3{dadd(q.p.x, dmul(q.n.x, r)), dadd(q.p.y, dmul(q.n.y, r)), dadd(q.p.z, dmul(q.n.z, r))};
}

// Leaf the best-overlap descent from the root reaches in the versioned tree
// (started at a node that contains the side's sphere, see sphere_start_v).
__device__ inline uint32_t descent_leaf_v(const NV &v, const Root &root, uint32_t start, uint32_t key,
                                          const SampleRef &q, int *err) {
    D3 endp = segment_end(q);
    uint32_t node = start;
    for (int guard = 0; guard < 4 * MAX_TREE_DEPTH; ++guard) {
        if (leaf_v(v, node, key)) return node;
        double sz = size_at(root.size, v.depth[node]);
        uint32_t b = best_child(v.nmin[node], sz, q.p, endp);
        if (b == INVALID) { *err = 2; return node; }
        node = v.children[node] + b;
    }
    *err = 3;
    return node;
}

// Round evaluation: status 1 = reliable (witness), 2 = writer.  Also counts
// each side's dependency pairs (1 for a witness; the rejected leaves plus the
// descent leaf for a writer).
// split_sides: the keys are both sides of consecutive samples in turn (the
// first round); threads then take all positive sides first and all negative
// sides after them, so the lanes of a warp search in the same direction
// (the two sides' searches differ, and a warp waits for its longest one).
// Results go to each side's own slot either way.
__global__ void k_sampling_eval(uint32_t m, const uint32_t *keys, NV v, Root root, const D3 *pos, const D3 *nrm,
                                const double *scale, double h_svo, uint8_t *status, uint32_t *witness,
                                uint32_t *dleaf, uint32_t *cnt, double margin, int *err, int split_sides) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const uint32_t half = (m + 1) / 2;
    const uint32_t i = split_sides ? (t < half ? 2 * t : 2 * (t - half) + 1) : t;
    uint32_t key = keys[i];
    SampleRef q = sample_side(key, pos, nrm, scale, h_svo);
    int e = 0;
    uint32_t reads = 0;
    uint32_t start = sphere_start_v(v, root, key, q, margin);
    uint32_t w = find_reliable_v(v, root, start, key, q, [&](uint32_t) { ++reads; }, &e);
    status[i] = (w != INVALID) ? 1 : 2;
    witness[i] = w;
    cnt[i] = (w != INVALID) ? 1u : reads + 1u;
    dleaf[i] = descent_leaf_v(v, root, start, key, q, &e);
    if (e) atomicExch(err, e);
}

// Conflict resolution of a round as a breadth-first search in key order.
// A side is unresolved when a leaf it depends on (its witness if reliable;
// every leaf its search read and its descent leaf if it is a writer) is
// claimed by an earlier writer or unresolved side; claims propagate wave by
// wave from the writers.  The result is the least fixed point, i.e. exactly
// what a sequential pass in key order computes.

// Each wave: members claim their descent leaf with their key (leaves whose
// claim dropped are recorded), then every side depending on a recorded leaf
// with a larger key becomes unresolved and joins the next wave.
//
// All waves of one round in one cooperative launch (grid-wide barriers
// instead of a host round trip per wave).  Counter pairs alternate by wave
// parity; the idle pair is cleared between the two barriers of a wave, when
// no thread can still be reading it.  The wave count is bounded.
__global__ void k_waves_coop(uint32_t nf0, uint32_t *front, uint32_t *next, const uint32_t *keys,
                             const uint32_t *dleaf, uint32_t *mark, uint32_t *touched, const uint32_t *seg_lo,
                             const uint32_t *seg_hi, const uint32_t *by_leaf, uint32_t *unres, uint32_t *ctr,
                             uint32_t max_waves, uint32_t *waves_out, int *err) {
    cg::grid_group grid = cg::this_grid();
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t gsize = gridDim.x * blockDim.x;
    const uint32_t lane = threadIdx.x & 31, gwarp = gtid >> 5, nwarps = gsize >> 5;
    uint32_t nf = nf0;
    uint32_t wave = 0;
    while (nf > 0) {
        if (wave >= max_waves) {
            if (gtid == 0) atomicExch(err, 7);
            break;
        }
        uint32_t *c = ctr + 2 * (wave & 1);        // this wave's (touched, next) counters
        uint32_t *c_idle = ctr + 2 * ((wave + 1) & 1);
        for (uint32_t i = gtid; i < nf; i += gsize) {
            uint32_t p = front[i];
            uint32_t x = dleaf[p], k = keys[p];
            uint32_t old = atomicMin(&mark[x], k);
            if (old > k) touched[atomicAdd(&c[0], 1u)] = x;
        }
        grid.sync();
        if (gtid == 0) { c_idle[0] = 0; c_idle[1] = 0; }
        const uint32_t nt = c[0];
        for (uint32_t j = gwarp; j < nt; j += nwarps) {
            uint32_t x = touched[j];
            uint32_t lo = seg_lo[x];
            if (lo == INVALID) continue;
            uint32_t hi = seg_hi[x], mk = mark[x];
            for (uint32_t q2 = lo + lane; q2 < hi; q2 += 32) {
                uint32_t q = by_leaf[q2];
                if (keys[q] > mk && atomicExch(&unres[q], 1u) == 0u) next[atomicAdd(&c[1], 1u)] = q;
            }
        }
        grid.sync();
        nf = c[1];
        uint32_t *tmp = front;
        front = next;
        next = tmp;
        ++wave;
    }
    if (gtid == 0) *waves_out += wave;   // running total over the rounds
}

// Dependency lists: the leaves each pending side depends on (its witness if
// reliable; the leaves its search read plus its descent leaf if a writer),
// written as (leaf, side) pairs at the offsets of the evaluation's counts.
__global__ void k_sens(uint32_t m, const uint32_t *keys, NV v, Root root, const D3 *pos, const D3 *nrm,
                       const double *scale, double h_svo, const uint8_t *status, const uint32_t *witness,
                       const uint32_t *dleaf, const uint32_t *off, uint32_t *skeys, uint32_t *svals, double margin,
                       int *err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    if (status[i] == 1) {
        skeys[off[i]] = witness[i];
        svals[off[i]] = i;
        return;
    }
    uint32_t key = keys[i];
    SampleRef q = sample_side(key, pos, nrm, scale, h_svo);
    int e = 0;
    uint32_t c = 0, o = off[i];
    find_reliable_v(v, root, sphere_start_v(v, root, key, q, margin), key, q, [&](uint32_t leaf) {
        skeys[o + c] = leaf;
        svals[o + c] = i;
        ++c;
    }, &e);
    skeys[o + c] = dleaf[i];
    svals[o + c] = i;
    if (e) atomicExch(err, e);
}

__global__ void k_writer_list(uint32_t m, const uint8_t *status, uint32_t *writers, uint32_t *nwri) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m && status[i] == 2) writers[atomicAdd(nwri, 1u)] = i;
}

__global__ void k_segments(uint32_t n, const uint32_t *sorted, uint32_t *seg_lo, uint32_t *seg_hi) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    uint32_t x = sorted[j];
    if (j == 0 || sorted[j - 1] != x) seg_lo[x] = j;
    if (j == n - 1 || sorted[j + 1] != x) seg_hi[x] = j + 1;
}

__global__ void k_segments_clear(uint32_t n, const uint32_t *sorted, uint32_t *seg_lo) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) seg_lo[sorted[j]] = INVALID;
}

__global__ void k_sampling_unmark(uint32_t m, const uint32_t *dleaf, uint32_t *mark) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) mark[dleaf[i]] = INVALID;
}

// Nodes::createNodesForSampling below the descent leaf (Nodes.cpp:285-336):
// the chain of splits is a function of geometry only, since every node below
// the first split is new.  Phase 0 counts splits, phase 1 materializes them.
__global__ void k_sampling_apply(uint32_t m, const uint32_t *keys, const uint8_t *status, const uint32_t *unres,
                                 const uint32_t *dleaf, NV v, Root root, const D3 *pos, const D3 *nrm,
                                 const double *scale, double h_svo, uint32_t *nsplit, const uint32_t *base,
                                 uint32_t start, int phase, int *err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    if (status[i] != 2 || unres[i]) {
        if (phase == 0) nsplit[i] = 0;
        return;
    }
    uint32_t key = keys[i];
    SampleRef q = sample_side(key, pos, nrm, scale, h_svo);
    D3 endp = segment_end(q);
    uint32_t node = dleaf[i];
    D3 mn = v.nmin[node];
    uint32_t d = v.depth[node];
    uint32_t splits = 0;
    uint32_t next = phase ? start + 8 * base[i] : 0;
    for (int guard = 0; guard < 4 * MAX_TREE_DEPTH; ++guard) {
        double sz = size_at(root.size, d);
        double cs = dmul(sz, 0.5);
        if (phase) {
            make_children(v, node, next, cs, key);
        }
        ++splits;
        // findReliableSamplingNode(scope) over the 8 fresh leaves
        bool found = false;
        for (uint32_t c = 0; c < 8 && !found; ++c) {
            D3 cmn = child_coords(mn, cs, c);
            if (!intersect_side(cmn, cs, q)) continue;
            if (leaf_reliable(cmn, cs, q)) found = true;
        }
        if (found) {
            if (phase == 0) nsplit[i] = splits;
            return;
        }
        uint32_t b = best_child(mn, sz, q.p, endp);
        if (b == INVALID) { atomicExch(err, 4); if (phase == 0) nsplit[i] = splits; return; }
        mn = child_coords(mn, cs, b);
        d += 1;
        if (d + 2 >= (uint32_t)MAX_TREE_DEPTH) { atomicExch(err, 6); if (phase == 0) nsplit[i] = splits; return; }
        if (phase) { node = next + b; next += 8; }
    }
    atomicExch(err, 5);
    if (phase == 0) nsplit[i] = splits;
}

// ---------------------------------------------------------------- balance
// Nodes::getNode (Nodes.cpp:145-184) from the root.
__device__ inline uint32_t get_node(const uint32_t *children, const D3 *nmin, const Root &root, const D3 &q,
                                    uint32_t max_depth, uint32_t *out_depth) {
    if (!node_contains(q, root.mn, root.size, 0.0)) { *out_depth = 0; return INVALID; }
    uint32_t node = 0, depth = 0;
    double size = root.size;
    D3 mn = root.mn;
    while (true) {
        if (children[node] == INVALID || depth == max_depth) break;
        double cs = dmul(size, 0.5);
        uint32_t c0 = children[node];
        bool moved = false;
        for (uint32_t c = 0; c < 8; ++c) {
            D3 cmn = child_coords(mn, cs, c);
            if (!node_contains(q, cmn, cs, 0.0)) continue;
            node = c0 + c;
            mn = cmn;
            size = cs;
            ++depth;
            moved = true;
            break;
        }
        if (!moved) break;
    }
    *out_depth = depth;
    return node;
}

// Nodes::createNodesForBalancing (Nodes.cpp:347-395) for a set of leaves: a
// face neighbour more than one level coarser must be split.
__global__ void k_balance_check(uint32_t m, const uint32_t *list, NV v, Root root, uint32_t *split_flag,
                                uint32_t *split_list, uint32_t *split_count, uint32_t *again_list,
                                uint32_t *again_count) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    uint32_t leaf = list[i];
    if (v.children[leaf] != INVALID) return;
    uint32_t d = v.depth[leaf];
    double size = size_at(root.size, d);
    D3 mn = v.nmin[leaf];
    bool marked = false;
    for (uint32_t side = 0; side < 6; ++side) {
        D3 tp = side_center(mn, size, side, dmul(size, 0.5));
        uint32_t nd;
        uint32_t nb = get_node(v.children, v.nmin, root, tp, d, &nd);
        if (nb == INVALID || v.children[nb] != INVALID) continue;
        if (d > nd + 1) {
            marked = true;
            if (atomicExch(&split_flag[nb], 1u) == 0u) split_list[atomicAdd(split_count, 1u)] = nb;
        }
    }
    if (marked) again_list[atomicAdd(again_count, 1u)] = leaf;
}

__global__ void k_balance_split(uint32_t m, const uint32_t *split_list, uint32_t *split_flag, NV v, Root root,
                                uint32_t base, uint32_t *next_list, uint32_t next_off) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    uint32_t node = split_list[i];
    split_flag[node] = 0;
    double cs = size_at(root.size, v.depth[node] + 1u);
    uint32_t b = base + 8 * i;
    make_children(v, node, b, cs, 0);
    for (uint32_t c = 0; c < 8; ++c) next_list[next_off + 8 * i + c] = b + c;
}

// --------------------------------------------------------------- relayout
__global__ void k_level_bounds(uint32_t n, const uint8_t *sorted_depth, uint32_t *level_start) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint8_t d = sorted_depth[i];
    if (i == 0 || sorted_depth[i - 1] != d) level_start[d] = i;
    if (i == n - 1) level_start[d + 1] = n;
}

// Subtree sizes (descendant nodes and leaves), one level bottom-up.
__global__ void k_subtree(uint32_t lo, uint32_t hi, const uint32_t *order, const uint32_t *children,
                          uint32_t *desc, uint32_t *nleaf) {
    uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hi) return;
    uint32_t n = order[i];
    uint32_t c0 = children[n];
    if (c0 == INVALID) { desc[n] = 0; nleaf[n] = 1; return; }
    uint32_t d = 8, l = 0;
    for (uint32_t c = 0; c < 8; ++c) { d += desc[c0 + c]; l += nleaf[c0 + c]; }
    desc[n] = d;
    nleaf[n] = l;
}

// Nodes::computeTargetIndices (Nodes.cpp:536-554) and Leaves::gatherScopes
// (Leaves.cpp:59-80), one level top-down: new index, children block start and
// first leaf index of every node.
__global__ void k_layout(uint32_t lo, uint32_t hi, const uint32_t *order, const uint32_t *children,
                         const uint32_t *desc, const uint32_t *nleaf, uint32_t *new_idx, uint32_t *block,
                         uint32_t *leaf_start) {
    uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hi) return;
    uint32_t n = order[i];
    uint32_t c0 = children[n];
    if (c0 == INVALID) return;
    uint32_t b = block[n], run = b + 8, ls = leaf_start[n];
    for (uint32_t c = 0; c < 8; ++c) {
        uint32_t ch = c0 + c;
        new_idx[ch] = b + c;
        block[ch] = run;
        leaf_start[ch] = ls;
        run += desc[ch];
        ls += nleaf[ch];
    }
}

__global__ void k_scatter_nodes(uint32_t n, NV v, const uint32_t *new_idx, const uint32_t *block,
                                const uint32_t *leaf_start, uint32_t *o_children, uint32_t *o_parents,
                                uint32_t *o_counts, uint8_t *o_depth, D3 *o_min, uint32_t *node_to_leaf,
                                D3 *leaf_min, uint32_t *leaf_node) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t ni = new_idx[i];
    bool leaf = v.children[i] == INVALID;
    o_children[ni] = leaf ? INVALID : block[i];
    uint32_t p = v.parents[i];
    o_parents[ni] = (p == INVALID) ? INVALID : new_idx[p];
    o_counts[ni] = v.cnt[i];
    o_depth[ni] = v.depth[i];
    o_min[ni] = v.nmin[i];
    if (leaf) {
        uint32_t l = leaf_start[i];
        node_to_leaf[ni] = l;
        leaf_min[l] = v.nmin[i];
        leaf_node[l] = ni;
    } else {
        node_to_leaf[ni] = INVALID;
    }
}

__global__ void k_sample_keys(uint32_t n, const uint32_t *container, const uint32_t *new_idx, uint32_t *keys,
                              uint32_t *vals) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    keys[s] = new_idx[container[s]];
    vals[s] = s;
}

__global__ void k_permute_samples(uint32_t n, uint32_t k, const uint32_t *old_of_new, uint32_t *target,
                                  const D3 *pos, const D3 *nrm, const double *scale, const double *conf,
                                  const uint32_t *links, D3 *opos, D3 *onrm, double *oscale, double *oconf,
                                  uint32_t *olinks) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    uint32_t s = old_of_new[t];
    target[s] = t;
    opos[t] = pos[s];
    onrm[t] = nrm[s];
    oscale[t] = scale[s];
    oconf[t] = conf[s];
    for (uint32_t j = 0; j < k; ++j) olinks[(size_t)t * k + j] = links[(size_t)s * k + j];
}

// -------------------------------------------------------------- neighbours
// Leaves::getUnresponsibleEdgeNeighbor (Leaves.cpp:159-180) for every
// (leaf, side); the edge event id is 6 * leaf + side.
__global__ void k_neighbor_events(uint32_t nl, const uint32_t *leaf_node, const D3 *leaf_min,
                                  const uint32_t *children, const D3 *nmin, const uint8_t *depth,
                                  const uint32_t *node_to_leaf, Root root, uint32_t *dst, uint32_t *row_count) {
    uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)nl * 6) return;
    uint32_t l = e / 6, side = e % 6;
    uint32_t node = leaf_node[l];
    uint32_t maxd = depth[node];
    double size = size_at(root.size, maxd);
    D3 tp = side_center(leaf_min[l], size, side, dmul(0.5, size));
    uint32_t nd;
    uint32_t nb = get_node(children, nmin, root, tp, maxd, &nd);
    uint32_t out = INVALID;
    if (nb != INVALID && children[nb] == INVALID && !(nd == maxd && nb < node)) out = node_to_leaf[nb];
    dst[e] = out;
    if (out != INVALID) {
        atomicAdd(&row_count[l], 1u);
        atomicAdd(&row_count[out], 1u);
    }
}

__global__ void k_neighbor_pairs(uint32_t ne, const uint32_t *dst, const uint32_t *slot, uint64_t *keys,
                                 uint32_t *vals) {
    uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    uint32_t o = dst[e];
    if (o == INVALID) return;
    uint32_t l = e / 6;
    uint32_t j = 2 * slot[e];
    keys[j] = ((uint64_t)l << 32) | e;
    vals[j] = o;
    keys[j + 1] = ((uint64_t)o << 32) | e;
    vals[j + 1] = l;
}

__global__ void k_valid_flags(uint32_t n, const uint32_t *dst, uint32_t *flag) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = dst[i] != INVALID ? 1u : 0u;
}

// -------------------------------------------------------------- dual cells
// Frames of the recursive enumeration of DualCells.cpp:49-357.  A frame
// carries the node indices of one call and the path of call ordinals that
// led to it (5 bits per call, 24 calls in two 64-bit words); sorting the
// emitted cells by that path reproduces the reference's emission order.
enum FrameType : uint8_t { F_NODE = 0, F_2X, F_2Y, F_2Z, F_4XY, F_4XZ, F_4YZ, F_V8 };

struct FrameBuf {
    DBuf<uint8_t> type;
    DBuf<uint32_t> nodes;   // 8 per frame
    DBuf<uint64_t> khi, klo;
};

__device__ inline void key_put(uint64_t &hi, uint64_t &lo, uint32_t level, uint32_t ord) {
    if (level < 12) hi |= (uint64_t)ord << (59 - 5 * level);
    else lo |= (uint64_t)ord << (59 - 5 * (level - 12));
}

__device__ inline bool is_leaf_n(const uint32_t *children, uint32_t n) { return children[n] == INVALID; }
__device__ inline uint32_t pickc(const uint32_t *children, uint32_t n, uint32_t c) {
    return children[n] == INVALID ? n : children[n] + c;
}

template <bool WRITE>
__device__ void expand_frame(uint8_t type, const uint32_t *nd, uint64_t khi, uint64_t klo, uint32_t level,
                             const uint32_t *children, const uint32_t *node_to_leaf, uint32_t &fo, uint32_t &co,
                             uint8_t *otype, uint32_t *onodes, uint64_t *okhi, uint64_t *oklo, uint32_t *cells,
                             uint64_t *ckhi, uint64_t *cklo) {
    auto push = [&](uint8_t t, uint32_t ord, const uint32_t *ns, int cnt) {
        // skip calls that return immediately
        if (t == F_NODE) { if (is_leaf_n(children, ns[0])) return; }
        else if (t != F_V8) {
            bool all = true;
            for (int j = 0; j < cnt; ++j) all &= is_leaf_n(children, ns[j]);
            if (all) return;
        }
        if (WRITE) {
            otype[fo] = t;
            for (int j = 0; j < 8; ++j) onodes[8 * (size_t)fo + j] = j < cnt ? ns[j] : INVALID;
            uint64_t h = khi, l = klo;
            key_put(h, l, level, ord);
            okhi[fo] = h;
            oklo[fo] = l;
        }
        ++fo;
    };
    uint32_t ch[8];
    auto faces_yz = [&](const uint32_t *c, uint32_t o) {
        uint32_t a[2];
        a[0] = c[0]; a[1] = c[1]; push(F_2X, o + 0, a, 2);
        a[0] = c[4]; a[1] = c[5]; push(F_2X, o + 1, a, 2);
        a[0] = c[2]; a[1] = c[3]; push(F_2X, o + 2, a, 2);
        a[0] = c[6]; a[1] = c[7]; push(F_2X, o + 3, a, 2);
    };
    auto faces_xz = [&](const uint32_t *c, uint32_t o) {
        uint32_t a[2];
        a[0] = c[2]; a[1] = c[0]; push(F_2Y, o + 0, a, 2);
        a[0] = c[3]; a[1] = c[1]; push(F_2Y, o + 1, a, 2);
        a[0] = c[6]; a[1] = c[4]; push(F_2Y, o + 2, a, 2);
        a[0] = c[7]; a[1] = c[5]; push(F_2Y, o + 3, a, 2);
    };
    auto faces_xy = [&](const uint32_t *c, uint32_t o) {
        uint32_t a[2];
        a[0] = c[0]; a[1] = c[4]; push(F_2Z, o + 0, a, 2);
        a[0] = c[1]; a[1] = c[5]; push(F_2Z, o + 1, a, 2);
        a[0] = c[2]; a[1] = c[6]; push(F_2Z, o + 2, a, 2);
        a[0] = c[3]; a[1] = c[7]; push(F_2Z, o + 3, a, 2);
    };
    auto edges_z = [&](const uint32_t *c, uint32_t o) {
        uint32_t a[4] = {c[0], c[1], c[2], c[3]};
        push(F_4XY, o, a, 4);
        uint32_t b[4] = {c[4], c[5], c[6], c[7]};
        push(F_4XY, o + 1, b, 4);
    };
    auto edges_y = [&](const uint32_t *c, uint32_t o) {
        uint32_t a[4] = {c[0], c[1], c[4], c[5]};
        push(F_4XZ, o, a, 4);
        uint32_t b[4] = {c[2], c[3], c[6], c[7]};
        push(F_4XZ, o + 1, b, 4);
    };
    auto edges_x = [&](const uint32_t *c, uint32_t o) {
        uint32_t a[4] = {c[0], c[2], c[4], c[6]};
        push(F_4YZ, o, a, 4);
        uint32_t b[4] = {c[1], c[3], c[5], c[7]};
        push(F_4YZ, o + 1, b, 4);
    };
    switch (type) {
        case F_NODE: {
            uint32_t c0 = children[nd[0]];
            for (uint32_t i = 0; i < 8; ++i) ch[i] = c0 + i;
            for (uint32_t i = 0; i < 8; ++i) push(F_NODE, i, &ch[i], 1);
            faces_yz(ch, 8); faces_xz(ch, 12); faces_xy(ch, 16);
            edges_z(ch, 20); edges_y(ch, 22); edges_x(ch, 24);
            push(F_V8, 26, ch, 8);
            break;
        }
        case F_2X: {
            uint32_t a = nd[0], b = nd[1];
            const uint32_t t[8] = {pickc(children, a, 1), pickc(children, b, 0), pickc(children, a, 3), pickc(children, b, 2),
                                   pickc(children, a, 5), pickc(children, b, 4), pickc(children, a, 7), pickc(children, b, 6)};
            faces_yz(t, 0); edges_z(t, 4); edges_y(t, 6); push(F_V8, 8, t, 8);
            break;
        }
        case F_2Y: {
            uint32_t a = nd[0], b = nd[1];
            const uint32_t t[8] = {pickc(children, b, 2), pickc(children, b, 3), pickc(children, a, 0), pickc(children, a, 1),
                                   pickc(children, b, 6), pickc(children, b, 7), pickc(children, a, 4), pickc(children, a, 5)};
            faces_xz(t, 0); edges_z(t, 4); edges_x(t, 6); push(F_V8, 8, t, 8);
            break;
        }
        case F_2Z: {
            uint32_t a = nd[0], b = nd[1];
            const uint32_t t[8] = {pickc(children, a, 4), pickc(children, a, 5), pickc(children, a, 6), pickc(children, a, 7),
                                   pickc(children, b, 0), pickc(children, b, 1), pickc(children, b, 2), pickc(children, b, 3)};
            faces_xy(t, 0); edges_y(t, 4); edges_x(t, 6); push(F_V8, 8, t, 8);
            break;
        }
        case F_4XY: {
            const uint32_t t[8] = {pickc(children, nd[0], 3), pickc(children, nd[1], 2), pickc(children, nd[2], 1), pickc(children, nd[3], 0),
                                   pickc(children, nd[0], 7), pickc(children, nd[1], 6), pickc(children, nd[2], 5), pickc(children, nd[3], 4)};
            edges_z(t, 0); push(F_V8, 2, t, 8);
            break;
        }
        case F_4XZ: {
            const uint32_t t[8] = {pickc(children, nd[0], 5), pickc(children, nd[1], 4), pickc(children, nd[0], 7), pickc(children, nd[1], 6),
                                   pickc(children, nd[2], 1), pickc(children, nd[3], 0), pickc(children, nd[2], 3), pickc(children, nd[3], 2)};
            edges_y(t, 0); push(F_V8, 2, t, 8);
            break;
        }
        case F_4YZ: {
            const uint32_t t[8] = {pickc(children, nd[0], 6), pickc(children, nd[0], 7), pickc(children, nd[1], 4), pickc(children, nd[1], 5),
                                   pickc(children, nd[2], 2), pickc(children, nd[2], 3), pickc(children, nd[3], 0), pickc(children, nd[3], 1)};
            edges_x(t, 0); push(F_V8, 2, t, 8);
            break;
        }
        default: {   // F_V8, DualCells.cpp:316-357
            bool only = true;
            for (int i = 0; i < 8; ++i) only &= is_leaf_n(children, nd[i]);
            if (only) {
                if (WRITE) {
                    for (int i = 0; i < 8; ++i) cells[8 * (size_t)co + i] = node_to_leaf[nd[i]];
                    ckhi[co] = khi;
                    cklo[co] = klo;
                }
                ++co;
                return;
            }
            uint32_t t[8];
            for (int i = 0; i < 8; ++i) t[i] = pickc(children, nd[i], 7 - i);
            push(F_V8, 0, t, 8);
        }
    }
}

__global__ void k_frames_count(uint32_t m, const uint8_t *type, const uint32_t *nodes, uint32_t level,
                               const uint32_t *children, const uint32_t *node_to_leaf, uint32_t *nf, uint32_t *nc) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    uint32_t fo = 0, co = 0;
    expand_frame<false>(type[i], nodes + 8 * (size_t)i, 0, 0, level, children, node_to_leaf, fo, co, nullptr, nullptr,
                        nullptr, nullptr, nullptr, nullptr, nullptr);
    nf[i] = fo;
    nc[i] = co;
}

__global__ void k_frames_write(uint32_t m, const uint8_t *type, const uint32_t *nodes, const uint64_t *khi,
                               const uint64_t *klo, uint32_t level, const uint32_t *children,
                               const uint32_t *node_to_leaf, const uint32_t *foff, const uint32_t *coff,
                               uint32_t cbase, uint8_t *otype, uint32_t *onodes, uint64_t *okhi, uint64_t *oklo,
                               uint32_t *cells, uint64_t *ckhi, uint64_t *cklo) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    uint32_t fo = foff[i], co = cbase + coff[i];
    expand_frame<true>(type[i], nodes + 8 * (size_t)i, khi[i], klo[i], level, children, node_to_leaf, fo, co, otype,
                       onodes, okhi, oklo, cells, ckhi, cklo);
}

__global__ void k_gather_cells(uint32_t nc, const uint32_t *order, const uint32_t *in, uint32_t *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    uint32_t s = order[i];
    for (int j = 0; j < 8; ++j) out[8 * (size_t)i + j] = in[8 * (size_t)s + j];
}

__global__ void k_gather_u64(uint32_t n, const uint32_t *order, const uint64_t *in, uint64_t *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[order[i]];
}

__global__ void k_map_order(uint32_t n, const uint32_t *order, const uint32_t *new_idx, uint32_t *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = new_idx[order[i]];
}

__global__ void k_iota(uint32_t n, uint32_t *a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

// ------------------------------------------------------------- cub helpers
template <class T>
void exclusive_scan(const T *in, T *out, uint32_t n, cudaStream_t st) {
    size_t tmp = 0;
    TSR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, st));
    DBuf<uint8_t> t(tmp, st);
    TSR_CUDA(cub::DeviceScan::ExclusiveSum(t.p, tmp, in, out, n, st));
}

template <class K, class V>
void sort_pairs(const K *kin, K *kout, const V *vin, V *vout, uint32_t n, cudaStream_t st, int end_bit = sizeof(K) * 8) {
    size_t tmp = 0;
    TSR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kin, kout, vin, vout, n, 0, end_bit, st));
    DBuf<uint8_t> t(tmp, st);
    TSR_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, kin, kout, vin, vout, n, 0, end_bit, st));
}

template <class T, class F>
uint32_t select_flagged(const T *in, const F *flags, T *out, uint32_t n, cudaStream_t st) {
    DBuf<uint32_t> cnt(1, st);
    size_t tmp = 0;
    TSR_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, in, flags, out, cnt.p, n, st));
    DBuf<uint8_t> t(tmp, st);
    TSR_CUDA(cub::DeviceSelect::Flagged(t.p, tmp, in, flags, out, cnt.p, n, st));
    return read_scalar(cnt.p, st);
}

__global__ void k_count_writers(uint32_t m, const uint8_t *status, const uint32_t *unres, unsigned long long *w) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m && status[i] == 2 && !unres[i]) atomicAdd(w, 1ull);
}

__global__ void k_keys_init(uint32_t m, uint32_t *keys) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) keys[i] = i + 1;
}

struct EventTimer {
    cudaEvent_t a{}, b{};
    cudaStream_t st;
    explicit EventTimer(cudaStream_t s) : st(s) {
        TSR_CUDA(cudaEventCreate(&a));
        TSR_CUDA(cudaEventCreate(&b));
        TSR_CUDA(cudaEventRecord(a, st));
    }
    float lap() {
        TSR_CUDA(cudaEventRecord(b, st));
        TSR_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        TSR_CUDA(cudaEventElapsedTime(&ms, a, b));
        std::swap(a, b);
        return ms;
    }
    ~EventTimer() { cudaEventDestroy(a); cudaEventDestroy(b); }
};

}  // namespace

// ====================================================================== API
namespace {

// ---- Tree::eraseSamples (Tree.cpp:50-53, Nodes.cpp:644-671) with
// Samples::compact for the tree's own copy of the samples.
// offsets[i] = erased samples before i (tree order), offsets[n] = total.
__global__ void k_erase_nodes(uint32_t nn, const uint32_t *offsets, uint32_t *counts, uint32_t *starts) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const uint32_t start = starts[i], end = start + counts[i];
    counts[i] -= offsets[end] - offsets[start];
    starts[i] = start - offsets[start];
}

__global__ void k_compact_samples(uint32_t n, uint32_t k, const uint8_t *inliers, const uint32_t *offsets,
                                  const D3 *pos, const D3 *nrm, const double *scale, const double *conf,
                                  const uint32_t *links, D3 *o_pos, D3 *o_nrm, double *o_scale, double *o_conf,
                                  uint32_t *o_links) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !inliers[i]) return;
    const uint32_t j = i - offsets[i];
    o_pos[j] = pos[i];
    o_nrm[j] = nrm[i];
    o_scale[j] = scale[i];
    o_conf[j] = conf[i];
    for (uint32_t c = 0; c < k; ++c) o_links[(size_t)j * k + c] = links[(size_t)i * k + c];
}

// target[input index] = tree-order index, INVALID once erased
__global__ void k_erase_targets(uint32_t n_in, const uint8_t *inliers, const uint32_t *offsets, uint32_t *target) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_in) return;
    const uint32_t t = target[i];
    if (t == INVALID) return;
    target[i] = inliers[t] ? t - offsets[t] : INVALID;
}

__global__ void k_outlier_flags(uint32_t n, const uint8_t *inliers, uint32_t *flags) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= n) flags[i] = (i < n && !inliers[i]) ? 1u : 0u;
}

}  // namespace

void erase_tree_samples(tsr_tree &t, const uint8_t *inliers) {
    cudaStream_t st = t.stream;
    const uint32_t n = t.n_samples, k = t.k, nn = t.n_nodes;
    DBuf<uint32_t> flags(n + 1, st), offsets(n + 1, st);
    k_outlier_flags<<<grid_for(n + 1, BLK), BLK, 0, st>>>(n, inliers, flags.p); ::tsr::note_launch();
    exclusive_scan(flags.p, offsets.p, n + 1, st);
    const uint32_t erased = read_scalar(offsets.p + n, st);
    k_erase_nodes<<<grid_for(nn, BLK), BLK, 0, st>>>(nn, offsets.p, t.counts.p, t.starts.p); ::tsr::note_launch();
    const uint32_t m = n - erased;
    DBuf<D3> pos(m, st), nrm(m, st);
    DBuf<double> scale(m, st), conf(m, st);
    DBuf<uint32_t> links((size_t)m * k, st);
    k_compact_samples<<<grid_for(n, BLK), BLK, 0, st>>>(n, k, inliers, offsets.p, t.pos.p, t.nrm.p, t.scale.p, t.conf.p,
                                                        t.links.p, pos.p, nrm.p, scale.p, conf.p, links.p);
    ::tsr::note_launch();
    k_erase_targets<<<grid_for(t.target.n, BLK), BLK, 0, st>>>((uint32_t)t.target.n, inliers, offsets.p,
                                                               t.target.p); ::tsr::note_launch();
    t.pos = std::move(pos);
    t.nrm = std::move(nrm);
    t.scale = std::move(scale);
    t.conf = std::move(conf);
    t.links = std::move(links);
    t.n_samples = m;
    TSR_CUDA(cudaGetLastError());
}

void build_tree(tsr_tree &t, const tsr_samples_view &sv, bool on_device) {
    cudaStream_t st = t.stream;
    const uint32_t n = sv.count, k = sv.cams_per_sample;
    const double h_svo = t.params.max_relative_sampling_distance;
    t.n_samples = n;
    t.k = k;
    // working set of the build: samples twice (input and tree order), the
    // sampling rounds' per-side buffers, the node store and its relayout
    reserve_pool((size_t)n * (700 + 8 * k) + (64u << 20), st);
    EventTimer timer(st);

    // ---- upload samples (FP64, Real = double)
    DBuf<D3> pos(n, st), nrm(n, st);
    DBuf<double> scale(n, st), conf(n, st);
    DBuf<uint32_t> links((size_t)n * k, st);
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    TSR_CUDA(cudaMemcpyAsync(pos.p, sv.positions, (size_t)n * 24, kind, st));
    TSR_CUDA(cudaMemcpyAsync(nrm.p, sv.normals, (size_t)n * 24, kind, st));
    TSR_CUDA(cudaMemcpyAsync(scale.p, sv.scales, (size_t)n * 8, kind, st));
    TSR_CUDA(cudaMemcpyAsync(conf.p, sv.confidences, (size_t)n * 8, kind, st));
    TSR_CUDA(cudaMemcpyAsync(links.p, sv.camera_links, (size_t)n * k * 4, kind, st));

    // ---- root scope (Tree.cpp:70-101)
    {
        unsigned g = std::min<unsigned>(grid_for(n, BLK), 1024);
        DBuf<double> part((size_t)g * 6, st);
        k_bounds<<<g, BLK, 0, st>>>(n, pos.p, scale.p, h_svo, part.p); ::tsr::note_launch();
        std::vector<double> h((size_t)g * 6);
        TSR_CUDA(cudaMemcpyAsync(h.data(), part.p, h.size() * 8, cudaMemcpyDeviceToHost, st));
        TSR_CUDA(cudaStreamSynchronize(st));
        double lo[3] = {REAL_MAX, REAL_MAX, REAL_MAX}, hi[3] = {-REAL_MAX, -REAL_MAX, -REAL_MAX};
        for (unsigned b = 0; b < g; ++b)
            for (int j = 0; j < 3; ++j) {
                lo[j] = std::min(lo[j], h[b * 6 + j]);
                hi[j] = std::max(hi[j], h[b * 6 + 3 + j]);
            }
        for (int j = 0; j < 3; ++j) {
            t.aabb[j] = lo[j];
            t.aabb[3 + j] = hi[j];
        }
        root_from_aabb(t);
    }
    Root root{D3{t.root_min[0], t.root_min[1], t.root_min[2]}, t.root_size};

    // ---- containment, level by level (Nodes.cpp:196-212)
    NodeStore S;
    S.st = st;
    S.ensure(std::max<uint64_t>(1024, (uint64_t)n * 4));
    {
        uint32_t init_children = INVALID, zero = 0;
        uint8_t d0 = 0;
        TSR_CUDA(cudaMemcpyAsync(S.children.p, &init_children, 4, cudaMemcpyHostToDevice, st));
        TSR_CUDA(cudaMemcpyAsync(S.parents.p, &init_children, 4, cudaMemcpyHostToDevice, st));
        TSR_CUDA(cudaMemcpyAsync(S.cc.p, &zero, 4, cudaMemcpyHostToDevice, st));
        TSR_CUDA(cudaMemcpyAsync(S.cnt.p, &zero, 4, cudaMemcpyHostToDevice, st));
        TSR_CUDA(cudaMemcpyAsync(S.depth.p, &d0, 1, cudaMemcpyHostToDevice, st));
        TSR_CUDA(cudaMemcpyAsync(S.nmin.p, &root.mn, 24, cudaMemcpyHostToDevice, st));
        TSR_CUDA(cudaStreamSynchronize(st));
        S.count = 1;
    }
    DBuf<uint32_t> cur(n, st), container(n, st);
    cur.zero();
    container.fill_bytes(0xFF);
    uint32_t lvl_lo = 0, lvl_hi = 1;
    for (uint32_t level = 0;; ++level) {
        if (level >= (uint32_t)MAX_TREE_DEPTH - 2) fail(TSR_ERR_OVERFLOW_U32, "tree deeper than supported");
        double size_l = size_at(root.size, level);
        uint32_t width = lvl_hi - lvl_lo;
        DBuf<uint32_t> need((size_t)S.cap + 1, st);
        TSR_CUDA(cudaMemsetAsync(need.p + lvl_lo, 0, ((size_t)width + 1) * 4, st));
        k_contain_mark<<<grid_for(n, BLK), BLK, 0, st>>>(n, scale.p, h_svo, size_l, cur.p, container.p, need.p, S.cnt.p); ::tsr::note_launch();
        DBuf<uint32_t> rank(width + 1, st);
        TSR_CUDA(cudaMemsetAsync(rank.p + width, 0, 4, st));
        exclusive_scan(need.p + lvl_lo, rank.p, width + 1, st);   // last entry = total
        uint32_t nneed = read_scalar(rank.p + width, st);
        if (nneed == 0) break;
        uint32_t base = S.count;
        // grow before allocating; need[] was sized to the old capacity
        S.ensure((uint64_t)S.count + 8ull * nneed);
        NV v = view(S);
        k_contain_alloc<<<grid_for(width, BLK), BLK, 0, st>>>(lvl_lo, lvl_hi, need.p, rank.p, v, base,
                                                               size_at(root.size, level + 1)); ::tsr::note_launch();
        k_contain_step<<<grid_for(n, BLK), BLK, 0, st>>>(n, pos.p, size_at(root.size, level + 1), cur.p, container.p, v); ::tsr::note_launch();
        S.count += 8 * nneed;
        lvl_lo = base;
        lvl_hi = S.count;
    }
    t.stage_ms[0] = timer.lap();

    // ---- sampling nodes, order-exact rounds (Nodes.cpp:213-219, 271-337)
    DBuf<int> derr(1, st);
    derr.zero();
    {
        if ((uint64_t)n * 2 >= INVALID) fail(TSR_ERR_OVERFLOW_U32, "too many samples");
        uint32_t m = 2 * n;
        DBuf<uint32_t> keys(m, st), keys2(m, st);
        k_keys_init<<<grid_for(m, BLK), BLK, 0, st>>>(m, keys.p); ::tsr::note_launch();
        DBuf<uint32_t> mark, seg_lo, seg_hi;
        mark.alloc(S.cap, st);
        mark.fill_bytes(0xFF);
        seg_lo.alloc(S.cap, st);
        seg_lo.fill_bytes(0xFF);
        seg_hi.alloc(S.cap, st);
        DBuf<unsigned long long> wcount(1, st);
        wcount.zero();
        DBuf<uint32_t> counters(4, st), waves_total(1, st);
        waves_total.zero();
        uint32_t rounds = 0, waves = 0;
        const double margin = 1e-12 * (std::max(std::max(std::fabs(root.mn.x), std::fabs(root.mn.y)),
                                                 std::fabs(root.mn.z)) + 2.0 * root.size);
        float eval_ms = 0, resolve_ms = 0;
        struct Events {   // destroyed on every exit, a failed round's included
            cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
            ~Events() { for (cudaEvent_t x : e) if (x) cudaEventDestroy(x); }
        } ev;
        for (cudaEvent_t &x : ev.e) TSR_CUDA(cudaEventCreate(&x));
        cudaEvent_t e0 = ev.e[0], e1 = ev.e[1], e2 = ev.e[2];
        unsigned coop_grid = 1;
        {
            int dev = 0, sms = 0, per_sm = 0;
            TSR_CUDA(cudaGetDevice(&dev));
            TSR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            TSR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_waves_coop, 256, 0));
            coop_grid = (unsigned)(sms * (per_sm > 0 ? per_sm : 1));
        }
        const uint32_t max_waves_used = limit_sampling_waves();
        while (m > 0) {
            if (++rounds > limit_rounds()) fail(TSR_ERR_TIMEOUT, "sampling rounds did not converge");
            NV v = view(S);
            DBuf<uint8_t> status(m, st);
            DBuf<uint32_t> unres(m, st), witness(m, st), dleaf(m, st);
            DBuf<uint32_t> scnt(m + 1, st), soff(m + 1, st), writers(m, st);
            unres.zero();
            TSR_CUDA(cudaMemsetAsync(scnt.p + m, 0, 4, st));
            TSR_CUDA(cudaEventRecord(e0, st));
            k_sampling_eval<<<grid_for(m, 128), 128, 0, st>>>(m, keys.p, v, root, pos.p, nrm.p, scale.p, h_svo,
                                                             status.p, witness.p, dleaf.p, scnt.p, margin, derr.p,
                                                             rounds == 1 ? 1 : 0);
            ::tsr::note_launch();
            TSR_CUDA(cudaEventRecord(e1, st));
            // dependency index (leaf -> sides) and the writer list
            exclusive_scan(scnt.p, soff.p, m + 1, st);
            counters.zero();
            k_writer_list<<<grid_for(m, BLK), BLK, 0, st>>>(m, status.p, writers.p, counters.p); ::tsr::note_launch();
            uint32_t cnt[2];
            TSR_CUDA(cudaMemcpyAsync(&cnt[0], soff.p + m, 4, cudaMemcpyDeviceToHost, st));
            TSR_CUDA(cudaMemcpyAsync(&cnt[1], counters.p, 4, cudaMemcpyDeviceToHost, st));
            TSR_CUDA(cudaStreamSynchronize(st));
            const uint32_t nsens = cnt[0], nwri = cnt[1];
            DBuf<uint32_t> skeys(nsens, st), svals(nsens, st), ssorted(nsens, st), by_leaf(nsens, st);
            if (nsens) {
                k_sens<<<grid_for(m, 128), 128, 0, st>>>(m, keys.p, v, root, pos.p, nrm.p, scale.p, h_svo, status.p,
                                                        witness.p, dleaf.p, soff.p, skeys.p, svals.p, margin,
                                                        derr.p); ::tsr::note_launch();
                int leaf_bits = 1;   // node indices stay below the node count
                while (leaf_bits < 32 && (1ull << leaf_bits) < (uint64_t)S.count) ++leaf_bits;
                sort_pairs(skeys.p, ssorted.p, svals.p, by_leaf.p, nsens, st, leaf_bits);
                k_segments<<<grid_for(nsens, BLK), BLK, 0, st>>>(nsens, ssorted.p, seg_lo.p, seg_hi.p); ::tsr::note_launch();
            }
            // waves: the frontier starts with every writer
            DBuf<uint32_t> front(m, st), next(m, st), touched(m, st);
            uint32_t nf = nwri;
            if (nwri) {
                TSR_CUDA(cudaMemcpyAsync(front.p, writers.p, (size_t)nwri * 4, cudaMemcpyDeviceToDevice, st));
                DBuf<uint32_t> ctr(4, st);
                ctr.zero();
                uint32_t max_waves = max_waves_used;
                uint32_t *fp = front.p, *np = next.p, *tp = touched.p, *kp = keys.p, *dp = dleaf.p, *mp = mark.p;
                uint32_t *slp = seg_lo.p, *shp = seg_hi.p, *blp = by_leaf.p, *up = unres.p, *cp = ctr.p;
                uint32_t *wp = waves_total.p;
                int *ep = derr.p;
                void *args[] = {&nf, &fp, &np, &kp, &dp, &mp, &tp, &slp, &shp, &blp, &up, &cp, &max_waves, &wp, &ep};
                TSR_CUDA(cudaLaunchCooperativeKernel((const void *)k_waves_coop, coop_grid, 256, args, 0, st));
                ::tsr::note_launch();
            }
            TSR_CUDA(cudaEventRecord(e2, st));
            if (nsens) k_segments_clear<<<grid_for(nsens, BLK), BLK, 0, st>>>(nsens, ssorted.p, seg_lo.p); ::tsr::note_launch();
            k_count_writers<<<grid_for(m, BLK), BLK, 0, st>>>(m, status.p, unres.p, wcount.p); ::tsr::note_launch();
            // commit resolved writers
            DBuf<uint32_t> nsplit(m + 1, st), base(m + 1, st);
            TSR_CUDA(cudaMemsetAsync(nsplit.p + m, 0, 4, st));
            k_sampling_apply<<<grid_for(m, 128), 128, 0, st>>>(m, keys.p, status.p, unres.p, dleaf.p, v, root, pos.p,
                                                              nrm.p, scale.p, h_svo, nsplit.p, nullptr, 0, 0, derr.p); ::tsr::note_launch();
            exclusive_scan(nsplit.p, base.p, m + 1, st);
            // the split total, and whether the waves ran out of their bound:
            // then the round's conflicts are unresolved and nothing is applied
            uint32_t total = 0;
            int round_err = 0;
            TSR_CUDA(cudaMemcpyAsync(&total, base.p + m, 4, cudaMemcpyDeviceToHost, st));
            TSR_CUDA(cudaMemcpyAsync(&round_err, derr.p, 4, cudaMemcpyDeviceToHost, st));
            TSR_CUDA(cudaStreamSynchronize(st));
            if (round_err == 7)
                fail(TSR_ERR_TIMEOUT, "sampling conflict resolution exceeded its bound of " +
                                          std::to_string(max_waves_used) + " waves in round " + std::to_string(rounds));
            float a = 0, b = 0;
            TSR_CUDA(cudaEventElapsedTime(&a, e0, e1));
            TSR_CUDA(cudaEventElapsedTime(&b, e1, e2));
            eval_ms += a;
            resolve_ms += b;
            if (total) {
                uint32_t old_cap = S.cap;
                S.ensure((uint64_t)S.count + 8ull * total);
                if (S.cap != old_cap) {
                    for (DBuf<uint32_t> *arr : {&mark, &seg_lo}) {
                        DBuf<uint32_t> nm(S.cap, st);
                        nm.fill_bytes(0xFF);
                        TSR_CUDA(cudaMemcpyAsync(nm.p, arr->p, (size_t)old_cap * 4, cudaMemcpyDeviceToDevice, st));
                        *arr = std::move(nm);
                    }
                    seg_hi.alloc(S.cap, st);
                }
                v = view(S);
                k_sampling_apply<<<grid_for(m, 128), 128, 0, st>>>(m, keys.p, status.p, unres.p, dleaf.p, v, root,
                                                                  pos.p, nrm.p, scale.p, h_svo, nsplit.p, base.p,
                                                                  S.count, 1, derr.p); ::tsr::note_launch();
                S.count += 8 * total;
            }
            k_sampling_unmark<<<grid_for(m, BLK), BLK, 0, st>>>(m, dleaf.p, mark.p); ::tsr::note_launch();
            // next round: unresolved sides only
            uint32_t m2 = select_flagged(keys.p, unres.p, keys2.p, m, st);
            std::swap(keys, keys2);
            m = m2;
        }
        t.sampling_rounds = rounds;
        t.stage_ms[6] = eval_ms;
        t.stage_ms[7] = resolve_ms;
        t.sampling_writers = read_scalar(wcount.p, st);
        waves = read_scalar(waves_total.p, st);
        t.sampling_waves = waves;
        // device-side failures of any round are reported once the rounds end
        // (every index a failing round leaves behind is still in range)
        int e = read_scalar(derr.p, st);
        if (e == 7) fail(TSR_ERR_TIMEOUT, "sampling conflict resolution did not converge");
        if (e) fail(TSR_ERR_DEVICE_ASSERT, "sampling traversal invariant broken (code " + std::to_string(e) + ")");
    }
    t.stage_ms[1] = timer.lap();

    // ---- balancing rounds (Nodes.cpp:339-395)
    {
        DBuf<uint32_t> list(S.count, st);
        k_iota<<<grid_for(S.count, BLK), BLK, 0, st>>>(S.count, list.p); ::tsr::note_launch();
        uint32_t m = S.count;
        DBuf<uint32_t> split_flag(S.cap, st);
        split_flag.zero();
        DBuf<uint32_t> counters(2, st);
        for (int round = 0;; ++round) {
            if ((uint32_t)round > limit_rounds()) fail(TSR_ERR_TIMEOUT, "balancing did not converge");
            NV v = view(S);
            DBuf<uint32_t> split_list(m * 6 < S.count ? m * 6 : S.count, st), again(m, st);
            counters.zero();
            k_balance_check<<<grid_for(m, 128), 128, 0, st>>>(m, list.p, v, root, split_flag.p, split_list.p,
                                                             counters.p, again.p, counters.p + 1); ::tsr::note_launch();
            uint32_t cnt[2];
            TSR_CUDA(cudaMemcpyAsync(cnt, counters.p, 8, cudaMemcpyDeviceToHost, st));
            TSR_CUDA(cudaStreamSynchronize(st));
            if (cnt[0] == 0) break;
            uint32_t old_cap = S.cap;
            S.ensure((uint64_t)S.count + 8ull * cnt[0]);
            if (S.cap != old_cap) {
                DBuf<uint32_t> nf(S.cap, st);
                nf.zero();
                TSR_CUDA(cudaMemcpyAsync(nf.p, split_flag.p, (size_t)old_cap * 4, cudaMemcpyDeviceToDevice, st));
                split_flag = std::move(nf);
            }
            v = view(S);
            uint32_t m2 = 8 * cnt[0] + cnt[1];
            DBuf<uint32_t> next(m2, st);
            k_balance_split<<<grid_for(cnt[0], BLK), BLK, 0, st>>>(cnt[0], split_list.p, split_flag.p, v, root, S.count,
                                                                  next.p, 0); ::tsr::note_launch();
            if (cnt[1]) TSR_CUDA(cudaMemcpyAsync(next.p + 8 * cnt[0], again.p, (size_t)cnt[1] * 4, cudaMemcpyDeviceToDevice, st));
            S.count += 8 * cnt[0];
            list = std::move(next);
            m = m2;
        }
    }
    t.stage_ms[2] = timer.lap();

    // ---- relayout (Nodes.cpp:519-592) + leaves (Leaves.cpp:44-80)
    const uint32_t nn = S.count;
    t.n_nodes = nn;
    NV v = view(S);
    DBuf<uint32_t> new_idx(nn, st), block(nn, st), leaf_start(nn, st);
    uint32_t max_depth = 0;
    {
        DBuf<uint32_t> iota(nn, st), order(nn, st);
        DBuf<uint8_t> sdepth(nn, st);
        k_iota<<<grid_for(nn, BLK), BLK, 0, st>>>(nn, iota.p); ::tsr::note_launch();
        sort_pairs(S.depth.p, sdepth.p, iota.p, order.p, nn, st, 8);
        uint8_t dmax = read_scalar(sdepth.p + nn - 1, st);
        max_depth = dmax;
        DBuf<uint32_t> lstart(dmax + 2, st);
        k_level_bounds<<<grid_for(nn, BLK), BLK, 0, st>>>(nn, sdepth.p, lstart.p); ::tsr::note_launch();
        std::vector<uint32_t> ls(dmax + 2);
        TSR_CUDA(cudaMemcpyAsync(ls.data(), lstart.p, (dmax + 2) * 4, cudaMemcpyDeviceToHost, st));
        TSR_CUDA(cudaStreamSynchronize(st));
        DBuf<uint32_t> desc(nn, st), nleaf(nn, st);
        for (int d = dmax; d >= 0; --d)
            k_subtree<<<grid_for(ls[d + 1] - ls[d], BLK), BLK, 0, st>>>(ls[d], ls[d + 1], order.p, S.children.p, desc.p, nleaf.p); ::tsr::note_launch();
        uint32_t zero = 0, one = 1;
        TSR_CUDA(cudaMemcpyAsync(new_idx.p, &zero, 4, cudaMemcpyHostToDevice, st));
        TSR_CUDA(cudaMemcpyAsync(block.p, &one, 4, cudaMemcpyHostToDevice, st));
        TSR_CUDA(cudaMemcpyAsync(leaf_start.p, &zero, 4, cudaMemcpyHostToDevice, st));
        for (uint32_t d = 0; d <= dmax; ++d)
            k_layout<<<grid_for(ls[d + 1] - ls[d], BLK), BLK, 0, st>>>(ls[d], ls[d + 1], order.p, S.children.p, desc.p,
                                                                     nleaf.p, new_idx.p, block.p, leaf_start.p); ::tsr::note_launch();
        t.n_leaves = read_scalar(nleaf.p + 0, st);
        // level lists in the final numbering, for bottom-up passes
        t.level_start.assign(ls.begin(), ls.end());
        t.level_order.alloc(nn, st);
        k_map_order<<<grid_for(nn, BLK), BLK, 0, st>>>(nn, order.p, new_idx.p, t.level_order.p); ::tsr::note_launch();
        TSR_CUDA(cudaStreamSynchronize(st));
    }
    t.max_depth = max_depth;
    t.children.alloc(nn, st); t.parents.alloc(nn, st); t.counts.alloc(nn, st); t.starts.alloc(nn, st);
    t.depth.alloc(nn, st); t.nmin.alloc(nn, st); t.node_to_leaf.alloc(nn, st);
    t.leaf_min.alloc(t.n_leaves, st); t.leaf_node.alloc(t.n_leaves, st);
    k_scatter_nodes<<<grid_for(nn, BLK), BLK, 0, st>>>(nn, v, new_idx.p, block.p, leaf_start.p, t.children.p, t.parents.p,
                                                      t.counts.p, t.depth.p, t.nmin.p, t.node_to_leaf.p, t.leaf_min.p,
                                                      t.leaf_node.p); ::tsr::note_launch();
    exclusive_scan(t.counts.p, t.starts.p, nn, st);

    // ---- sample reorder (Nodes.cpp:594-636, Samples.cpp:825-835)
    {
        DBuf<uint32_t> keys(n, st), vals(n, st), skeys(n, st), old_of_new(n, st);
        k_sample_keys<<<grid_for(n, BLK), BLK, 0, st>>>(n, container.p, new_idx.p, keys.p, vals.p); ::tsr::note_launch();
        sort_pairs(keys.p, skeys.p, vals.p, old_of_new.p, n, st);
        t.target.alloc(n, st); t.pos.alloc(n, st); t.nrm.alloc(n, st); t.scale.alloc(n, st); t.conf.alloc(n, st);
        t.links.alloc((size_t)n * k, st);
        k_permute_samples<<<grid_for(n, BLK), BLK, 0, st>>>(n, k, old_of_new.p, t.target.p, pos.p, nrm.p, scale.p, conf.p,
                                                           links.p, t.pos.p, t.nrm.p, t.scale.p, t.conf.p, t.links.p); ::tsr::note_launch();
    }
    t.stage_ms[3] = timer.lap();

    // ---- leaf neighbours (Leaves.cpp:82-157)
    {
        uint32_t nl = t.n_leaves;
        uint64_t ne64 = (uint64_t)nl * 6;
        if (ne64 >= INVALID) fail(TSR_ERR_OVERFLOW_U32, "too many leaves for the neighbour graph");
        uint32_t ne = (uint32_t)ne64;
        DBuf<uint32_t> dst(ne, st), rowc(nl + 1, st), flag(ne + 1, st), slot(ne + 1, st);
        rowc.zero();
        k_neighbor_events<<<grid_for(ne, 128), 128, 0, st>>>(nl, t.leaf_node.p, t.leaf_min.p, t.children.p, t.nmin.p,
                                                            t.depth.p, t.node_to_leaf.p, root, dst.p, rowc.p); ::tsr::note_launch();
        t.nb_off.alloc(nl + 1, st);
        exclusive_scan(rowc.p, t.nb_off.p, nl + 1, st);
        k_valid_flags<<<grid_for(ne, BLK), BLK, 0, st>>>(ne, dst.p, flag.p); ::tsr::note_launch();
        TSR_CUDA(cudaMemsetAsync(flag.p + ne, 0, 4, st));
        exclusive_scan(flag.p, slot.p, ne + 1, st);
        uint32_t nev = read_scalar(slot.p + ne, st);
        uint64_t nent = 2ull * nev;
        t.n_nb = nent;
        DBuf<uint64_t> keys(nent, st), skeys(nent, st);
        DBuf<uint32_t> vals(nent, st);
        t.nbs.alloc(nent, st);
        k_neighbor_pairs<<<grid_for(ne, BLK), BLK, 0, st>>>(ne, dst.p, slot.p, keys.p, vals.p); ::tsr::note_launch();
        if (nent) sort_pairs(keys.p, skeys.p, vals.p, t.nbs.p, (uint32_t)nent, st);
    }
    t.stage_ms[4] = timer.lap();

    // ---- dual cells (DualCells.cpp:21-31, 49-357)
    {
        if (max_depth + 1 > 24) fail(TSR_ERR_OVERFLOW_U32, "tree too deep for the dual-cell path keys");
        DBuf<uint32_t> all_cells;
        DBuf<uint64_t> all_hi, all_lo;
        uint32_t ncells = 0, ccap = 0;
        FrameBuf cur_f;
        uint32_t nf = 0;
        if (t.n_nodes > 1) {
            cur_f.type.alloc(1, st); cur_f.nodes.alloc(8, st); cur_f.khi.alloc(1, st); cur_f.klo.alloc(1, st);
            uint8_t ty = F_NODE;
            uint32_t nd8[8] = {0, INVALID, INVALID, INVALID, INVALID, INVALID, INVALID, INVALID};
            uint64_t z = 0;
            TSR_CUDA(cudaMemcpyAsync(cur_f.type.p, &ty, 1, cudaMemcpyHostToDevice, st));
            TSR_CUDA(cudaMemcpyAsync(cur_f.nodes.p, nd8, 32, cudaMemcpyHostToDevice, st));
            TSR_CUDA(cudaMemcpyAsync(cur_f.khi.p, &z, 8, cudaMemcpyHostToDevice, st));
            TSR_CUDA(cudaMemcpyAsync(cur_f.klo.p, &z, 8, cudaMemcpyHostToDevice, st));
            TSR_CUDA(cudaStreamSynchronize(st));
            nf = 1;
        }
        for (uint32_t level = 0; nf > 0; ++level) {
            if (level >= 24) fail(TSR_ERR_OVERFLOW_U32, "dual-cell recursion deeper than supported");
            DBuf<uint32_t> cf(nf + 1, st), cc(nf + 1, st), of(nf + 1, st), oc(nf + 1, st);
            TSR_CUDA(cudaMemsetAsync(cf.p + nf, 0, 4, st));
            TSR_CUDA(cudaMemsetAsync(cc.p + nf, 0, 4, st));
            k_frames_count<<<grid_for(nf, 128), 128, 0, st>>>(nf, cur_f.type.p, cur_f.nodes.p, level, t.children.p,
                                                             t.node_to_leaf.p, cf.p, cc.p); ::tsr::note_launch();
            exclusive_scan(cf.p, of.p, nf + 1, st);
            exclusive_scan(cc.p, oc.p, nf + 1, st);
            uint32_t tot[2];
            TSR_CUDA(cudaMemcpyAsync(&tot[0], of.p + nf, 4, cudaMemcpyDeviceToHost, st));
            TSR_CUDA(cudaMemcpyAsync(&tot[1], oc.p + nf, 4, cudaMemcpyDeviceToHost, st));
            TSR_CUDA(cudaStreamSynchronize(st));
            if ((uint64_t)ncells + tot[1] > ccap) {
                uint64_t ncap = std::max<uint64_t>((uint64_t)ncells + tot[1], (uint64_t)ccap * 2);
                if (ncap * 8 >= INVALID) fail(TSR_ERR_OVERFLOW_U32, "too many dual cells");
                DBuf<uint32_t> a(ncap * 8, st);
                DBuf<uint64_t> h(ncap, st), l(ncap, st);
                if (ncells) {
                    TSR_CUDA(cudaMemcpyAsync(a.p, all_cells.p, (size_t)ncells * 32, cudaMemcpyDeviceToDevice, st));
                    TSR_CUDA(cudaMemcpyAsync(h.p, all_hi.p, (size_t)ncells * 8, cudaMemcpyDeviceToDevice, st));
                    TSR_CUDA(cudaMemcpyAsync(l.p, all_lo.p, (size_t)ncells * 8, cudaMemcpyDeviceToDevice, st));
                }
                all_cells = std::move(a); all_hi = std::move(h); all_lo = std::move(l);
                ccap = (uint32_t)ncap;
            }
            FrameBuf nx;
            nx.type.alloc(tot[0], st); nx.nodes.alloc((size_t)tot[0] * 8, st); nx.khi.alloc(tot[0], st); nx.klo.alloc(tot[0], st);
            k_frames_write<<<grid_for(nf, 128), 128, 0, st>>>(nf, cur_f.type.p, cur_f.nodes.p, cur_f.khi.p, cur_f.klo.p,
                                                             level, t.children.p, t.node_to_leaf.p, of.p, oc.p, ncells,
                                                             nx.type.p, nx.nodes.p, nx.khi.p, nx.klo.p, all_cells.p,
                                                             all_hi.p, all_lo.p); ::tsr::note_launch();
            ncells += tot[1];
            cur_f = std::move(nx);
            nf = tot[0];
        }
        t.n_cells = ncells;
        t.cells.alloc((size_t)ncells * 8, st);
        if (ncells) {
            DBuf<uint32_t> idx(ncells, st), idx2(ncells, st), idx3(ncells, st);
            DBuf<uint64_t> k2(ncells, st), k3(ncells, st);
            k_iota<<<grid_for(ncells, BLK), BLK, 0, st>>>(ncells, idx.p); ::tsr::note_launch();
            // LSD: stable sort by the low word, then by the high word
            sort_pairs(all_lo.p, k2.p, idx.p, idx2.p, ncells, st);
            DBuf<uint64_t> hi_sorted(ncells, st);
            k_gather_u64<<<grid_for(ncells, BLK), BLK, 0, st>>>(ncells, idx2.p, all_hi.p, hi_sorted.p); ::tsr::note_launch();
            sort_pairs(hi_sorted.p, k3.p, idx2.p, idx3.p, ncells, st);
            k_gather_cells<<<grid_for(ncells, BLK), BLK, 0, st>>>(ncells, idx3.p, all_cells.p, t.cells.p); ::tsr::note_launch();
        }
    }
    t.stage_ms[5] = timer.lap();
    TSR_CUDA(cudaStreamSynchronize(st));
    TSR_CUDA(cudaGetLastError());
}

}  // namespace tsr
