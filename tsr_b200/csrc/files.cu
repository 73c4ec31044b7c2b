// files.cu -- the reference's on-disk formats for the tree and the field:
// Nodes::saveToFile/loadFromFile (Nodes.cpp:770-807), Leaves (Leaves.cpp:
// 230-292), DualCells (DualCells.cpp:359-385), Occupancy (Occupancy.cpp:
// 663-766), Samples::saveToFile (Samples.cpp:733-765), with the file
// endings of FileNaming.cpp:21-29.
//
// Each body has the reference's order and widths with Real = double:
//   .nodes      u32 nodeCount; u32 children[], parents[], samplesPerNode[],
//               sampleStartIndices[] (nodeCount each)
//   .leaves     u32 {nodeCount, leafCount, neighbourCount}; u32 nodeToLeaf[];
//               Scope[leafCount] = {f64 min xyz, f64 size, u32 node, u32 pad};
//               u32 neighbourOffsets[leafCount + 1], neighbours[]
//   .dualCells  u32 indexCount; u32 indices[] (8 per cell)
//   .occupancy  u32 {leafCount, nodeCount}; for EMPTINESS then SAMPLENESS:
//               f64 coneLengths[], kernelSums[]; f64 priorsForEmptiness[];
//               u32 nodeStates[]; f64 coneCount
//   .samples    u32 sampleCount, camerasPerSample; f64 AABB min xyz, max xyz;
//               f64 colors[3 n], normals[3 n], positions[3 n], confidences[n],
//               scales[n]; u32 parentCameras[K n]
// The reference writes BaseProject's File header before each body; that
// library is not available here, so its header is replaced by a fixed
// 16-byte one: "TSRF", u32 format 1, u32 the reference's FILE_VERSION (0),
// u32 kind (1 nodes, 2 leaves, 3 dual cells, 4 occupancy, 5 samples).
// Little endian.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "handles.h"

namespace tsr {

namespace {

constexpr uint32_t FORMAT = 1, REF_FILE_VERSION = 0;
enum Kind : uint32_t { NODES = 1, LEAVES = 2, DUAL_CELLS = 3, OCCUPANCY = 4, SAMPLES = 5 };

struct ScopeRecord {   // Scope.h with Real = double
    double min[3];
    double size;
    uint32_t node;
    uint32_t pad;
};
static_assert(sizeof(ScopeRecord) == 40, "Scope record layout");

struct Writer {
    FILE *f = nullptr;
    std::string path;
    Writer(const std::string &p, uint32_t kind) : path(p) {
        f = std::fopen(p.c_str(), "wb");
        if (!f) fail(TSR_ERR_INVALID_ARG, "cannot create " + p);
        const char magic[4] = {'T', 'S', 'R', 'F'};
        put(magic, 4);
        const uint32_t h[3] = {FORMAT, REF_FILE_VERSION, kind};
        put(h, sizeof(h));
    }
    ~Writer() { if (f) std::fclose(f); }
    void put(const void *p, size_t bytes) {
        if (bytes && std::fwrite(p, 1, bytes, f) != bytes) fail(TSR_ERR_INVALID_ARG, "cannot write " + path);
    }
    template <class T> void put_vec(const std::vector<T> &v) { put(v.data(), v.size() * sizeof(T)); }
    void close() {
        if (std::fclose(f) != 0) { f = nullptr; fail(TSR_ERR_INVALID_ARG, "cannot write " + path); }
        f = nullptr;
    }
};

struct Reader {
    FILE *f = nullptr;
    std::string path;
    uint64_t left = 0;   // bytes not read yet: counts are checked against it before any allocation
    Reader(const std::string &p, uint32_t kind) : path(p) {
        f = std::fopen(p.c_str(), "rb");
        if (!f) fail(TSR_ERR_INVALID_ARG, "cannot open " + p);
        if (std::fseek(f, 0, SEEK_END) != 0) fail(TSR_ERR_INVALID_ARG, "cannot read " + p);
        const long size = std::ftell(f);
        if (size < 0 || std::fseek(f, 0, SEEK_SET) != 0) fail(TSR_ERR_INVALID_ARG, "cannot read " + p);
        left = (uint64_t)size;
        char magic[4];
        uint32_t h[3];
        get(magic, 4);
        get(h, sizeof(h));
        if (std::memcmp(magic, "TSRF", 4) != 0 || h[0] != FORMAT || h[1] != REF_FILE_VERSION || h[2] != kind)
            fail(TSR_ERR_INVALID_ARG, "not a file of the expected kind and version: " + p);
    }
    ~Reader() { if (f) std::fclose(f); }
    void get(void *p, size_t bytes) {
        if (bytes > left || (bytes && std::fread(p, 1, bytes, f) != bytes))
            fail(TSR_ERR_INVALID_ARG, "truncated file " + path);
        left -= bytes;
    }
    template <class T> void get_vec(std::vector<T> &v, size_t n) {
        if (n > left / sizeof(T)) fail(TSR_ERR_INVALID_ARG, "truncated file " + path);
        v.resize(n);
        get(v.data(), n * sizeof(T));
    }
    void expect_end() {
        if (left != 0) fail(TSR_ERR_INVALID_ARG, "trailing data in " + path);
    }
};

template <class T>
std::vector<T> download(const DBuf<T> &b, size_t n, cudaStream_t st) {
    std::vector<T> h(n);
    if (n) TSR_CUDA(cudaMemcpyAsync(h.data(), b.p, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    return h;
}

template <class T>
void upload(DBuf<T> &b, const std::vector<T> &h, cudaStream_t st) {
    b.alloc(h.size(), st);
    if (!h.empty()) TSR_CUDA(cudaMemcpyAsync(b.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

}  // namespace

void save_tree(const tsr_tree &t, const std::string &prefix) {
    if (t.n_nb >= INVALID) fail(TSR_ERR_OVERFLOW_U32, "neighbour count beyond the format's 32-bit count");
    cudaStream_t st = t.stream;
    const uint32_t nn = t.n_nodes, nl = t.n_leaves;
    auto children = download(t.children, nn, st), parents = download(t.parents, nn, st);
    auto counts = download(t.counts, nn, st), starts = download(t.starts, nn, st);
    auto node_to_leaf = download(t.node_to_leaf, nn, st), leaf_node = download(t.leaf_node, nl, st);
    auto leaf_min = download(t.leaf_min, nl, st);
    auto depth = download(t.depth, nn, st);
    auto nb_off = download(t.nb_off, (size_t)nl + 1, st), nbs = download(t.nbs, t.n_nb, st);
    auto cells = download(t.cells, (size_t)t.n_cells * 8, st);
    TSR_CUDA(cudaStreamSynchronize(st));
    {
        Writer w(prefix + ".nodes", NODES);
        w.put(&nn, 4);
        w.put_vec(children); w.put_vec(parents); w.put_vec(counts); w.put_vec(starts);
        w.close();
    }
    {
        Writer w(prefix + ".leaves", LEAVES);
        const uint32_t c[3] = {nn, nl, (uint32_t)t.n_nb};
        w.put(c, sizeof(c));
        w.put_vec(node_to_leaf);
        std::vector<ScopeRecord> scopes(nl);
        for (uint32_t l = 0; l < nl; ++l) {
            const uint32_t node = leaf_node[l];
            scopes[l] = ScopeRecord{{leaf_min[l].x, leaf_min[l].y, leaf_min[l].z}, size_at(t.root_size, depth[node]),
                                    node, 0};
        }
        w.put_vec(scopes);
        w.put_vec(nb_off);
        w.put_vec(nbs);
        w.close();
    }
    {
        Writer w(prefix + ".dualCells", DUAL_CELLS);
        const uint32_t ic = (uint32_t)cells.size();
        w.put(&ic, 4);
        w.put_vec(cells);
        w.close();
    }
}

// Tree::getRootScope (Tree.cpp:70-101): the cube around the samples' AABB.
void root_from_aabb(tsr_tree &t) {
    const double *lo = t.aabb, *hi = t.aabb + 3;
    const double ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    const double size = std::max(std::max(ext[0], ext[1]), ext[2]);
    const double half = size * 0.5;
    for (int j = 0; j < 3; ++j) t.root_min[j] = (lo[j] + hi[j]) * 0.5 - half;
    t.root_size = size;
}

// Tree::loadFromFile (Tree.cpp:118-127): the saved arrays plus what the
// build derives from them (depths, node corners by the build's own FP64
// recurrence, the level lists).  The root scope comes from the samples'
// AABB like the reference's (Samples::mAABBWS, stored in the samples file,
// Samples.cpp:705): the caller's, or when aabb is null computed from the
// samples exactly as the build computes it.  The samples come in tree order
// (the order they were saved in).
void load_tree(tsr_tree &t, const std::string &prefix, const tsr_samples_view &sv, const double *aabb) {
    cudaStream_t st = t.stream;
    std::vector<uint32_t> children, parents, counts, starts, node_to_leaf, nb_off, nbs, cells;
    std::vector<ScopeRecord> scopes;
    uint32_t nn = 0, nl = 0, nnb = 0;
    {
        Reader r(prefix + ".nodes", NODES);
        r.get(&nn, 4);
        if (nn == 0 || nn >= INVALID) fail(TSR_ERR_INVALID_ARG, "bad node count in " + r.path);
        r.get_vec(children, nn); r.get_vec(parents, nn); r.get_vec(counts, nn); r.get_vec(starts, nn);
        r.expect_end();
    }
    {
        Reader r(prefix + ".leaves", LEAVES);
        uint32_t c[3];
        r.get(c, sizeof(c));
        if (c[0] != nn) fail(TSR_ERR_INVALID_ARG, "leaves file of another tree: " + r.path);
        nl = c[1];
        nnb = c[2];
        r.get_vec(node_to_leaf, nn);
        r.get_vec(scopes, nl);
        r.get_vec(nb_off, (size_t)nl + 1);
        r.get_vec(nbs, nnb);
        r.expect_end();
    }
    {
        Reader r(prefix + ".dualCells", DUAL_CELLS);
        uint32_t ic = 0;
        r.get(&ic, 4);
        if (ic % 8) fail(TSR_ERR_INVALID_ARG, "dual cell indices not a multiple of 8 in " + r.path);
        r.get_vec(cells, ic);
        r.expect_end();
    }
    // Consistency, so that no kernel indexes out of range on a damaged file:
    // parents precede children, child blocks are whole 8-node blocks at
    // 1 + 8k that point back at their parent, sample ranges stay inside the
    // sample arrays, and leaves are exactly the childless nodes.
    uint64_t total = 0;
    for (uint32_t i = 0; i < nn; ++i) {
        if (i == 0 ? parents[i] != INVALID : parents[i] >= i)
            fail(TSR_ERR_INVALID_ARG, "nodes file: a parent must precede its children");
        const uint32_t c = children[i];
        if (c != INVALID) {
            if (c <= i || (uint64_t)c + 8 > nn || (c - 1) % 8 != 0)
                fail(TSR_ERR_INVALID_ARG, "nodes file: child block out of range");
            for (uint32_t j = 0; j < 8; ++j)
                if (parents[c + j] != i) fail(TSR_ERR_INVALID_ARG, "nodes file: child and parent links disagree");
        }
        if ((uint64_t)starts[i] + counts[i] > sv.count)
            fail(TSR_ERR_INVALID_ARG, "nodes file: a node's samples lie outside the sample arrays");
        if ((c == INVALID) != (node_to_leaf[i] != INVALID) || (node_to_leaf[i] != INVALID && node_to_leaf[i] >= nl))
            fail(TSR_ERR_INVALID_ARG, "leaves file: leaves must be exactly the childless nodes");
        total += counts[i];
    }
    if (total != sv.count) fail(TSR_ERR_INVALID_ARG, "nodes file holds another sample count");
    for (uint32_t l = 0; l < nl; ++l)
        if (scopes[l].node >= nn || node_to_leaf[scopes[l].node] != l)
            fail(TSR_ERR_INVALID_ARG, "leaves file: scope and node links disagree");
    if (nb_off[0] != 0 || nb_off[nl] != nnb) fail(TSR_ERR_INVALID_ARG, "leaves file: neighbour offsets disagree");
    for (uint32_t l = 0; l < nl; ++l)
        if (nb_off[l] > nb_off[l + 1]) fail(TSR_ERR_INVALID_ARG, "leaves file: neighbour offsets decrease");
    for (uint32_t x : nbs) if (x >= nl) fail(TSR_ERR_INVALID_ARG, "leaves file: neighbour out of range");
    for (uint32_t x : cells) if (x >= nl) fail(TSR_ERR_INVALID_ARG, "dual cells file: leaf out of range");

    if (aabb) {
        for (int j = 0; j < 3; ++j)
            if (!std::isfinite(aabb[j]) || !std::isfinite(aabb[3 + j]) || !(aabb[j] <= aabb[3 + j]))
                fail(TSR_ERR_INVALID_ARG, "AABB must be finite with min <= max");
        std::copy(aabb, aabb + 6, t.aabb);
    } else {
        // Samples::computeAABB (Samples.cpp:290-298, 442-449), as the build computes it
        const double h = t.params.max_relative_sampling_distance;
        double lo[3] = {REAL_MAX, REAL_MAX, REAL_MAX}, hi[3] = {-REAL_MAX, -REAL_MAX, -REAL_MAX};
        for (uint32_t s = 0; s < sv.count; ++s) {
            const double r = dadd(dmul(sv.scales[s], h), EPS);
            for (int j = 0; j < 3; ++j) {
                const double p = sv.positions[3 * (size_t)s + j];
                lo[j] = std::min(lo[j], dsub(p, r));
                hi[j] = std::max(hi[j], dadd(p, r));
            }
        }
        for (int j = 0; j < 3; ++j) {
            t.aabb[j] = lo[j];
            t.aabb[3 + j] = hi[j];
        }
    }
    root_from_aabb(t);

    // depths and corners in index order (parents come first)
    std::vector<uint8_t> depth(nn, 0);
    std::vector<D3> nmin(nn);
    nmin[0] = D3{t.root_min[0], t.root_min[1], t.root_min[2]};
    uint32_t max_depth = 0;
    for (uint32_t i = 1; i < nn; ++i) {
        const uint32_t p = parents[i];
        const uint32_t d = depth[p] + 1u;
        if (d > MAX_TREE_DEPTH) fail(TSR_ERR_INVALID_ARG, "nodes file: tree deeper than supported");
        depth[i] = (uint8_t)d;
        max_depth = std::max(max_depth, d);
        const uint32_t cp = children[p];
        if (cp == INVALID || i < cp || i - cp >= 8) fail(TSR_ERR_INVALID_ARG, "nodes file: a node outside its parent's block");
        nmin[i] = child_coords(nmin[p], size_at(t.root_size, d), i - cp);
    }
    for (uint32_t l = 0; l < nl; ++l) {
        const ScopeRecord &sc = scopes[l];
        const D3 m = nmin[sc.node];
        if (m.x != sc.min[0] || m.y != sc.min[1] || m.z != sc.min[2] || sc.size != size_at(t.root_size, depth[sc.node]))
            fail(TSR_ERR_INVALID_ARG, "leaves file: scopes do not match the root scope of this AABB");
    }
    // level lists (nodes by depth, index order within a depth)
    std::vector<uint32_t> level_start(max_depth + 2, 0), order(nn);
    for (uint32_t i = 0; i < nn; ++i) ++level_start[depth[i] + 1];
    for (uint32_t d = 0; d <= max_depth; ++d) level_start[d + 1] += level_start[d];
    {
        std::vector<uint32_t> fill(level_start.begin(), level_start.end() - 1);
        for (uint32_t i = 0; i < nn; ++i) order[fill[depth[i]]++] = i;
    }
    std::vector<D3> leaf_min(nl);
    std::vector<uint32_t> leaf_node(nl);
    for (uint32_t l = 0; l < nl; ++l) {
        leaf_min[l] = D3{scopes[l].min[0], scopes[l].min[1], scopes[l].min[2]};
        leaf_node[l] = scopes[l].node;
    }
    std::vector<uint32_t> target(sv.count);
    for (uint32_t s = 0; s < sv.count; ++s) target[s] = s;

    t.n_samples = sv.count;
    t.k = sv.cams_per_sample;
    t.n_nodes = nn;
    t.n_leaves = nl;
    t.max_depth = max_depth;
    t.n_cells = (uint32_t)(cells.size() / 8);
    t.n_nb = nnb;
    upload(t.children, children, st); upload(t.parents, parents, st);
    upload(t.counts, counts, st); upload(t.starts, starts, st);
    upload(t.depth, depth, st); upload(t.nmin, nmin, st);
    upload(t.level_order, order, st);
    t.level_start = level_start;
    upload(t.node_to_leaf, node_to_leaf, st); upload(t.leaf_min, leaf_min, st); upload(t.leaf_node, leaf_node, st);
    upload(t.nb_off, nb_off, st); upload(t.nbs, nbs, st); upload(t.cells, cells, st);
    upload(t.target, target, st);
    const size_t n = sv.count, k = sv.cams_per_sample;
    t.pos.alloc(n, st); t.nrm.alloc(n, st); t.scale.alloc(n, st); t.conf.alloc(n, st); t.links.alloc(n * k, st);
    TSR_CUDA(cudaMemcpyAsync(t.pos.p, sv.positions, n * 24, cudaMemcpyHostToDevice, st));
    TSR_CUDA(cudaMemcpyAsync(t.nrm.p, sv.normals, n * 24, cudaMemcpyHostToDevice, st));
    TSR_CUDA(cudaMemcpyAsync(t.scale.p, sv.scales, n * 8, cudaMemcpyHostToDevice, st));
    TSR_CUDA(cudaMemcpyAsync(t.conf.p, sv.confidences, n * 8, cudaMemcpyHostToDevice, st));
    TSR_CUDA(cudaMemcpyAsync(t.links.p, sv.camera_links, n * k * 4, cudaMemcpyHostToDevice, st));
    TSR_CUDA(cudaStreamSynchronize(st));   // the host vectors go out of scope
}

// Samples::saveToFile (Samples.cpp:733-765, the .samples branch): the
// tree's samples in tree order with the AABB the tree was built over.
// Colours are not part of this library's samples; the caller passes them
// (3 per sample, tree order) or gets zeros.
void save_samples(const tsr_tree &t, const double *colors, const std::string &path) {
    cudaStream_t st = t.stream;
    const size_t n = t.n_samples, k = t.k;
    auto nrm = download(t.nrm, n, st), pos = download(t.pos, n, st);
    auto conf = download(t.conf, n, st), scale = download(t.scale, n, st);
    auto links = download(t.links, n * k, st);
    TSR_CUDA(cudaStreamSynchronize(st));
    Writer w(path, SAMPLES);
    const uint32_t c[2] = {t.n_samples, t.k};
    w.put(c, sizeof(c));
    w.put(t.aabb, sizeof(t.aabb));
    if (colors) {
        w.put(colors, n * 24);
    } else {
        const std::vector<double> zeros(3 * n, 0.0);
        w.put_vec(zeros);
    }
    w.put_vec(nrm); w.put_vec(pos); w.put_vec(conf); w.put_vec(scale); w.put_vec(links);
    w.close();
}

void save_occupancy(const tsr_occupancy &o, const std::string &path) {
    cudaStream_t st = o.stream;
    const uint32_t nl = o.n_leaves, nn = o.n_nodes;
    auto elen = download(o.e_len, nl, st), esum = download(o.e_sum, nl, st);
    auto slen = download(o.s_len, nl, st), ssum = download(o.s_sum, nl, st);
    auto prior = download(o.prior, nl, st);
    auto states = download(o.states, nn, st);
    TSR_CUDA(cudaStreamSynchronize(st));
    Writer w(path, OCCUPANCY);
    const uint32_t c[2] = {nl, nn};
    w.put(c, sizeof(c));
    w.put_vec(elen); w.put_vec(esum);   // EMPTINESS
    w.put_vec(slen); w.put_vec(ssum);   // SAMPLENESS
    w.put_vec(prior);
    w.put_vec(states);
    w.put(&o.cone_count, 8);
    w.close();
}

void load_occupancy(const tsr_tree &t, tsr_occupancy &o, const std::string &path, const tsr_params &p) {
    cudaStream_t st = o.stream;
    Reader r(path, OCCUPANCY);
    uint32_t c[2];
    r.get(c, sizeof(c));
    if (c[0] != t.n_leaves || c[1] != t.n_nodes) fail(TSR_ERR_INVALID_ARG, "occupancy file of another tree: " + path);
    std::vector<double> elen, esum, slen, ssum, prior;
    std::vector<uint32_t> states;
    r.get_vec(elen, c[0]); r.get_vec(esum, c[0]);
    r.get_vec(slen, c[0]); r.get_vec(ssum, c[0]);
    r.get_vec(prior, c[0]);
    r.get_vec(states, c[1]);
    r.get(&o.cone_count, 8);
    r.expect_end();
    o.n_leaves = c[0];
    o.n_nodes = c[1];
    o.confidence_threshold = p.confidence_threshold;
    upload(o.e_len, elen, st); upload(o.e_sum, esum, st);
    upload(o.s_len, slen, st); upload(o.s_sum, ssum, st);
    upload(o.prior, prior, st);
    upload(o.states, states, st);
    finalize_field(o, p);
    TSR_CUDA(cudaStreamSynchronize(st));
}

}  // namespace tsr
