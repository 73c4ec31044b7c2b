/*
 * tsr_oracle.cpp -- FP64 CPU restatement of the reference's volumetric core.
 *
 * TEST INFRASTRUCTURE ONLY (parity checker + timed CPU baseline); see
 * tsr_oracle.h.  Paths cited below are relative to
 * SurfaceReconstruction/SurfaceReconstruction/ in the reference.
 *
 * Real = double.  Built with -ffp-contract=off so every expression rounds
 * exactly as written; the GPU tree build evaluates the same expressions in
 * the same operation order with explicitly round-to-nearest FP64 intrinsics
 * (__dadd_rn, __dmul_rn, ...; tsr_b200/csrc/common.cuh), which the compiler
 * never fuses, so that topology decisions agree bit for bit.
 *
 * Pinned to the reference: tests/test_ref_pin.py compares every tree,
 * field and DMC array of this restatement with the reference's own sources
 * built against the BaseProject shim (oracle/ref_driver.cpp, `make ref`).
 */
#include "tsr_oracle.h"
#include "tsr_geom.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace tsrg;

namespace {

const uint32_t INVALID = 0xFFFFFFFFu;
const uint32_t CHILD_COUNT = 8;
const uint32_t SIDE_COUNT = 6;
const uint32_t MAX_DEPTH_DIFFERENCE = 3;       // Occupancy.cpp:72
const uint32_t FLAG_SAMPLENESS = 1u << 0;      // Occupancy.h:38
const uint32_t FLAG_EMPTINESS = 1u << 1;       // Occupancy.h:39
enum { EMPTINESS = 0, SAMPLENESS = 1 };        // Occupancy.h:29-34

struct Scope {
    V3 mn;
    double size;
    uint32_t idx;
    V3 center() const { double h = 0.5 * size; return V3{mn.x + h, mn.y + h, mn.z + h}; }
    V3 mx() const { return V3{mn.x + size, mn.y + size, mn.z + size}; }
};

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct tsro_scene {
    uint32_t N = 0, K = 0, C = 0;
    std::vector<V3> pos, nrm;
    std::vector<double> scale, conf;
    std::vector<uint32_t> links;
    std::vector<V3> cams;
    double h_svo = 2.0, h_o = 2.0, conf_thresh = 100.0, prior_rel = 25.0, rel_cone = 1.0;

    V3 aabb[2];
    Scope root{};

    // Nodes.h:144-147
    std::vector<uint32_t> children, parents, counts, starts;
    std::vector<uint32_t> target;   // sample permutation, Nodes.cpp:594-636
    uint64_t writers = 0, sampling_splits = 0;

    // Leaves.h:90-98
    std::vector<Scope> leaves;
    std::vector<uint32_t> node_to_leaf, nb_off, nbs;
    // DualCells.h:67
    std::vector<uint32_t> cells;

    // Occupancy.h:135-148
    std::vector<double> ksum[2], clen[2], prior;
    std::vector<uint32_t> states;
    double cone_count = 0.0;
    std::vector<double> occ;

    // DMC
    std::vector<uint8_t> cases;
    std::vector<double> vpos, vscale;
    std::vector<uint32_t> vkeys, tris;

    double stage[10] = {0};

    // ---------------------------------------------------------------- samples
    double max_dist(uint32_t s) const { return scale[s] * h_svo; }   // Samples.h:409-412
    double plane_dist(const V3 &x, uint32_t s) const { return sample_plane_distance(pos[s], nrm[s], x); }

    // Samples.cpp:290-298, 442-449; Tree.cpp:70-101
    void compute_root() {
        aabb[0] = V3{DBL_MAX_, DBL_MAX_, DBL_MAX_};
        aabb[1] = V3{-DBL_MAX_, -DBL_MAX_, -DBL_MAX_};
        for (uint32_t s = 0; s < N; ++s) {
            const V3 &p = pos[s];
            double r = max_dist(s) + EPS;
            V3 lo{p.x - r, p.y - r, p.z - r}, hi{p.x + r, p.y + r, p.z + r};
            aabb[0] = vmin(aabb[0], lo);
            aabb[1] = vmax(aabb[1], hi);
        }
        V3 ext = sub(aabb[1], aabb[0]);
        double size = std::max(std::max(ext.x, ext.y), ext.z);
        V3 center = mul(add(aabb[0], aabb[1]), 0.5);
        double half = size * 0.5;
        root.mn = V3{center.x - half, center.y - half, center.z - half};
        root.size = size;
        root.idx = 0;
    }

    // Tree.cpp:86-91
    uint32_t sample_depth(uint32_t s) const {
        double temp = root.size / max_dist(s);
        return (uint32_t)std::ceil(std::log2(temp));
    }

    // ------------------------------------------------------------------ nodes
    uint32_t count() const { return (uint32_t)children.size(); }
    bool is_leaf(uint32_t i) const { return i != INVALID && children[i] == INVALID; }   // Nodes.h:203-208

    void resize(uint32_t n) {   // Nodes.cpp:425-431
        children.resize(n, INVALID);
        parents.resize(n, INVALID);
        counts.resize(n, 0);
        starts.resize(n, INVALID);
    }

    void create_children(uint32_t idx) {   // Nodes.cpp:397-415
        uint32_t old = count();
        if ((uint64_t)old + CHILD_COUNT >= (uint64_t)INVALID)
            throw std::runtime_error("node count overflow");
        resize(old + CHILD_COUNT);
        children[idx] = old;
        for (uint32_t c = 0; c < CHILD_COUNT; ++c) parents[old + c] = idx;
    }

    Scope child_scope(const Scope &sc, uint32_t c, double child_size) const {   // Nodes.h:184-191
        return Scope{child_coords(sc.mn, child_size, c), child_size, children[sc.idx] + c};
    }

    uint32_t depth_of(uint32_t idx) const {   // Nodes.cpp:133-143
        uint32_t d = 0;
        for (uint32_t c = parents[idx]; c != INVALID; c = parents[c]) ++d;
        return d;
    }

    // Nodes.cpp:231-269
    bool find_container(Scope &sc, uint32_t s) const {
        const V3 &p = pos[s];
        double r = max_dist(s);
        if (!node_contains(p, sc.mn, sc.size, EPS))
            throw std::runtime_error("sample outside start node");
        while (true) {
            if (sc.size <= r) return true;
            if (is_leaf(sc.idx)) return false;
            double child_size = sc.size * 0.5;
            V3 center{sc.mn.x + child_size, sc.mn.y + child_size, sc.mn.z + child_size};
            V3 off = sub(p, center);
            uint32_t c = child_index_for_offset(off);
            sc = child_scope(sc, c, child_size);
        }
    }

    // Nodes.cpp:471-488
    bool fitting_center(const V3 &node_min, double child_size, bool positive, uint32_t s) const {
        V3 c{node_min.x + child_size, node_min.y + child_size, node_min.z + child_size};
        double d2 = len2(sub(c, pos[s]));
        double r = max_dist(s);
        if (d2 > r * r) return false;
        bool on_pos = plane_dist(c, s) > 0.0;
        return on_pos == positive;
    }

    // Nodes.cpp:490-517
    bool intersect(const Scope &sc, bool positive, uint32_t s) const {
        bool all_wrong = true;
        for (uint32_t i = 0; i < CHILD_COUNT; ++i) {
            V3 corner = child_coords(sc.mn, sc.size, i);
            bool in_pos = plane_dist(corner, s) > 0.0;
            if (in_pos != positive) continue;
            all_wrong = false;
            break;
        }
        if (all_wrong) return false;
        return aabb_sphere(sc.mn, sc.mx(), pos[s], max_dist(s));
    }

    // Nodes.cpp:433-469
    uint32_t find_reliable(const Scope &sc, bool positive, uint32_t s) const {
        double child_size = sc.size * 0.5;
        if (is_leaf(sc.idx)) {
            bool fit = fitting_center(sc.mn, child_size, positive, s);
            double grand = child_size * 0.5;
            if (fit)
                for (uint32_t i = 0; i < CHILD_COUNT; ++i)
                    if (fitting_center(child_coords(sc.mn, child_size, i), grand, positive, s)) return sc.idx;
            return INVALID;
        }
        for (uint32_t c = 0; c < CHILD_COUNT; ++c) {
            Scope cs = child_scope(sc, c, child_size);
            if (!intersect(cs, positive, s)) continue;
            uint32_t r = find_reliable(cs, positive, s);
            if (r != INVALID) return r;
        }
        return INVALID;
    }

    // Nodes.cpp:271-337
    void create_for_sampling(Scope sc, bool positive, uint32_t s) {
        if (find_reliable(sc, positive, s) != INVALID) return;
        ++writers;
        const V3 &p = pos[s];
        const V3 &n = nrm[s];
        double r = max_dist(s);
        V3 endp = add(p, mul(n, positive ? r : -r));
        for (int guard = 0; guard < 200; ++guard) {
            if (is_leaf(sc.idx)) {
                create_children(sc.idx);
                ++sampling_splits;
                if (find_reliable(sc, positive, s) != INVALID) return;
            }
            double child_size = sc.size * 0.5;
            if (child_size == 0.0) throw std::runtime_error("zero node size");
            double score = -DBL_MAX_;
            uint32_t best = INVALID;
            for (uint32_t c = 0; c < CHILD_COUNT; ++c) {
                V3 bmin = child_coords(sc.mn, child_size, c);
                V3 bmax{bmin.x + child_size, bmin.y + child_size, bmin.z + child_size};
                double t0, t1;
                if (!segment_aabb(t0, t1, p, endp, bmin, bmax)) continue;
                double ov = t1 - t0;
                if (ov <= score) continue;
                score = ov;
                best = c;
                if (ov >= 1.0 - EPS) break;
            }
            if (best == INVALID) throw std::runtime_error("sampling descent left the segment");
            sc = child_scope(sc, best, child_size);
        }
        throw std::runtime_error("sampling descent did not terminate");
    }

    // Nodes.cpp:145-184
    uint32_t get_node(Scope &sc, const V3 &q, uint32_t max_depth) const {
        uint32_t depth = depth_of(sc.idx);
        if (depth > max_depth || !node_contains(q, sc.mn, sc.size, 0.0)) {
            sc.idx = INVALID;
            return depth;
        }
        while (true) {
            if (is_leaf(sc.idx)) return depth;
            if (depth == max_depth) return depth;
            for (uint32_t c = 0; c < CHILD_COUNT; ++c) {
                double child_size = sc.size * 0.5;
                V3 cc = child_coords(sc.mn, child_size, c);
                if (!node_contains(q, cc, child_size, 0.0)) continue;
                sc.idx = children[sc.idx] + c;
                sc.mn = cc;
                sc.size = child_size;
                ++depth;
                break;
            }
        }
    }

    // Nodes.cpp:347-395
    bool balance_pass(uint32_t depth, const Scope &sc) {
        if (!is_leaf(sc.idx)) {
            double child_size = 0.5 * sc.size;
            bool created = false;
            for (uint32_t c = 0; c < CHILD_COUNT; ++c) {
                Scope cs = child_scope(sc, c, child_size);
                created |= balance_pass(depth + 1, cs);
            }
            return created;
        }
        bool created = false;
        for (uint32_t side = 0; side < SIDE_COUNT; ++side) {
            V3 target_pos = side_center(sc.mn, sc.size, side, sc.size * 0.5);
            Scope nb = root;
            uint32_t nd = get_node(nb, target_pos, depth);
            if (nb.idx == INVALID) continue;
            if (!is_leaf(nb.idx)) continue;
            while (depth > nd + 1) {
                create_children(nb.idx);
                nd = get_node(nb, target_pos, depth);
                created = true;
            }
        }
        return created;
    }

    // Nodes.cpp:536-554
    uint32_t target_indices(std::vector<uint32_t> &t, uint32_t node, uint32_t next_free) const {
        if (is_leaf(node)) return next_free;
        uint32_t block = children[node];
        uint32_t nn = next_free + CHILD_COUNT;
        for (uint32_t c = 0; c < CHILD_COUNT; ++c) {
            t[block + c] = next_free + c;
            nn = target_indices(t, block + c, nn);
        }
        return nn;
    }

    // Nodes.cpp:519-534, 556-592
    void reorder_nodes() {
        uint32_t n = count();
        std::vector<uint32_t> t(n, INVALID);
        t[0] = 0;
        target_indices(t, 0, 1);
        std::vector<uint32_t> tmp(n);
        for (std::vector<uint32_t> *links : {&children, &parents}) {
            for (uint32_t i = 0; i < n; ++i) {
                uint32_t old = (*links)[i];
                tmp[t[i]] = (old == INVALID ? old : t[old]);
            }
            links->swap(tmp);
        }
        for (uint32_t i = 0; i < n; ++i) tmp[t[i]] = counts[i];
        counts.swap(tmp);
        uint32_t acc = 0;
        for (uint32_t i = 0; i < n; ++i) { starts[i] = acc; acc += counts[i]; }
        std::fill(counts.begin(), counts.end(), 0u);
    }

    // Nodes.cpp:594-636 (sequential: samples keep their input order inside
    // each node, one of the orders the reference's omp critical can produce)
    void reorder_samples() {
        target.assign(N, INVALID);
        for (uint32_t s = 0; s < N; ++s) {
            Scope sc = root;
            if (!find_container(sc, s)) throw std::runtime_error("sample not inserted");
            uint32_t off = counts[sc.idx]++;
            target[s] = starts[sc.idx] + off;
        }
        // Samples.cpp:825-835
        std::vector<V3> p2(N), n2(N);
        std::vector<double> s2(N), c2(N);
        std::vector<uint32_t> l2((size_t)N * K);
        for (uint32_t s = 0; s < N; ++s) {
            uint32_t t = target[s];
            p2[t] = pos[s]; n2[t] = nrm[s]; s2[t] = scale[s]; c2[t] = conf[s];
            for (uint32_t k = 0; k < K; ++k) l2[(size_t)t * K + k] = links[(size_t)s * K + k];
        }
        pos.swap(p2); nrm.swap(n2); scale.swap(s2); conf.swap(c2); links.swap(l2);
    }

    // Leaves.cpp:44-80
    void gather(const Scope &sc) {
        if (is_leaf(sc.idx)) {
            node_to_leaf[sc.idx] = (uint32_t)leaves.size();
            leaves.push_back(sc);
            return;
        }
        uint32_t c0 = children[sc.idx];
        double cs = sc.size * 0.5;
        for (uint32_t i = 0; i < CHILD_COUNT; ++i)
            gather(Scope{child_coords(sc.mn, cs, i), cs, c0 + i});
    }

    // Leaves.cpp:159-180
    uint32_t unresponsible_neighbor(const Scope &leaf, uint32_t side) const {
        V3 tp = side_center(leaf.mn, leaf.size, side, 0.5 * leaf.size);
        uint32_t maxd = depth_of(leaf.idx);
        Scope nb = root;
        uint32_t nd = get_node(nb, tp, maxd);
        if (nb.idx == INVALID) return INVALID;
        if (!is_leaf(nb.idx)) return INVALID;
        if (nd == maxd && nb.idx < leaf.idx) return INVALID;
        return nb.idx;
    }

    // Leaves.cpp:82-157
    void neighbors() {
        uint32_t L = (uint32_t)leaves.size();
        nb_off.assign(L + 1, 0);
        for (uint32_t l = 0; l < L; ++l)
            for (uint32_t side = 0; side < SIDE_COUNT; ++side) {
                uint32_t n = unresponsible_neighbor(leaves[l], side);
                if (n == INVALID) continue;
                ++nb_off[l];
                ++nb_off[node_to_leaf[n]];
            }
        uint32_t e = 0;
        for (uint32_t i = 0; i < L + 1; ++i) { uint32_t sz = nb_off[i]; nb_off[i] = e; e += sz; }
        nbs.assign(e, INVALID);
        std::vector<uint32_t> fill(L, 0);
        for (uint32_t l = 0; l < L; ++l)
            for (uint32_t side = 0; side < SIDE_COUNT; ++side) {
                uint32_t n = unresponsible_neighbor(leaves[l], side);
                if (n == INVALID) continue;
                uint32_t nl = node_to_leaf[n];
                nbs[nb_off[l] + fill[l]++] = nl;
                nbs[nb_off[nl] + fill[nl]++] = l;
            }
    }

    // DualCells.cpp:49-357
    uint32_t cb(uint32_t n) const { return children[n]; }
    void dc_node(uint32_t n) {
        if (is_leaf(n)) return;
        uint32_t c0 = cb(n);
        uint32_t ch[8] = {c0, c0 + 1, c0 + 2, c0 + 3, c0 + 4, c0 + 5, c0 + 6, c0 + 7};
        for (uint32_t i = 0; i < 8; ++i) dc_node(ch[i]);
        faces_yz(ch); faces_xz(ch); faces_xy(ch);
        edges_z(ch); edges_y(ch); edges_x(ch);
        dc_vertex(ch);
    }
    uint32_t pick(uint32_t n, bool leaf, uint32_t c) const { return leaf ? n : cb(n) + c; }
    void dc_2x(uint32_t a, uint32_t b) {
        bool la = is_leaf(a), lb = is_leaf(b);
        if (la && lb) return;
        uint32_t ch[8] = {pick(a, la, 1), pick(b, lb, 0), pick(a, la, 3), pick(b, lb, 2),
                          pick(a, la, 5), pick(b, lb, 4), pick(a, la, 7), pick(b, lb, 6)};
        faces_yz(ch); edges_z(ch); edges_y(ch); dc_vertex(ch);
    }
    void dc_2y(uint32_t a, uint32_t b) {
        bool la = is_leaf(a), lb = is_leaf(b);
        if (la && lb) return;
        uint32_t ch[8] = {pick(b, lb, 2), pick(b, lb, 3), pick(a, la, 0), pick(a, la, 1),
                          pick(b, lb, 6), pick(b, lb, 7), pick(a, la, 4), pick(a, la, 5)};
        faces_xz(ch); edges_z(ch); edges_x(ch); dc_vertex(ch);
    }
    void dc_2z(uint32_t a, uint32_t b) {
        bool la = is_leaf(a), lb = is_leaf(b);
        if (la && lb) return;
        uint32_t ch[8] = {pick(a, la, 4), pick(a, la, 5), pick(a, la, 6), pick(a, la, 7),
                          pick(b, lb, 0), pick(b, lb, 1), pick(b, lb, 2), pick(b, lb, 3)};
        faces_xy(ch); edges_y(ch); edges_x(ch); dc_vertex(ch);
    }
    void dc_4xy(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
        bool l0 = is_leaf(a), l1 = is_leaf(b), l2 = is_leaf(c), l3 = is_leaf(d);
        if (l0 && l1 && l2 && l3) return;
        uint32_t ch[8] = {pick(a, l0, 3), pick(b, l1, 2), pick(c, l2, 1), pick(d, l3, 0),
                          pick(a, l0, 7), pick(b, l1, 6), pick(c, l2, 5), pick(d, l3, 4)};
        edges_z(ch); dc_vertex(ch);
    }
    void dc_4xz(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
        bool l0 = is_leaf(a), l1 = is_leaf(b), l2 = is_leaf(c), l3 = is_leaf(d);
        if (l0 && l1 && l2 && l3) return;
        uint32_t ch[8] = {pick(a, l0, 5), pick(b, l1, 4), pick(a, l0, 7), pick(b, l1, 6),
                          pick(c, l2, 1), pick(d, l3, 0), pick(c, l2, 3), pick(d, l3, 2)};
        edges_y(ch); dc_vertex(ch);
    }
    void dc_4yz(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
        bool l0 = is_leaf(a), l1 = is_leaf(b), l2 = is_leaf(c), l3 = is_leaf(d);
        if (l0 && l1 && l2 && l3) return;
        uint32_t ch[8] = {pick(a, l0, 6), pick(a, l0, 7), pick(b, l1, 4), pick(b, l1, 5),
                          pick(c, l2, 2), pick(c, l2, 3), pick(d, l3, 0), pick(d, l3, 1)};
        edges_x(ch); dc_vertex(ch);
    }
    void edges_z(const uint32_t *c) { dc_4xy(c[0], c[1], c[2], c[3]); dc_4xy(c[4], c[5], c[6], c[7]); }
    void edges_y(const uint32_t *c) { dc_4xz(c[0], c[1], c[4], c[5]); dc_4xz(c[2], c[3], c[6], c[7]); }
    void edges_x(const uint32_t *c) { dc_4yz(c[0], c[2], c[4], c[6]); dc_4yz(c[1], c[3], c[5], c[7]); }
    void faces_yz(const uint32_t *c) { dc_2x(c[0], c[1]); dc_2x(c[4], c[5]); dc_2x(c[2], c[3]); dc_2x(c[6], c[7]); }
    void faces_xz(const uint32_t *c) { dc_2y(c[2], c[0]); dc_2y(c[3], c[1]); dc_2y(c[6], c[4]); dc_2y(c[7], c[5]); }
    void faces_xy(const uint32_t *c) { dc_2z(c[0], c[4]); dc_2z(c[1], c[5]); dc_2z(c[2], c[6]); dc_2z(c[3], c[7]); }
    void dc_vertex(const uint32_t *n) {
        bool lf[8];
        bool only = true;
        for (int i = 0; i < 8; ++i) { lf[i] = is_leaf(n[i]); only &= lf[i]; }
        if (only) {
            for (int i = 0; i < 8; ++i) cells.push_back(node_to_leaf[n[i]]);
            return;
        }
        uint32_t ch[8];
        for (int i = 0; i < 8; ++i) ch[i] = pick(n[i], lf[i], 7 - i);
        dc_vertex(ch);
    }

    // ---------------------------------------------------------------------
    // Round-parallel schedule of the sampling pass (Nodes.cpp:214-219).
    //
    // The reference processes sample sides sequentially (key k = 2 s + side + 1,
    // positive side first).  Each node records the key of the sample that
    // created its children (0 = containment), so "the tree as sample k saw it"
    // is every node whose parent's children were created by a key < k.  A
    // round evaluates all pending sides against their own versions of the
    // tree; a side whose sensitive leaves (its witness if reliable; every leaf
    // its search read plus the leaf its descent ends in if it is a writer) are
    // untouched by any earlier writer or unresolved side is final.  Writers
    // then split their descent leaf.  This reproduces the sequential tree
    // exactly and is the schedule the GPU build executes; the oracle runs it
    // to prove both claims on real scenes (stop_after = 4 / 5).
    std::vector<uint64_t> ccreator;
    uint64_t rounds = 0, max_contagion = 0;

    bool leaf_v(uint32_t n, uint64_t key) const {
        return children[n] == INVALID || ccreator[n] >= key;
    }
    void split_v(uint32_t n, uint64_t key) {
        create_children(n);
        ccreator.resize(count(), 0);
        ccreator[n] = key;
    }
    uint32_t find_reliable_v(const Scope &sc, bool positive, uint32_t s, uint64_t key,
                             std::vector<uint32_t> *reads) const {
        double child_size = sc.size * 0.5;
        if (leaf_v(sc.idx, key)) {
            bool fit = fitting_center(sc.mn, child_size, positive, s);
            double grand = child_size * 0.5;
            if (fit)
                for (uint32_t i = 0; i < CHILD_COUNT; ++i)
                    if (fitting_center(child_coords(sc.mn, child_size, i), grand, positive, s)) return sc.idx;
            if (reads) reads->push_back(sc.idx);
            return INVALID;
        }
        for (uint32_t c = 0; c < CHILD_COUNT; ++c) {
            Scope cs = child_scope(sc, c, child_size);
            if (!intersect(cs, positive, s)) continue;
            uint32_t r = find_reliable_v(cs, positive, s, key, reads);
            if (r != INVALID) return r;
        }
        return INVALID;
    }
    uint32_t best_child(const Scope &sc, const V3 &p, const V3 &endp) const {
        double child_size = sc.size * 0.5;
        double score = -DBL_MAX_;
        uint32_t best = INVALID;
        for (uint32_t c = 0; c < CHILD_COUNT; ++c) {
            V3 bmin = child_coords(sc.mn, child_size, c);
            V3 bmax{bmin.x + child_size, bmin.y + child_size, bmin.z + child_size};
            double t0, t1;
            if (!segment_aabb(t0, t1, p, endp, bmin, bmax)) continue;
            double ov = t1 - t0;
            if (ov <= score) continue;
            score = ov;
            best = c;
            if (ov >= 1.0 - EPS) break;
        }
        if (best == INVALID) throw std::runtime_error("sampling descent left the segment");
        return best;
    }
    Scope descent_leaf_v(bool positive, uint32_t s, uint64_t key) const {
        const V3 &p = pos[s];
        double r = max_dist(s);
        V3 endp = add(p, mul(nrm[s], positive ? r : -r));
        Scope sc = root;
        while (!leaf_v(sc.idx, key)) sc = child_scope(sc, best_child(sc, p, endp), sc.size * 0.5);
        return sc;
    }
    void apply_sampling(Scope sc, bool positive, uint32_t s, uint64_t key) {
        const V3 &p = pos[s];
        double r = max_dist(s);
        V3 endp = add(p, mul(nrm[s], positive ? r : -r));
        for (int guard = 0; guard < 200; ++guard) {
            if (leaf_v(sc.idx, key + 1)) {
                split_v(sc.idx, key);
                ++sampling_splits;
                if (find_reliable_v(sc, positive, s, key + 1, nullptr) != INVALID) return;
            }
            sc = child_scope(sc, best_child(sc, p, endp), sc.size * 0.5);
        }
        throw std::runtime_error("sampling descent did not terminate");
    }
    void sampling_rounds() {
        ccreator.assign(count(), 0);
        std::vector<uint64_t> pending;
        pending.reserve((size_t)2 * N);
        for (uint64_t k = 1; k <= (uint64_t)2 * N; ++k) pending.push_back(k);
        std::vector<uint64_t> mark;
        std::vector<uint32_t> level;
        struct Ev { bool reliable; uint32_t witness; Scope d; std::vector<uint32_t> reads; };
        std::vector<Ev> ev;
        rounds = 0;
        max_contagion = 0;
        while (!pending.empty()) {
            ++rounds;
            ev.assign(pending.size(), Ev{});
#pragma omp parallel for schedule(dynamic, 64)
            for (int64_t i = 0; i < (int64_t)pending.size(); ++i) {
                uint64_t k = pending[(size_t)i];
                uint32_t s = (uint32_t)((k - 1) / 2);
                bool positive = ((k - 1) & 1) == 0;
                Ev &e = ev[(size_t)i];
                uint32_t w = find_reliable_v(root, positive, s, k, &e.reads);
                e.reliable = (w != INVALID);
                e.witness = w;
                e.d = descent_leaf_v(positive, s, k);
            }
            mark.assign(count(), UINT64_MAX);
            level.assign(count(), 0);
            std::vector<size_t> commit;
            std::vector<uint64_t> next;
            for (size_t i = 0; i < pending.size(); ++i) {
                uint64_t k = pending[i];
                Ev &e = ev[i];
                bool conflict = false;
                uint32_t lv = 0;
                auto chk = [&](uint32_t x) {
                    if (mark[x] < k) { conflict = true; lv = std::max(lv, level[x] + 1); }
                };
                if (e.reliable) chk(e.witness);
                else { for (uint32_t x : e.reads) chk(x); chk(e.d.idx); }
                if (conflict || !e.reliable) {
                    if (mark[e.d.idx] == UINT64_MAX) mark[e.d.idx] = k;
                    level[e.d.idx] = std::max(level[e.d.idx], lv);
                    max_contagion = std::max<uint64_t>(max_contagion, lv);
                }
                if (conflict) next.push_back(k);
                else if (!e.reliable) { commit.push_back(i); ++writers; }
            }
            for (size_t i : commit) {
                uint64_t k = pending[i];
                apply_sampling(ev[i].d, ((k - 1) & 1) == 0, (uint32_t)((k - 1) / 2), k);
            }
            pending.swap(next);
        }
    }

    int build(int stop_after) {
        compute_root();
        children.clear(); parents.clear(); counts.clear(); starts.clear();
        writers = sampling_splits = 0;
        resize(1);
        double t0 = now();
        // Nodes.cpp:196-229
        for (uint32_t s = 0; s < N; ++s) {
            Scope sc = root;
            while (!find_container(sc, s)) create_children(sc.idx);
            ++counts[sc.idx];
        }
        double t1 = now();
        stage[0] = t1 - t0;
        if (stop_after == 1) return 0;
        if (stop_after >= 4) {
            sampling_rounds();
        } else {
            for (uint32_t s = 0; s < N; ++s) {
                create_for_sampling(root, true, s);
                create_for_sampling(root, false, s);
            }
        }
        double t2 = now();
        stage[1] = t2 - t1;
        if (stop_after == 2 || stop_after == 5) return 0;
        while (balance_pass(0, root)) {}   // Nodes.cpp:339-345
        double t3 = now();
        stage[2] = t3 - t2;
        if (stop_after == 3) return 0;
        reorder_nodes();
        reorder_samples();
        double t4 = now();
        stage[3] = t4 - t3;
        // Leaves.cpp:22-28
        leaves.clear();
        node_to_leaf.assign(count(), INVALID);
        gather(root);
        neighbors();
        double t5 = now();
        stage[4] = t5 - t4;
        cells.clear();
        cells.reserve(leaves.size() * 8);
        dc_node(0);
        stage[5] = now() - t5;
        return 0;
    }

    // ------------------------------------------------------------- occupancy
    // Recursive restatement of LeavesIterator + a NodesChecker
    // (NodesIterator.cpp:17-86, LeavesIterator.cpp:16-31).
    template <class Ignored, class Visit>
    void for_leaves(const Scope &sc, uint32_t depth, uint32_t max_depth, const Ignored &ignored, const Visit &visit) const {
        if (is_leaf(sc.idx)) { visit(sc); return; }
        if (depth + 1 > max_depth) return;
        double cs = sc.size * 0.5;
        for (uint32_t c = 0; c < CHILD_COUNT; ++c) {
            Scope ch = child_scope(sc, c, cs);
            if (ignored(ch, depth + 1)) continue;
            for_leaves(ch, depth + 1, max_depth, ignored, visit);
        }
    }

    // Occupancy.cpp:138-248 for links [first, last), or with `chosen` for the
    // links of the chosen samples (link l: sample chosen[l / K], slot l % K,
    // Occupancy.cpp:262-266); removal negates the kernel values, the cone
    // lengths and the cone count and sets no flags (Occupancy.cpp:210-234,
    // 335-341).
    void update_kernels(int type, uint64_t first, uint64_t last, int prune, const uint32_t *chosen = nullptr,
                        bool removal = false) {
        if (type == EMPTINESS) forward_flag(0, FLAG_SAMPLENESS);
        uint32_t leaf_flag = (type == EMPTINESS) ? FLAG_EMPTINESS : FLAG_SAMPLENESS;
        uint32_t req = (type == EMPTINESS) ? FLAG_SAMPLENESS : 0u;
        double count_sum = 0.0;
        double *ks = ksum[type].data();
        double *cl = clen[type].data();
        uint32_t *st = states.data();
#pragma omp parallel for schedule(dynamic, 128) reduction(+ : count_sum)
        for (int64_t l = (int64_t)first; l < (int64_t)last; ++l) {
            uint32_t s = chosen ? chosen[l / K] : (uint32_t)(l / K);
            uint32_t cam = chosen ? links[(size_t)s * K + (size_t)(l % K)] : links[(size_t)l];
            if (cam == INVALID || cam >= C) continue;   // Occupancy.cpp:250-277
            const V3 &cw = cams[cam];
            V3 normal = neg(nrm[s]);
            const V3 &p = pos[s];
            double kernel_r = h_o * scale[s];
            double cone_len = DBL_MAX_;
            V3 end = p;
            if (type == SAMPLENESS) {
                V3 cs = sub(p, cw);
                double total = len(cs);
                V3 dir = divv(cs, total);
                cone_len = kernel_r * rel_cone;
                end = add(end, mul(dir, cone_len * 0.5));
            }
            Cone cone;
            cone_init(cone, cw, normal, end, kernel_r, cone_len);
            if (cone_degenerated(cone)) continue;
            uint32_t max_depth = MAX_DEPTH_DIFFERENCE + sample_depth(s);   // Occupancy.cpp:518-521
            double c = conf[s];
            double wlen = (removal ? -1.0 : 1.0) * c * cone.length;
            if (type == EMPTINESS) count_sum += removal ? -c : c;
            auto ignored = [&](const Scope &sc, uint32_t depth) {   // ConeNodesChecker.cpp:50-66
                if (depth > max_depth) return true;
                if (req != (req & st[sc.idx])) return true;
                if (!prune) return false;
                return cone_box_separated(cone, sc.mn, sc.size);
            };
            auto visit = [&](const Scope &sc) {
                V3 center = sc.center();
                double val;
                if (!add_kernel(val, center, cone, type == SAMPLENESS, c)) return;
                if (removal) val = -val;
                uint32_t leaf = node_to_leaf[sc.idx];
#pragma omp atomic
                ks[leaf] += val;
#pragma omp atomic
                cl[leaf] += wlen;
                if (!removal) {
#pragma omp atomic
                    st[sc.idx] |= leaf_flag;
                }
            };
            if (!ignored(root, 0)) for_leaves(root, 0, max_depth, ignored, visit);
        }
        if (type == EMPTINESS) cone_count += count_sum;
    }

    // Occupancy.cpp:491-516
    uint32_t forward_flag(uint32_t n, uint32_t flag) {
        uint32_t &state = states[n];
        if (is_leaf(n)) return state;
        state &= ~flag;
        uint32_t c0 = children[n];
        for (uint32_t c = 0; c < CHILD_COUNT; ++c) {
            uint32_t cs = forward_flag(c0 + c, flag);
            if (flag & cs) state |= flag;
        }
        return state;
    }

    // Occupancy.cpp:530-568
    void compute_priors() {
        uint32_t L = (uint32_t)leaves.size();
        const uint32_t *st = states.data();
#pragma omp parallel for schedule(dynamic, 512)
        for (int64_t i = 0; i < (int64_t)L; ++i) {
            const Scope &sc = leaves[(size_t)i];
            V3 center = sc.center();
            double radius = sc.size * prior_rel;
            uint32_t max_depth = depth_of(sc.idx) + MAX_DEPTH_DIFFERENCE;
            double eL = 0.0, sL = 0.0;
            auto ignored = [&](const Scope &s2, uint32_t depth) {   // SphereNodeStatesChecker.cpp:28-36
                if (FLAG_SAMPLENESS != (FLAG_SAMPLENESS & st[s2.idx])) return true;
                if (depth > max_depth) return true;
                return !aabb_sphere(s2.mn, s2.mx(), center, radius);
            };
            auto visit = [&](const Scope &s2) {
                uint32_t leaf = node_to_leaf[s2.idx];
                eL += clen[EMPTINESS][leaf];
                sL += clen[SAMPLENESS][leaf];
            };
            if (!ignored(root, 0)) for_leaves(root, 0, max_depth, ignored, visit);
            prior[(size_t)i] = eL / (eL + sL);
        }
    }

    // Occupancy.cpp:570-587
    double get_occupancy(uint32_t l) const {
        double e = ksum[EMPTINESS][l], s = ksum[SAMPLENESS][l];
        if ((e + s) < conf_thresh) return -EPS;
        double pe = prior[l] * (e / cone_count);
        double ps = (1.0 - prior[l]) * (s / cone_count);
        if (pe >= ps) return -EPS;
        return ps - pe;
    }

    void occupancy_reset() {
        uint32_t L = (uint32_t)leaves.size();
        for (int t = 0; t < 2; ++t) { ksum[t].assign(L, 0.0); clen[t].assign(L, 0.0); }
        prior.assign(L, 0.0);
        states.assign(count(), 0u);
        cone_count = 0.0;
    }

    int occupancy(int nthreads, int prune, uint64_t first, uint64_t cnt) {
#ifdef _OPENMP
        if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
        occupancy_reset();
        uint64_t nl = (uint64_t)N * K;
        uint64_t last = std::min<uint64_t>(nl, first + cnt);
        double t0 = now();
        update_kernels(SAMPLENESS, first, last, prune);
        double t1 = now();
        update_kernels(EMPTINESS, first, last, prune);
        double t2 = now();
        compute_priors();
        double t3 = now();
        stage[6] = t1 - t0; stage[7] = t2 - t1; stage[8] = t3 - t2;
        uint32_t L = (uint32_t)leaves.size();
        occ.resize(L);
        for (uint32_t l = 0; l < L; ++l) occ[l] = get_occupancy(l);
        return 0;
    }

    // Occupancy::addSamples / eraseSamples (Occupancy.h:167-175) ->
    // onSamplesChanged -> update (Occupancy.cpp:129-136, Occupancy.h:222-227):
    // both cone passes over the chosen samples' links, then the priors; the
    // occupancy values follow from the updated sums.
    int update(int nthreads, const uint32_t *chosen, uint32_t count, bool removal) {
#ifdef _OPENMP
        if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
        for (uint32_t i = 0; i < count; ++i)
            if (chosen[i] >= N) return -1;
        const uint64_t nl = (uint64_t)count * K;
        update_kernels(SAMPLENESS, 0, nl, 1, chosen, removal);
        update_kernels(EMPTINESS, 0, nl, 1, chosen, removal);
        compute_priors();
        uint32_t L = (uint32_t)leaves.size();
        occ.resize(L);
        for (uint32_t l = 0; l < L; ++l) occ[l] = get_occupancy(l);
        return 0;
    }

    // ------------------------------------------------------------------- DMC
    // DualMarchingCells.cpp:61-169, DualMarchingCell.cpp:34-101
    int dmc() {
        double t0 = now();
        uint32_t nc = (uint32_t)(cells.size() / 8);
        cases.assign(nc, 0);
        vpos.clear(); vscale.clear(); vkeys.clear(); tris.clear();
        std::map<std::pair<uint32_t, uint32_t>, uint32_t> evi;
        for (uint32_t ci = 0; ci < nc; ++ci) {
            const uint32_t *dc = &cells[(size_t)ci * 8];
            V3 cp[8]; double cd[8], csz[8]; uint32_t cl_[8];
            for (int i = 0; i < 8; ++i) {
                uint32_t leaf = dc[MC_CORNER_REORDERING[i]];
                const Scope &sc = leaves[leaf];
                cp[i] = sc.center();
                cd[i] = occ[leaf];
                csz[i] = sc.size;
                cl_[i] = leaf;
            }
            uint32_t code = 0;
            for (int i = 0; i < 8; ++i) if (cd[i] > 0.0) code |= (1u << i);
            cases[ci] = (uint8_t)code;
            uint32_t cut = mc_edge_cuttings(code);
            if (!cut) continue;
            V3 ip[12]; double is[12];
            for (int e = 0; e < 12; ++e) {
                if (!(cut & (1u << e))) continue;
                int a = MC_EDGE_ENDS[e][0], b = MC_EDGE_ENDS[e][1];
                double f = interpolation_factor(cd[a], cd[b]);
                ip[e] = add(cp[a], mul(sub(cp[b], cp[a]), f));
                is[e] = csz[a] + (csz[b] - csz[a]) * f;
            }
            const int8_t *tri = mc_triangles(code);
            for (int t = 0; tri[t] != -1; t += 3) {
                if (degenerated_triangle(&tri[t], cl_)) continue;
                uint32_t out[3];
                for (int j = 0; j < 3; ++j) {
                    int e = tri[t + j];
                    uint32_t l0 = cl_[MC_EDGE_ENDS[e][0]], l1 = cl_[MC_EDGE_ENDS[e][1]];
                    std::pair<uint32_t, uint32_t> key(std::min(l0, l1), std::max(l0, l1));
                    auto it = evi.find(key);
                    if (it != evi.end()) { out[j] = it->second; continue; }
                    uint32_t vi = (uint32_t)vscale.size();
                    vpos.push_back(ip[e].x); vpos.push_back(ip[e].y); vpos.push_back(ip[e].z);
                    vscale.push_back(is[e]);
                    vkeys.push_back(key.first); vkeys.push_back(key.second);
                    evi.emplace(key, vi);
                    out[j] = vi;
                }
                tris.push_back(out[0]); tris.push_back(out[1]); tris.push_back(out[2]);
            }
        }
        stage[9] = now() - t0;
        return 0;
    }
};

extern "C" {

tsro_scene *tsro_create(uint32_t n, uint32_t k, const double *pos, const double *nrm,
                        const double *scale, const double *conf, const uint32_t *links,
                        uint32_t ncams, const double *cams, const double *params) {
    tsro_scene *s = new tsro_scene();
    s->N = n; s->K = k; s->C = ncams;
    s->pos.resize(n); s->nrm.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        s->pos[i] = V3{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        s->nrm[i] = V3{nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]};
    }
    s->scale.assign(scale, scale + n);
    s->conf.assign(conf, conf + n);
    s->links.assign(links, links + (size_t)n * k);
    s->cams.resize(ncams);
    for (uint32_t i = 0; i < ncams; ++i) s->cams[i] = V3{cams[3 * i], cams[3 * i + 1], cams[3 * i + 2]};
    if (params) {
        s->h_svo = params[0]; s->h_o = params[1]; s->conf_thresh = params[2];
        s->prior_rel = params[3]; s->rel_cone = params[4];
    }
    return s;
}

void tsro_free(tsro_scene *s) { delete s; }

int tsro_build_tree(tsro_scene *s, int stop_after) {
    try { return s->build(stop_after); } catch (const std::exception &) { return -1; }
}

void tsro_counts(const tsro_scene *s, uint64_t *c) {
    c[0] = s->children.size(); c[1] = s->leaves.size(); c[2] = s->cells.size() / 8;
    c[3] = s->nbs.size(); c[4] = s->vscale.size(); c[5] = s->tris.size() / 3;
    c[6] = s->writers; c[7] = s->sampling_splits; c[8] = s->rounds; c[9] = s->max_contagion;
}

void tsro_root(const tsro_scene *s, double *m) {
    m[0] = s->root.mn.x; m[1] = s->root.mn.y; m[2] = s->root.mn.z; m[3] = s->root.size;
}

void tsro_get_nodes(const tsro_scene *s, uint32_t *ch, uint32_t *pa, uint32_t *co, uint32_t *st) {
    size_t n = s->children.size();
    if (ch) std::memcpy(ch, s->children.data(), n * 4);
    if (pa) std::memcpy(pa, s->parents.data(), n * 4);
    if (co) std::memcpy(co, s->counts.data(), n * 4);
    if (st) std::memcpy(st, s->starts.data(), n * 4);
}

void tsro_get_permutation(const tsro_scene *s, uint32_t *t) {
    std::memcpy(t, s->target.data(), s->target.size() * 4);
}

void tsro_get_leaves(const tsro_scene *s, double *ms, uint32_t *ni, uint32_t *n2l, uint32_t *off, uint32_t *nbs) {
    size_t L = s->leaves.size();
    for (size_t i = 0; i < L; ++i) {
        const Scope &sc = s->leaves[i];
        if (ms) { ms[4 * i] = sc.mn.x; ms[4 * i + 1] = sc.mn.y; ms[4 * i + 2] = sc.mn.z; ms[4 * i + 3] = sc.size; }
        if (ni) ni[i] = sc.idx;
    }
    if (n2l) std::memcpy(n2l, s->node_to_leaf.data(), s->node_to_leaf.size() * 4);
    if (off) std::memcpy(off, s->nb_off.data(), s->nb_off.size() * 4);
    if (nbs) std::memcpy(nbs, s->nbs.data(), s->nbs.size() * 4);
}

void tsro_get_dual_cells(const tsro_scene *s, uint32_t *c) {
    std::memcpy(c, s->cells.data(), s->cells.size() * 4);
}

void tsro_get_sample_depths(const tsro_scene *s, uint32_t *d) {
    for (uint32_t i = 0; i < s->N; ++i) d[i] = s->sample_depth(i);
}

int tsro_occupancy(tsro_scene *s, int nthreads, int prune) {
    try { return s->occupancy(nthreads, prune, 0, (uint64_t)s->N * s->K); } catch (const std::exception &) { return -1; }
}

int tsro_occupancy_update(tsro_scene *s, int nthreads, const uint32_t *samples, uint32_t count, int removal) {
    try { return s->update(nthreads, samples, count, removal != 0); } catch (const std::exception &) { return -1; }
}

int tsro_occupancy_links(tsro_scene *s, int nthreads, uint64_t first, uint64_t count) {
    try { return s->occupancy(nthreads, 1, first, count); } catch (const std::exception &) { return -1; }
}

void tsro_get_occupancy(const tsro_scene *s, double *es, double *ss, double *el, double *sl,
                        double *pr, double *oc, uint32_t *st, double *cc) {
    size_t L = s->leaves.size();
    if (es) std::memcpy(es, s->ksum[EMPTINESS].data(), L * 8);
    if (ss) std::memcpy(ss, s->ksum[SAMPLENESS].data(), L * 8);
    if (el) std::memcpy(el, s->clen[EMPTINESS].data(), L * 8);
    if (sl) std::memcpy(sl, s->clen[SAMPLENESS].data(), L * 8);
    if (pr) std::memcpy(pr, s->prior.data(), L * 8);
    if (oc) std::memcpy(oc, s->occ.data(), L * 8);
    if (st) std::memcpy(st, s->states.data(), s->states.size() * 4);
    if (cc) *cc = s->cone_count;
}

int tsro_set_occupancy(tsro_scene *s, const double *occ) {
    s->occ.assign(occ, occ + s->leaves.size());
    return 0;
}

int tsro_dmc(tsro_scene *s) {
    try { return s->dmc(); } catch (const std::exception &) { return -1; }
}

void tsro_get_mesh(const tsro_scene *s, uint8_t *cases, double *vpos, double *vscale, uint32_t *vkeys, uint32_t *tris) {
    if (cases) std::memcpy(cases, s->cases.data(), s->cases.size());
    if (vpos) std::memcpy(vpos, s->vpos.data(), s->vpos.size() * 8);
    if (vscale) std::memcpy(vscale, s->vscale.data(), s->vscale.size() * 8);
    if (vkeys) std::memcpy(vkeys, s->vkeys.data(), s->vkeys.size() * 4);
    if (tris) std::memcpy(tris, s->tris.data(), s->tris.size() * 4);
}

double tsro_stage_seconds(const tsro_scene *s, int stage) {
    return (stage >= 0 && stage < 10) ? s->stage[stage] : 0.0;
}

}  // extern "C"
