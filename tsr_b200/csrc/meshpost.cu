// meshpost.cu -- sm_100a post-processing of an extracted surface, the steps
// DualMarchingCells runs after extractMesh (DualMarchingCells.cpp:26-39):
//   1. FlexibleMesh::deleteIsolatedGeometry with IslesEraser (FlexibleMesh.cpp:
//      1411-1556, IslesEraser.cpp:23-205): vertices connected by edges form an
//      isle; isles of fewer than minIsleSize vertices are deleted, and the
//      rest is compacted in order.
//   2. FlexibleMesh::fillHoles (FlexibleMesh.cpp:1580-1931): border edges,
//      oriented like their triangle, are chained into rings; each ring is
//      closed by concentric rings of new vertices down to <= 5 border edges.
//   3. Mesh::computeNormalsWeightedByAngles (Mesh.cpp:145-203).
//
// The mesh's edges are never stored: a radix sort of the 3 corner edges of
// every triangle by (smaller vertex, larger vertex) gives, per edge, its
// triangles (one: a border edge; three or more: the reference throws,
// FlexibleMesh.cpp:1227-1259).  Isles come from a lock-free union-find over
// the sorted edges whose roots are each isle's smallest vertex index -- the
// labels the reference's propagation converges to.  Hole border edges are
// taken in the order a single thread of the reference finds them (edge index
// order, which for border edges is (triangle, corner) order); the reference
// gathers them in an OpenMP loop with a critical section, so there the order
// depends on thread timing.  The rings are then chained by one thread that
// replays the reference's greedy search exactly (FlexibleMesh.cpp:1650-1709:
// the first unused edge, in the current order of the edge list, that starts
// where the ring ends, swapped behind the ring), with a tail-sorted index of
// the border edges in place of its linear scans; border edges are few (tens
// on the benchmark scenes).  One block per ring builds the fill rings level
// by level with the reference's FP64 expression order.
#include <cub/cub.cuh>

#include "handles.h"

namespace tsr {
namespace {

constexpr unsigned BLK = 256;
constexpr unsigned FILL_BLK = 128;
constexpr uint32_t UF_MAX_STEPS = 1u << 26;   // far above any real path length; a bound, not a budget

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t *p) { return *(const volatile uint32_t *)p; }

// Root of x; parents only ever decrease, so the walk ends.  Path halving by
// CAS keeps that property under concurrent writers.
__device__ uint32_t uf_find(uint32_t *parent, uint32_t x, int *err) {
    for (uint32_t step = 0; step < UF_MAX_STEPS; ++step) {
        const uint32_t p = ld_volatile(parent + x);
        if (p == x) return x;
        const uint32_t g = ld_volatile(parent + p);
        if (g != p) atomicCAS(parent + x, p, g);
        x = p;
    }
    atomicExch(err, 2);
    return x;
}

// Hooks the larger root under the smaller one, so every isle's root ends up
// its smallest vertex index.
__device__ void uf_unite(uint32_t *parent, uint32_t a, uint32_t b, int *err) {
    for (uint32_t step = 0; step < UF_MAX_STEPS; ++step) {
        a = uf_find(parent, a, err);
        b = uf_find(parent, b, err);
        if (a == b) return;
        if (a > b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(parent + b, b, a) == b) return;
    }
    atomicExch(err, 2);
}

__global__ void k_edge_keys(uint32_t nc, const uint32_t *tris, uint64_t *keys, uint32_t *vals) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const uint32_t t = c / 3, k = c - 3 * t;
    const uint32_t a = tris[c], b = tris[3 * t + (k == 2 ? 0 : k + 1)];
    keys[c] = ((uint64_t)min(a, b) << 32) | max(a, b);
    vals[c] = c;
}

__global__ void k_iota_u32(uint32_t n, uint32_t *x) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = i;
}

// One thread per sorted corner edge; the first of each run of equal keys
// classifies the edge and joins its vertices' isles.
__global__ void k_edge_runs(uint32_t nc, const uint64_t *skeys, const uint32_t *svals, uint8_t *border,
                            uint32_t *parent, int *err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    const uint64_t key = skeys[i];
    if (i > 0 && skeys[i - 1] == key) return;
    uint32_t run = 1;
    if (i + 1 < nc && skeys[i + 1] == key) ++run;
    if (i + 2 < nc && skeys[i + 2] == key) ++run;
    if (run >= 3) atomicExch(err, 1);
    if (run == 1) border[svals[i]] = 1;
    uf_unite(parent, (uint32_t)(key >> 32), (uint32_t)key, err);
}

__global__ void k_labels(uint32_t nv, uint32_t *parent, uint32_t *label, uint32_t *size, int *err) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const uint32_t r = uf_find(parent, v, err);
    label[v] = r;
    atomicAdd(size + r, 1u);
}

__global__ void k_keep_vertices(uint32_t nv, const uint32_t *label, const uint32_t *size, uint32_t min_size,
                                uint32_t *keep, uint32_t *any_small) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const bool small = size[label[v]] < min_size;
    keep[v] = small ? 0u : 1u;
    if (small && label[v] == v) atomicOr(any_small, 1u);
}

// A triangle's corners share one isle, so its first corner decides.
__global__ void k_keep_triangles(uint32_t nt, const uint32_t *tris, const uint32_t *keepv, uint32_t *keept) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nt) keept[t] = keepv[tris[3 * t]];
}

__global__ void k_compact_vertices(uint32_t nv, const uint32_t *keep, const uint32_t *vnew, const double *pos,
                                   const double *scale, const uint32_t *vkeys, double *pos2, double *scale2,
                                   uint32_t *vkeys2) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv || !keep[v]) return;
    const uint32_t d = vnew[v];
    for (int j = 0; j < 3; ++j) pos2[3 * (size_t)d + j] = pos[3 * (size_t)v + j];
    scale2[d] = scale[v];
    vkeys2[2 * (size_t)d] = vkeys[2 * (size_t)v];
    vkeys2[2 * (size_t)d + 1] = vkeys[2 * (size_t)v + 1];
}

__global__ void k_compact_triangles(uint32_t nt, const uint32_t *keept, const uint32_t *tnew, const uint32_t *vnew,
                                    const uint32_t *tris, const uint8_t *border, uint32_t *tris2, uint8_t *border2) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt || !keept[t]) return;
    const uint32_t d = tnew[t];
    for (int k = 0; k < 3; ++k) {
        tris2[3 * (size_t)d + k] = vnew[tris[3 * (size_t)t + k]];
        border2[3 * (size_t)d + k] = border[3 * (size_t)t + k];
    }
}

// Border edge j as its triangle passes it (Triangle::getVerticesInWindingOrder).
__global__ void k_border_edges(uint32_t nb, const uint32_t *corners, const uint32_t *tris, uint32_t *tail,
                               uint32_t *head) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nb) return;
    const uint32_t c = corners[j], t = c / 3, k = c - 3 * t;
    tail[j] = tris[c];
    head[j] = tris[3 * t + (k == 2 ? 0 : k + 1)];
}

struct RingOut {
    uint32_t rings, holes, skipped, add_v, add_t;
};

__device__ __forceinline__ void fill_counts(uint32_t n, uint32_t &va, uint32_t &ta) {
    va = 0;
    ta = 0;
    uint32_t s = n;
    while (s > 5) {
        const uint32_t a = s / 2;
        va += a;
        ta += s + a;
        s = a;
    }
    ta += s - 2;
}

// FlexibleMesh::findBorderRings / findBorderRing / extendBorderRing /
// removeDuplicatesInRings (FlexibleMesh.cpp:1617-1732), replayed by one
// thread.  order[] is the current order of the edge list (position -> edge),
// pos[] its inverse; the candidates that continue a ring at vertex v are the
// unused edges starting at v (stails/sids: edges sorted by tail, stable), and
// the reference takes the one at the smallest current position.  A set that
// cannot be closed stays one ring, as in the reference.  Ring vertices are
// the edge tails in ring order; rings of fewer than 3 vertices are counted
// and not filled (the reference reads past them, FlexibleMesh.cpp:1905-1916).
__global__ void k_rings(uint32_t nb, const uint32_t *tail, const uint32_t *head, const uint32_t *stails,
                        const uint32_t *sids, uint32_t *order, uint32_t *pos, uint8_t *used, uint32_t *ring_start,
                        uint32_t *ring_len, uint32_t *ring_verts, uint32_t *ring_vofs, uint32_t *ring_tofs,
                        RingOut *out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (uint32_t j = 0; j < nb; ++j) {
        order[j] = j;
        pos[j] = j;
        used[j] = 0;
    }
    uint32_t rings = 0, holes = 0, skipped = 0, add_v = 0, add_t = 0, s0 = 0;
    while (s0 < nb) {
        const uint32_t start = tail[order[s0]];
        used[order[s0]] = 1;
        uint32_t r = s0 + 1;
        bool closed = false;
        while (r < nb) {
            const uint32_t end = head[order[r - 1]];
            // edges starting at `end`: lower bound in the tail-sorted index
            uint32_t lo = 0, hi = nb;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (stails[mid] < end) lo = mid + 1; else hi = mid;
            }
            uint32_t best = 0xFFFFFFFFu;
            for (uint32_t q = lo; q < nb && stails[q] == end; ++q) {
                const uint32_t id = sids[q];
                if (!used[id] && pos[id] < best) best = pos[id];
            }
            if (best == 0xFFFFFFFFu) break;
            const uint32_t id = order[best], other = order[r];
            order[r] = id;
            pos[id] = r;
            order[best] = other;
            pos[other] = best;
            used[id] = 1;
            ++r;
            if (head[id] == start) {
                closed = true;
                break;
            }
        }
        const uint32_t stop = closed ? r : nb;   // an unclosed set stays whole
        const uint32_t n = stop - s0;
        ring_start[rings] = s0;
        ring_len[rings] = n;
        for (uint32_t p = s0; p < stop; ++p) ring_verts[p] = tail[order[p]];
        uint32_t va = 0, ta = 0;
        if (n >= 3) {
            fill_counts(n, va, ta);
            ++holes;
        } else {
            ++skipped;
        }
        ring_vofs[rings] = add_v;
        ring_tofs[rings] = add_t;
        add_v += va;
        add_t += ta;
        ++rings;
        s0 = stop;
    }
    out->rings = rings;
    out->holes = holes;
    out->skipped = skipped;
    out->add_v = add_v;
    out->add_t = add_t;
}

struct RingView {
    const uint32_t *verts;   // explicit border ring, or null for consecutive new vertices
    uint32_t base;
    __device__ __forceinline__ uint32_t operator()(uint32_t j) const { return verts ? verts[j] : base + j; }
};

// FlexibleMesh::fillHoles(rings) / fillHole / createHoleFillingRingVertices /
// connectHoleFillingRings (FlexibleMesh.cpp:1734-1931), one block per ring.
__global__ void __launch_bounds__(FILL_BLK)
k_fill(const uint32_t *ring_start, const uint32_t *ring_len, const uint32_t *ring_verts, const uint32_t *ring_vofs,
       const uint32_t *ring_tofs, uint32_t nv0, uint32_t nt0, double *vpos, uint32_t *tris) {
    const uint32_t r = blockIdx.x;
    uint32_t n = ring_len[r];
    if (n < 3) return;
    __shared__ double center[3];
    RingView R{ring_verts + ring_start[r], 0};
    if (threadIdx.x == 0) {
        double c[3] = {0.0, 0.0, 0.0};
        for (uint32_t j = 0; j < n; ++j)
            for (int d = 0; d < 3; ++d) c[d] = __dadd_rn(c[d], vpos[3 * (size_t)R(j) + d]);
        for (int d = 0; d < 3; ++d) center[d] = __ddiv_rn(c[d], (double)n);
    }
    __syncthreads();
    uint32_t cur_v = nv0 + ring_vofs[r], cur_t = nt0 + ring_tofs[r];
    while (n > 5) {
        const uint32_t a = n / 2;
        const bool odd = (n & 1u) != 0;
        const uint32_t rl = 31u - (uint32_t)__clz((int)n);   // remaining ring count: bit length - 1
        const double f0 = __ddiv_rn((double)(rl - 1u), (double)rl);
        const double f1 = (double)__fdiv_rn(1.0f, (float)rl);   // a float division in the reference
        const double s = __ddiv_rn(f0, 3.0);
        for (uint32_t i = threadIdx.x; i < a; i += blockDim.x) {
            const uint32_t v0 = R(2 * i), v1 = R(2 * i + 1), v2 = (i == a - 1) ? R(0) : R(2 * i + 2);
            const size_t dst = 3 * (size_t)(cur_v + i);
            for (int d = 0; d < 3; ++d) {
                const double p = __dadd_rn(__dadd_rn(vpos[3 * (size_t)v0 + d], vpos[3 * (size_t)v1 + d]),
                                           vpos[3 * (size_t)v2 + d]);
                vpos[dst + d] = __dadd_rn(__dmul_rn(p, s), __dmul_rn(center[d], f1));
            }
            const uint32_t o2 = (!odd && i == a - 1) ? R(0) : R(2 * i + 2);
            uint32_t *t0 = tris + 3 * (size_t)(cur_t + 2 * i);
            t0[0] = v0; t0[1] = v1; t0[2] = cur_v + i;
            t0[3] = v1; t0[4] = o2; t0[5] = cur_v + i;
            uint32_t *ti = tris + 3 * (size_t)(cur_t + 2 * a + (odd ? 1 : 0) + i);
            ti[0] = cur_v + i;
            ti[1] = (i + 1 == a) ? R(0) : R(2 * (i + 1));
            ti[2] = (i + 1 == a) ? cur_v : cur_v + i + 1;
        }
        if (odd && threadIdx.x == 0) {
            uint32_t *to = tris + 3 * (size_t)(cur_t + 2 * a);
            to[0] = R(n - 1); to[1] = R(0); to[2] = cur_v + a - 1;
        }
        __syncthreads();   // this level's positions are read by the next one
        R = RingView{nullptr, cur_v};
        cur_t += n + a;
        cur_v += a;
        n = a;
    }
    if (threadIdx.x == 0) {   // FlexibleMesh::fillHole(borderVertices, <= 5)
        uint32_t *t = tris + 3 * (size_t)cur_t;
        t[0] = R(0); t[1] = R(1); t[2] = R(2);
        if (n >= 4) { t[3] = R(2); t[4] = R(3); t[5] = R(0); }
        if (n == 5) { t[6] = R(3); t[7] = R(4); t[8] = R(0); }
    }
}

__device__ __forceinline__ void norm3(double *v) {
    const double l = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(v[0], v[0]), __dmul_rn(v[1], v[1])), __dmul_rn(v[2], v[2])));
    if (l > 0.0)
        for (int d = 0; d < 3; ++d) v[d] = __ddiv_rn(v[d], l);
}

__device__ __forceinline__ double dot3(const double *a, const double *b) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1])), __dmul_rn(a[2], b[2]));
}

// Mesh::computeNormalsWeightedByAngles (Mesh.cpp:145-203): every triangle adds
// its unit normal times the corner angle to its three vertices.
__global__ void k_angle_normals(uint32_t nt, const uint32_t *tris, const double *vpos, double *nrm) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const uint32_t i0 = tris[3 * (size_t)t], i1 = tris[3 * (size_t)t + 1], i2 = tris[3 * (size_t)t + 2];
    double p0[3], p1[3], p2[3];
    for (int d = 0; d < 3; ++d) {
        p0[d] = vpos[3 * (size_t)i0 + d];
        p1[d] = vpos[3 * (size_t)i1 + d];
        p2[d] = vpos[3 * (size_t)i2 + d];
    }
    double d0[3], d1[3], d2[3], n[3];
    for (int d = 0; d < 3; ++d) {
        d0[d] = __dsub_rn(p1[d], p0[d]);
        d1[d] = __dsub_rn(p2[d], p1[d]);
        d2[d] = __dsub_rn(p2[d], p0[d]);
    }
    n[0] = __dsub_rn(__dmul_rn(d0[1], d2[2]), __dmul_rn(d0[2], d2[1]));
    n[1] = __dsub_rn(__dmul_rn(d0[2], d2[0]), __dmul_rn(d0[0], d2[2]));
    n[2] = __dsub_rn(__dmul_rn(d0[0], d2[1]), __dmul_rn(d0[1], d2[0]));
    norm3(d0);
    norm3(d1);
    norm3(d2);
    norm3(n);
    const double md2[3] = {-d2[0], -d2[1], -d2[2]};
    const double c[3] = {dot3(d0, d2), -dot3(d0, d1), -dot3(d1, md2)};
    const uint32_t idx[3] = {i0, i1, i2};
    for (int k = 0; k < 3; ++k) {
        const double ang = acos(fmin(1.0, fmax(-1.0, c[k])));
        for (int d = 0; d < 3; ++d) atomicAdd(nrm + 3 * (size_t)idx[k] + d, __dmul_rn(n[d], ang));
    }
}

__global__ void k_normalize(uint32_t nv, double *nrm) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < nv) norm3(nrm + 3 * (size_t)v);
}

template <class T>
void excl_scan(const T *in, T *out, uint32_t n, cudaStream_t st) {
    size_t tmp = 0;
    TSR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, st));
    DBuf<uint8_t> t(tmp, st);
    TSR_CUDA(cub::DeviceScan::ExclusiveSum(t.p, tmp, in, out, n, st));
}

template <class K, class V>
void sort_kv(const K *kin, K *kout, const V *vin, V *vout, uint32_t n, int bits, cudaStream_t st) {
    size_t tmp = 0;
    TSR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kin, kout, vin, vout, n, 0, bits, st));
    DBuf<uint8_t> t(tmp, st);
    TSR_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, kin, kout, vin, vout, n, 0, bits, st));
}

int bits_for(uint32_t maxval) {
    int b = 1;
    while (b < 32 && (maxval >> b)) ++b;
    return b;
}

}  // namespace

// Mesh::computeNormalsWeightedByAngles (Mesh.cpp:145-203) into nrm, which
// must hold zeros.
void angle_weighted_normals(const uint32_t *tris, uint32_t nt, const double *pos, uint32_t nv, double *nrm,
                            cudaStream_t st) {
    if (nt) k_angle_normals<<<grid_for(nt, BLK), BLK, 0, st>>>(nt, tris, pos, nrm); ::tsr::note_launch();
    if (nv) k_normalize<<<grid_for(nv, BLK), BLK, 0, st>>>(nv, nrm); ::tsr::note_launch();
}

void postprocess_mesh(tsr_mesh &m, uint32_t min_isle_size, tsr_mesh_post_counts &pc) {
    cudaStream_t st = m.stream;
    pc = tsr_mesh_post_counts{};
    const uint32_t nv = (uint32_t)m.n_verts, nt = (uint32_t)m.n_tris;
    const uint64_t nc64 = 3ull * nt;
    if (nc64 >= INVALID) fail(TSR_ERR_OVERFLOW_U32, "too many triangle corners");
    const uint32_t nc = (uint32_t)nc64;
    // ---- edges, isles (IslesEraser::computeVerticesToIsles)
    DBuf<uint8_t> border(nc, st);
    border.zero();
    DBuf<uint32_t> parent(nv, st), label(nv, st), size(nv, st), keepv(nv + 1, st), vnew(nv + 1, st);
    DBuf<int> err(1, st);
    err.zero();
    DBuf<uint32_t> flag(1, st);
    flag.zero();
    if (nv) {
        k_iota_u32<<<grid_for(nv, BLK), BLK, 0, st>>>(nv, parent.p); ::tsr::note_launch();
        size.zero();
    }
    if (nc) {
        DBuf<uint64_t> keys(nc, st), skeys(nc, st);
        DBuf<uint32_t> vals(nc, st), svals(nc, st);
        k_edge_keys<<<grid_for(nc, BLK), BLK, 0, st>>>(nc, m.tris.p, keys.p, vals.p); ::tsr::note_launch();
        sort_kv(keys.p, skeys.p, vals.p, svals.p, nc, 64, st);
        k_edge_runs<<<grid_for(nc, BLK), BLK, 0, st>>>(nc, skeys.p, svals.p, border.p, parent.p, err.p); ::tsr::note_launch();
    }
    if (nv) {
        k_labels<<<grid_for(nv, BLK), BLK, 0, st>>>(nv, parent.p, label.p, size.p, err.p); ::tsr::note_launch();
        k_keep_vertices<<<grid_for(nv, BLK), BLK, 0, st>>>(nv, label.p, size.p, min_isle_size, keepv.p, flag.p); ::tsr::note_launch();
    }
    const int e = read_scalar(err.p, st);
    if (e == 1) fail(TSR_ERR_STATE, "an edge is shared by more than two triangles (FlexibleMesh.cpp:1227-1259 throws)");
    if (e) fail(TSR_ERR_DEVICE_ASSERT, "isle search exceeded its step bound");
    const bool any_small = read_scalar(flag.p, st) != 0;

    // ---- deleteGeometry: order-keeping compaction (FlexibleMesh.cpp:1428-1556).
    // The mesh itself is replaced only at the very end, so a failure on the
    // way leaves it as it was.
    uint32_t nvk = nv, ntk = nt;
    DBuf<uint32_t> tris_k, vkeys_k;
    DBuf<uint8_t> border_k;
    DBuf<double> pos_k, scale_k;
    const double *pos_p = m.vpos.p, *scale_p = m.vscale.p;
    const uint32_t *vkeys_p = m.vkeys.p, *tris_p = m.tris.p;
    const uint8_t *border_p = border.p;
    if (any_small) {
        DBuf<uint32_t> keept(nt + 1, st), tnew(nt + 1, st);
        TSR_CUDA(cudaMemsetAsync(keepv.p + nv, 0, 4, st));
        excl_scan(keepv.p, vnew.p, nv + 1, st);
        if (nt) k_keep_triangles<<<grid_for(nt, BLK), BLK, 0, st>>>(nt, m.tris.p, keepv.p, keept.p); ::tsr::note_launch();
        TSR_CUDA(cudaMemsetAsync(keept.p + nt, 0, 4, st));
        excl_scan(keept.p, tnew.p, nt + 1, st);
        nvk = read_scalar(vnew.p + nv, st);
        ntk = read_scalar(tnew.p + nt, st);
        pos_k.alloc(3ull * nvk, st);
        scale_k.alloc(nvk, st);
        vkeys_k.alloc(2ull * nvk, st);
        tris_k.alloc(3ull * ntk, st);
        border_k.alloc(3ull * ntk, st);
        if (nv)
            k_compact_vertices<<<grid_for(nv, BLK), BLK, 0, st>>>(nv, keepv.p, vnew.p, m.vpos.p, m.vscale.p, m.vkeys.p,
                                                                 pos_k.p, scale_k.p, vkeys_k.p); ::tsr::note_launch();
        if (nt)
            k_compact_triangles<<<grid_for(nt, BLK), BLK, 0, st>>>(nt, keept.p, tnew.p, vnew.p, m.tris.p, border.p,
                                                                  tris_k.p, border_k.p); ::tsr::note_launch();
        pos_p = pos_k.p;
        scale_p = scale_k.p;
        vkeys_p = vkeys_k.p;
        tris_p = tris_k.p;
        border_p = border_k.p;
        pc.isle_vertices = nv - nvk;
        pc.isle_triangles = nt - ntk;
    }

    RingOut ro{0, 0, 0, 0, 0};
    DBuf<uint32_t> ring_start, ring_len, ring_verts, ring_vofs, ring_tofs;
    // DualMarchingCells.cpp:32-33: with no vertex or no triangle left, no
    // holes are filled and no normals computed
    const bool rest = nvk != 0 && ntk != 0;
    if (rest) {
        // ---- hole border edges in (triangle, corner) order, and their rings
        const uint32_t nck = 3 * ntk;
        DBuf<uint32_t> corners(nck, st), nsel(1, st), ids(nck, st);
        k_iota_u32<<<grid_for(nck, BLK), BLK, 0, st>>>(nck, ids.p); ::tsr::note_launch();
        {
            size_t tmp = 0;
            TSR_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, ids.p, border_p, corners.p, nsel.p, (int)nck, st));
            DBuf<uint8_t> tb(tmp, st);
            TSR_CUDA(cub::DeviceSelect::Flagged(tb.p, tmp, ids.p, border_p, corners.p, nsel.p, (int)nck, st));
        }
        const uint32_t nb = read_scalar(nsel.p, st);
        pc.border_edges = nb;
        if (nb) {
            DBuf<uint32_t> tail(nb, st), head(nb, st), stails(nb, st), sids(nb, st), iota(nb, st), order(nb, st),
                posn(nb, st);
            DBuf<uint8_t> used(nb, st);
            ring_start.alloc(nb, st); ring_len.alloc(nb, st); ring_verts.alloc(nb, st);
            ring_vofs.alloc(nb, st); ring_tofs.alloc(nb, st);
            DBuf<RingOut> out(1, st);
            k_border_edges<<<grid_for(nb, BLK), BLK, 0, st>>>(nb, corners.p, tris_p, tail.p, head.p); ::tsr::note_launch();
            k_iota_u32<<<grid_for(nb, BLK), BLK, 0, st>>>(nb, iota.p); ::tsr::note_launch();
            sort_kv(tail.p, stails.p, iota.p, sids.p, nb, bits_for(nvk), st);
            k_rings<<<1, 1, 0, st>>>(nb, tail.p, head.p, stails.p, sids.p, order.p, posn.p, used.p, ring_start.p,
                                     ring_len.p, ring_verts.p, ring_vofs.p, ring_tofs.p, out.p); ::tsr::note_launch();
            ro = read_scalar(out.p, st);
        }
        pc.holes = ro.holes;
        pc.skipped_rings = ro.skipped;
        pc.hole_vertices = ro.add_v;
        pc.hole_triangles = ro.add_t;
    }

    // ---- final arrays: kept elements, then every ring's fill in ring order
    const uint64_t nv2_64 = (uint64_t)nvk + ro.add_v, nt2_64 = (uint64_t)ntk + ro.add_t;
    if (nv2_64 >= INVALID || 3 * nt2_64 >= INVALID) fail(TSR_ERR_OVERFLOW_U32, "filled mesh exceeds 32-bit indices");
    const uint32_t nv2 = (uint32_t)nv2_64, nt2 = (uint32_t)nt2_64;
    DBuf<double> pos2, scale2, nrm(3ull * nv2, st);
    DBuf<uint32_t> vkeys2, tris2;
    const bool grow = ro.add_v || ro.add_t;
    if (grow) {
        pos2.alloc(3ull * nv2, st);
        scale2.alloc(nv2, st);
        vkeys2.alloc(2ull * nv2, st);
        tris2.alloc(3ull * nt2, st);
        TSR_CUDA(cudaMemcpyAsync(pos2.p, pos_p, 24ull * nvk, cudaMemcpyDeviceToDevice, st));
        TSR_CUDA(cudaMemcpyAsync(scale2.p, scale_p, 8ull * nvk, cudaMemcpyDeviceToDevice, st));
        TSR_CUDA(cudaMemcpyAsync(vkeys2.p, vkeys_p, 8ull * nvk, cudaMemcpyDeviceToDevice, st));
        TSR_CUDA(cudaMemcpyAsync(tris2.p, tris_p, 12ull * ntk, cudaMemcpyDeviceToDevice, st));
        if (ro.add_v) {
            TSR_CUDA(cudaMemsetAsync(scale2.p + nvk, 0, 8ull * ro.add_v, st));
            TSR_CUDA(cudaMemsetAsync(vkeys2.p + 2ull * nvk, 0xFF, 8ull * ro.add_v, st));
        }
        k_fill<<<ro.rings, FILL_BLK, 0, st>>>(ring_start.p, ring_len.p, ring_verts.p, ring_vofs.p, ring_tofs.p, nvk,
                                              ntk, pos2.p, tris2.p); ::tsr::note_launch();
        pos_p = pos2.p;
        tris_p = tris2.p;
    }
    // ---- normals (Mesh.cpp:145-203); zeros when nothing is left
    nrm.zero();
    if (rest) angle_weighted_normals(tris_p, nt2, pos_p, nv2, nrm.p, st);
    TSR_CUDA(cudaStreamSynchronize(st));   // every step ran: from here on nothing can fail
    if (grow) {
        m.vpos = std::move(pos2);
        m.vscale = std::move(scale2);
        m.vkeys = std::move(vkeys2);
        m.tris = std::move(tris2);
    } else if (any_small) {
        m.vpos = std::move(pos_k);
        m.vscale = std::move(scale_k);
        m.vkeys = std::move(vkeys_k);
        m.tris = std::move(tris_k);
    }
    m.vnrm = std::move(nrm);
    m.n_verts = nv2;
    m.n_tris = nt2;
    // a depth-map mesh's colours and pixel map describe the old vertices
    m.vcol.release();
    m.pix2v.release();
    m.width = m.height = 0;
}

}  // namespace tsr
