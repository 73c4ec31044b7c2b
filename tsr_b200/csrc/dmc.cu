// dmc.cu -- sm_100a dual marching cells of the TSR volumetric core.
//
// Reproduces DualMarchingCells::extractSurfaces (SurfaceExtraction/
// DualMarchingCells.cpp:61-169) with DualMarchingCell::getCuttingsIdx,
// getInterpolationFactor and isDegeneratedTriangle (DualMarchingCell.cpp:
// 34-101) and the EdgeVertexIndex de-duplication (EdgeVertexIndex.cpp:15-33).
//
// The reference walks the cells sequentially and numbers a vertex when an
// undirected leaf pair is first used.  Here every cell is classified in
// parallel, triangle corners are emitted into a compacted array in (cell,
// triangle, corner) order, and a stable radix sort by leaf-pair key finds the
// first use of each pair; ranking the first uses reproduces the sequential
// numbering exactly, and each vertex is interpolated from the corner that
// first used it (FP64, same expression order as the reference).
#include <cub/cub.cuh>

#include "handles.h"
#include "mc_tables.h"

namespace tsr {
namespace {

constexpr unsigned BLK = 256;

__constant__ uint8_t c_reorder[8] = TSR_MC_CORNER_REORDERING_INIT;
__constant__ uint8_t c_ends[12][2] = TSR_MC_EDGE_ENDS_INIT;
__constant__ int8_t c_tris[256][16] = TSR_MC_TRIANGLES_INIT;

__device__ inline bool degenerated(const int8_t *e, const uint32_t *leaf) {
    for (int i = 0; i < 3; ++i)
        if (leaf[c_ends[e[i]][0]] == leaf[c_ends[e[i]][1]]) return true;
    for (int i = 0; i < 3; ++i) {
        const uint8_t *a = c_ends[e[i]];
        const uint8_t *b = c_ends[e[(i + 1) % 3]];
        if (leaf[a[0]] == leaf[b[0]] && leaf[a[1]] == leaf[b[1]]) return true;
        if (leaf[a[0]] == leaf[b[1]] && leaf[a[1]] == leaf[b[0]]) return true;
    }
    return false;
}

__device__ inline void load_cell(const uint32_t *cells, uint32_t c, const double *occ, uint32_t *leaf, uint32_t &code) {
    code = 0;
    for (int i = 0; i < 8; ++i) {
        uint32_t l = cells[8 * (size_t)c + c_reorder[i]];
        leaf[i] = l;
        if (occ[l] > 0.0) code |= 1u << i;
    }
}

__global__ void k_classify(uint32_t nc, const uint32_t *cells, const double *occ, uint8_t *cases, uint32_t *ntri,
                           uint32_t *active) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    uint32_t leaf[8], code;
    load_cell(cells, c, occ, leaf, code);
    cases[c] = (uint8_t)code;
    uint32_t cnt = 0;
    if (code != 0 && code != 255) {
        atomicAdd(active, 1u);
        const int8_t *t = c_tris[code];
        for (int i = 0; t[i] != -1; i += 3)
            if (!degenerated(&t[i], leaf)) ++cnt;
    }
    ntri[c] = cnt;
}

__global__ void k_emit(uint32_t nc, const uint32_t *cells, const double *occ, const uint32_t *toff,
                       uint64_t *keys, uint32_t *vals, uint32_t *ends) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    uint32_t leaf[8], code;
    load_cell(cells, c, occ, leaf, code);
    if (code == 0 || code == 255) return;
    uint32_t slot = toff[c];
    const int8_t *t = c_tris[code];
    for (int i = 0; t[i] != -1; i += 3) {
        if (degenerated(&t[i], leaf)) continue;
        for (int j = 0; j < 3; ++j) {
            int e = t[i + j];
            uint32_t l0 = leaf[c_ends[e][0]], l1 = leaf[c_ends[e][1]];
            uint32_t g = 3 * slot + j;
            uint32_t lo = l0 < l1 ? l0 : l1, hi = l0 < l1 ? l1 : l0;
            keys[g] = ((uint64_t)hi << 32) | lo;   // EdgeVertexIndex ordering: max leaf, then min leaf
            vals[g] = g;
            ends[2 * (size_t)g] = l0;
            ends[2 * (size_t)g + 1] = l1;
        }
        ++slot;
    }
}

__global__ void k_heads(uint32_t m, const uint64_t *skeys, const uint32_t *svals, uint32_t *head,
                        uint32_t *first_use) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    bool h = (i == 0) || (skeys[i] != skeys[i - 1]);
    head[i] = h ? 1u : 0u;
    if (h) first_use[i] = svals[i];
}

__global__ void k_seg_first(uint32_t m, const uint32_t *head, const uint32_t *segid, const uint32_t *svals,
                            uint32_t *seg_first, uint32_t *seg_iota) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || !head[i]) return;
    uint32_t s = segid[i] - 1;   // inclusive scan of heads is 1-based
    seg_first[s] = svals[i];
    seg_iota[s] = s;
}

__global__ void k_rank(uint32_t nv, const uint32_t *order, uint32_t *vert_of_seg) {
    uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < nv) vert_of_seg[order[v]] = v;
}

__global__ void k_tris(uint32_t m, const uint32_t *svals, const uint32_t *segid, const uint32_t *vert_of_seg,
                       uint32_t *tris) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) tris[svals[i]] = vert_of_seg[segid[i] - 1];
}

// DualMarchingCell.cpp:51-71 and DualMarchingCells.cpp:132-151 (FP64)
__device__ inline double interp_factor(double d0, double d1) {
    if (EPS >= fabs(dsub(d1, d0))) return 0.5;
    if (EPS >= fabs(d0)) return 0.0;
    if (EPS >= fabs(d1)) return 1.0;
    return dsub(0.0, d0) / dsub(d1, d0);
}

__global__ void k_vertices(uint32_t nv, const uint32_t *order, const uint32_t *seg_first, const uint32_t *ends,
                           const D3 *leaf_min, const uint32_t *leaf_node, const uint8_t *depth, double root_size,
                           const double *occ, double *vpos, double *vscale, uint32_t *vkeys) {
    uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    uint32_t g = seg_first[order[v]];
    uint32_t l0 = ends[2 * (size_t)g], l1 = ends[2 * (size_t)g + 1];
    double s0 = size_at(root_size, depth[leaf_node[l0]]);
    double s1 = size_at(root_size, depth[leaf_node[l1]]);
    D3 m0 = leaf_min[l0], m1 = leaf_min[l1];
    double h0 = dmul(0.5, s0), h1 = dmul(0.5, s1);
    D3 p0{dadd(m0.x, h0), dadd(m0.y, h0), dadd(m0.z, h0)};
    D3 p1{dadd(m1.x, h1), dadd(m1.y, h1), dadd(m1.z, h1)};
    double f = interp_factor(occ[l0], occ[l1]);
    vpos[3 * (size_t)v + 0] = dadd(p0.x, dmul(dsub(p1.x, p0.x), f));
    vpos[3 * (size_t)v + 1] = dadd(p0.y, dmul(dsub(p1.y, p0.y), f));
    vpos[3 * (size_t)v + 2] = dadd(p0.z, dmul(dsub(p1.z, p0.z), f));
    vscale[v] = dadd(s0, dmul(dsub(s1, s0), f));
    vkeys[2 * (size_t)v] = l0 < l1 ? l0 : l1;
    vkeys[2 * (size_t)v + 1] = l0 < l1 ? l1 : l0;
}

template <class T>
void exscan(const T *in, T *out, uint32_t n, cudaStream_t st) {
    size_t tmp = 0;
    TSR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, st));
    DBuf<uint8_t> t(tmp, st);
    TSR_CUDA(cub::DeviceScan::ExclusiveSum(t.p, tmp, in, out, n, st));
}

template <class K, class V>
void sortp(const K *kin, K *kout, const V *vin, V *vout, uint32_t n, cudaStream_t st) {
    size_t tmp = 0;
    TSR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kin, kout, vin, vout, n, 0, sizeof(K) * 8, st));
    DBuf<uint8_t> t(tmp, st);
    TSR_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, kin, kout, vin, vout, n, 0, sizeof(K) * 8, st));
}

}  // namespace

void extract_dmc(const tsr_tree &t, const tsr_occupancy &o, tsr_mesh &m) {
    cudaStream_t st = m.stream;
    const uint32_t nc = t.n_cells;
    m.n_cells = nc;
    m.cases.alloc(nc, st);
    DBuf<uint32_t> ntri(nc + 1, st), toff(nc + 1, st), active(1, st);
    active.zero();
    TSR_CUDA(cudaMemsetAsync(ntri.p + nc, 0, 4, st));
    if (nc) k_classify<<<grid_for(nc, BLK), BLK, 0, st>>>(nc, t.cells.p, o.occ.p, m.cases.p, ntri.p, active.p); ::tsr::note_launch();
    exscan(ntri.p, toff.p, nc + 1, st);
    uint32_t ntr = read_scalar(toff.p + nc, st);
    m.n_active = read_scalar(active.p, st);
    m.n_tris = ntr;
    uint64_t mc64 = 3ull * ntr;
    if (mc64 >= INVALID) fail(TSR_ERR_OVERFLOW_U32, "too many triangle corners");
    uint32_t mc = (uint32_t)mc64;
    m.tris.alloc(mc, st);
    if (mc == 0) {
        m.n_verts = 0;
        return;
    }
    DBuf<uint64_t> keys(mc, st), skeys(mc, st);
    DBuf<uint32_t> vals(mc, st), svals(mc, st), ends(2ull * mc, st);
    k_emit<<<grid_for(nc, BLK), BLK, 0, st>>>(nc, t.cells.p, o.occ.p, toff.p, keys.p, vals.p, ends.p); ::tsr::note_launch();
    sortp(keys.p, skeys.p, vals.p, svals.p, mc, st);
    DBuf<uint32_t> head(mc, st), segid(mc, st), first(mc, st);
    k_heads<<<grid_for(mc, BLK), BLK, 0, st>>>(mc, skeys.p, svals.p, head.p, first.p); ::tsr::note_launch();
    {
        size_t tmp = 0;
        TSR_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, head.p, segid.p, mc, st));
        DBuf<uint8_t> tb(tmp, st);
        TSR_CUDA(cub::DeviceScan::InclusiveSum(tb.p, tmp, head.p, segid.p, mc, st));
    }
    uint32_t nv = read_scalar(segid.p + mc - 1, st);
    m.n_verts = nv;
    DBuf<uint32_t> seg_first(nv, st), seg_iota(nv, st), sfirst(nv, st), order(nv, st), vert_of_seg(nv, st);
    k_seg_first<<<grid_for(mc, BLK), BLK, 0, st>>>(mc, head.p, segid.p, svals.p, seg_first.p, seg_iota.p); ::tsr::note_launch();
    sortp(seg_first.p, sfirst.p, seg_iota.p, order.p, nv, st);
    k_rank<<<grid_for(nv, BLK), BLK, 0, st>>>(nv, order.p, vert_of_seg.p); ::tsr::note_launch();
    k_tris<<<grid_for(mc, BLK), BLK, 0, st>>>(mc, svals.p, segid.p, vert_of_seg.p, m.tris.p); ::tsr::note_launch();
    m.vpos.alloc(3ull * nv, st);
    m.vscale.alloc(nv, st);
    m.vkeys.alloc(2ull * nv, st);
    k_vertices<<<grid_for(nv, BLK), BLK, 0, st>>>(nv, order.p, seg_first.p, ends.p, t.leaf_min.p, t.leaf_node.p,
                                                 t.depth.p, t.root_size, o.occ.p, m.vpos.p, m.vscale.p, m.vkeys.p); ::tsr::note_launch();
    TSR_CUDA(cudaGetLastError());
}

}  // namespace tsr
