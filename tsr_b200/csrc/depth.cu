// depth.cu -- sm_100a triangulation of a depth map into a mesh whose
// vertices become samples: DepthImage::triangulate and createFlexibleMesh
// (Image/DepthImage.cpp:186-461), FlexibleMesh::findVertexNeighbors
// (FlexibleMesh.cpp:137-171) and Mesh::computeVertexScales (Mesh.cpp:63-123).
//
// The reference walks the 2x2 pixel blocks row by row, emits up to two
// triangles per block and numbers a pixel's vertex when a triangle first
// uses it.  Here every block is classified in parallel, the triangle corners
// are written in (block, triangle, corner) order after a scan, a pixel's
// first use is the smallest corner position naming it (atomicMin), and a scan
// over "this corner is its pixel's first use" ranks the first uses: the
// reference's numbering exactly.  A vertex's neighbour list is kept in the
// order findVertexNeighbors builds it (first appearance over the triangles'
// edges), by two stable radix sorts of the directed edge events, so the mean
// neighbour distance sums in the reference's order.
//
// The camera enters as the two 3x3 matrices the reference computes from its
// PinholeCamera (BaseProject, absent here): hPSToNNRayDirVS = inverse
// viewport x inverse projection, and hPSToNNRayDirWS = that x inverse
// rotation (DepthImage.cpp:189-194).  A homogeneous pixel (x, y, 1) times a
// matrix is taken as a row vector times it.
#include <cub/cub.cuh>

#include "handles.h"

namespace tsr {
namespace {

constexpr unsigned BLK = 256;
constexpr double SQRT_TWO = 1.4142135623730951;     // Math::SQRT_TWO
constexpr double DEPTH_DIFFERENCE_FACTOR = 5.0;     // DepthImage.cpp:25
constexpr uint32_t NONE = 0xFFFFFFFFu;

struct Mat3 {
    double m[9];   // row major: m[3 * i + j]
};

__constant__ uint8_t c_block_tris[4][3] = {{0, 2, 1}, {0, 3, 1}, {0, 2, 3}, {1, 2, 3}};

// (x, y, z) times M: out_j = (x m0j + y m1j) + z m2j
__device__ __forceinline__ void row_times(double x, double y, double z, const Mat3 &M, double *o) {
    for (int j = 0; j < 3; ++j)
        o[j] = __dadd_rn(__dadd_rn(__dmul_rn(x, M.m[j]), __dmul_rn(y, M.m[3 + j])), __dmul_rn(z, M.m[6 + j]));
}

__device__ __forceinline__ double length3(const double *v) {
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(v[0], v[0]), __dmul_rn(v[1], v[1])), __dmul_rn(v[2], v[2])));
}

// DepthImage::triangulateBlock (DepthImage.cpp:218-383) without the output:
// the block's triangles as indices into c_block_tris (0xF: none).
__device__ uint32_t block_triangles(const double *depths, uint32_t W, uint32_t x, uint32_t y, const Mat3 &Mvs) {
    const uint32_t p = W * y + x;
    const double d[4] = {depths[p], depths[p + 1], depths[p + W], depths[p + W + 1]};
    uint32_t mask = 0, avail = 0;
    for (uint32_t i = 0; i < 4; ++i)
        if (!(0.0 >= d[i])) {
            mask |= 1u << i;
            ++avail;
        }
    if (avail < 3) return 0xFFu;
    uint32_t t[2] = {0xFu, 0xFu};
    switch (mask) {
        case 7: t[0] = 0; break;
        case 11: t[0] = 1; break;
        case 13: t[0] = 2; break;
        case 14: t[0] = 3; break;
        case 15:
            if (fabs(__dsub_rn(d[0], d[3])) < fabs(__dsub_rn(d[1], d[2]))) { t[0] = 1; t[1] = 2; }
            else { t[0] = 0; t[1] = 3; }
            break;
        default: return 0xFFu;
    }
    double fp[4] = {0.0, 0.0, 0.0, 0.0};
    for (uint32_t i = 0; i < 4; ++i) {
        if (0.0 >= d[i]) continue;
        double v[3];
        row_times((double)(x + i % 2), (double)(y + i / 2), 1.0, Mvs, v);
        fp[i] = __ddiv_rn(__dmul_rn(Mvs.m[0], d[i]), length3(v));
    }
    for (int k = 0; k < 2; ++k) {
        if (t[k] == 0xFu) continue;
        for (uint32_t e = 0; e < 3; ++e) {   // DepthImage::isDepthDiscontinuity (DepthImage.cpp:385-400)
            const uint32_t v0 = c_block_tris[t[k]][e], v1 = c_block_tris[t[k]][(e + 1) % 3];
            const uint32_t closer = d[v0] < d[v1] ? v0 : v1, further = d[v0] < d[v1] ? v1 : v0;
            const double f = (v0 + v1 == 3) ? __dmul_rn(DEPTH_DIFFERENCE_FACTOR, SQRT_TWO) : DEPTH_DIFFERENCE_FACTOR;
            if (__dsub_rn(d[further], d[closer]) > __dmul_rn(fp[closer], f)) {
                t[k] = 0xFu;
                break;
            }
        }
    }
    return t[0] | (t[1] << 4);
}

__global__ void k_classify_blocks(const double *depths, uint32_t W, uint32_t H, Mat3 Mvs, uint8_t *code,
                                  uint32_t *ntri) {
    const uint32_t bw = W - 1, nb = bw * (H - 1);
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const uint32_t c = block_triangles(depths, W, b % bw, b / bw, Mvs);
    code[b] = (uint8_t)c;
    ntri[b] = ((c & 0xFu) != 0xFu ? 1u : 0u) + ((c >> 4) != 0xFu ? 1u : 0u);
}

// Corner pixels in (block, triangle, corner) order, and every pixel's first
// corner (the smallest corner position naming it).
__global__ void k_emit_corners(uint32_t W, uint32_t H, const uint8_t *code, const uint32_t *toff, uint32_t *corner_pix,
                               uint32_t *first) {
    const uint32_t bw = W - 1, nb = bw * (H - 1);
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const uint32_t c = code[b];
    if (c == 0xFFu) return;
    const uint32_t p = W * (b / bw) + b % bw;
    uint32_t out = 3 * toff[b];
    for (int k = 0; k < 2; ++k) {
        const uint32_t t = (c >> (4 * k)) & 0xFu;
        if (t == 0xFu) continue;
        for (int j = 0; j < 3; ++j) {
            const uint32_t v = c_block_tris[t][j];
            const uint32_t q = p + (v / 2) * W + v % 2;
            corner_pix[out] = q;
            atomicMin(first + q, out);
            ++out;
        }
    }
}

__global__ void k_first_flags(uint32_t nc, const uint32_t *corner_pix, const uint32_t *first, uint32_t *flag) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) flag[c] = first[corner_pix[c]] == c ? 1u : 0u;
}

__global__ void k_pixel_vertices(uint32_t np, const uint32_t *first, const uint32_t *rank, uint32_t *pix2v) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < np) pix2v[p] = first[p] == NONE ? NONE : rank[first[p]];
}

__global__ void k_corner_vertices(uint32_t nc, const uint32_t *corner_pix, const uint32_t *pix2v, uint32_t *tris) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) tris[c] = pix2v[corner_pix[c]];
}

// DepthImage::setVertexPositions / setVertexColors (DepthImage.cpp:402-461)
__global__ void k_depth_vertices(uint32_t W, uint32_t np, const uint32_t *pix2v, const double *depths, Mat3 Mws,
                                 double cx, double cy, double cz, const double *colors, double *pos, double *col) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const uint32_t v = pix2v[p];
    if (v == NONE) return;
    double dir[3];
    row_times((double)(p % W), (double)(p / W), 1.0, Mws, dir);
    const double l = length3(dir);
    if (l > 0.0)
        for (int j = 0; j < 3; ++j) dir[j] = __ddiv_rn(dir[j], l);
    const double dep = depths[p];
    pos[3 * (size_t)v] = __dadd_rn(cx, __dmul_rn(dir[0], dep));
    pos[3 * (size_t)v + 1] = __dadd_rn(cy, __dmul_rn(dir[1], dep));
    pos[3 * (size_t)v + 2] = __dadd_rn(cz, __dmul_rn(dir[2], dep));
    for (int j = 0; j < 3; ++j) col[3 * (size_t)v + j] = colors ? colors[3 * (size_t)p + j] : 0.5;
}

// FlexibleMesh::findVertexNeighbors (FlexibleMesh.cpp:137-171) visits, per
// triangle (i0, i1, i2), the edges (i0, i1), (i1, i2), (i2, i0) and adds each
// end to the other's list unless present: event 6t + 2e is "owner i_e gets
// i_e+1", 6t + 2e + 1 the reverse.
__global__ void k_neighbor_events(uint32_t nt, const uint32_t *tris, uint64_t *key, uint32_t *pos) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 6 * nt) return;
    const uint32_t t = e / 6, r = e - 6 * t, k = r / 2;
    const uint32_t a = tris[3 * t + k], b = tris[3 * t + (k + 1) % 3];
    const uint32_t owner = (r & 1) ? b : a, nb = (r & 1) ? a : b;
    key[e] = ((uint64_t)owner << 32) | nb;
    pos[e] = e;
}

// The first event of each (owner, neighbour) run, keyed by (owner, event).
__global__ void k_first_events(uint32_t ne, const uint64_t *skey, const uint32_t *spos, uint64_t *key2, uint32_t *nb2,
                               uint32_t *flag) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ne) return;
    const bool head = i == 0 || skey[i - 1] != skey[i];
    flag[i] = head ? 1u : 0u;
    key2[i] = head ? ((skey[i] >> 32) << 32) | spos[i] : ~0ull;
    nb2[i] = (uint32_t)skey[i];
}

__global__ void k_count_owners(uint32_t n, const uint64_t *key, uint32_t *cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(cnt + (uint32_t)(key[i] >> 32), 1u);
}

// Mesh::computeAverageDistance (Mesh.cpp:100-123) over the neighbour list in
// findVertexNeighbors order.
__global__ void k_vertex_scales(uint32_t nv, const uint32_t *off, const uint32_t *nbs, const double *pos, double *scale) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const uint32_t b = off[v], e = off[v + 1];
    uint32_t count = e - b;
    double sum = 0.0;
    const double c[3] = {pos[3 * (size_t)v], pos[3 * (size_t)v + 1], pos[3 * (size_t)v + 2]};
    for (uint32_t i = b; i < e; ++i) {
        const uint32_t q = nbs[i];
        if (q == v) {
            --count;
            continue;
        }
        const double d[3] = {__dsub_rn(pos[3 * (size_t)q], c[0]), __dsub_rn(pos[3 * (size_t)q + 1], c[1]),
                             __dsub_rn(pos[3 * (size_t)q + 2], c[2])};
        sum = __dadd_rn(sum, length3(d));
    }
    scale[v] = count == 0 ? -REAL_MAX : __ddiv_rn(sum, (double)count);
}

template <class T>
void excl_scan(const T *in, T *out, uint32_t n, cudaStream_t st) {
    size_t tmp = 0;
    TSR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, st));
    DBuf<uint8_t> t(tmp, st);
    TSR_CUDA(cub::DeviceScan::ExclusiveSum(t.p, tmp, in, out, n, st));
}

template <class K, class V>
void sort_kv(const K *kin, K *kout, const V *vin, V *vout, uint32_t n, cudaStream_t st) {
    size_t tmp = 0;
    TSR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kin, kout, vin, vout, n, 0, (int)sizeof(K) * 8, st));
    DBuf<uint8_t> t(tmp, st);
    TSR_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, kin, kout, vin, vout, n, 0, (int)sizeof(K) * 8, st));
}

}  // namespace

void triangulate_depth(const double *depths_host, uint32_t W, uint32_t H, const double *hps_to_ray_vs,
                       const double *hps_to_ray_ws, const double *center, const double *colors_host, tsr_mesh &m) {
    cudaStream_t st = m.stream;
    const uint64_t np64 = (uint64_t)W * H;
    if (W < 2 || H < 2) fail(TSR_ERR_INVALID_ARG, "a depth map needs at least 2 x 2 pixels");
    // up to 2 triangles per pixel and 6 neighbour events per triangle stay below 2^32
    if (12 * np64 >= NONE) fail(TSR_ERR_OVERFLOW_U32, "depth map too large for 32-bit neighbour event indices");
    const uint32_t np = (uint32_t)np64, nblocks = (W - 1) * (H - 1);
    Mat3 Mvs, Mws;
    for (int i = 0; i < 9; ++i) {
        Mvs.m[i] = hps_to_ray_vs[i];
        Mws.m[i] = hps_to_ray_ws[i];
    }
    DBuf<double> depths(np, st), colors;
    TSR_CUDA(cudaMemcpyAsync(depths.p, depths_host, 8ull * np, cudaMemcpyHostToDevice, st));
    if (colors_host) {
        colors.alloc(3ull * np, st);
        TSR_CUDA(cudaMemcpyAsync(colors.p, colors_host, 24ull * np, cudaMemcpyHostToDevice, st));
    }
    // ---- triangles per block, corners, first uses
    DBuf<uint8_t> code(nblocks, st);
    DBuf<uint32_t> ntri(nblocks + 1, st), toff(nblocks + 1, st), first(np, st);
    TSR_CUDA(cudaMemsetAsync(ntri.p + nblocks, 0, 4, st));
    first.fill_bytes(0xFF);
    k_classify_blocks<<<grid_for(nblocks, BLK), BLK, 0, st>>>(depths.p, W, H, Mvs, code.p, ntri.p); ::tsr::note_launch();
    excl_scan(ntri.p, toff.p, nblocks + 1, st);
    const uint32_t nt = read_scalar(toff.p + nblocks, st), nc = 3 * nt;
    DBuf<uint32_t> corner_pix(nc, st), flag(nc + 1, st), rank(nc + 1, st);
    m.pix2v.alloc(np, st);
    m.width = W;
    m.height = H;
    m.tris.alloc(nc, st);
    if (nt) {
        k_emit_corners<<<grid_for(nblocks, BLK), BLK, 0, st>>>(W, H, code.p, toff.p, corner_pix.p, first.p); ::tsr::note_launch();
        k_first_flags<<<grid_for(nc, BLK), BLK, 0, st>>>(nc, corner_pix.p, first.p, flag.p); ::tsr::note_launch();
    }
    TSR_CUDA(cudaMemsetAsync(flag.p + nc, 0, 4, st));
    excl_scan(flag.p, rank.p, nc + 1, st);
    const uint32_t nv = read_scalar(rank.p + nc, st);
    k_pixel_vertices<<<grid_for(np, BLK), BLK, 0, st>>>(np, first.p, rank.p, m.pix2v.p); ::tsr::note_launch();
    if (nt) k_corner_vertices<<<grid_for(nc, BLK), BLK, 0, st>>>(nc, corner_pix.p, m.pix2v.p, m.tris.p); ::tsr::note_launch();
    m.n_tris = nt;
    m.n_verts = nv;
    m.n_cells = 0;
    // ---- vertex positions and colours
    m.vpos.alloc(3ull * nv, st);
    m.vcol.alloc(3ull * nv, st);
    m.vscale.alloc(nv, st);
    m.vkeys.alloc(2ull * nv, st);
    m.vkeys.fill_bytes(0xFF);
    m.vnrm.alloc(3ull * nv, st);
    m.vnrm.zero();
    k_depth_vertices<<<grid_for(np, BLK), BLK, 0, st>>>(W, np, m.pix2v.p, depths.p, Mws, center[0], center[1], center[2],
                                                        colors.p, m.vpos.p, m.vcol.p); ::tsr::note_launch();
    // ---- normals (createFlexibleMesh: computeNormalsWeightedByAngles)
    angle_weighted_normals(m.tris.p, nt, m.vpos.p, nv, m.vnrm.p, st);
    // ---- neighbour lists in findVertexNeighbors order, scales
    DBuf<uint32_t> noff(nv + 1, st), ncnt(nv + 1, st);
    ncnt.zero();
    DBuf<uint32_t> nbs;
    if (nt) {
        const uint32_t ne = 6 * nt;
        DBuf<uint64_t> key(ne, st), skey(ne, st), key2(ne, st), skey2(ne, st);
        DBuf<uint32_t> pos(ne, st), spos(ne, st), nb2(ne, st), snb2(ne, st), hflag(ne, st);
        k_neighbor_events<<<grid_for(ne, BLK), BLK, 0, st>>>(nt, m.tris.p, key.p, pos.p); ::tsr::note_launch();
        sort_kv(key.p, skey.p, pos.p, spos.p, ne, st);
        k_first_events<<<grid_for(ne, BLK), BLK, 0, st>>>(ne, skey.p, spos.p, key2.p, nb2.p, hflag.p); ::tsr::note_launch();
        sort_kv(key2.p, skey2.p, nb2.p, snb2.p, ne, st);   // non-heads (~0) sort last
        size_t tmp = 0;
        DBuf<uint32_t> nheads(1, st);
        TSR_CUDA(cub::DeviceReduce::Sum(nullptr, tmp, hflag.p, nheads.p, ne, st));
        {
            DBuf<uint8_t> tb(tmp, st);
            TSR_CUDA(cub::DeviceReduce::Sum(tb.p, tmp, hflag.p, nheads.p, ne, st));
        }
        const uint32_t nn = read_scalar(nheads.p, st);
        k_count_owners<<<grid_for(nn, BLK), BLK, 0, st>>>(nn, skey2.p, ncnt.p); ::tsr::note_launch();
        nbs = std::move(snb2);
    }
    excl_scan(ncnt.p, noff.p, nv + 1, st);
    if (nv)
        k_vertex_scales<<<grid_for(nv, BLK), BLK, 0, st>>>(nv, noff.p, nbs.p, m.vpos.p, m.vscale.p); ::tsr::note_launch();
    TSR_CUDA(cudaStreamSynchronize(st));
    TSR_CUDA(cudaGetLastError());
}

}  // namespace tsr
