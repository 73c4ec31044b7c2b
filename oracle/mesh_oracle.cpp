// mesh_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the FP64 CPU restatement of
// the mesh post-processing DualMarchingCells runs after extracting a mesh
// (DualMarchingCells.cpp:26-39): FlexibleMesh::deleteIsolatedGeometry with
// IslesEraser, FlexibleMesh::fillHoles and
// Mesh::computeNormalsWeightedByAngles; and of the depth-map triangulation
// that creates samples (DepthImage::triangulate, DepthImage.cpp:186-461).
// It is the parity checker of the GPU versions and nothing else; only tests/
// load it.
//
// Paths below are relative to SurfaceReconstruction/SurfaceReconstruction/
// of the reference.  The reference's Vector3 (BaseProject, absent from the
// reference tree) is restated as componentwise double arithmetic with
// division for `/=` and `normalize` = division by the Euclidean length; a
// zero-length vector is left zero.  PARITY UNPINNED: no reference-produced
// output backs this restatement (the reference does not build here).
//
// The reference gathers hole border edges inside an OpenMP parallel loop
// with a critical section (FlexibleMesh.cpp:1586-1609), so their order -- and
// with it which ring is filled first and which vertex a ring starts at --
// depends on thread timing.  This restatement uses the order a single
// thread gives (edge index order), which is the order the GPU reproduces.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace {

constexpr uint32_t INVALID = 0xFFFFFFFFu;

struct V3 {
    double x = 0, y = 0, z = 0;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline void normalize(V3 &a) {
    const double l = std::sqrt(dot(a, a));
    if (l > 0) a = {a.x / l, a.y / l, a.z / l};
}

// Edge.h: the two vertices (smaller first) and up to two triangles.
struct Edge {
    uint32_t v[2];
    uint32_t t[2];
};

struct Mesh {
    std::vector<V3> pos, nrm;
    std::vector<double> scale;
    std::vector<uint32_t> tri;               // 3 per triangle
    std::vector<Edge> edges;
    std::vector<std::vector<uint32_t>> v2e;  // mVerticesToEdges
    int error = 0;                           // 1: edge conflict (FlexibleMesh.cpp:1227-1259 throws)
    // statistics
    uint32_t isle_vertices = 0, isle_triangles = 0, border_edges = 0, holes = 0;
    uint32_t hole_vertices = 0, hole_triangles = 0, skipped_rings = 0;

    uint32_t nv() const { return (uint32_t)pos.size(); }
    uint32_t nt() const { return (uint32_t)(tri.size() / 3); }

    // FlexibleMesh::getEdgeIndex (FlexibleMesh.cpp:1110-1126)
    uint32_t edge_index(uint32_t a, uint32_t b) const {
        for (uint32_t e : v2e[a]) {
            const Edge &E = edges[e];
            if ((E.v[0] == a && E.v[1] == b) || (E.v[0] == b && E.v[1] == a)) return e;
        }
        return INVALID;
    }

    // FlexibleMesh::addEdge / createEdge / addEdgeConflict (FlexibleMesh.cpp:1184-1259)
    void add_edge(uint32_t t, uint32_t local) {
        const uint32_t a = tri[3 * t + local], b = tri[3 * t + (local + 1) % 3];
        const uint32_t v0 = a < b ? a : b, v1 = a < b ? b : a;
        const uint32_t e = edge_index(v0, v1);
        if (e == INVALID) {
            const uint32_t n = (uint32_t)edges.size();
            v2e[v0].push_back(n);
            v2e[v1].push_back(n);
            edges.push_back(Edge{{v0, v1}, {t, INVALID}});
            return;
        }
        if (edges[e].t[1] == INVALID) {
            edges[e].t[1] = t;
            return;
        }
        error = 1;
    }

    // FlexibleMesh::findAdjacencies (FlexibleMesh.cpp:1137-1156)
    void find_adjacencies() {
        edges.clear();
        v2e.assign(nv(), {});
        for (uint32_t t = 0; t < nt(); ++t)
            for (uint32_t e = 0; e < 3; ++e) add_edge(t, e);
    }

    void add_triangle(uint32_t a, uint32_t b, uint32_t c) {
        tri.push_back(a);
        tri.push_back(b);
        tri.push_back(c);
        ++hole_triangles;
    }
};

// IslesEraser (IslesEraser.cpp:23-205): vertices connected by edges form an
// isle; an isle with fewer than minIsleSize vertices is deleted.  The
// reference converges its parallel label propagation to the smallest vertex
// index of each isle; a union-find with the same labels restates it.
bool isle_offsets(const Mesh &m, uint32_t min_size, std::vector<uint32_t> &vdoom, std::vector<uint32_t> &edoom,
                  std::vector<uint32_t> &tdoom) {
    const uint32_t nv = m.nv();
    std::vector<uint32_t> parent(nv);
    std::iota(parent.begin(), parent.end(), 0u);
    auto find = [&](uint32_t x) {
        while (parent[x] != x) x = parent[x] = parent[parent[x]];
        return x;
    };
    for (const Edge &e : m.edges) {
        uint32_t a = find(e.v[0]), b = find(e.v[1]);
        if (a == b) continue;
        if (a < b) parent[b] = a; else parent[a] = b;
    }
    std::vector<uint32_t> size(nv, 0), label(nv);
    for (uint32_t v = 0; v < nv; ++v) ++size[label[v] = find(v)];
    bool small = false;   // IslesEraser::hasFoundTooSmallIsle
    for (uint32_t v = 0; v < nv; ++v)
        if (label[v] == v && size[v] < min_size) small = true;
    if (!small) return false;
    // FlexibleMesh::computeOffsetsForFiltering (FlexibleMesh.cpp:25-104)
    vdoom.assign(nv, 0);
    edoom.assign(m.edges.size(), 0);
    tdoom.assign(m.nt(), 0);
    for (uint32_t v = 0; v < nv; ++v) {
        if (size[label[v]] >= min_size) continue;
        vdoom[v] = 1;
        for (uint32_t e : m.v2e[v]) {
            edoom[e] = 1;
            for (int s = 0; s < 2; ++s)
                if (m.edges[e].t[s] != INVALID) tdoom[m.edges[e].t[s]] = 1;
        }
    }
    for (uint32_t t = 0; t < m.nt(); ++t) {
        if (!tdoom[t]) continue;
        for (uint32_t k = 0; k < 3; ++k) {
            const uint32_t e = m.edge_index(m.tri[3 * t + k], m.tri[3 * t + (k + 1) % 3]);
            const Edge &E = m.edges[e];
            const uint32_t other = E.t[0] == t ? E.t[1] : E.t[0];
            if (other == INVALID || tdoom[other]) edoom[e] = 1;
        }
    }
    return true;
}

// FlexibleMesh::deleteGeometry (FlexibleMesh.cpp:1428-1556): order-keeping
// compaction of vertices, edges and triangles with every index remapped.
void delete_geometry(Mesh &m, const std::vector<uint32_t> &vdoom, const std::vector<uint32_t> &edoom,
                     const std::vector<uint32_t> &tdoom) {
    const uint32_t nv = m.nv(), ne = (uint32_t)m.edges.size(), nt = m.nt();
    std::vector<uint32_t> vnew(nv, INVALID), enew(ne, INVALID), tnew(nt, INVALID);
    uint32_t k = 0;
    for (uint32_t v = 0; v < nv; ++v) if (!vdoom[v]) vnew[v] = k++;
    k = 0;
    for (uint32_t e = 0; e < ne; ++e) if (!edoom[e]) enew[e] = k++;
    k = 0;
    for (uint32_t t = 0; t < nt; ++t) if (!tdoom[t]) tnew[t] = k++;
    Mesh out;
    out.isle_vertices = m.isle_vertices;
    out.isle_triangles = m.isle_triangles;
    for (uint32_t v = 0; v < nv; ++v) {
        if (vdoom[v]) { ++out.isle_vertices; continue; }
        out.pos.push_back(m.pos[v]);
        out.nrm.push_back(m.nrm[v]);
        out.scale.push_back(m.scale[v]);
        std::vector<uint32_t> links;
        for (uint32_t e : m.v2e[v]) if (!edoom[e]) links.push_back(enew[e]);
        out.v2e.push_back(links);
    }
    for (uint32_t e = 0; e < ne; ++e) {
        if (edoom[e]) continue;
        Edge E = m.edges[e];
        for (int s = 0; s < 2; ++s) {
            E.v[s] = vnew[E.v[s]];
            E.t[s] = (E.t[s] == INVALID || tdoom[E.t[s]]) ? INVALID : tnew[E.t[s]];
        }
        if (E.t[0] == INVALID) std::swap(E.t[0], E.t[1]);
        out.edges.push_back(E);
    }
    for (uint32_t t = 0; t < nt; ++t) {
        if (tdoom[t]) { ++out.isle_triangles; continue; }
        for (int c = 0; c < 3; ++c) out.tri.push_back(vnew[m.tri[3 * t + c]]);
    }
    out.error = m.error;
    m = std::move(out);
}

// FlexibleMesh::findBorderRing / extendBorderRing (FlexibleMesh.cpp:1650-1709),
// literally: scan for the first edge (from the ring's end onwards) that
// starts where the ring ends, swap it behind the ring, until the ring closes.
void find_border_ring(std::vector<uint32_t> &remaining, std::vector<uint32_t> &set) {
    remaining.clear();
    const uint32_t start = set[0];
    uint32_t size = 2;
    const uint32_t n = (uint32_t)set.size();
    for (uint32_t i = size; i < n;) {
        const uint32_t e0 = set[i], e1 = set[i + 1];
        const uint32_t end = set[size - 1];
        if (e0 != end) {
            i += 2;
            continue;
        }
        set[i] = set[size];
        set[i + 1] = set[size + 1];
        set[size] = e0;
        set[size + 1] = e1;
        size += 2;
        i = size;
        if (e1 != start) continue;
        if (n == size) return;
        remaining.assign(set.begin() + size, set.end());
        set.resize(size);
        return;
    }
}

// FlexibleMesh::findBorderRings + removeDuplicatesInRings (FlexibleMesh.cpp:1617-1732)
std::vector<std::vector<uint32_t>> find_border_rings(std::vector<uint32_t> border) {
    std::vector<std::vector<uint32_t>> sets;
    if (!border.empty()) sets.push_back(border);
    sets.emplace_back();
    for (size_t i = 0; i + 1 < sets.size(); ++i) {
        std::vector<uint32_t> rest;
        find_border_ring(rest, sets[i]);
        sets.back() = rest;
        if (!sets.back().empty()) sets.emplace_back();
    }
    if (sets.back().empty()) sets.pop_back();
    for (auto &ring : sets) {
        std::vector<uint32_t> r;
        for (size_t j = 0; j < ring.size(); j += 2) r.push_back(ring[j]);
        ring = r;
    }
    return sets;
}

// FlexibleMesh::fillHole for <= 5 border edges (FlexibleMesh.cpp:1902-1931)
void fill_small(Mesh &m, const uint32_t *ring, uint32_t n) {
    uint32_t idx[5];
    if (ring) {
        std::memcpy(idx, ring, sizeof(uint32_t) * n);
    } else {
        const uint32_t start = m.nv() - n;
        for (uint32_t i = 0; i < n; ++i) idx[i] = start + i;
    }
    m.add_triangle(idx[0], idx[1], idx[2]);
    if (n == 3) return;
    m.add_triangle(idx[2], idx[3], idx[0]);
    if (n == 4) return;
    m.add_triangle(idx[3], idx[4], idx[0]);
}

// FlexibleMesh::fillHole / createHoleFillingRingVertices /
// connectHoleFillingRings (FlexibleMesh.cpp:1766-1900)
void fill_hole(Mesh &m, const uint32_t *ring, uint32_t n, V3 center) {
    if (n <= 5) {
        fill_small(m, ring, n);
        return;
    }
    const uint32_t old_nv = m.nv(), add = n / 2, new_nv = old_nv + add;
    // createHoleFillingRingVertices
    uint32_t rings_left = 0;
    for (uint32_t x = n; x; x >>= 1) ++rings_left;
    rings_left -= 1;
    const double f0 = (rings_left - 1) / (double)rings_left;
    const double f1 = (double)(1.0f / (float)rings_left);   // a float division in the reference
    const uint32_t prev = old_nv - n, last = new_nv - 1;
    m.pos.resize(new_nv);
    m.nrm.resize(new_nv);
    m.scale.resize(new_nv, 0.0);
    m.hole_vertices += add;
    uint32_t b = ring ? 0 : prev;
    for (uint32_t v = old_nv; v < new_nv; ++v) {
        const uint32_t v0 = ring ? ring[b] : b;
        ++b;
        const uint32_t v1 = ring ? ring[b] : b;
        ++b;
        const uint32_t v2 = (v == last) ? (ring ? ring[0] : prev) : (ring ? ring[b] : b);
        V3 p = m.pos[v0] + m.pos[v1] + m.pos[v2];
        m.pos[v] = p * (f0 / 3.0) + center * f1;
    }
    // connectHoleFillingRings
    const uint32_t outer = ring ? 0 : old_nv - n;
    const bool odd = (n & 1) == 1;
    for (uint32_t o = outer, i = 0; i < add; ++i) {
        const uint32_t a = ring ? ring[o] : o;
        ++o;
        const uint32_t c = ring ? ring[o] : o;
        ++o;
        const uint32_t d = (!odd && i == add - 1) ? (ring ? ring[outer] : outer) : (ring ? ring[o] : o);
        m.add_triangle(a, c, old_nv + i);
        m.add_triangle(c, d, old_nv + i);
    }
    if (odd) {
        if (ring) m.add_triangle(ring[n - 1], ring[0], m.nv() - 1);
        else m.add_triangle(old_nv - 1, outer, m.nv() - 1);
    }
    for (uint32_t o = outer + 2, i = 0; i < add; o += 2) {
        const uint32_t i0 = old_nv + i;
        uint32_t i1, ov;
        ++i;
        if (i == add) {
            i1 = old_nv;
            ov = ring ? ring[outer] : outer;
        } else {
            i1 = old_nv + i;
            ov = ring ? ring[o] : o;
        }
        m.add_triangle(i0, ov, i1);
    }
    fill_hole(m, nullptr, add, center);
}

// FlexibleMesh::fillHoles (FlexibleMesh.cpp:1580-1615, 1734-1764)
void fill_holes(Mesh &m) {
    std::vector<uint32_t> border;
    for (const Edge &e : m.edges) {
        if (e.t[0] != INVALID && e.t[1] != INVALID) continue;
        const uint32_t *t = &m.tri[3 * (e.t[1] != INVALID ? e.t[1] : e.t[0])];
        // Triangle::getVerticesInWindingOrder: the edge as the triangle passes it
        for (int k = 0; k < 3; ++k) {
            const uint32_t a = t[k], b = t[(k + 1) % 3];
            if ((a == e.v[0] && b == e.v[1]) || (a == e.v[1] && b == e.v[0])) {
                border.push_back(a);
                border.push_back(b);
                break;
            }
        }
    }
    m.border_edges = (uint32_t)(border.size() / 2);
    auto rings = find_border_rings(border);
    for (const auto &ring : rings) {
        const uint32_t n = (uint32_t)ring.size();
        if (n < 3) {   // the reference reads past such a ring (FlexibleMesh.cpp:1905-1916)
            ++m.skipped_rings;
            continue;
        }
        ++m.holes;
        V3 c;
        for (uint32_t v : ring) c = c + m.pos[v];
        c = V3{c.x / (double)n, c.y / (double)n, c.z / (double)n};
        fill_hole(m, ring.data(), n, c);
    }
}

// Mesh::computeNormalsWeightedByAngles (Mesh.cpp:145-203)
void normals(Mesh &m) {
    for (V3 &n : m.nrm) n = V3{};
    for (uint32_t t = 0; t < m.nt(); ++t) {
        const uint32_t *tr = &m.tri[3 * t];
        const V3 v0 = m.pos[tr[0]], v1 = m.pos[tr[1]], v2 = m.pos[tr[2]];
        V3 d0 = v1 - v0, d1 = v2 - v1, d2 = v2 - v0;
        V3 n = cross(d0, d2);
        normalize(d0);
        normalize(d1);
        normalize(d2);
        normalize(n);
        const double c[3] = {dot(d0, d2), -dot(d0, d1), -dot(d1, V3{-d2.x, -d2.y, -d2.z})};
        for (int k = 0; k < 3; ++k) {
            const double a = std::acos(std::fmin(1.0, std::fmax(-1.0, c[k])));
            m.nrm[tr[k]] = m.nrm[tr[k]] + n * a;
        }
    }
    for (V3 &n : m.nrm) normalize(n);
}

// ---- DepthImage::triangulate (DepthImage.cpp:186-461)
// Vector3 * Matrix3x3 is taken as a row vector times the matrix,
// out_j = (x m0j + y m1j) + z m2j; Math::SQRT_TWO as sqrt(2) rounded to double.
constexpr double SQRT_TWO = 1.4142135623730951;
constexpr double DEPTH_DIFFERENCE_FACTOR = 5.0;   // DepthImage.cpp:25

V3 row_times(V3 v, const double *M) {
    return {v.x * M[0] + v.y * M[3] + v.z * M[6], v.x * M[1] + v.y * M[4] + v.z * M[7],
            v.x * M[2] + v.y * M[5] + v.z * M[8]};
}

inline double length(V3 a) { return std::sqrt(dot(a, a)); }

// DepthImage::isDepthDiscontinuity (DepthImage.cpp:385-400)
bool discontinuity(const double fp[4], const double d[4], uint32_t v0, uint32_t v1) {
    const uint32_t closer = d[v0] < d[v1] ? v0 : v1, further = d[v0] < d[v1] ? v1 : v0;
    double f = DEPTH_DIFFERENCE_FACTOR;
    if (v0 + v1 == 3) f *= SQRT_TWO;
    return d[further] - d[closer] > fp[closer] * f;
}

// DepthImage::triangulateBlock (DepthImage.cpp:218-383)
uint32_t triangulate_block(std::vector<uint32_t> &indices, std::vector<uint32_t> &pix2v, uint32_t nv, uint32_t x,
                           uint32_t y, const double *depths, uint32_t W, const double *Mvs) {
    static const uint32_t tri_of[4][3] = {{0, 2, 1}, {0, 3, 1}, {0, 2, 3}, {1, 2, 3}};
    const uint32_t p = W * y + x;
    const double d[4] = {depths[p], depths[p + 1], depths[p + W], depths[p + W + 1]};
    uint32_t mask = 0, avail = 0;
    for (uint32_t i = 0; i < 4; ++i) {
        if (0.0 >= d[i]) continue;
        mask |= 1u << i;
        ++avail;
    }
    if (avail < 3) return nv;
    uint32_t t[2] = {INVALID, INVALID};
    switch (mask) {
        case 7: t[0] = 0; break;
        case 11: t[0] = 1; break;
        case 13: t[0] = 2; break;
        case 14: t[0] = 3; break;
        case 15:
            if (std::fabs(d[0] - d[3]) < std::fabs(d[1] - d[2])) { t[0] = 1; t[1] = 2; }
            else { t[0] = 0; t[1] = 3; }
            break;
        default: return nv;
    }
    double fp[4] = {0, 0, 0, 0};
    for (uint32_t i = 0; i < 4; ++i) {
        if (0.0 >= d[i]) continue;
        const V3 v = row_times(V3{(double)(x + i % 2), (double)(y + i / 2), 1.0}, Mvs);
        fp[i] = Mvs[0] * d[i] / length(v);
    }
    for (auto &ti : t) {
        if (ti == INVALID) continue;
        for (uint32_t e = 0; e < 3 && ti != INVALID; ++e)
            if (discontinuity(fp, d, tri_of[ti][e], tri_of[ti][(e + 1) % 3])) ti = INVALID;
    }
    for (uint32_t ti : t) {
        if (ti == INVALID) continue;
        for (uint32_t c = 0; c < 3; ++c) {
            const uint32_t q = p + (tri_of[ti][c] / 2) * W + tri_of[ti][c] % 2;
            if (pix2v[q] == INVALID) pix2v[q] = nv++;
            indices.push_back(pix2v[q]);
        }
    }
    return nv;
}

// Mesh::computeAverageDistance (Mesh.cpp:100-123)
double average_distance(V3 c, const std::vector<V3> &pos, const std::vector<uint32_t> &nbs, uint32_t skip) {
    uint32_t count = (uint32_t)nbs.size();
    double sum = 0.0;
    for (uint32_t n : nbs) {
        if (n == skip) { --count; continue; }
        sum += length(pos[n] - c);
    }
    if (count == 0) return -1.7976931348623157e308;
    return sum / count;
}

}  // namespace

extern "C" {

struct tsro_mesh {
    Mesh m;
    std::vector<V3> colors;   // depth meshes only
};

// DualMarchingCells::DualMarchingCells after extractMesh (DualMarchingCells.cpp:
// 26-39): isles, then -- unless nothing is left -- holes and normals.
tsro_mesh *tsro_mesh_postprocess(uint32_t nv, const double *positions, const double *scales, uint32_t nt,
                                 const uint32_t *triangles, uint32_t min_isle_size) {
    auto *h = new tsro_mesh();
    Mesh &m = h->m;
    m.pos.resize(nv);
    m.nrm.resize(nv);
    m.scale.assign(nv, 0.0);
    for (uint32_t v = 0; v < nv; ++v) {
        m.pos[v] = V3{positions[3 * v], positions[3 * v + 1], positions[3 * v + 2]};
        if (scales) m.scale[v] = scales[v];
    }
    m.tri.assign(triangles, triangles + 3 * (size_t)nt);
    m.find_adjacencies();
    if (m.error) return h;
    std::vector<uint32_t> vd, ed, td;
    if (isle_offsets(m, min_isle_size, vd, ed, td)) delete_geometry(m, vd, ed, td);
    if (m.nv() == 0 || m.tri.empty()) return h;
    fill_holes(m);
    normals(m);
    return h;
}

void tsro_mesh_free(tsro_mesh *h) { delete h; }

// DepthImage::triangulate + createFlexibleMesh (DepthImage.cpp:186-216,
// 402-461): triangles of the pixel grid, vertex positions along the pixel
// rays, colours (given per pixel, or 0.5 grey), angle-weighted normals and
// each vertex's mean distance to its neighbours (FlexibleMesh::
// findVertexNeighbors, FlexibleMesh.cpp:137-171; Mesh::computeVertexScales,
// Mesh.cpp:63-98).  pix2v (W*H) receives the vertex of every pixel.
tsro_mesh *tsro_depth_triangulate(const double *depths, uint32_t W, uint32_t H, const double *Mvs, const double *Mws,
                                  const double *center, const double *colors, uint32_t *pix2v_out) {
    auto *h = new tsro_mesh();
    Mesh &m = h->m;
    std::vector<uint32_t> pix2v((size_t)W * H, INVALID);
    uint32_t nv = 0;
    for (uint32_t y = 0; y + 1 < H; ++y)
        for (uint32_t x = 0; x + 1 < W; ++x) nv = triangulate_block(m.tri, pix2v, nv, x, y, depths, W, Mvs);
    // findVertexNeighbors
    std::vector<std::vector<uint32_t>> nbs(nv);
    auto add = [&](uint32_t a, uint32_t b) {
        for (uint32_t q : nbs[a]) if (q == b) return;
        nbs[a].push_back(b);
    };
    for (size_t t = 0; t + 2 < m.tri.size(); t += 3) {
        uint32_t e0 = m.tri[t], e1 = m.tri[t + 1];
        for (uint32_t k = 0; k < 3; ++k) {
            add(e0, e1);
            add(e1, e0);
            e0 = e1;
            e1 = m.tri[t + (k + 2) % 3];
        }
    }
    // setVertexPositions / setVertexColors
    m.pos.resize(nv);
    m.nrm.resize(nv);
    m.scale.assign(nv, 0.0);
    h->colors.assign(nv, V3{0.5, 0.5, 0.5});
    const V3 c{center[0], center[1], center[2]};
    for (uint32_t p = 0; p < W * H; ++p) {
        const uint32_t v = pix2v[p];
        if (v == INVALID) continue;
        V3 dir = row_times(V3{(double)(p % W), (double)(p / W), 1.0}, Mws);
        normalize(dir);
        m.pos[v] = c + dir * depths[p];
        if (colors) h->colors[v] = V3{colors[3 * (size_t)p], colors[3 * (size_t)p + 1], colors[3 * (size_t)p + 2]};
    }
    normals(m);
    for (uint32_t v = 0; v < nv; ++v) m.scale[v] = average_distance(m.pos[v], m.pos, nbs[v], v);
    if (pix2v_out) std::memcpy(pix2v_out, pix2v.data(), pix2v.size() * sizeof(uint32_t));
    return h;
}

void tsro_mesh_colors(const tsro_mesh *h, double *colors) {
    for (size_t v = 0; v < h->colors.size(); ++v) {
        colors[3 * v] = h->colors[v].x;
        colors[3 * v + 1] = h->colors[v].y;
        colors[3 * v + 2] = h->colors[v].z;
    }
}

// The ring search alone: nb border edges (tail, head pairs in list order)
// into rings of tail vertices; returns the ring count.  ring_verts holds nb
// entries, ring_lens one per ring (at most nb).
uint32_t tsro_border_rings(uint32_t nb, const uint32_t *edges, uint32_t *ring_verts, uint32_t *ring_lens) {
    std::vector<uint32_t> border(edges, edges + 2 * (size_t)nb);
    const auto rings = find_border_rings(border);
    uint32_t k = 0;
    for (size_t r = 0; r < rings.size(); ++r) {
        ring_lens[r] = (uint32_t)rings[r].size();
        for (uint32_t v : rings[r]) ring_verts[k++] = v;
    }
    return (uint32_t)rings.size();
}

// counts: vertices, triangles, error, isle vertices, isle triangles, border
// edges, holes, hole vertices, hole triangles, skipped rings
void tsro_mesh_counts(const tsro_mesh *h, uint64_t *c) {
    const Mesh &m = h->m;
    c[0] = m.nv();
    c[1] = m.nt();
    c[2] = (uint64_t)m.error;
    c[3] = m.isle_vertices;
    c[4] = m.isle_triangles;
    c[5] = m.border_edges;
    c[6] = m.holes;
    c[7] = m.hole_vertices;
    c[8] = m.hole_triangles;
    c[9] = m.skipped_rings;
}

void tsro_mesh_get(const tsro_mesh *h, double *positions, double *normals_out, double *scales, uint32_t *triangles) {
    const Mesh &m = h->m;
    for (uint32_t v = 0; v < m.nv(); ++v) {
        if (positions) {
            positions[3 * v] = m.pos[v].x;
            positions[3 * v + 1] = m.pos[v].y;
            positions[3 * v + 2] = m.pos[v].z;
        }
        if (normals_out) {
            normals_out[3 * v] = m.nrm[v].x;
            normals_out[3 * v + 1] = m.nrm[v].y;
            normals_out[3 * v + 2] = m.nrm[v].z;
        }
        if (scales) scales[v] = m.scale[v];
    }
    if (triangles) std::memcpy(triangles, m.tri.data(), m.tri.size() * sizeof(uint32_t));
}

}  // extern "C"
