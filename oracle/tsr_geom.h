/*
 * tsr_geom.h -- FP64 geometry helpers of the CPU oracle (test infrastructure).
 *
 * Vector arithmetic and the geometry predicates the reference's hot path calls.
 * The predicates marked "BaseProject" live in a library that is not part of the
 * reference tree; they are restated here from their call sites and comments
 * (parity at that boundary is unpinned; the reference build's shim,
 * oracle/ref_shim/, calls these same functions).  Operation order is fixed so that the
 * GPU tree build, which repeats these expressions in FP64, rounds identically.
 */
#ifndef TSR_ORACLE_GEOM_H
#define TSR_ORACLE_GEOM_H

#include <cmath>
#include <cstdint>

#include "../tsr_b200/csrc/mc_tables.h"

namespace tsrg {

// Math::EPSILON and REAL_MAX for Real = double.  BaseProject's values are not in
// the reference tree; these are the values this project fixes for both sides.
constexpr double EPS = 1e-6;
constexpr double DBL_MAX_ = 1.7976931348623157e308;
constexpr double PI = 3.14159265358979323846;

struct V3 { double x, y, z; };

inline V3 add(const V3 &a, const V3 &b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(const V3 &a, const V3 &b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 mul(const V3 &a, double s) { return V3{a.x * s, a.y * s, a.z * s}; }
inline V3 divv(const V3 &a, double s) { return V3{a.x / s, a.y / s, a.z / s}; }
inline V3 neg(const V3 &a) { return V3{-a.x, -a.y, -a.z}; }
inline double dot(const V3 &a, const V3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double len2(const V3 &a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline double len(const V3 &a) { return std::sqrt(len2(a)); }
inline V3 vmin(const V3 &a, const V3 &b) { return V3{a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z}; }
inline V3 vmax(const V3 &a, const V3 &b) { return V3{a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z}; }

// Nodes.h:154-162 (half-open containment with a tolerance)
inline bool node_contains(const V3 &p, const V3 &mn, double size, double tol) {
    return p.x >= mn.x - tol && p.x < mn.x + size + tol &&
           p.y >= mn.y - tol && p.y < mn.y + size + tol &&
           p.z >= mn.z - tol && p.z < mn.z + size + tol;
}

// Nodes.cpp:32-44
inline uint32_t child_index_for_offset(const V3 &o) {
    uint32_t i = 0;
    if (o.x >= 0.0) i |= 1u;
    if (o.y >= 0.0) i |= 2u;
    if (o.z >= 0.0) i |= 4u;
    return i;
}

// Nodes.cpp:46-58
inline V3 child_coords(const V3 &mn, double step, uint32_t i) {
    V3 c = mn;
    if (i & 1u) c.x += step;
    if (i & 2u) c.y += step;
    if (i & 4u) c.z += step;
    return c;
}

// Nodes.cpp:60-84
inline V3 side_center(const V3 &mn, double size, uint32_t side, double step) {
    double half = size * 0.5;
    V3 p{mn.x + half, mn.y + half, mn.z + half};
    double d = half + step;
    switch (side) {
        case 0: p.x -= d; break;
        case 1: p.x += d; break;
        case 2: p.y -= d; break;
        case 3: p.y += d; break;
        case 4: p.z -= d; break;
        default: p.z += d; break;
    }
    return p;
}

// Samples.cpp:451-455: signed distance to the sample's tangent plane
// (BaseProject Plane with a unit normal): dot(x - p, n).
inline double sample_plane_distance(const V3 &p, const V3 &n, const V3 &x) {
    return dot(sub(x, p), n);
}

// BaseProject intersectAABBWithSphere (called at Nodes.cpp:121,516,
// SphereNodesChecker.cpp:39): closed test, squared box distance <= r^2.
inline bool aabb_sphere(const V3 &mn, const V3 &mx, const V3 &c, double r) {
    double d2 = 0.0;
    if (c.x < mn.x) { double t = c.x - mn.x; d2 += t * t; } else if (c.x > mx.x) { double t = c.x - mx.x; d2 += t * t; }
    if (c.y < mn.y) { double t = c.y - mn.y; d2 += t * t; } else if (c.y > mx.y) { double t = c.y - mx.y; d2 += t * t; }
    if (c.z < mn.z) { double t = c.z - mn.z; d2 += t * t; } else if (c.z > mx.z) { double t = c.z - mx.z; d2 += t * t; }
    return d2 <= r * r;
}

// BaseProject intersectAABBWithLineSegment (called at Nodes.cpp:319): slab
// clipping of the segment s + t (e - s), t in [0, 1]; entry/exit are the
// clipped parameters, so exit - entry is the fraction of the segment inside.
inline bool segment_aabb(double &t0, double &t1, const V3 &s, const V3 &e, const V3 &mn, const V3 &mx) {
    double lo = 0.0, hi = 1.0;
    const double sv[3] = {s.x, s.y, s.z};
    const double dv[3] = {e.x - s.x, e.y - s.y, e.z - s.z};
    const double bmn[3] = {mn.x, mn.y, mn.z};
    const double bmx[3] = {mx.x, mx.y, mx.z};
    for (int a = 0; a < 3; ++a) {
        if (dv[a] == 0.0) {
            if (sv[a] < bmn[a] || sv[a] > bmx[a]) return false;
            continue;
        }
        double inv = 1.0 / dv[a];
        double ta = (bmn[a] - sv[a]) * inv;
        double tb = (bmx[a] - sv[a]) * inv;
        if (ta > tb) { double t = ta; ta = tb; tb = t; }
        if (ta > lo) lo = ta;
        if (tb < hi) hi = tb;
        if (lo > hi) return false;
    }
    t0 = lo;
    t1 = hi;
    return true;
}

// BaseProject ObliqueCircularCone, restated from its uses in
// ConeNodesChecker.h:24-29 and Occupancy.cpp:199-206,288-314:
// apex a, end-disc centre e, end-disc normal m (pointing out of the cone),
// end radius R.  Every disc of the cone is parallel to the end disc; the disc
// whose plane meets the axis at parameter t (apex = 0, end = 1) is centred at
// a + t (e - a) with radius t R.  `length` cuts the cone: only the last
// `length` of the axis (measured back from e) belongs to it; REAL_MAX keeps
// the complete cone.
struct Cone {
    V3 apex, end, normal, axis;   // axis = end - apex
    double radius, full, length;  // full = |axis|, length = min(cut, full)
    double denom;                 // dot(axis, normal)
    double t_start;               // 1 - length / full
};

inline void cone_init(Cone &c, const V3 &apex, const V3 &normal, const V3 &end, double radius, double length) {
    c.apex = apex; c.end = end; c.normal = normal; c.radius = radius;
    c.axis = sub(end, apex);
    c.full = len(c.axis);
    c.length = length < c.full ? length : c.full;
    c.denom = dot(c.axis, normal);
    c.t_start = (c.full > 0.0) ? 1.0 - c.length / c.full : 0.0;
}

// Degenerate when the axis has no length, the disc planes contain the axis
// direction (no plane/axis intersection) or the cone has no width.
inline bool cone_degenerated(const Cone &c) {
    if (!(c.full > EPS) || !(c.radius > 0.0)) return true;
    return std::fabs(c.denom) <= EPS * c.full;
}

inline double cone_t_complete(const Cone &c, const V3 &x) { return dot(sub(x, c.apex), c.normal) / c.denom; }
inline double cone_t_cut(const Cone &c, double tc) { return (tc * c.full - (c.full - c.length)) / c.length; }

// Conservative replacement for ObliqueCircularCone::haveSeparatingAxis
// (ConeNodesChecker.cpp:65): returns true only when no point of the box lies
// in the cut cone.  Occupancy::addKernel re-tests each leaf centre exactly, so
// any conservative test yields the same sums; tsro_occupancy(prune = 0) checks
// this on small scenes.
inline bool cone_box_separated(const Cone &c, const V3 &mn, double size) {
    double h = 0.5 * size;
    V3 ctr{mn.x + h, mn.y + h, mn.z + h};
    double n1 = std::fabs(c.normal.x) + std::fabs(c.normal.y) + std::fabs(c.normal.z);
    double tmid = cone_t_complete(c, ctr);
    double dt = h * n1 / std::fabs(c.denom);
    double slack = 1e-9;
    if (tmid + dt < c.t_start - slack || tmid - dt >= 1.0 + slack) return true;
    if (tmid + dt <= 0.0) return true;
    V3 q = sub(sub(ctr, c.apex), mul(c.axis, tmid));
    double qn = len(q);
    double tmax = tmid + dt < 1.0 ? tmid + dt : 1.0;
    double bound = qn - h * 1.7320508075688772 - dt * c.full;
    return bound > tmax * c.radius * (1.0 + slack) + slack * c.radius;
}

// Occupancy.cpp:348-400 (CONE_PCD_KERNEL_NEG_PARABLE)
inline double disc_kernel_sq(double r2, double R) {
    double R2 = R * R;
    if (r2 >= R2) return 0.0;
    double not_normed = 1.0 - r2 / R2;
    return (2.0 / (PI * R2)) * not_normed;
}

// Occupancy.cpp:429-439 (CONE_RAY_KERNEL_NEG_PARABLE)
inline double ray_kernel(double z, double Z) {
    if (z < 0.0 || z >= Z) return 0.0;
    double z2 = z * z, Z2 = Z * Z;
    return (3.0 / (2.0 * Z)) * (-z2 / Z2 + 1.0);
}

// Occupancy.cpp:279-346; returns the confidence-scaled kernel value in `out`.
inline bool add_kernel(double &out, const V3 &x, const Cone &c, bool sampleness, double confidence) {
    double tc = cone_t_complete(c, x);
    double tcut = cone_t_cut(c, tc);
    if (tcut < 0.0 || tcut >= 1.0) return false;
    V3 pcd = add(c.apex, mul(c.axis, tc));
    double pr = c.radius * tc;
    double r2 = len2(sub(x, pcd));
    if (r2 >= pr * pr) return false;
    double Z, z, norm;
    if (!sampleness) { Z = c.length; z = tcut * Z; norm = 1.0; }
    else { double tcen = std::fabs(tcut - 0.5) * 2.0; Z = 0.5 * c.length; z = tcen * Z; norm = 0.5; }
    double kv = ray_kernel(z, Z) * norm * disc_kernel_sq(r2, pr);
    if (EPS > kv) return false;
    double scaled = confidence * kv;
    if (EPS > scaled) return false;
    out = scaled;
    return true;
}

// DualMarchingCell.cpp:51-71
inline double interpolation_factor(double d0, double d1) {
    if (EPS >= std::fabs(d1 - d0)) return 0.5;
    if (EPS >= std::fabs(d0)) return 0.0;
    if (EPS >= std::fabs(d1)) return 1.0;
    return (0.0 - d0) / (d1 - d0);
}

// DualMarchingCell.cpp:73-101
inline bool degenerated_triangle(const int8_t *edges, const uint32_t *leaf) {
    for (int i = 0; i < 3; ++i) {
        const uint8_t *e = MC_EDGE_ENDS[edges[i]];
        if (leaf[e[0]] == leaf[e[1]]) return true;
    }
    for (int i = 0; i < 3; ++i) {
        const uint8_t *a = MC_EDGE_ENDS[edges[i]];
        const uint8_t *b = MC_EDGE_ENDS[edges[(i + 1) % 3]];
        if (leaf[a[0]] == leaf[b[0]] && leaf[a[1]] == leaf[b[1]]) return true;
        if (leaf[a[0]] == leaf[b[1]] && leaf[a[1]] == leaf[b[0]]) return true;
    }
    return false;
}

// Edge cuttings derived from the corner signs: edge e is cut when its two
// ends differ (equals the reference's MC_EDGE_CUTTINGS_TABLE).
inline uint32_t mc_edge_cuttings(uint32_t code) {
    uint32_t cut = 0;
    for (int e = 0; e < 12; ++e)
        if (((code >> MC_EDGE_ENDS[e][0]) ^ (code >> MC_EDGE_ENDS[e][1])) & 1u) cut |= 1u << e;
    return cut;
}

}  // namespace tsrg

#endif
