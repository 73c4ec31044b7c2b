// occupancy.cu -- sm_100a occupancy field of the TSR volumetric core.
//
// Reproduces Occupancy::computeOccupancy (SurfaceExtraction/Occupancy.cpp:
// 105-127): the SAMPLENESS and EMPTINESS cone-kernel passes over every
// camera-to-sample link (updateKernels :138-248, addKernel :279-346), the
// bottom-up SAMPLENESS flag propagation (forwardAnyChildStateFlag :491-516),
// the semi-local Bayesian priors (computePriors :530-568) and the per-leaf
// occupancy value (getOccupancy :570-587).
//
// Precision: the per-link cone set-up, the depth cap, the cone length and the
// cone count are FP64 (as the reference's Real = double); kernel evaluation
// runs in FP32 in a frame centred on the sample, and every per-leaf sum is an
// FP64 accumulator updated by FP64 atomic adds whose result is not used (no
// round trip per accepted pair).  Priors and occupancy are evaluated in FP64;
// the prior's sphere / box membership test is the same FP64 expression as the
// tree build's, so the set of leaves each prior sums over is exact.
#include <cub/cub.cuh>

#include <vector>

#include "handles.h"

namespace tsr {
namespace {

constexpr unsigned BLK = 256;
enum { EMPTINESS = 0, SAMPLENESS = 1 };

struct F3 {
    float x, y, z;
};
__device__ inline F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ inline F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ inline F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ inline F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ inline float fdot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Cone in the sample-centred FP32 frame.  t is measured from the end disc:
// te = dot(x - end, m) / denom = tComplete - 1, which keeps the arithmetic
// near the sample (where the kernels are evaluated) well conditioned.
struct ConeF {
    F3 end, axis, m;   // m = end-disc normal
    float radius, full, inv_denom, a_over_l, t_start_e;
    float ray_k;       // 3 / (2 L), L = cone length
    float n1;          // |m|_1
};

struct LinkIn {
    const D3 *pos, *nrm;
    const double *scale, *conf;
    const uint32_t *links;
    const D3 *cams;
    uint32_t k, ncams;
    double h_svo, h_o, rel_cone, root_size;
};

struct TreeIn {
    const D3 *nmin;   // node min corners (FP64), for the start-node descent
};


// Occupancy::addKernel (Occupancy.cpp:279-346) at a leaf centre x, given
// te = dot(x - end, m) / denom (= tComplete - 1) and r2 = |x - PCD centre|^2:
// the confidence-scaled kernel value, or 0 where addKernel adds nothing.
// Straight-line code (no early exits), so that the lanes of a warp testing
// different children stay together.
__device__ __forceinline__ float kernel_value(const ConeF &c, float te, float r2, bool sampleness, float conf) {
    const float tcut_m1 = te * c.a_over_l;         // tCut - 1
    const float tcut = 1.0f + tcut_m1;
    const float pr = c.radius * (1.0f + te);       // PCD radius at tComplete
    const float pr2 = pr * pr;
    bool ok = (tcut >= 0.0f) & (tcut < 1.0f) & (r2 < pr2);
    float f;   // ray factor: 3/(2Z)(1 - (z/Z)^2) with the 3/(2 L) part in ray_k
    if (sampleness) {
        const float tcen = fabsf(tcut - 0.5f) * 2.0f;
        f = 1.0f - tcen * tcen;
        ok &= tcen < 1.0f;
    } else {
        f = (-tcut_m1) * (1.0f + tcut);            // (1 - tCut)(1 + tCut)
    }
    const float inv = __frcp_rn(pr2);
    const float kv = c.ray_k * f * (0.63661977236758134f * inv) * (1.0f - r2 * inv);
    const float scaled = conf * kv;
    ok &= (kv >= (float)EPS) & (scaled >= (float)EPS);
    return ok ? scaled : 0.0f;
}

// Cone-frame coordinates of point x: te, the offset q from the axis point of
// the same te, and |q|^2.
__device__ __forceinline__ void cone_coords(const ConeF &c, F3 x, float &te, F3 &q, float &r2) {
    F3 u = x - c.end;
    te = fdot(u, c.m) * c.inv_denom;
    q = u - c.axis * te;
    r2 = fdot(q, q);
}

__device__ inline float eval_kernel(const ConeF &c, F3 x, bool sampleness, float conf) {
    float te, r2;
    F3 q;
    cone_coords(c, x, te, q, r2);
    return kernel_value(c, te, r2, sampleness, conf);
}

__device__ inline F3 rel(const D3 &a, const D3 &origin) {
    return f3((float)(a.x - origin.x), (float)(a.y - origin.y), (float)(a.z - origin.z));
}

// ------------------------------------------------------ cone traversal
// Conservative cone/box rejection (stands in for ObliqueCircularCone::
// haveSeparatingAxis, ConeNodesChecker.cpp:65).  Pruning can only skip boxes
// that contain no point of the cut cone, so the sums do not depend on it.
// Conservative box test with an absolute slack for the FP32 box recurrence.
__device__ inline bool cone_box_separated_pt(const ConeF &c, F3 bmin, float size) {
    float h = 0.5f * size;
    F3 ctr = bmin + f3(h, h, h);
    float mag = fabsf(ctr.x) + fabsf(ctr.y) + fabsf(ctr.z);
    float hs = h + 2e-6f * mag;
    F3 u = ctr - c.end;
    float te = fdot(u, c.m) * c.inv_denom;
    float dt = hs * c.n1 * fabsf(c.inv_denom);
    float slack = 1e-4f * (dt + fabsf(te)) + 1e-6f;
    if (te + dt < c.t_start_e - slack) return true;
    if (te - dt >= slack) return true;
    if (1.0f + te + dt <= 0.0f) return true;
    F3 q = u - c.axis * te;
    float qn = sqrtf(fdot(q, q));
    float tmax = fminf(1.0f + te + dt, 1.0f);
    float bound = qn - hs * 1.7320508f - dt * c.full;
    return bound > tmax * c.radius * 1.0001f + 1e-4f * (qn + hs + dt * c.full);
}

// The same test for a box of centre coordinates (te, q, r2 = |q|^2; q is
// the offset from the axis point of the same te) and half size hs already
// widened by the recurrence slack; dt = hs * |m|_1 * |1/denom|.  A box point
// ctr + d has te + (d.m)/denom and offset q + d - axis (d.m)/denom, whose
// length is at least |q| + d.w with w = (q - (q.axis / denom) m) / |q|, so
// every box point is at least |q| - hs |w|_1 from the axis: the exact
// support of the box in that direction, with the axis shift over the box's
// te range folded in.  Straight-line code; |q| = 0 never separates.
__device__ __forceinline__ bool separated_at(const ConeF &c, float te, F3 q, float r2, float hs, float dt) {
    const float slack = 1e-4f * (dt + fabsf(te)) + 1e-6f;
    bool sep = (te + dt < c.t_start_e - slack) | (te - dt >= slack) | (1.0f + te + dt <= 0.0f);
    const float tmax = fminf(1.0f + te + dt, 1.0f);
    const float inv = rsqrtf(r2);
    const float qn = r2 * inv;
    const F3 v = q - c.m * (fdot(q, c.axis) * c.inv_denom);
    const float v1 = fabsf(v.x) + fabsf(v.y) + fabsf(v.z);
    const float rest = tmax * c.radius * 1.0001f + 1e-4f * (hs + dt * c.full);
    sep |= (qn * 0.9999f - hs * v1 * inv) > rest;
    return sep;
}

constexpr int PT_BLOCK = 128;
// Resident blocks per SM the persistent traversals are compiled for (the
// register budget: 65536 / (128 threads x blocks)).
#ifndef TSR_CONE_E_BLOCKS
#define TSR_CONE_E_BLOCKS 6
#endif
#ifndef TSR_CONE_S_BLOCKS
#define TSR_CONE_S_BLOCKS 5
#endif
#ifndef TSR_PRIOR_BLOCKS
#define TSR_PRIOR_BLOCKS 1
#endif

// ------------------------------------------- block-expansion cone traversal
// Thread-per-link depth-first traversal (the per-link LeavesIterator with a
// ConeNodesChecker) run by persistent threads: a lane whose traversal ends
// takes the next link, fetched per warp in one atomic batch, so lanes do not
// idle behind the warp's longest link.  Child boxes are derived from the
// parent's box in the link's FP32 frame.  The traversal is organised around
// children blocks: every step expands one node, loading its eight children's records in one 64-byte
// line and testing all eight at once, then descends straight into the first
// surviving child; only nodes with further surviving children go on the
// stack.  One dependent load per expanded node replaces one per visited
// child.  Leaf flags are not written here: a leaf got a kernel exactly when
// its sum is non-zero (every accepted value is >= EPSILON), so they are set
// afterwards from the sums.
//
// Node records: rec[i + 7] = (first child or INVALID, leaf index or
// REC_NOLEAF, with the node's SAMPLENESS flag in bit 31).  Children blocks
// start at 1 + 8k (root 0, then whole blocks of 8), so a block's records
// start on a 64-byte boundary.
constexpr uint32_t REC_FLAG = 0x80000000u, REC_NOLEAF = 0x7FFFFFFFu;
constexpr uint32_t REC_OFFSET = 7;

__global__ void k_pack_rec(uint32_t nn, const uint32_t *children, const uint32_t *node_to_leaf,
                           const uint32_t *states, uint2 *rec) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    uint32_t c = children[i];
    uint32_t y = (c == INVALID) ? node_to_leaf[i] : REC_NOLEAF;
    if (states && (states[i] & FLAG_SAMPLENESS)) y |= REC_FLAG;
    rec[i + REC_OFFSET] = make_uint2(c, y);
}

// Pruned field: which leaves need their prior.  Only a reliable leaf
// (E + S >= confidenceThreshold) uses it, and with E == 0 or S == 0 its sign
// is fixed without it (need 0).  A leaf near a predicted sign change
// (PRED_KEEP), or one whose sign the network is unsure of, is queried
// (need 1); any other leaf is a candidate for skipping (need 2): its sign is
// then certified from bounds of its prior (k_certify) or it is queried after
// all.
constexpr uint8_t NEED_NONE = 0, NEED_QUERY = 1, NEED_CERTIFY = 2;


__global__ void k_prior_needed(uint32_t nl, const uint8_t *pred, const double *esum, const double *ssum,
                               double threshold, uint8_t *need) {
    uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    const double e = esum[l], s = ssum[l];
    const uint8_t pr = pred[l];
    uint8_t n = NEED_NONE;
    if (!((e + s) < threshold) && e > 0.0 && s > 0.0)
        n = ((pr & PRED_KEEP) || !(pr & (PRED_POS | PRED_NEG))) ? NEED_QUERY : NEED_CERTIFY;
    else if (!((e + s) < threshold) && (pr & PRED_KEEP))
        n = NEED_QUERY;
    need[l] = n;
}

// The sign of a skip candidate from bounds [lo, hi] of its prior p: the
// occupancy is positive iff (1 - p) S > p E (Occupancy.cpp:570-587; the
// common factor 1 / coneCount dropped), which decreases in p.  Positive when
// it holds at p = hi, negative when it fails at p = lo, each with a relative
// margin of 1e-9 that covers the rounding of the sums and of the exact
// formula; otherwise the leaf is queried (need 1).  A certified leaf's sign
// goes to its PRED_POS / PRED_NEG bits, which the pruned k_finalize uses.
//
// A positive leaf's value (1 - p) S / coneCount - p E / coneCount is also
// placed against EPSILON when the bounds decide it (PRED_HIGH / PRED_LOW,
// same margin): DMC snaps a vertex to the end of an edge whose value is
// within EPSILON of zero, and a negative leaf's value is -EPSILON, so that
// side is all the mesh takes from a positive leaf's value.
__global__ void k_certify(uint32_t n, const uint32_t *list, const double *esum, const double *ssum,
                          const double2 *bounds, const double *cone_count, uint8_t *pred, uint8_t *need,
                          unsigned long long *certified) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool ok = false;
    if (i < n) {
        const uint32_t l = list[i];
        const double e = esum[l], s = ssum[l];
        const double2 b = bounds[i];
        const double margin = 1e-9 * (s + e);
        const double at_hi = (1.0 - b.y) * s - b.y * e, at_lo = (1.0 - b.x) * s - b.x * e;
        const bool pos = at_hi > margin;
        const bool neg = at_lo < -margin;
        const uint8_t keep = pred[l] & PRED_KEEP;
        const double eps_cc = EPS * *cone_count;
        if (pos) pred[l] = keep | PRED_POS | (at_hi > eps_cc + margin ? PRED_HIGH : 0) |
                           (at_lo < eps_cc - margin ? PRED_LOW : 0);
        else if (neg) pred[l] = keep | PRED_NEG;
        ok = pos || neg;
        need[l] = ok ? NEED_NONE : NEED_QUERY;
    }
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(certified, (unsigned long long)__popc(m));
}

__device__ __forceinline__ F3 child_min(F3 pmin, uint32_t ci, float size) {
    return f3((ci & 1u) ? pmin.x + size : pmin.x, (ci & 2u) ? pmin.y + size : pmin.y,
              (ci & 4u) ? pmin.z + size : pmin.z);
}

// Per-link set-up of the traversal, precomputed by one thread per link so
// that the persistent traversal below never runs this long FP64 stretch for a
// few lanes of a warp while the others wait.  c0 == INVALID: nothing to
// traverse (no camera, degenerated cone, pruned start, or a start leaf that
// the set-up kernel has already visited).
struct __align__(16) LinkRec {
    float end[3], axis[3], m[3];
    float radius, full, ray_k, inv_denom, a_over_l, t_start_e, n1;
    float smin[3], fconf;     // start node corner in the sample's frame; confidence
    double wlen;              // confidence * cone length
    uint32_t c0;              // children block of the start node
    uint32_t depths;          // depth of those children | max depth << 8
    double spos[3];           // the sample: origin of the FP32 frame
    uint64_t pad;
};

__device__ __forceinline__ ConeF cone_of(const LinkRec &r) {
    ConeF c;
    c.end = f3(r.end[0], r.end[1], r.end[2]);
    c.axis = f3(r.axis[0], r.axis[1], r.axis[2]);
    c.m = f3(r.m[0], r.m[1], r.m[2]);
    c.radius = r.radius;
    c.full = r.full;
    c.ray_k = r.ray_k;
    c.inv_denom = r.inv_denom;
    c.a_over_l = r.a_over_l;
    c.t_start_e = r.t_start_e;
    c.n1 = r.n1;
    return c;
}

// Set-up of link order[i] (Occupancy.cpp:174-201), FP64, and the start of its
// traversal: the deepest node containing the cut cone's bounding box.
// sign: +1 adds the links' kernels, -1 removes them (Occupancy::updateKernels
// with forRemoval, Occupancy.cpp:138-248: the same acceptance, negated
// values, cone lengths and cone count).
template <int TYPE>
__global__ void __launch_bounds__(128) k_link_setup(uint64_t nlinks, const uint32_t *order, LinkIn in, TreeIn tr,
                                                    const uint2 *rec, LinkRec *out, double *ksum, double *clen,
                                                    double *cone_count, unsigned long long *accepted, double sign) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double count = 0.0;
    unsigned long long acc = 0;
    if (i < nlinks) {
        LinkRec r;
        r.c0 = INVALID;
        r.depths = 0;
        do {
            uint64_t l = order ? order[i] : i;
            uint32_t s = (uint32_t)(l / in.k);
            uint32_t cam = in.links[l];
            if (cam == INVALID || cam >= in.ncams) break;
            D3 p = in.pos[s];
            D3 n = in.nrm[s];
            D3 cwp = in.cams[cam];
            double kernel_r = in.h_o * in.scale[s];
            D3 apex_d{cwp.x - p.x, cwp.y - p.y, cwp.z - p.z};
            D3 end_d{0.0, 0.0, 0.0};
            double cone_len = REAL_MAX;
            if (TYPE == SAMPLENESS) {
                D3 cs{-apex_d.x, -apex_d.y, -apex_d.z};
                double total = sqrt(cs.x * cs.x + cs.y * cs.y + cs.z * cs.z);
                cone_len = kernel_r * in.rel_cone;
                double hh = cone_len * 0.5;
                end_d = D3{cs.x / total * hh, cs.y / total * hh, cs.z / total * hh};
            }
            D3 m{-n.x, -n.y, -n.z};
            D3 axis{end_d.x - apex_d.x, end_d.y - apex_d.y, end_d.z - apex_d.z};
            double full = sqrt(axis.x * axis.x + axis.y * axis.y + axis.z * axis.z);
            double length = cone_len < full ? cone_len : full;
            double denom = axis.x * m.x + axis.y * m.y + axis.z * m.z;
            if (!(full > EPS) || !(kernel_r > 0.0) || fabs(denom) <= EPS * full) break;   // isDegenerated
            double conf = in.conf[s];
            if (TYPE == EMPTINESS) count += sign * conf;
            const double wlen = conf * length;
            const float fconf = (float)conf;
            const uint32_t max_depth =
                (uint32_t)ceil(log2(in.root_size / (in.scale[s] * in.h_svo))) + MAX_DEPTH_DIFFERENCE;
            ConeF c;
            c.end = f3((float)end_d.x, (float)end_d.y, (float)end_d.z);
            c.axis = f3((float)axis.x, (float)axis.y, (float)axis.z);
            c.m = f3((float)m.x, (float)m.y, (float)m.z);
            c.radius = (float)kernel_r;
            c.full = (float)full;
            c.ray_k = (float)(1.5 / length);
            c.inv_denom = (float)(1.0 / denom);
            c.a_over_l = (float)(full / length);
            c.t_start_e = (float)(-length / full);
            c.n1 = fabsf(c.m.x) + fabsf(c.m.y) + fabsf(c.m.z);
            F3 p0 = c.end + c.axis * c.t_start_e;
            F3 lo = f3(fminf(p0.x, c.end.x) - c.radius, fminf(p0.y, c.end.y) - c.radius, fminf(p0.z, c.end.z) - c.radius);
            F3 hi = f3(fmaxf(p0.x, c.end.x) + c.radius, fmaxf(p0.y, c.end.y) + c.radius, fmaxf(p0.z, c.end.z) + c.radius);
            const float root_size_f = (float)in.root_size;
            uint32_t start = 0, base = 0;
            uint2 srec = __ldg(&rec[REC_OFFSET]);
            F3 smin = rel(tr.nmin[0], p);
            float ssize = root_size_f;
            while (srec.x != INVALID && base + 1 <= max_depth) {
                float cs = 0.5f * ssize;
                float margin = 1e-5f * ssize;
                F3 ctr = smin + f3(cs, cs, cs);
                const float l3[3] = {lo.x, lo.y, lo.z}, h3[3] = {hi.x, hi.y, hi.z}, c3[3] = {ctr.x, ctr.y, ctr.z};
                uint32_t digit = 0;
                bool inside = true;
                for (int a = 0; a < 3; ++a) {
                    if (h3[a] < c3[a] - margin) continue;
                    if (l3[a] > c3[a] + margin) { digit |= 1u << a; continue; }
                    inside = false;
                }
                if (!inside) break;
                start = srec.x + digit;
                srec = __ldg(&rec[start + REC_OFFSET]);
                smin = rel(tr.nmin[start], p);
                ssize = cs;
                ++base;
            }
            if (TYPE == EMPTINESS && !(srec.y & REC_FLAG)) break;
            if (cone_box_separated_pt(c, smin, ssize)) break;
            if (srec.x == INVALID) {   // the start is a leaf: visit it here
                float h = 0.5f * ssize;
                float val = eval_kernel(c, smin + f3(h, h, h), TYPE == SAMPLENESS, fconf);
                if (val > 0.0f) {
                    uint32_t leaf = srec.y & REC_NOLEAF;
                    atomicAdd(&ksum[leaf], sign * (double)val);
                    atomicAdd(&clen[leaf], sign * wlen);
                    ++acc;
                }
                break;
            }
            if (base + 1 > max_depth) break;
            r.end[0] = c.end.x; r.end[1] = c.end.y; r.end[2] = c.end.z;
            r.axis[0] = c.axis.x; r.axis[1] = c.axis.y; r.axis[2] = c.axis.z;
            r.m[0] = c.m.x; r.m[1] = c.m.y; r.m[2] = c.m.z;
            r.radius = c.radius; r.full = c.full; r.ray_k = c.ray_k; r.inv_denom = c.inv_denom;
            r.a_over_l = c.a_over_l; r.t_start_e = c.t_start_e; r.n1 = c.n1;
            r.smin[0] = smin.x; r.smin[1] = smin.y; r.smin[2] = smin.z;
            r.fconf = fconf;
            r.wlen = sign * wlen;
            r.c0 = srec.x;
            r.depths = (base + 1) | (max_depth << 8);
            r.spos[0] = p.x; r.spos[1] = p.y; r.spos[2] = p.z;
            r.pad = 0;
        } while (0);
        out[i] = r;
    }
    typedef cub::BlockReduce<double, 128> BR;
    typedef cub::BlockReduce<unsigned long long, 128> BRU;
    __shared__ typename BR::TempStorage tmp;
    __shared__ typename BRU::TempStorage tmpu;
    double bc = BR(tmp).Sum(count);
    unsigned long long ba = BRU(tmpu).Sum(acc);
    if (threadIdx.x == 0) {
        if (TYPE == EMPTINESS && bc != 0.0) atomicAdd(cone_count, bc);
        if (ba) atomicAdd(accepted, ba);
    }
}

template <int TYPE>
__global__ void __launch_bounds__(PT_BLOCK, (TYPE == 0) ? TSR_CONE_E_BLOCKS : TSR_CONE_S_BLOCKS) k_cone_x(uint64_t nlinks, const LinkRec *links,
                                                                         TreeIn tr, const uint2 *rec,
                                                                         float root_size_f, double *ksum,
                                                                         double *clen, unsigned long long *accepted,
                                                                         unsigned long long *next_link,
                                                                         unsigned long long *visits, int *err,
                                                                         double sign) {
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31;
    // stack of expanded nodes that still have children to descend into
    uint64_t st[MAX_TREE_DEPTH];   // children block | mask << 32 | depth << 40
    int sp = 0;
    D3 spos{0.0, 0.0, 0.0};        // the link's sample: origin of the FP32 frame
    // the node to expand next: its children block, box corner and depth
    bool have = false;
    uint32_t x_c0 = 0, x_d = 0;
    F3 x_min = f3(0.f, 0.f, 0.f);
    uint32_t max_depth = 0;
    ConeF c;
    double wlen = 0.0;
    float fconf = 0.f;
    bool done = false;
    unsigned long long acc = 0, nvis = 0;

    while (true) {
        // resume the deepest expanded node that has children left
        if (!have && sp > 0) {
            uint64_t e = st[sp - 1];
            uint32_t m = (uint32_t)(e >> 32) & 0xFFu;
            uint32_t node = (uint32_t)e + (uint32_t)(__ffs(m) - 1);
            m &= m - 1;
            if (m) st[sp - 1] = (e & ~(0xFFull << 32)) | ((uint64_t)m << 32); else --sp;
            x_c0 = __ldg(&rec[node + REC_OFFSET]).x;
            x_min = rel(tr.nmin[node], spos);
            x_d = (uint32_t)(e >> 40) + 1;
            have = true;
        }
        bool need = !have && !done;
        unsigned nm = __ballot_sync(FULL, need);
        if (nm) {
            int leader = __ffs(nm) - 1;
            unsigned long long b = 0;
            if ((int)lane == leader) b = atomicAdd(next_link, (unsigned long long)__popc(nm));
            b = __shfl_sync(FULL, b, leader);
            if (need) {
                uint64_t i = b + __popc(nm & ((1u << lane) - 1u));
                if (i >= nlinks) {
                    done = true;
                } else {
                    const LinkRec r = links[i];
                    if (r.c0 != INVALID) {
                        c = cone_of(r);
                        wlen = r.wlen;
                        fconf = r.fconf;
                        max_depth = r.depths >> 8;
                        spos = D3{r.spos[0], r.spos[1], r.spos[2]};
                        x_c0 = r.c0;
                        x_min = f3(r.smin[0], r.smin[1], r.smin[2]);
                        x_d = r.depths & 0xFFu;
                        have = true;
                    }
                }
            }
        }
        if (__all_sync(FULL, done && !have && sp == 0)) break;
        if (!have) continue;
        // ---- expand: test the eight children of the node (NodesIterator.cpp:38-86)
        have = false;
        if ((x_c0 & 7u) != 1u || x_c0 > 0xFFFFFFF0u) {   // children blocks start at 1 + 8k
            atomicExch(err, 3);
            continue;
        }
        const uint4 *line = reinterpret_cast<const uint4 *>(rec + x_c0 + REC_OFFSET);
        uint4 q0 = __ldg(line), q1 = __ldg(line + 1), q2 = __ldg(line + 2), q3 = __ldg(line + 3);
        const uint32_t rx[8] = {q0.x, q0.z, q1.x, q1.z, q2.x, q2.z, q3.x, q3.z};
        const uint32_t ry[8] = {q0.y, q0.w, q1.y, q1.w, q2.y, q2.w, q3.y, q3.w};
        const float size = ldexpf(root_size_f, -(int)x_d);
        const bool can_descend = x_d + 1 <= max_depth;
        // one widened half size for all eight boxes: covers the FP32 corner
        // error of every child centre (|centre|_1 <= |x_min|_1 + 4.5 size)
        const float h = 0.5f * size;
        const float hs = h + 2e-6f * (fabsf(x_min.x) + fabsf(x_min.y) + fabsf(x_min.z) + 4.5f * size);
        const float dt = hs * c.n1 * fabsf(c.inv_denom);
        const F3 ctr0 = x_min + f3(h, h, h);
        uint32_t mask = 0;
        nvis += 8;
#pragma unroll
        for (int ci = 0; ci < 8; ++ci) {
            // both tests for every child, without branches; only the outcome
            // (a leaf's kernel, or a child to descend into) is conditional
            const bool flagged = TYPE == SAMPLENESS || (ry[ci] & REC_FLAG);
            const bool leaf = rx[ci] == INVALID;
            F3 ctr = f3((ci & 1) ? ctr0.x + size : ctr0.x, (ci & 2) ? ctr0.y + size : ctr0.y,
                        (ci & 4) ? ctr0.z + size : ctr0.z);
            float te, r2;
            F3 q;
            cone_coords(c, ctr, te, q, r2);
            const float val = kernel_value(c, te, r2, TYPE == SAMPLENESS, fconf);
            const bool sep = separated_at(c, te, q, r2, hs, dt);
            // a leaf: addKernel's exact test decides, no box test needed
            if (flagged && leaf && val > 0.0f) {
                uint32_t lf = ry[ci] & REC_NOLEAF;
                atomicAdd(&ksum[lf], sign * (double)val);
                atomicAdd(&clen[lf], wlen);   // wlen carries the sign
                ++acc;
            }
            if (flagged && !leaf && can_descend && !sep) mask |= 1u << ci;
        }
        if (mask) {
            uint32_t ci = __ffs(mask) - 1;
            uint32_t rest = mask & (mask - 1);
            if (rest) {
                if (sp >= MAX_TREE_DEPTH) {
                    atomicExch(err, 1);
                    continue;
                }
                st[sp++] = (uint64_t)x_c0 | ((uint64_t)rest << 32) | ((uint64_t)x_d << 40);
            }
            uint32_t nc = rx[0];
#pragma unroll
            for (int k = 1; k < 8; ++k)
                if (ci == (uint32_t)k) nc = rx[k];
            x_min = child_min(x_min, ci, size);
            x_c0 = nc;
            x_d += 1;
            have = true;
        }
    }
    for (int o = 16; o; o >>= 1) {
        acc += __shfl_xor_sync(FULL, acc, o);
        nvis += __shfl_xor_sync(FULL, nvis, o);
    }
    if (lane == 0) {
        if (acc) atomicAdd(accepted, acc);
        if (nvis) atomicAdd(visits, nvis);
    }
}

// Pruned field repair: skipped reliable leaves (need == 0, E + S >= the
// threshold) that are positive and share a face with a negative leaf, and
// whose value's side of EPSILON is not proved.  DMC interpolates along
// dual-cell edges, which join face neighbours, so only the two ends of a
// sign change matter; the negative end's value is -EPS whatever its prior
// (Occupancy.cpp:570-587), and with one end at -EPS the vertex snaps to an
// end, decided by whether the positive end's value exceeds EPS
// (DualMarchingCell.cpp:51-71).
__global__ void k_repair_mark(uint32_t nl, const uint32_t *nb_off, const uint32_t *nbs, const double *occ,
                              const uint8_t *need, const uint8_t *pred, const double *esum, const double *ssum,
                              double threshold, uint8_t *mark) {
    uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    auto skipped = [&](uint32_t x) {
        return !need[x] && !((esum[x] + ssum[x]) < threshold) && !(pred[x] & (PRED_HIGH | PRED_LOW));
    };
    const bool pl = occ[l] > 0.0;
    for (uint32_t e = nb_off[l]; e < nb_off[l + 1]; ++e) {
        const uint32_t m = nbs[e];
        if ((occ[m] > 0.0) == pl) continue;
        const uint32_t positive = pl ? l : m;
        if (skipped(positive)) mark[positive] = 1;
    }
}

__global__ void k_flag_equal(uint32_t n, const uint8_t *v, uint8_t value, uint8_t *flag) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = v[i] == value ? 1 : 0;
}

__global__ void k_set_needed(uint32_t n, const uint32_t *list, uint8_t *need) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) need[list[i]] = 1;
}

// Depth of every listed leaf (list == null: leaves 0 .. n-1) as a sort key.
__global__ void k_leaf_depth_keys(uint32_t n, const uint32_t *list, const uint32_t *leaf_node, const uint8_t *depth,
                                  uint32_t *keys, uint32_t *vals) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t l = list ? list[i] : i;
    keys[i] = depth[leaf_node[l]];
    vals[i] = l;
}

__global__ void k_iota(uint32_t n, uint32_t *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = i;
}

// A leaf carries a type's flag exactly when it received a kernel of that type.
__global__ void k_leaf_flags(uint32_t nl, const uint32_t *leaf_node, const double *ksum, uint32_t *states,
                             uint32_t flag) {
    uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    if (ksum[l] > 0.0) states[leaf_node[l]] |= flag;
}

// Camera of every listed link (list == null: links 0 .. nlinks-1), as sort keys.
__global__ void k_link_cameras(uint64_t nlinks, const uint32_t *list, const uint32_t *links, uint32_t ncams,
                               uint32_t *keys, uint32_t *vals) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nlinks) return;
    const uint32_t l = list ? list[i] : (uint32_t)i;
    uint32_t c = links[l];
    keys[i] = (c == INVALID || c >= ncams) ? ncams : c;
    vals[i] = l;
}

// The links of the chosen samples: sample s has links s K .. s K + K - 1.
__global__ void k_sample_links(uint32_t count, const uint32_t *samples, uint32_t k, uint32_t *out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)count * k) return;
    out[i] = samples[i / k] * k + (uint32_t)(i % k);
}

// forwardAnyChildStateFlag, one level bottom-up.
__global__ void k_forward_flag(uint32_t lo, uint32_t hi, const uint32_t *order, const uint32_t *children,
                               uint32_t *states, uint32_t flag) {
    uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hi) return;
    uint32_t n = order[i];
    uint32_t c0 = children[n];
    if (c0 == INVALID) return;
    uint32_t s = states[n] & ~flag;
    for (uint32_t c = 0; c < 8; ++c)
        if (states[c0 + c] & flag) s |= flag;
    states[n] = s;
}

// Cumulative prior sums per node: psum[k * nn + node] = sum of (emptiness,
// sampleness) cone lengths over SAMPLENESS-flagged leaves of the node's
// subtree at most k levels below the node.  Built bottom-up, one level per
// launch.  Rows are k-major so that the eight siblings of a children block
// share one 128-byte line per k.
constexpr int PK = 8;

__global__ void k_prior_sums(uint32_t lo, uint32_t hi, uint32_t nn, const uint32_t *order,
                             const uint32_t *children, const uint32_t *node_to_leaf, const uint32_t *states,
                             const double *elen, const double *slen, double2 *psum) {
    uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hi) return;
    uint32_t n = order[i];
    uint32_t c0 = children[n];
    if (c0 == INVALID) {
        double2 v = make_double2(0.0, 0.0);
        if (states[n] & FLAG_SAMPLENESS) {
            uint32_t l = node_to_leaf[n];
            v = make_double2(elen[l], slen[l]);
        }
        for (int k = 0; k < PK; ++k) psum[(size_t)k * nn + n] = v;
        return;
    }
    psum[n] = make_double2(0.0, 0.0);
    for (int k = 1; k < PK; ++k) {
        const double2 *row = psum + (size_t)(k - 1) * nn + c0;
        double e = 0.0, s = 0.0;
        for (uint32_t c = 0; c < 8; ++c) {
            double2 v = row[c];
            e += v.x;
            s += v.y;
        }
        psum[(size_t)k * nn + n] = make_double2(e, s);
    }
}

// intersectAABBWithSphere as the tree build evaluates it (aabb_sphere), with
// the per-axis branches turned into selects: an axis where the centre lies
// within the box adds an exact +0, so the sum is bit-identical.
__device__ __forceinline__ bool sphere_meets_box(const D3 &mn, const D3 &mx, const D3 &c, double r) {
    const double tx = c.x < mn.x ? dsub(c.x, mn.x) : (c.x > mx.x ? dsub(c.x, mx.x) : 0.0);
    const double ty = c.y < mn.y ? dsub(c.y, mn.y) : (c.y > mx.y ? dsub(c.y, mx.y) : 0.0);
    const double tz = c.z < mn.z ? dsub(c.z, mn.z) : (c.z > mx.z ? dsub(c.z, mx.z) : 0.0);
    const double d2 = dadd(dadd(dmul(tx, tx), dmul(ty, ty)), dmul(tz, tz));
    return d2 <= dmul(r, r);
}

// Box entirely inside the sphere, with a strict relative margin so that every
// leaf below certainly passes the closed sphere/box test.
__device__ inline bool box_inside_sphere(const D3 &mn, double sz, const D3 &c, double r) {
    double dx = fmax(fabs(c.x - mn.x), fabs(mn.x + sz - c.x));
    double dy = fmax(fabs(c.y - mn.y), fabs(mn.y + sz - c.y));
    double dz = fmax(fabs(c.z - mn.z), fabs(mn.z + sz - c.z));
    return dx * dx + dy * dy + dz * dz <= r * r * (1.0 - 1e-9);
}

// Occupancy::computePriors (Occupancy.cpp:530-568) with a
// SphereNodeStatesChecker (SphereNodeStatesChecker.cpp:28-36).  The set of
// summed leaves is the reference's: SAMPLENESS-flagged leaves at most three
// levels below the query leaf whose box meets the sphere (the exact FP64
// test); subtrees wholly inside the sphere are added from psum, whose row 0
// of a leaf is the leaf's own (emptiness, sampleness) cone-length pair.
//
// Run by persistent threads over the traversal records of the cone passes,
// expanding one node per step: its eight children's records come in one
// 64-byte line and their FP64 boxes are derived from the parent's corner with
// the tree build's own recurrence (child_coords, exact), so no node geometry
// is loaded inside the loop.
//
// BOUNDS (the pruned field's sign certificates): a node that straddles the
// sphere at depth >= the query leaf's depth - coarse_up is not descended;
// its whole subtree row is added to an undecided pair (eU, sU) instead, so
// the query ends early with eL <= E <= eL + eU and sL <= S <= sL + sU for
// the exact sums E, S, and writes bounds[i] = (eL / (eL + sL + sU),
// (eL + eU) / (eL + eU + sL)) around the prior E / (E + S).
template <bool BOUNDS>
__global__ void __launch_bounds__(PT_BLOCK, TSR_PRIOR_BLOCKS) k_priors_x(uint32_t nl, uint32_t nn, const uint32_t *list,
                                                      const uint32_t *leaf_node, const D3 *leaf_min,
                                                      const uint8_t *depth, const D3 *nmin, const uint2 *rec,
                                                      const double2 *psum, double root_size, double rel_radius,
                                                      double *prior, unsigned long long *next_leaf,
                                                      unsigned long long *visits, int *err, double2 *bounds,
                                                      uint32_t coarse_up) {
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31;
    uint64_t st[MAX_TREE_DEPTH];   // children block | mask << 32 | depth << 40
    int sp = 0;
    bool have = false, active = false, done = false;
    uint32_t x_c0 = 0, x_d = 0;
    D3 x_min{0.0, 0.0, 0.0};
    uint32_t l = 0, max_depth = 0, qi = 0, stop_depth = 0;
    D3 center{0.0, 0.0, 0.0};
    double radius = 0.0, eL = 0.0, sL = 0.0, eU = 0.0, sU = 0.0;
    float r2f = 0.0f;
    unsigned long long nvis = 0;
    auto add_row = [&](uint32_t n, uint32_t k) {
        double2 v = psum[(size_t)k * nn + n];
        eL += v.x;
        sL += v.y;
    };
    while (true) {
        if (!have && sp > 0) {
            uint64_t e = st[sp - 1];
            uint32_t m = (uint32_t)(e >> 32) & 0xFFu;
            uint32_t node = (uint32_t)e + (uint32_t)(__ffs(m) - 1);
            m &= m - 1;
            if (m) st[sp - 1] = (e & ~(0xFFull << 32)) | ((uint64_t)m << 32); else --sp;
            x_c0 = __ldg(&rec[node + REC_OFFSET]).x;
            x_min = nmin[node];   // the build's own FP64 corner of that node
            x_d = (uint32_t)(e >> 40) + 1;
            have = true;
        }
        if (!have && active) {   // query finished
            if (BOUNDS)
                bounds[qi] = make_double2(eL / (eL + sL + sU), (eL + eU) / (eL + eU + sL));
            else
                prior[l] = eL / (eL + sL);
            active = false;
        }
        bool need = !have && !done;
        unsigned nm = __ballot_sync(FULL, need);
        if (nm) {
            int leader = __ffs(nm) - 1;
            unsigned long long b = 0;
            if ((int)lane == leader) b = atomicAdd(next_leaf, (unsigned long long)__popc(nm));
            b = __shfl_sync(FULL, b, leader);
            if (need) {
                uint64_t i = b + __popc(nm & ((1u << lane) - 1u));
                if (i >= nl) {
                    done = true;
                } else {
                    qi = (uint32_t)i;
                    l = list ? list[i] : (uint32_t)i;
                    uint32_t node = leaf_node[l];
                    uint32_t ld = depth[node];
                    stop_depth = ld > coarse_up + 1 ? ld - coarse_up : 1;
                    double size = size_at(root_size, ld);
                    D3 mn = leaf_min[l];
                    double half = dmul(0.5, size);
                    center = D3{dadd(mn.x, half), dadd(mn.y, half), dadd(mn.z, half)};
                    radius = dmul(size, rel_radius);
                    r2f = (float)dmul(radius, radius);
                    max_depth = ld + MAX_DEPTH_DIFFERENCE;
                    eL = sL = eU = sU = 0.0;
                    active = true;
                    // the root (SphereNodeStatesChecker on node 0)
                    uint2 r0 = __ldg(&rec[REC_OFFSET]);
                    D3 bmn = nmin[0];
                    D3 bmx{dadd(bmn.x, root_size), dadd(bmn.y, root_size), dadd(bmn.z, root_size)};
                    if ((r0.y & REC_FLAG) && aabb_sphere(bmn, bmx, center, radius)) {
                        if (max_depth < (uint32_t)PK && box_inside_sphere(bmn, root_size, center, radius)) {
                            add_row(0, max_depth);
                        } else if (r0.x == INVALID) {
                            add_row(0, 0);
                        } else if (1 <= max_depth) {
                            x_c0 = r0.x;
                            x_min = bmn;
                            x_d = 1;
                            have = true;
                        }
                    }
                }
            }
        }
        if (__all_sync(FULL, done && !have && sp == 0 && !active)) break;
        if (!have) continue;
        have = false;
        if ((x_c0 & 7u) != 1u || x_c0 > 0xFFFFFFF0u) {
            atomicExch(err, 3);
            continue;
        }
        const uint4 *line = reinterpret_cast<const uint4 *>(rec + x_c0 + REC_OFFSET);
        uint4 q0 = __ldg(line), q1 = __ldg(line + 1), q2 = __ldg(line + 2), q3 = __ldg(line + 3);
        const uint32_t rx[8] = {q0.x, q0.z, q1.x, q1.z, q2.x, q2.z, q3.x, q3.z};
        const uint32_t ry[8] = {q0.y, q0.w, q1.y, q1.w, q2.y, q2.w, q3.y, q3.w};
        const double cs = ldexp(root_size, -(int)x_d);
        const uint32_t d = x_d;
        const bool can_descend = d + 1 <= max_depth;
        const bool can_add = d <= max_depth && max_depth - d < (uint32_t)PK;
        uint32_t mask = 0;
        nvis += 8;
        if (d <= max_depth) {
            // Every test for every child without branches; only the outcome
            // (a row to add, or a child to descend into) is conditional.  The
            // exact FP64 tests run only where an FP32 estimate in the query
            // centre's frame cannot decide: its error is bounded by e_a per
            // axis (rounding of the frame offset and of two FP32 adds) plus
            // 4e-7 of the squared distances, and a decision needs a margin
            // of 1e-6 r^2 beyond that.  The rows of all eight children are
            // loaded before any is added, so their L2 latencies overlap
            // (adding 0 for the others is exact).
            const float csf = (float)cs;
            const float rx0 = (float)dsub(x_min.x, center.x), ry0 = (float)dsub(x_min.y, center.y),
                        rz0 = (float)dsub(x_min.z, center.z);
            const float ex = 4e-7f * (fabsf(rx0) + 2.0f * csf), ey = 4e-7f * (fabsf(ry0) + 2.0f * csf),
                        ez = 4e-7f * (fabsf(rz0) + 2.0f * csf);
            // Every child reads row krow: an added subtree needs row
            // max_depth - d (< PK wherever one is added), and a leaf's rows
            // are all equal, so the eight children's pairs come from one
            // 128-byte line.
            const uint32_t krow = max_depth - d < (uint32_t)PK ? max_depth - d : (uint32_t)PK - 1u;
            double2 v[8];
            uint32_t umask = 0;
#pragma unroll
            for (int ci = 0; ci < 8; ++ci) {
                const bool flagged = (ry[ci] & REC_FLAG) != 0;
                const bool leaf = rx[ci] == INVALID;
                const float lx = (ci & 1) ? rx0 + csf : rx0, ly = (ci & 2) ? ry0 + csf : ry0,
                            lz = (ci & 4) ? rz0 + csf : rz0;
                const float hx = lx + csf, hy = ly + csf, hz = lz + csf;
                const float tx = lx > 0.0f ? lx : (hx < 0.0f ? -hx : 0.0f);
                const float ty = ly > 0.0f ? ly : (hy < 0.0f ? -hy : 0.0f);
                const float tz = lz > 0.0f ? lz : (hz < 0.0f ? -hz : 0.0f);
                const float d2 = tx * tx + ty * ty + tz * tz;
                const float b1 = 2.0f * ((tx + ex) * ex + (ty + ey) * ey + (tz + ez) * ez) + 4e-7f * d2;
                const float fx = fmaxf(fabsf(lx), fabsf(hx)), fy = fmaxf(fabsf(ly), fabsf(hy)),
                            fz = fmaxf(fabsf(lz), fabsf(hz));
                const float D2 = fx * fx + fy * fy + fz * fz;
                const float b2 = 2.0f * ((fx + ex) * ex + (fy + ey) * ey + (fz + ez) * ez) + 4e-7f * D2;
                bool meets = d2 + b1 < r2f * (1.0f - 1e-6f);
                bool inside = can_add && (D2 + b2 < r2f * (1.0f - 2e-6f));
                const bool meets_unsure = !meets && !(d2 - b1 > r2f * (1.0f + 1e-6f));
                const bool inside_unsure = can_add && !inside && !(D2 - b2 > r2f * (1.0f + 1e-6f));
                if (flagged && (meets_unsure || ((meets || meets_unsure) && inside_unsure))) {
                    const D3 bmn = child_coords(x_min, cs, (uint32_t)ci);
                    const D3 bmx{dadd(bmn.x, cs), dadd(bmn.y, cs), dadd(bmn.z, cs)};
                    meets = sphere_meets_box(bmn, bmx, center, radius);
                    inside = can_add && box_inside_sphere(bmn, cs, center, radius);
                }
                meets = meets && flagged;
                // BOUNDS: a straddling node at or below the stop depth is undecided
                // (max_depth - d <= 3 + coarse_up < PK there)
                const bool unc = BOUNDS && meets && !inside && !leaf && d >= stop_depth;
                const size_t row = (size_t)krow * nn + x_c0 + ci;
                v[ci] = (meets && (inside || leaf || unc)) ? __ldg(&psum[row]) : make_double2(0.0, 0.0);
                if (unc) umask |= 1u << ci;
                if (meets && !inside && !leaf && can_descend && !unc) mask |= 1u << ci;
            }
#pragma unroll
            for (int ci = 0; ci < 8; ++ci) {
                if (BOUNDS && ((umask >> ci) & 1u)) {
                    eU += v[ci].x;
                    sU += v[ci].y;
                } else {
                    eL += v[ci].x;
                    sL += v[ci].y;
                }
            }
        }
        if (mask) {
            uint32_t ci = __ffs(mask) - 1;
            uint32_t rest = mask & (mask - 1);
            if (rest) {
                if (sp >= MAX_TREE_DEPTH) {
                    atomicExch(err, 2);
                    continue;
                }
                st[sp++] = (uint64_t)x_c0 | ((uint64_t)rest << 32) | ((uint64_t)d << 40);
            }
            uint32_t nc = rx[0];
#pragma unroll
            for (int k = 1; k < 8; ++k)
                if (ci == (uint32_t)k) nc = rx[k];
            x_min = child_coords(x_min, cs, ci);
            x_c0 = nc;
            x_d = d + 1;
            have = true;
        }
    }
    for (int o = 16; o; o >>= 1) nvis += __shfl_xor_sync(FULL, nvis, o);
    if (lane == 0 && nvis) atomicAdd(visits, nvis);
}

// Occupancy::getOccupancy (Occupancy.cpp:570-587), FP64.
// Occupancy::getOccupancy (Occupancy.cpp:570-587), FP64.  In a pruned field
// (pred != null) a reliable leaf whose prior was not queried (need == 0)
// gets its sign from E == 0 / S == 0 or from the pruner, and the value
// 0.5 (S - E) / coneCount for a positive sign (the value at prior 1/2), so
// only leaves away from a predicted sign change carry an approximate value.
__global__ void k_finalize(uint32_t nl, const double *esum, const double *ssum, const double *elen,
                           const double *slen, const double *prior, double cone_count, double threshold,
                           const uint8_t *pred, const uint8_t *need, double *o_esum, double *o_ssum,
                           double *o_elen, double *o_slen, double *occ) {
    uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    double e = esum[l], s = ssum[l];
    o_esum[l] = e;
    o_ssum[l] = s;
    o_elen[l] = elen[l];
    o_slen[l] = slen[l];
    double v;
    if ((e + s) < threshold) {
        v = -EPS;
    } else if (pred && !need[l]) {
        const bool pos = (e == 0.0) ? true : (s == 0.0) ? false : (pred[l] & PRED_POS) != 0;
        const double approx = 0.5 * (s - e) / cone_count;
        if (pos && (pred[l] & PRED_HIGH))
            v = approx > 2.0 * EPS ? approx : 2.0 * EPS;   // above EPSILON, like the exact value
        else if (pos && (pred[l] & PRED_LOW))
            v = EPS;                                       // at most EPSILON, like the exact value
        else
            v = (pos && approx > 0.0) ? approx : (pos ? EPS : -EPS);
    } else {
        double pr = prior[l];
        double pe = pr * (e / cone_count);
        double ps = (1.0 - pr) * (s / cone_count);
        v = (pe >= ps) ? -EPS : ps - pe;
    }
    occ[l] = v;
}

struct Timer {
    cudaEvent_t a{}, b{};
    cudaStream_t st;
    explicit Timer(cudaStream_t s) : st(s) {
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
    ~Timer() { cudaEventDestroy(a); cudaEventDestroy(b); }
};

// Prior queries in order of leaf depth, coarsest first, tree order within a
// depth (a stable radix sort of 6-bit keys).  A coarse leaf's sphere is wide
// and its query long; taking those first keeps the persistent lanes from
// ending on a tail of long queries, and a warp's lanes share one radius.
static_assert(MAX_TREE_DEPTH <= 64, "depth keys are 6 bits");
DBuf<uint32_t> depth_ordered(uint32_t n, const uint32_t *list, const uint32_t *leaf_node, const uint8_t *depth,
                             cudaStream_t st) {
    DBuf<uint32_t> out(n, st);
    if (n == 0) return out;
    DBuf<uint32_t> k1(n, st), k2(n, st), v1(n, st);
    k_leaf_depth_keys<<<grid_for(n, BLK), BLK, 0, st>>>(n, list, leaf_node, depth, k1.p, v1.p);
    ::tsr::note_launch();
    size_t tmp = 0;
    TSR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k1.p, k2.p, v1.p, out.p, (int)n, 0, 6, st));
    DBuf<uint8_t> tb(tmp, st);
    TSR_CUDA(cub::DeviceRadixSort::SortPairs(tb.p, tmp, k1.p, k2.p, v1.p, out.p, (int)n, 0, 6, st));
    return out;
}

}  // namespace

// The field of all links (update == false), or an update of an existing
// field by the links of `chosen` samples (device indices, tree order) added
// (sign +1) or removed (sign -1): Occupancy::update (Occupancy.h:222-227)
// after onSamplesChanged (Occupancy.cpp:129-136) -- both cone passes over the
// chosen links into the field's sums, node flags set only when adding, then
// the priors and the occupancy of every leaf again.
void compute_occupancy(const tsr_tree &t, const tsr_cameras_view &cv, const tsr_params &p, int mode,
                       tsr_occupancy &o, const tsr_pruner *pruner, const uint32_t *chosen, uint32_t nchosen,
                       double sign, bool update) {
    (void)mode;
    cudaStream_t st = o.stream;
    const uint32_t nl = t.n_leaves, nn = t.n_nodes;
    o.n_leaves = nl;
    o.n_nodes = nn;
    o.confidence_threshold = p.confidence_threshold;
    const uint64_t nlinks = update ? (uint64_t)nchosen * t.k : (uint64_t)t.n_samples * t.k;
    // working set: per link the set-up record, keys and order; per node the
    // traversal records, states and the prior table; per leaf the sums
    reserve_pool((size_t)nlinks * 160 + (size_t)nn * 200 + (size_t)nl * 120 + (64u << 20), o.stream);
    Timer timer(st);
    DBuf<D3> cams(cv.count, st);
    if (cv.count) TSR_CUDA(cudaMemcpyAsync(cams.p, cv.positions, (size_t)cv.count * 24, cudaMemcpyHostToDevice, st));
    DBuf<double> acc;   // esum, ssum, elen, slen of a new field
    double *esum, *ssum, *elen, *slen;
    DBuf<uint32_t> link_list;
    if (update) {
        esum = o.e_sum.p; ssum = o.s_sum.p; elen = o.e_len.p; slen = o.s_len.p;
        link_list.alloc(nlinks, st);
        k_sample_links<<<grid_for(nlinks, BLK), BLK, 0, st>>>(nchosen, chosen, t.k, link_list.p); ::tsr::note_launch();
    } else {
        acc.alloc(4ull * nl, st);
        acc.zero();
        esum = acc.p; ssum = acc.p + nl; elen = acc.p + 2ull * nl; slen = acc.p + 3ull * nl;
        o.states.alloc(nn, st);
        o.states.zero();
    }
    DBuf<double> cone_count(1, st);
    cone_count.zero();
    DBuf<unsigned long long> accepted(5, st);   // accepted E, S; visits E, S; prior visits
    accepted.zero();
    DBuf<int> err(1, st);
    err.zero();

    LinkIn in{t.pos.p, t.nrm.p, t.scale.p, t.conf.p, t.links.p, cams.p, t.k, cv.count,
              p.max_relative_sampling_distance, p.bandwidth_factor, p.relative_sample_cone_length, t.root_size};
    TreeIn tr{t.nmin.p};
    if (!update) o.links = nlinks;
    DBuf<unsigned long long> next_link(1, st);
    unsigned x_grid = 0, prior_grid = 0;
    {
        int dev = 0, sms = 0, per_sm = 0;
        TSR_CUDA(cudaGetDevice(&dev));
        TSR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        TSR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cone_x<EMPTINESS>, PT_BLOCK, 0));
        x_grid = (unsigned)(sms * (per_sm > 0 ? per_sm : 1));
        TSR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_priors_x<false>, PT_BLOCK, 0));
        prior_grid = (unsigned)(sms * (per_sm > 0 ? per_sm : 1));
    }
    if (nl > REC_NOLEAF) fail(TSR_ERR_OVERFLOW_U32, "leaf count must stay below 2^31 - 1 for the traversal records");
    DBuf<uint2> recs((size_t)nn + 8, st);
    if (reinterpret_cast<uintptr_t>(recs.p) % 16) fail(TSR_ERR_CUDA, "traversal records are not 16-byte aligned");
    next_link.zero();
    k_pack_rec<<<grid_for(nn, BLK), BLK, 0, st>>>(nn, t.children.p, t.node_to_leaf.p, nullptr, recs.p); ::tsr::note_launch();
    DBuf<LinkRec> lrec((size_t)nlinks, st);
    if (nlinks) {
        k_link_setup<SAMPLENESS><<<grid_for(nlinks, 128), 128, 0, st>>>(nlinks, link_list.p, in, tr, recs.p, lrec.p,
                                                                        ssum, slen, cone_count.p, accepted.p + 1,
                                                                        sign);
        ::tsr::note_launch();
        k_cone_x<SAMPLENESS><<<x_grid, PT_BLOCK, 0, st>>>(nlinks, lrec.p, tr, recs.p, (float)t.root_size, ssum, slen,
                                                         accepted.p + 1, next_link.p, accepted.p + 3, err.p, sign);
        ::tsr::note_launch();
    }
    // flags mark leaves that received a kernel; removal leaves them set (Occupancy.cpp:232)
    if (sign > 0.0) {
        k_leaf_flags<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, t.leaf_node.p, ssum, o.states.p, FLAG_SAMPLENESS);
        ::tsr::note_launch();
    }
    o.stage_ms[0] = timer.lap();
    // EMPTINESS links grouped by camera (stable, so sample order is kept
    // within a camera): a warp's cones then share their apex
    DBuf<uint32_t> order((size_t)nlinks, st);
    {
        DBuf<uint32_t> ckeys((size_t)nlinks, st), ckeys2((size_t)nlinks, st), vals((size_t)nlinks, st);
        if (nlinks) {
            k_link_cameras<<<grid_for(nlinks, BLK), BLK, 0, st>>>(nlinks, link_list.p, t.links.p, cv.count, ckeys.p,
                                                                  vals.p); ::tsr::note_launch();
        }
        int bits = 1;
        while ((1u << bits) <= cv.count) ++bits;
        size_t tmp = 0;
        if (nlinks) {
            TSR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, ckeys.p, ckeys2.p, vals.p, order.p, (int)nlinks, 0,
                                                     bits, st));
            DBuf<uint8_t> tb(tmp, st);
            TSR_CUDA(cub::DeviceRadixSort::SortPairs(tb.p, tmp, ckeys.p, ckeys2.p, vals.p, order.p, (int)nlinks, 0,
                                                     bits, st));
        }
    }
    // forwardAnyChildStateFlag(0, SAMPLENESS) before the EMPTINESS pass (Occupancy.cpp:141-142)
    for (int d = (int)t.level_start.size() - 2; d >= 0; --d) {
        uint32_t lo = t.level_start[d], hi = t.level_start[d + 1];
        k_forward_flag<<<grid_for(hi - lo, BLK), BLK, 0, st>>>(lo, hi, t.level_order.p, t.children.p, o.states.p,
                                                              FLAG_SAMPLENESS); ::tsr::note_launch();
    }
    k_pack_rec<<<grid_for(nn, BLK), BLK, 0, st>>>(nn, t.children.p, t.node_to_leaf.p, o.states.p, recs.p);
    ::tsr::note_launch();
    o.stage_ms[1] = timer.lap();
    next_link.zero();
    if (nlinks) {
        k_link_setup<EMPTINESS><<<grid_for(nlinks, 128), 128, 0, st>>>(nlinks, order.p, in, tr, recs.p, lrec.p, esum,
                                                                       elen, cone_count.p, accepted.p, sign);
        ::tsr::note_launch();
        k_cone_x<EMPTINESS><<<x_grid, PT_BLOCK, 0, st>>>(nlinks, lrec.p, tr, recs.p, (float)t.root_size, esum, elen,
                                                        accepted.p, next_link.p, accepted.p + 2, err.p, sign);
        ::tsr::note_launch();
    }
    if (sign > 0.0) {
        k_leaf_flags<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, t.leaf_node.p, esum, o.states.p, FLAG_EMPTINESS);
        ::tsr::note_launch();
    }
    o.stage_ms[2] = timer.lap();
    o.prior.alloc(nl, st);
    DBuf<uint8_t> need;   // pruned field: leaves whose prior is queried
    DBuf<uint8_t> pred_buf;
    if (pruner) pruner_predict(t, *pruner, esum, ssum, p.confidence_threshold, pred_buf, st);
    const uint8_t *pred = pred_buf.p;
    if (pred) {
        o.prior.fill_bytes(0xFF);   // NaN: no prior where the query was skipped
        need.alloc(nl, st);
        k_prior_needed<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, pred, esum, ssum, p.confidence_threshold, need.p);
        ::tsr::note_launch();
    }
    DBuf<double2> psum;   // cumulative prior sums (kept for the pruned field's repairs)
    {
        // the queried leaves: all of them, or the selected ones of a pruned field
        DBuf<uint32_t> list;
        uint32_t nq = nl;
        psum.alloc((size_t)nn * PK, st);
        for (int d = (int)t.level_start.size() - 2; d >= 0; --d) {
            uint32_t lo = t.level_start[d], hi = t.level_start[d + 1];
            k_prior_sums<<<grid_for(hi - lo, BLK), BLK, 0, st>>>(lo, hi, nn, t.level_order.p, t.children.p,
                                                                t.node_to_leaf.p, o.states.p, elen, slen, psum.p); ::tsr::note_launch();
        }
        if (pred) {
            DBuf<uint32_t> ids(nl, st), nsel(1, st), clist(nl, st);
            DBuf<uint8_t> cflag(nl, st);
            DBuf<unsigned long long> ncert(1, st);
            ncert.zero();
            list.alloc(nl, st);
            k_iota<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, ids.p); ::tsr::note_launch();
            size_t tmp = 0;
            TSR_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, ids.p, need.p, list.p, nsel.p, (int)nl, st));
            DBuf<uint8_t> tb(tmp, st);
            // skip candidates: certify their signs from bounds of their priors
            k_flag_equal<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, need.p, NEED_CERTIFY, cflag.p); ::tsr::note_launch();
            TSR_CUDA(cub::DeviceSelect::Flagged(tb.p, tmp, ids.p, cflag.p, clist.p, nsel.p, (int)nl, st));
            const uint32_t nc = read_scalar(nsel.p, st);
            if (nc) {
                clist = depth_ordered(nc, clist.p, t.leaf_node.p, t.depth.p, st);
                DBuf<double2> bnd(nc, st);
                next_link.zero();
                k_priors_x<true><<<prior_grid, PT_BLOCK, 0, st>>>(nc, nn, clist.p, t.leaf_node.p, t.leaf_min.p,
                                                                  t.depth.p, t.nmin.p, recs.p, psum.p, t.root_size,
                                                                  p.relative_radius_for_priors, nullptr, next_link.p,
                                                                  accepted.p + 4, err.p, bnd.p, pruner->bound_levels);
                ::tsr::note_launch();
                k_certify<<<grid_for(nc, BLK), BLK, 0, st>>>(nc, clist.p, esum, ssum, bnd.p, cone_count.p,
                                                            pred_buf.p, need.p,
                                                            ncert.p); ::tsr::note_launch();
                o.certified = read_scalar(ncert.p, st);
            }
            // every leaf still needing its prior (need 1) is queried
            TSR_CUDA(cub::DeviceSelect::Flagged(tb.p, tmp, ids.p, need.p, list.p, nsel.p, (int)nl, st));
            nq = read_scalar(nsel.p, st);
            o.pruned = nl - nq;
        }
        list = depth_ordered(nq, list.p, t.leaf_node.p, t.depth.p, st);
        next_link.zero();
        k_priors_x<false><<<prior_grid, PT_BLOCK, 0, st>>>(nq, nn, list.p, t.leaf_node.p, t.leaf_min.p, t.depth.p,
                                                          t.nmin.p, recs.p, psum.p, t.root_size,
                                                          p.relative_radius_for_priors, o.prior.p, next_link.p,
                                                          accepted.p + 4, err.p, nullptr, 0);
        ::tsr::note_launch();
    }
    o.stage_ms[3] = timer.lap();
    if (update) {
        o.cone_count += read_scalar(cone_count.p, st);
    } else {
        o.cone_count = read_scalar(cone_count.p, st);
        o.e_sum.alloc(nl, st); o.s_sum.alloc(nl, st); o.e_len.alloc(nl, st); o.s_len.alloc(nl, st);
        o.occ.alloc(nl, st);
    }
    k_finalize<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, esum, ssum, elen, slen, o.prior.p, o.cone_count,
                                                 p.confidence_threshold, pred, need.p, o.e_sum.p, o.s_sum.p,
                                                 o.e_len.p, o.s_len.p, o.occ.p); ::tsr::note_launch();
    if (pred) {
        // Repair: a skipped positive leaf next to a negative one carries a
        // value the surface uses (the signs themselves are exact); query its
        // prior and recompute it, until no such leaf is left (one round
        // queries them all; the next finds none).
        DBuf<uint8_t> mark(nl, st);
        DBuf<uint32_t> ids(nl, st), flist(nl, st), nsel(1, st);
        k_iota<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, ids.p); ::tsr::note_launch();
        size_t tmp = 0;
        TSR_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, ids.p, mark.p, flist.p, nsel.p, (int)nl, st));
        DBuf<uint8_t> tb(tmp, st);
        for (int round = 0; round < 64; ++round) {
            mark.zero();
            k_repair_mark<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, t.nb_off.p, t.nbs.p, o.occ.p, need.p, pred, esum, ssum,
                                                            p.confidence_threshold, mark.p); ::tsr::note_launch();
            TSR_CUDA(cub::DeviceSelect::Flagged(tb.p, tmp, ids.p, mark.p, flist.p, nsel.p, (int)nl, st));
            const uint32_t nf = read_scalar(nsel.p, st);
            if (nf == 0) break;
            k_set_needed<<<grid_for(nf, BLK), BLK, 0, st>>>(nf, flist.p, need.p); ::tsr::note_launch();
            DBuf<uint32_t> fq = depth_ordered(nf, flist.p, t.leaf_node.p, t.depth.p, st);
            next_link.zero();
            k_priors_x<false><<<prior_grid, PT_BLOCK, 0, st>>>(nf, nn, fq.p, t.leaf_node.p, t.leaf_min.p,
                                                              t.depth.p, t.nmin.p, recs.p, psum.p, t.root_size,
                                                              p.relative_radius_for_priors, o.prior.p, next_link.p,
                                                              accepted.p + 4, err.p, nullptr, 0); ::tsr::note_launch();
            k_finalize<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, esum, ssum, elen, slen, o.prior.p, o.cone_count,
                                                         p.confidence_threshold, pred, need.p, o.e_sum.p, o.s_sum.p,
                                                         o.e_len.p, o.s_len.p, o.occ.p); ::tsr::note_launch();
            o.pruned -= nf;
            o.repaired += nf;
        }
    }
    o.stage_ms[4] = timer.lap();
    unsigned long long a[5];
    TSR_CUDA(cudaMemcpyAsync(a, accepted.p, sizeof(a), cudaMemcpyDeviceToHost, st));
    int e = read_scalar(err.p, st);
    o.accepted[0] = a[0];
    o.accepted[1] = a[1];
    o.visits[0] = a[2];
    o.visits[1] = a[3];
    o.visits[2] = a[4];
    if (e == 3) fail(TSR_ERR_DEVICE_ASSERT, "occupancy traversal met a children block off its 8-node alignment");
    if (e) fail(TSR_ERR_DEVICE_ASSERT, "occupancy traversal exceeded its stack bound");
    TSR_CUDA(cudaGetLastError());
}

// The occupancy of every leaf from sums, cone lengths, priors and cone count
// already in the field's buffers (a field read from a file): the plain
// formula of k_finalize, sums copied onto themselves.
void finalize_field(tsr_occupancy &o, const tsr_params &p) {
    const uint32_t nl = o.n_leaves;
    o.occ.alloc(nl, o.stream);
    if (!nl) return;
    k_finalize<<<grid_for(nl, BLK), BLK, 0, o.stream>>>(nl, o.e_sum.p, o.s_sum.p, o.e_len.p, o.s_len.p, o.prior.p,
                                                       o.cone_count, p.confidence_threshold, nullptr, nullptr,
                                                       o.e_sum.p, o.s_sum.p, o.e_len.p, o.s_len.p, o.occ.p);
    ::tsr::note_launch();
    TSR_CUDA(cudaGetLastError());
}

}  // namespace tsr
