// common.cuh -- shared plumbing and FP64 geometry of the TSR sm_100a core.
//
// FP64 geometry below is written with explicit round-to-nearest intrinsics
// (__dadd_rn, __dmul_rn, ...) so no multiply-add contraction can change a
// rounding: tree topology decisions must match an FP64 CPU evaluation of the
// same expressions bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/tsr_core.h"

namespace tsr {

constexpr uint32_t INVALID = 0xFFFFFFFFu;
constexpr double EPS = 1e-6;                       // Math::EPSILON (Real = double)
constexpr double REAL_MAX = 1.7976931348623157e308;
constexpr uint32_t MAX_DEPTH_DIFFERENCE = 3;       // Occupancy.cpp:72
constexpr uint32_t FLAG_SAMPLENESS = 1u;           // Occupancy.h:38
constexpr uint32_t FLAG_EMPTINESS = 2u;            // Occupancy.h:39
// per-leaf predictions of the learned pruner: near a sign change (or within
// the dilation ring), confidently positive, confidently not positive
constexpr uint8_t PRED_KEEP = 1, PRED_POS = 2, PRED_NEG = 4;
// A certified positive leaf whose value is proved above EPSILON / at most EPSILON.
constexpr uint8_t PRED_HIGH = 8, PRED_LOW = 16;
constexpr int MAX_TREE_DEPTH = 40;                 // stack bound of the traversals

struct Error {
    tsr_status status;
    std::string msg;
};

[[noreturn]] void fail(tsr_status st, const std::string &msg);
void note_launch();   // counts this library's kernel launches (instrumentation)
// Iteration bounds of the tree build (tsr_set_iteration_limits): conflict
// waves per sampling round (a device-side loop) and host rounds.
uint32_t limit_sampling_waves();
uint32_t limit_rounds();
void check_cuda(cudaError_t e, const char *what);
#define TSR_CUDA(call) ::tsr::check_cuda((call), #call)

// Stream-ordered device buffer.
template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaStream_t st = nullptr;
    DBuf() = default;
    DBuf(size_t count, cudaStream_t s) { alloc(count, s); }
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    DBuf(DBuf &&o) noexcept : p(o.p), n(o.n), st(o.st) { o.p = nullptr; o.n = 0; }
    DBuf &operator=(DBuf &&o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; st = o.st; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DBuf() { release(); }
    void alloc(size_t count, cudaStream_t s) {
        release();
        st = s;
        n = count;
        if (count) {
            cudaError_t e = cudaMallocAsync((void **)&p, count * sizeof(T), s);
            if (e != cudaSuccess) {
                p = nullptr;
                n = 0;
                (void)cudaGetLastError();
                fail(TSR_ERR_OOM, std::string("device allocation failed: ") + cudaGetErrorString(e));
            }
        }
    }
    void release() {
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        n = 0;
    }
    void zero() { if (n) TSR_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), st)); }
    void fill_bytes(int v) { if (n) TSR_CUDA(cudaMemsetAsync(p, v, n * sizeof(T), st)); }
    T *get() const { return p; }
};

template <class T>
inline T read_scalar(const T *dev, cudaStream_t st) {
    T v;
    TSR_CUDA(cudaMemcpyAsync(&v, dev, sizeof(T), cudaMemcpyDeviceToHost, st));
    TSR_CUDA(cudaStreamSynchronize(st));
    return v;
}

inline unsigned grid_for(size_t n, unsigned block) {
    size_t g = (n + block - 1) / block;
    return (unsigned)(g ? g : 1);
}

// ------------------------------------------------------------ FP64 geometry
struct D3 {
    double x, y, z;
};

__host__ __device__ inline double dadd(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ inline double dsub(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
__host__ __device__ inline double dmul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}

__host__ __device__ inline D3 d3sub(const D3 &a, const D3 &b) { return D3{dsub(a.x, b.x), dsub(a.y, b.y), dsub(a.z, b.z)}; }
__host__ __device__ inline double d3dot(const D3 &a, const D3 &b) {
    return dadd(dadd(dmul(a.x, b.x), dmul(a.y, b.y)), dmul(a.z, b.z));
}
__host__ __device__ inline double d3len2(const D3 &a) { return d3dot(a, a); }

// Nodes.h:154-162
__host__ __device__ inline bool node_contains(const D3 &p, const D3 &mn, double size, double tol) {
    return p.x >= dsub(mn.x, tol) && p.x < dadd(dadd(mn.x, size), tol) &&
           p.y >= dsub(mn.y, tol) && p.y < dadd(dadd(mn.y, size), tol) &&
           p.z >= dsub(mn.z, tol) && p.z < dadd(dadd(mn.z, size), tol);
}

// Nodes.cpp:46-58
__host__ __device__ inline D3 child_coords(const D3 &mn, double step, uint32_t i) {
    D3 c = mn;
    if (i & 1u) c.x = dadd(c.x, step);
    if (i & 2u) c.y = dadd(c.y, step);
    if (i & 4u) c.z = dadd(c.z, step);
    return c;
}

// Nodes.cpp:60-84
__host__ __device__ inline D3 side_center(const D3 &mn, double size, uint32_t side, double step) {
    double half = dmul(size, 0.5);
    D3 p{dadd(mn.x, half), dadd(mn.y, half), dadd(mn.z, half)};
    double d = dadd(half, step);
    switch (side) {
        case 0: p.x = dsub(p.x, d); break;
        case 1: p.x = dadd(p.x, d); break;
        case 2: p.y = dsub(p.y, d); break;
        case 3: p.y = dadd(p.y, d); break;
        case 4: p.z = dsub(p.z, d); break;
        default: p.z = dadd(p.z, d); break;
    }
    return p;
}

// Signed distance to the sample's tangent plane (Samples.cpp:451-455).
__host__ __device__ inline double plane_distance(const D3 &p, const D3 &n, const D3 &x) {
    return d3dot(d3sub(x, p), n);
}

// Closed sphere / AABB overlap (squared box distance <= r^2).
__host__ __device__ inline bool aabb_sphere(const D3 &mn, const D3 &mx, const D3 &c, double r) {
    double d2 = 0.0;
    if (c.x < mn.x) { double t = dsub(c.x, mn.x); d2 = dadd(d2, dmul(t, t)); }
    else if (c.x > mx.x) { double t = dsub(c.x, mx.x); d2 = dadd(d2, dmul(t, t)); }
    if (c.y < mn.y) { double t = dsub(c.y, mn.y); d2 = dadd(d2, dmul(t, t)); }
    else if (c.y > mx.y) { double t = dsub(c.y, mx.y); d2 = dadd(d2, dmul(t, t)); }
    if (c.z < mn.z) { double t = dsub(c.z, mn.z); d2 = dadd(d2, dmul(t, t)); }
    else if (c.z > mx.z) { double t = dsub(c.z, mx.z); d2 = dadd(d2, dmul(t, t)); }
    return d2 <= dmul(r, r);
}

// Slab clipping of s + t (e - s), t in [0, 1].
__host__ __device__ inline bool segment_aabb(double &t0, double &t1, const D3 &s, const D3 &e,
                                             const D3 &mn, const D3 &mx) {
    double lo = 0.0, hi = 1.0;
    const double sv[3] = {s.x, s.y, s.z};
    const double dv[3] = {dsub(e.x, s.x), dsub(e.y, s.y), dsub(e.z, s.z)};
    const double bmn[3] = {mn.x, mn.y, mn.z};
    const double bmx[3] = {mx.x, mx.y, mx.z};
    for (int a = 0; a < 3; ++a) {
        if (dv[a] == 0.0) {
            if (sv[a] < bmn[a] || sv[a] > bmx[a]) return false;
            continue;
        }
        double inv = 1.0 / dv[a];
        double ta = dmul(dsub(bmn[a], sv[a]), inv);
        double tb = dmul(dsub(bmx[a], sv[a]), inv);
        if (ta > tb) { double t = ta; ta = tb; tb = t; }
        if (ta > lo) lo = ta;
        if (tb < hi) hi = tb;
        if (lo > hi) return false;
    }
    t0 = lo;
    t1 = hi;
    return true;
}

// Node edge length at a depth: repeated exact halving of the root size.
__host__ __device__ inline double size_at(double root_size, uint32_t depth) {
    double s = root_size;
    for (uint32_t i = 0; i < depth; ++i) s = dmul(s, 0.5);
    return s;
}

}  // namespace tsr
