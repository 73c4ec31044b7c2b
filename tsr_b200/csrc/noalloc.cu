// noalloc.cu -- the root scope of a device-resident sample set, computed with
// no memory allocation at all (tsr_samples_root_scope_noalloc).
//
// Why it exists: the tree build allocates stream-ordered buffers throughout.
// Some callers cannot allow that for a step they run on their own stream: a
// host process that has already handed every byte of HBM to its own pool, or
// a pipeline whose memory use must stay fixed after start-up so that its peak
// is known in advance.  For them this entry point computes the first step of
// Tree::Tree -- the root node's scope, the cube around every sample's
// sampling-distance box -- into a buffer the caller owns.  Its only working
// memory is the fixed-size file-scope array below; it never calls cudaMalloc,
// cudaMallocAsync, cudaFree or any library routine that allocates, and on
// success it makes no host allocation either.
//
// Set-up: the first call on each device looks the scratch array's address up
// with cudaGetSymbolAddress and queries the kernel's attributes, with that
// device current.  Both may make the CUDA runtime load this library's device
// code onto that device, so make one call on each device before any stream
// capture begins; later calls only validate, clear one counter and launch.
//
// Concurrency: every call on a device shares the one scratch array, so two
// calls on the same device that can overlap in time (different streams with
// no ordering between them) race and give wrong scopes.  Order them on one
// stream or with events.
#include <mutex>

#include "handles.h"

namespace tsr {
namespace {

constexpr unsigned RS_BLOCK = 256;
// One partial box per block; 1184 = 8 resident 256-thread blocks on each of
// the 148 SMs, enough to fill the GPU for any count thanks to the grid-stride
// loop.  Scratch size: 1184 * 48 B + 4 B = 56,836 B per device.
constexpr unsigned RS_MAX_BLOCKS = 1184;
constexpr int RS_MAX_DEVICES = 64;

struct RootScratch {
    double part[RS_MAX_BLOCKS][6];   // per-block lo xyz, hi xyz; written before read, no init needed
    unsigned int done;               // blocks finished; MUST be 0 when the kernel starts
};

static __device__ __align__(256) RootScratch g_root_scratch;

__device__ __forceinline__ double dmin_(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double dmax_(double a, double b) { return b > a ? b : a; }

// Block-wide min/max of six values through shared memory; every thread gets
// the result.
__device__ void block_box(double v[6], double (*sm)[RS_BLOCK]) {
    for (int j = 0; j < 6; ++j) sm[j][threadIdx.x] = v[j];
    __syncthreads();
    for (unsigned o = RS_BLOCK / 2; o; o >>= 1) {
        if (threadIdx.x < o)
            for (int j = 0; j < 6; ++j) {
                double a = sm[j][threadIdx.x], b = sm[j][threadIdx.x + o];
                sm[j][threadIdx.x] = j < 3 ? dmin_(a, b) : dmax_(a, b);
            }
        __syncthreads();
    }
    for (int j = 0; j < 6; ++j) v[j] = sm[j][0];
    __syncthreads();
}

// Same per-sample box and same root cube as the tree build's bounds pass
// (Samples.cpp:442-449 for the box, Nodes.cpp root scope); min and max are
// order independent and the last steps use correctly rounded intrinsics, so
// the result is bit-identical to tsr_tree_root_scope of a tree built from the
// same samples.  The last block to finish reduces the partials.
__global__ void __launch_bounds__(RS_BLOCK)
k_root_scope_noalloc(uint64_t n, const double *pos, const double *scale, double h_svo,
                     RootScratch *scr, double *out) {
    __shared__ double sm[6][RS_BLOCK];
    __shared__ bool last;
    double v[6] = {REAL_MAX, REAL_MAX, REAL_MAX, -REAL_MAX, -REAL_MAX, -REAL_MAX};
    for (uint64_t s = (uint64_t)blockIdx.x * RS_BLOCK + threadIdx.x; s < n; s += (uint64_t)gridDim.x * RS_BLOCK) {
        double r = dadd(dmul(scale[s], h_svo), EPS);
        for (int j = 0; j < 3; ++j) {
            double p = pos[3 * s + j];
            v[j] = dmin_(v[j], dsub(p, r));
            v[3 + j] = dmax_(v[3 + j], dadd(p, r));
        }
    }
    block_box(v, sm);
    if (threadIdx.x == 0) {
        for (int j = 0; j < 6; ++j) scr->part[blockIdx.x][j] = v[j];
        __threadfence();
        last = atomicAdd(&scr->done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double w[6] = {REAL_MAX, REAL_MAX, REAL_MAX, -REAL_MAX, -REAL_MAX, -REAL_MAX};
    for (unsigned b = threadIdx.x; b < gridDim.x; b += RS_BLOCK)
        for (int j = 0; j < 6; ++j) {
            double x = ((volatile double *)scr->part[b])[j];
            w[j] = j < 3 ? dmin_(w[j], x) : dmax_(w[j], x);
        }
    block_box(w, sm);
    if (threadIdx.x == 0) {
        // the build's root_from_aabb: max(max(extent x, extent y), extent z)
        const double size = dmax_(dmax_(dsub(w[3], w[0]), dsub(w[4], w[1])), dsub(w[5], w[2]));
        double half = dmul(size, 0.5);
        for (int j = 0; j < 3; ++j) out[j] = dsub(dmul(dadd(w[j], w[3 + j]), 0.5), half);
        out[3] = size;
        scr->done = 0;
    }
}

struct DeviceSetup {
    RootScratch *scratch = nullptr;
    int max_blocks = 0;
};

DeviceSetup g_setup[RS_MAX_DEVICES];
std::mutex g_setup_mu;

// One-time per-device set-up with `dev` current (see the file comment).
const DeviceSetup &setup_for(int dev) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    DeviceSetup &d = g_setup[dev];
    if (d.scratch) return d;
    void *p = nullptr;
    TSR_CUDA(cudaGetSymbolAddress(&p, g_root_scratch));
    cudaFuncAttributes fa;
    TSR_CUDA(cudaFuncGetAttributes(&fa, k_root_scope_noalloc));
    int sms = 0, per_sm = 0;
    TSR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    TSR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_root_scope_noalloc, RS_BLOCK, 0));
    long long g = (long long)sms * (per_sm > 0 ? per_sm : 1);
    d.max_blocks = (int)(g < (long long)RS_MAX_BLOCKS ? g : RS_MAX_BLOCKS);
    d.scratch = static_cast<RootScratch *>(p);
    return d;
}

// Device memory of device `dev`, or managed memory.
bool on_device(const void *p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice && a.device == dev) || a.type == cudaMemoryTypeManaged;
}

}  // namespace

void root_scope_noalloc(uint64_t count, const double *positions, const double *scales, double h_svo,
                        double *out_min_xyz_size, cudaStream_t st) {
    if (!positions || !scales || !out_min_xyz_size) fail(TSR_ERR_INVALID_ARG, "null argument");
    if (count == 0) fail(TSR_ERR_INVALID_ARG, "no samples to compute a root scope for");
    if (count * 2 >= (uint64_t)INVALID)   // the tree build's limit (two sides per sample)
        fail(TSR_ERR_OVERFLOW_U32, "sample count above the tree build's limit of 2^31 - 1");
    if (!(h_svo > 0)) fail(TSR_ERR_INVALID_ARG, "parameters must be positive");
    if (((uintptr_t)positions | (uintptr_t)scales | (uintptr_t)out_min_xyz_size) & 7)
        fail(TSR_ERR_INVALID_ARG, "arrays must be 8-byte aligned doubles");
    int dev = 0;
    TSR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= RS_MAX_DEVICES) fail(TSR_ERR_INVALID_ARG, "device ordinal above 63");
    if (!on_device(positions, dev) || !on_device(scales, dev) || !on_device(out_min_xyz_size, dev))
        fail(TSR_ERR_INVALID_ARG, "positions, scales and the output must be memory of the current device");
    const DeviceSetup &d = setup_for(dev);
    uint64_t want = (count + RS_BLOCK - 1) / RS_BLOCK;
    unsigned grid = (unsigned)(want < (uint64_t)d.max_blocks ? want : (uint64_t)d.max_blocks);
    TSR_CUDA(cudaMemsetAsync(&d.scratch->done, 0, sizeof(unsigned int), st));
    k_root_scope_noalloc<<<grid, RS_BLOCK, 0, st>>>(count, positions, scales, h_svo, d.scratch,
                                                    out_min_xyz_size);
    note_launch();
    TSR_CUDA(cudaGetLastError());
}

}  // namespace tsr
