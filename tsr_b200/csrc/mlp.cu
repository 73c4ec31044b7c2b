// mlp.cu -- the learned pruner of the occupancy field.
//
// A small MLP (10 leaf features -> 64 -> 64 -> 2 logits: "occupancy > 0" and
// "near a sign change") is trained on fields the plain method computes and
// then decides, per leaf, whether the most expensive per-leaf step, the
// prior query, can be skipped.  This file holds:
//   * the per-leaf feature kernels (local sample statistics of the tree and
//     the cone passes' sums, with neighbour extremes),
//   * FP32 training kernels (forward + backward with block-level gradient
//     reductions, Adam), driven from the host through the C ABI,
//   * the BF16 tensor-core inference kernel (mma.sync m16n8k16, FP32
//     accumulation; the three layers chain through registers),
//   * the keep mask of the pruned field (thresholds + neighbour dilation).
// None of this has a counterpart in the reference; the features only read
// the tree and the sums the field computation produced.
#include <cuda_bf16.h>

#include <cmath>
#include <vector>

#include "handles.h"

namespace tsr {

namespace {

constexpr int NF = TSR_MLP_FEATURES;   // 10
constexpr int NH = TSR_MLP_HIDDEN;     // 64
constexpr int NO = TSR_MLP_OUTPUTS;    // 2
// parameter blob offsets (FP32): W1 [NF][NH], b1, W2 [NH][NH], b2, W3 [NH][NO], b3
constexpr int OW1 = 0, OB1 = OW1 + NF * NH, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH,
              OB3 = OW3 + NH * NO, NPARAM = OB3 + NO;
static_assert(NPARAM == TSR_MLP_PARAMS, "parameter layout");

constexpr unsigned BLK = 256;

// ------------------------------------------------------------- features
// Per leaf, from the tree's samples and the two cone passes' sums (what is
// known before the prior queries): log1p(samples in the leaf), log(mean
// sample scale / leaf size), normal spread 1 - |mean normal|, depth / 16,
// log1p(E), log1p(S), r = S / (E + S) (-1 when both are 0), reliability
// (E + S >= confidenceThreshold), and the smallest and largest r among the
// face neighbours (the leaf's own r without neighbours).
__global__ void k_leaf_features(uint32_t nl, const uint32_t *leaf_node, const uint32_t *counts,
                                const uint32_t *starts, const uint8_t *depth, const double *scale, const D3 *nrm,
                                double root_size, const double *esum, const double *ssum, double threshold,
                                float *out, int *rmin, int *rmax) {
    uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    const uint32_t node = leaf_node[l];
    const uint32_t cnt = counts[node], s0 = starts[node];
    const double size = ldexp(root_size, -(int)depth[node]);
    double ssum_sc = 0.0, nx = 0.0, ny = 0.0, nz = 0.0;
    for (uint32_t j = 0; j < cnt; ++j) {
        const uint32_t s = s0 + j;
        ssum_sc += scale[s];
        const D3 n = nrm[s];
        nx += n.x; ny += n.y; nz += n.z;
    }
    const double e = esum[l], sv = ssum[l];
    const float r = (e + sv) > 0.0 ? (float)(sv / (e + sv)) : -1.0f;
    float *f = out + (size_t)l * NF;
    f[0] = log1pf((float)cnt);
    f[1] = cnt ? (float)log(ssum_sc / cnt / size) : 0.0f;
    f[2] = cnt ? (float)(1.0 - sqrt(nx * nx + ny * ny + nz * nz) / cnt) : 0.0f;
    f[3] = (float)depth[node] * (1.0f / 16.0f);
    f[4] = (float)log1p(e);
    f[5] = (float)log1p(sv);
    f[6] = r;
    f[7] = (e + sv) < threshold ? 0.0f : 1.0f;
    // r + 2 > 0, so its float bits order like the values (for the atomics)
    const int key = __float_as_int(r + 2.0f);
    rmin[l] = key;
    rmax[l] = key;
}

// Neighbour extremes of r over the face-neighbour CSR (each pair once, so
// both directions are updated).
__global__ void k_neighbour_r(uint32_t nl, const uint32_t *nb_off, const uint32_t *nbs, const float *feat,
                              int *rmin, int *rmax) {
    uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    const int kl = __float_as_int(feat[(size_t)l * NF + 6] + 2.0f);
    for (uint32_t e = nb_off[l]; e < nb_off[l + 1]; ++e) {
        const uint32_t m = nbs[e];
        const int km = __float_as_int(feat[(size_t)m * NF + 6] + 2.0f);
        atomicMin(&rmin[l], km);
        atomicMax(&rmax[l], km);
        atomicMin(&rmin[m], kl);
        atomicMax(&rmax[m], kl);
    }
}

__global__ void k_feature_minmax(uint32_t nl, const int *rmin, const int *rmax, float *feat) {
    uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    feat[(size_t)l * NF + 8] = __int_as_float(rmin[l]) - 2.0f;
    feat[(size_t)l * NF + 9] = __int_as_float(rmax[l]) - 2.0f;
}

// ------------------------------------------------------------- training
// One block of TR_ROWS threads takes TR_ROWS rows: every thread runs its
// row's forward and backward pass (activations and their gradients go to
// shared memory), then the block reduces the weight gradients over its rows
// as small GEMMs and adds them to the global gradient with one atomic per
// entry.  Loss: binary cross-entropy with logits on both outputs, positive
// rows weighted by pos_weight[k].
constexpr int TR_ROWS = 64;
constexpr int LD = NH + 1;   // row stride of the activation tiles (no bank conflicts)

__device__ __forceinline__ float sigmoidf_(float z) { return 1.0f / (1.0f + expf(-z)); }
// log(1 + exp(-|z|)) + max(z, 0) - z y  (stable BCE with logits)
__device__ __forceinline__ float bce_logits(float z, float y) {
    return fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z)));
}

__global__ void __launch_bounds__(TR_ROWS) k_mlp_train(uint32_t n, const float *x, const float *y,
                                                     const float *params, float *grads, float *loss,
                                                     float pw0, float pw1) {
    extern __shared__ float sm[];
    float *P = sm;                          // NPARAM
    float *X = P + NPARAM;                  // TR_ROWS * NF
    float *H1 = X + TR_ROWS * NF;           // TR_ROWS * LD
    float *H2 = H1 + TR_ROWS * LD;          // TR_ROWS * LD
    float *D2 = H2 + TR_ROWS * LD;          // dL/d(pre-activation of layer 2), TR_ROWS * LD
    float *D1 = D2 + TR_ROWS * LD;          // dL/d(pre-activation of layer 1), TR_ROWS * LD
    float *DO = D1 + TR_ROWS * LD;          // TR_ROWS * NO
    __shared__ float red[TR_ROWS];
    const int t = threadIdx.x;
    for (int i = t; i < NPARAM; i += TR_ROWS) P[i] = params[i];
    const uint32_t row = blockIdx.x * TR_ROWS + t;
    const bool valid = row < n;
    for (int f = 0; f < NF; ++f) X[t * NF + f] = valid ? x[(size_t)row * NF + f] : 0.0f;
    __syncthreads();
    float l = 0.0f;
    {
        // forward
        for (int h = 0; h < NH; ++h) {
            float a = P[OB1 + h];
            for (int f = 0; f < NF; ++f) a += X[t * NF + f] * P[OW1 + f * NH + h];
            H1[t * LD + h] = fmaxf(a, 0.0f);
        }
        for (int h = 0; h < NH; ++h) {
            float a = P[OB2 + h];
            for (int j = 0; j < NH; ++j) a += H1[t * LD + j] * P[OW2 + j * NH + h];
            H2[t * LD + h] = fmaxf(a, 0.0f);
        }
        float o[NO];
        for (int k = 0; k < NO; ++k) {
            float a = P[OB3 + k];
            for (int j = 0; j < NH; ++j) a += H2[t * LD + j] * P[OW3 + j * NO + k];
            o[k] = a;
        }
        // loss and its gradient
        for (int k = 0; k < NO; ++k) {
            const float yk = valid ? y[(size_t)row * NO + k] : 0.0f;
            const float w = yk > 0.5f ? (k == 0 ? pw0 : pw1) : 1.0f;
            l += valid ? w * bce_logits(o[k], yk) : 0.0f;
            DO[t * NO + k] = valid ? w * (sigmoidf_(o[k]) - yk) : 0.0f;
        }
        // backward through the hidden layers
        for (int h = 0; h < NH; ++h) {
            float g = 0.0f;
            for (int k = 0; k < NO; ++k) g += P[OW3 + h * NO + k] * DO[t * NO + k];
            D2[t * LD + h] = H2[t * LD + h] > 0.0f ? g : 0.0f;
        }
        for (int h = 0; h < NH; ++h) {
            float g = 0.0f;
            for (int j = 0; j < NH; ++j) g += P[OW2 + h * NH + j] * D2[t * LD + j];
            D1[t * LD + h] = H1[t * LD + h] > 0.0f ? g : 0.0f;
        }
    }
    red[t] = l;
    __syncthreads();
    if (t == 0) {
        float s = 0.0f;
        for (int i = 0; i < TR_ROWS; ++i) s += red[i];
        atomicAdd(loss, s);
    }
    // weight gradients: sums over the block's rows
    for (int e = t; e < NPARAM; e += TR_ROWS) {
        float g = 0.0f;
        if (e < OB1) {                       // W1[f][h]
            const int f = e / NH, h = e % NH;
            for (int r = 0; r < TR_ROWS; ++r) g += X[r * NF + f] * D1[r * LD + h];
        } else if (e < OW2) {                // b1[h]
            const int h = e - OB1;
            for (int r = 0; r < TR_ROWS; ++r) g += D1[r * LD + h];
        } else if (e < OB2) {                // W2[j][h]
            const int j = (e - OW2) / NH, h = (e - OW2) % NH;
            for (int r = 0; r < TR_ROWS; ++r) g += H1[r * LD + j] * D2[r * LD + h];
        } else if (e < OW3) {                // b2[h]
            const int h = e - OB2;
            for (int r = 0; r < TR_ROWS; ++r) g += D2[r * LD + h];
        } else if (e < OB3) {                // W3[j][k]
            const int j = (e - OW3) / NO, k = (e - OW3) % NO;
            for (int r = 0; r < TR_ROWS; ++r) g += H2[r * LD + j] * DO[r * NO + k];
        } else {                             // b3[k]
            const int k = e - OB3;
            for (int r = 0; r < TR_ROWS; ++r) g += DO[r * NO + k];
        }
        if (g != 0.0f) atomicAdd(&grads[e], g);
    }
}

__global__ void k_adam(uint32_t np, float *p, const float *g, float *m, float *v, float lr, float b1, float b2,
                       float eps, float c1, float c2, float gscale) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const float gi = g[i] * gscale;
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// FP32 forward pass, one thread per row (for evaluation and as the reference
// of the BF16 kernel).
__global__ void k_mlp_forward(uint32_t n, const float *x, const float *params, float *out) {
    __shared__ float P[NPARAM];
    for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    float xin[NF], h1[NH];
    for (int f = 0; f < NF; ++f) xin[f] = x[(size_t)row * NF + f];
    for (int h = 0; h < NH; ++h) {
        float a = P[OB1 + h];
        for (int f = 0; f < NF; ++f) a += xin[f] * P[OW1 + f * NH + h];
        h1[h] = fmaxf(a, 0.0f);
    }
    float o[NO];
    for (int k = 0; k < NO; ++k) o[k] = P[OB3 + k];
    for (int h = 0; h < NH; ++h) {
        float a = P[OB2 + h];
        for (int j = 0; j < NH; ++j) a += h1[j] * P[OW2 + j * NH + h];
        a = fmaxf(a, 0.0f);
        for (int k = 0; k < NO; ++k) o[k] += a * P[OW3 + h * NO + k];
    }
    for (int k = 0; k < NO; ++k) out[(size_t)row * NO + k] = o[k];
}

// ------------------------------------------------- BF16 tensor-core inference
// Weights as mma.sync B fragments (K x N, "col"), BF16 pairs, laid out
// [layer tiles][register][lane] so that a warp's loads are conflict-free:
//   layer 1: K = 16 (10 features, zero padded), N = 64  -> 1 x 8 tiles
//   layer 2: K = 64, N = 64                            -> 4 x 8 tiles
//   layer 3: K = 64, N = 8 (2 outputs, zero padded)    -> 4 x 1 tiles
// Fragment of tile (t, j), lane L: reg 0 = W[16t + 2(L%4) + {0,1}][8j + L/4],
// reg 1 = W[16t + 8 + 2(L%4) + {0,1}][8j + L/4].
constexpr int FRAG1 = 1 * 8 * 2 * 32, FRAG2 = 4 * 8 * 2 * 32, FRAG3 = 4 * 1 * 2 * 32;
constexpr int NFRAG = FRAG1 + FRAG2 + FRAG3;

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Builds the fragment table from the FP32 parameters (one thread per word).
__global__ void k_mlp_pack_frags(const float *P, uint32_t *frag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NFRAG) return;
    int rel = i, K, N, ow, nt;
    if (rel < FRAG1) { K = NF; N = NH; ow = OW1; nt = 8; }
    else if ((rel -= FRAG1) < FRAG2) { K = NH; N = NH; ow = OW2; nt = 8; }
    else { rel -= FRAG2; K = NH; N = NO; ow = OW3; nt = 1; }
    const int lane = rel % 32, reg = (rel / 32) % 2, tile = rel / 64;
    const int t = tile / nt, j = tile % nt;
    const int n = 8 * j + lane / 4;
    const int k0 = 16 * t + 8 * reg + 2 * (lane % 4);
    const float lo = (k0 < K && n < N) ? P[ow + k0 * N + n] : 0.0f;
    const float hi = (k0 + 1 < K && n < N) ? P[ow + (k0 + 1) * N + n] : 0.0f;
    frag[i] = pack_bf16(lo, hi);
}

// Logits of n rows of normalized features; each warp takes 16 rows at a time.
__global__ void __launch_bounds__(128) k_mlp_infer(uint32_t n, const float *x, const uint32_t *frag_g,
                                                 const float *params, float *out) {
    __shared__ uint32_t frag[NFRAG];
    __shared__ float bias[NH + NH + 8];
    for (int i = threadIdx.x; i < NFRAG; i += blockDim.x) frag[i] = frag_g[i];
    for (int i = threadIdx.x; i < NH; i += blockDim.x) {
        bias[i] = params[OB1 + i];
        bias[NH + i] = params[OB2 + i];
    }
    if (threadIdx.x < 8) bias[2 * NH + threadIdx.x] = threadIdx.x < NO ? params[OB3 + threadIdx.x] : 0.0f;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t r = lane >> 2, cpair = 2 * (lane & 3);
    const uint32_t *F1 = frag, *F2 = frag + FRAG1, *F3 = frag + FRAG1 + FRAG2;
    for (uint32_t base = warp * 16; base < n; base += nwarps * 16) {
        // layer 1: A = features (16 x 16, columns >= NF are zero)
        const uint32_t r0 = base + r, r1 = base + r + 8;
        auto xv = [&](uint32_t row, uint32_t col) -> float {
            return (row < n && col < (uint32_t)NF) ? x[(size_t)row * NF + col] : 0.0f;
        };
        uint32_t a[4];
        a[0] = pack_bf16(xv(r0, cpair), xv(r0, cpair + 1));
        a[1] = pack_bf16(xv(r1, cpair), xv(r1, cpair + 1));
        a[2] = pack_bf16(xv(r0, cpair + 8), xv(r0, cpair + 9));
        a[3] = pack_bf16(xv(r1, cpair + 8), xv(r1, cpair + 9));
        float c1[8][4];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            c1[j][0] = c1[j][1] = c1[j][2] = c1[j][3] = 0.0f;
            mma_bf16(c1[j], a, F1[(j * 2 + 0) * 32 + lane], F1[(j * 2 + 1) * 32 + lane]);
        }
        // bias + ReLU, then the C fragments of tiles 2t, 2t+1 are the A fragment of k-step t
        uint32_t a2[4][4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = 2 * t + h;
                const float b0 = bias[8 * j + cpair], b1 = bias[8 * j + cpair + 1];
                a2[t][2 * h + 0] = pack_bf16(fmaxf(c1[j][0] + b0, 0.0f), fmaxf(c1[j][1] + b1, 0.0f));
                a2[t][2 * h + 1] = pack_bf16(fmaxf(c1[j][2] + b0, 0.0f), fmaxf(c1[j][3] + b1, 0.0f));
            }
        }
        float c2[8][4];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            c2[j][0] = c2[j][1] = c2[j][2] = c2[j][3] = 0.0f;
#pragma unroll
            for (int t = 0; t < 4; ++t)
                mma_bf16(c2[j], a2[t], F2[((t * 8 + j) * 2 + 0) * 32 + lane], F2[((t * 8 + j) * 2 + 1) * 32 + lane]);
        }
        uint32_t a3[4][4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = 2 * t + h;
                const float b0 = bias[NH + 8 * j + cpair], b1 = bias[NH + 8 * j + cpair + 1];
                a3[t][2 * h + 0] = pack_bf16(fmaxf(c2[j][0] + b0, 0.0f), fmaxf(c2[j][1] + b1, 0.0f));
                a3[t][2 * h + 1] = pack_bf16(fmaxf(c2[j][2] + b0, 0.0f), fmaxf(c2[j][3] + b1, 0.0f));
            }
        }
        float c3[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int t = 0; t < 4; ++t) mma_bf16(c3, a3[t], F3[(t * 2 + 0) * 32 + lane], F3[(t * 2 + 1) * 32 + lane]);
        if ((lane & 3) == 0) {   // columns 0 and 1 are the two logits
            if (r0 < n) {
                out[(size_t)r0 * NO + 0] = c3[0] + bias[2 * NH + 0];
                out[(size_t)r0 * NO + 1] = c3[1] + bias[2 * NH + 1];
            }
            if (r1 < n) {
                out[(size_t)r1 * NO + 0] = c3[2] + bias[2 * NH + 0];
                out[(size_t)r1 * NO + 1] = c3[3] + bias[2 * NH + 1];
            }
        }
    }
}

// ----------------------------------------------------------- keep mask
__global__ void k_normalize(uint32_t nl, float *feat, const float *mean, const float *istd) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)nl * NF) return;
    const int f = i % NF;
    feat[i] = (feat[i] - mean[f]) * istd[f];
}

// Per-leaf prediction: PRED_KEEP when P(near a sign change) >= band_p,
// PRED_POS / PRED_NEG when P(occupancy > 0) is above 1 - sign_p / below sign_p.
__global__ void k_predict(uint32_t nl, const float *logits, float band_logit, float sign_logit, uint8_t *pred) {
    uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    const float zs = logits[(size_t)l * NO + 0], zb = logits[(size_t)l * NO + 1];
    uint8_t p = 0;
    if (zb >= band_logit) p |= PRED_KEEP;
    if (zs >= -sign_logit) p |= PRED_POS;       // P >= 1 - sign_p
    if (zs <= sign_logit) p |= PRED_NEG;        // P <= sign_p
    pred[l] = p;
}

// One ring of face neighbours around every PRED_KEEP leaf (the neighbour
// CSR stores each pair once, so both directions are written here).
__global__ void k_dilate(uint32_t nl, const uint32_t *nb_off, const uint32_t *nbs, const uint8_t *pred,
                         uint8_t *out) {
    uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    const bool kl = pred[l] & PRED_KEEP;
    uint8_t mine = pred[l];
    for (uint32_t e = nb_off[l]; e < nb_off[l + 1]; ++e) {
        const uint32_t m = nbs[e];
        if (kl) atomicOr(reinterpret_cast<unsigned int *>(out + (m & ~3u)), (unsigned)PRED_KEEP << (8 * (m & 3u)));
        if (pred[m] & PRED_KEEP) mine |= PRED_KEEP;
    }
    atomicOr(reinterpret_cast<unsigned int *>(out + (l & ~3u)), (unsigned)mine << (8 * (l & 3u)));
}

}  // namespace

// ------------------------------------------------------------ host side
void leaf_features(const tsr_tree &t, const double *esum, const double *ssum, double threshold, DBuf<float> &feat,
                   cudaStream_t st) {
    const uint32_t nl = t.n_leaves;
    feat.alloc((size_t)nl * NF, st);
    DBuf<int> rmin(nl, st), rmax(nl, st);
    k_leaf_features<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, t.leaf_node.p, t.counts.p, t.starts.p, t.depth.p,
                                                       t.scale.p, t.nrm.p, t.root_size, esum, ssum, threshold,
                                                       feat.p, rmin.p, rmax.p); ::tsr::note_launch();
    k_neighbour_r<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, t.nb_off.p, t.nbs.p, feat.p, rmin.p, rmax.p);
    ::tsr::note_launch();
    k_feature_minmax<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, rmin.p, rmax.p, feat.p); ::tsr::note_launch();
    TSR_CUDA(cudaGetLastError());
}

void mlp_train_batch(const float *x, const float *y, uint32_t n, const float *params, float *grads, float *loss,
                     float pw0, float pw1, cudaStream_t st) {
    if (n == 0) return;
    const size_t smem = (size_t)(NPARAM + TR_ROWS * NF + 4 * TR_ROWS * LD + TR_ROWS * NO) * sizeof(float);
    static bool attr_set = false;
    if (!attr_set) {
        TSR_CUDA(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set = true;
    }
    k_mlp_train<<<(n + TR_ROWS - 1) / TR_ROWS, TR_ROWS, smem, st>>>(n, x, y, params, grads, loss, pw0, pw1);
    ::tsr::note_launch();
    TSR_CUDA(cudaGetLastError());
}

void mlp_adam(float *p, const float *g, float *m, float *v, uint32_t step, float lr, float gscale,
              cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)step), c2 = 1.0f - std::pow(b2, (float)step);
    k_adam<<<grid_for(NPARAM, BLK), BLK, 0, st>>>(NPARAM, p, g, m, v, lr, b1, b2, 1e-8f, c1, c2, gscale);
    ::tsr::note_launch();
    TSR_CUDA(cudaGetLastError());
}

void mlp_forward(const float *x, uint32_t n, const float *params, float *out, cudaStream_t st) {
    if (n == 0) return;
    k_mlp_forward<<<grid_for(n, 128), 128, 0, st>>>(n, x, params, out); ::tsr::note_launch();
    TSR_CUDA(cudaGetLastError());
}

void mlp_infer_bf16(const float *x, uint32_t n, const float *params, float *out, cudaStream_t st) {
    if (n == 0) return;
    DBuf<uint32_t> frag(NFRAG, st);
    k_mlp_pack_frags<<<grid_for(NFRAG, BLK), BLK, 0, st>>>(params, frag.p); ::tsr::note_launch();
    int dev = 0, sms = 0;
    TSR_CUDA(cudaGetDevice(&dev));
    TSR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint64_t tiles = (n + 15) / 16;
    uint64_t blocks = (tiles + 3) / 4;
    const uint64_t cap = (uint64_t)sms * 8;
    if (blocks > cap) blocks = cap;
    k_mlp_infer<<<(unsigned)blocks, 128, 0, st>>>(n, x, frag.p, params, out); ::tsr::note_launch();
    TSR_CUDA(cudaGetLastError());
}

void pruner_predict(const tsr_tree &t, const tsr_pruner &pr, const double *esum, const double *ssum,
                    double threshold, DBuf<uint8_t> &pred, cudaStream_t st) {
    const uint32_t nl = t.n_leaves;
    DBuf<float> feat;
    leaf_features(t, esum, ssum, threshold, feat, st);
    DBuf<float> norm(2 * NF, st), params(NPARAM, st), logits((size_t)nl * NO, st);
    float hnorm[2 * NF];
    for (int f = 0; f < NF; ++f) { hnorm[f] = pr.feature_mean[f]; hnorm[NF + f] = pr.feature_inv_std[f]; }
    TSR_CUDA(cudaMemcpyAsync(norm.p, hnorm, sizeof(hnorm), cudaMemcpyHostToDevice, st));
    TSR_CUDA(cudaMemcpyAsync(params.p, pr.weights, NPARAM * sizeof(float), cudaMemcpyHostToDevice, st));
    k_normalize<<<grid_for((size_t)nl * NF, BLK), BLK, 0, st>>>(nl, feat.p, norm.p, norm.p + NF); ::tsr::note_launch();
    mlp_infer_bf16(feat.p, nl, params.p, logits.p, st);
    auto logit = [](float p) { return std::log(p / (1.0f - p)); };
    // padded to whole 32-bit words for the dilation's byte-wise atomics
    const size_t nw = ((size_t)nl + 3) & ~(size_t)3;
    DBuf<uint8_t> p0(nw, st);
    k_predict<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, logits.p, logit(pr.band_threshold), logit(pr.sign_threshold),
                                                 p0.p); ::tsr::note_launch();
    for (uint32_t r = 0; r < pr.dilation; ++r) {
        DBuf<uint8_t> p1(nw, st);
        p1.zero();
        k_dilate<<<grid_for(nl, BLK), BLK, 0, st>>>(nl, t.nb_off.p, t.nbs.p, p0.p, p1.p); ::tsr::note_launch();
        p0 = std::move(p1);
    }
    pred = std::move(p0);
    TSR_CUDA(cudaGetLastError());
}

}  // namespace tsr
