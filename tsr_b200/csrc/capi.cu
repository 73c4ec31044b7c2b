// capi.cu -- extern "C" entry points of include/tsr_core.h.
//
// Each call validates its arguments, runs on the caller's stream, converts
// internal failures into a tsr_status and keeps the message for
// tsr_last_error_message() (the reference throws FailureHandling::Exception).
#include <atomic>
#include <cstring>
#include <new>
#include <string>

#include "handles.h"

namespace tsr {

static thread_local std::string g_last_error;
static std::atomic<unsigned long long> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

constexpr uint32_t DEFAULT_SAMPLING_WAVES = 1u << 22, DEFAULT_ROUNDS = 100000;
static std::atomic<uint32_t> g_limit_waves{DEFAULT_SAMPLING_WAVES}, g_limit_rounds{DEFAULT_ROUNDS};
uint32_t limit_sampling_waves() { return g_limit_waves.load(std::memory_order_relaxed); }
uint32_t limit_rounds() { return g_limit_rounds.load(std::memory_order_relaxed); }

void fail(tsr_status st, const std::string &msg) { throw Error{st, msg}; }

void check_cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return;
    (void)cudaGetLastError();
    tsr_status st = (e == cudaErrorMemoryAllocation) ? TSR_ERR_OOM : TSR_ERR_CUDA;
    fail(st, std::string(what) + ": " + cudaGetErrorString(e));
}

// The build allocates and frees large stream-ordered buffers many times per
// call; keep freed memory in the current device's default pool instead of
// unmapping it at every synchronization (once per device).
static void keep_pool_memory() {
    static std::atomic<uint64_t> done_mask{0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= 64) { (void)cudaGetLastError(); return; }
    uint64_t bit = 1ull << dev;
    if (done_mask.load() & bit) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t threshold = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    (void)cudaGetLastError();
    done_mask.fetch_or(bit);
}

// Grows the device's default pool in one step to hold a call's working set.
// Without it the pool grew piecemeal during the call whenever a large request
// found no free block of its size, and each growth (mapping fresh memory)
// stalled the host for 5-200 ms in the middle of a reconstruction.  The pool
// keeps the memory (see keep_pool_memory), so later calls find it free.
void reserve_pool(size_t want, cudaStream_t st) {
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return;
    }
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) {
        (void)cudaGetLastError();
        return;
    }
    if (reserved >= used && reserved - used >= want) return;
    void *p = nullptr;
    if (cudaMallocAsync(&p, want, st) == cudaSuccess) {
        (void)cudaFreeAsync(p, st);
    } else {
        (void)cudaGetLastError();   // not enough memory for the reservation: allocate as we go
    }
}

template <class F>
static tsr_status guarded(F &&f) {
    try {
        keep_pool_memory();
        f();
        return TSR_OK;
    } catch (const Error &e) {
        g_last_error = e.msg;
        return e.status;
    } catch (const std::bad_alloc &) {
        g_last_error = "host allocation failed";
        return TSR_ERR_OOM;
    } catch (...) {
        g_last_error = "unexpected failure";
        return TSR_ERR_CUDA;
    }
}

static void check_params(const tsr_params &p) {
    if (!(p.max_relative_sampling_distance > 0) || !(p.bandwidth_factor > 0) ||
        !(p.relative_radius_for_priors > 0) || !(p.relative_sample_cone_length > 0))
        fail(TSR_ERR_INVALID_ARG, "parameters must be positive");
}

template <class T>
static void to_host(const DBuf<T> &b, size_t n, void *dst, cudaStream_t st) {
    if (!dst || n == 0) return;
    TSR_CUDA(cudaMemcpyAsync(dst, b.p, n * sizeof(T), cudaMemcpyDeviceToHost, st));
}

}  // namespace tsr

using namespace tsr;

extern "C" {

void tsr_params_default(tsr_params *out) {
    if (!out) return;
    out->max_relative_sampling_distance = 2.0;
    out->bandwidth_factor = 2.0;
    out->confidence_threshold = 100.0;
    out->relative_radius_for_priors = 25.0;
    out->relative_sample_cone_length = 1.0;
}

const char *tsr_last_error_message(void) { return g_last_error.c_str(); }

const char *tsr_version(void) { return "tsr_b200 core 0.1 (sm_100a)"; }

static void check_samples(const tsr_samples_view &sv, bool on_device) {
    if (sv.count == 0) fail(TSR_ERR_INVALID_ARG, "no samples to build a tree from (Scene.cpp:141-146)");
    if (sv.cams_per_sample == 0) fail(TSR_ERR_INVALID_ARG, "cams_per_sample must be >= 1");
    if (!sv.positions || !sv.normals || !sv.scales || !sv.confidences || !sv.camera_links)
        fail(TSR_ERR_INVALID_ARG, "null sample array");
    if ((uint64_t)sv.count * sv.cams_per_sample >= 0xFFFFFFFFull)
        fail(TSR_ERR_OVERFLOW_U32, "link count must stay below 2^32 - 1 (Samples.h:395-402)");
    if (!on_device)
        for (uint32_t i = 0; i < sv.count; ++i)
            if (!(sv.scales[i] > 0.0))   // Samples.cpp:280-288
                fail(TSR_ERR_INVALID_ARG, "invalid (non-positive) sample scale at index " + std::to_string(i));
}

static tsr_status tree_build_impl(const tsr_samples_view *samples, const tsr_params *params, void *cuda_stream,
                                  tsr_tree **out_tree, bool on_device) {
    if (out_tree) *out_tree = nullptr;
    return guarded([&] {
        if (!samples || !out_tree) fail(TSR_ERR_INVALID_ARG, "null argument");
        check_samples(*samples, on_device);
        tsr_params p;
        tsr_params_default(&p);
        if (params) p = *params;
        check_params(p);
        tsr_tree *t = new tsr_tree();
        t->stream = (cudaStream_t)cuda_stream;
        t->params = p;
        try {
            build_tree(*t, *samples, on_device);
        } catch (...) {
            delete t;
            throw;
        }
        *out_tree = t;
    });
}

tsr_status tsr_tree_build(const tsr_samples_view *samples, const tsr_params *params, void *cuda_stream,
                          tsr_tree **out_tree) {
    return tree_build_impl(samples, params, cuda_stream, out_tree, false);
}

tsr_status tsr_tree_build_device(const tsr_samples_view *samples, const tsr_params *params, void *cuda_stream,
                                 tsr_tree **out_tree) {
    return tree_build_impl(samples, params, cuda_stream, out_tree, true);
}

unsigned long long tsr_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

void tsr_set_iteration_limits(uint32_t max_sampling_waves, uint32_t max_rounds) {
    tsr::g_limit_waves.store(max_sampling_waves ? max_sampling_waves : tsr::DEFAULT_SAMPLING_WAVES);
    tsr::g_limit_rounds.store(max_rounds ? max_rounds : tsr::DEFAULT_ROUNDS);
}

void tsr_tree_free(tsr_tree *tree) { delete tree; }

tsr_status tsr_tree_get_counts(const tsr_tree *t, tsr_tree_counts *out) {
    return guarded([&] {
        if (!t || !out) fail(TSR_ERR_INVALID_ARG, "null argument");
        out->nodes = t->n_nodes;
        out->leaves = t->n_leaves;
        out->dual_cells = t->n_cells;
        out->neighbor_entries = t->n_nb;
        out->max_depth = t->max_depth;
        out->sampling_rounds = t->sampling_rounds;
        out->sampling_writers = t->sampling_writers;
        out->sampling_waves = t->sampling_waves;
        out->reserved = 0;
    });
}

tsr_status tsr_tree_root_scope(const tsr_tree *t, double m[4]) {
    return guarded([&] {
        if (!t || !m) fail(TSR_ERR_INVALID_ARG, "null argument");
        m[0] = t->root_min[0]; m[1] = t->root_min[1]; m[2] = t->root_min[2]; m[3] = t->root_size;
    });
}

tsr_status tsr_samples_root_scope_noalloc(uint64_t count, const double *positions, const double *scales,
                                          const tsr_params *params, double *out_min_xyz_size, void *cuda_stream) {
    return guarded([&] {
        if (!params) fail(TSR_ERR_INVALID_ARG, "null argument");
        root_scope_noalloc(count, positions, scales, params->max_relative_sampling_distance, out_min_xyz_size,
                           static_cast<cudaStream_t>(cuda_stream));
    });
}

tsr_status tsr_tree_copy_nodes(const tsr_tree *t, uint32_t *children, uint32_t *parents, uint32_t *sample_counts,
                               uint32_t *sample_starts) {
    return guarded([&] {
        if (!t) fail(TSR_ERR_INVALID_ARG, "null tree");
        to_host(t->children, t->n_nodes, children, t->stream);
        to_host(t->parents, t->n_nodes, parents, t->stream);
        to_host(t->counts, t->n_nodes, sample_counts, t->stream);
        to_host(t->starts, t->n_nodes, sample_starts, t->stream);
        TSR_CUDA(cudaStreamSynchronize(t->stream));
    });
}

tsr_status tsr_tree_copy_samples(const tsr_tree *t, double *positions, double *normals, double *scales,
                                 double *confidences, uint32_t *camera_links) {
    return guarded([&] {
        if (!t) fail(TSR_ERR_INVALID_ARG, "null tree");
        to_host(t->pos, t->n_samples, positions, t->stream);
        to_host(t->nrm, t->n_samples, normals, t->stream);
        to_host(t->scale, t->n_samples, scales, t->stream);
        to_host(t->conf, t->n_samples, confidences, t->stream);
        to_host(t->links, (size_t)t->n_samples * t->k, camera_links, t->stream);
        TSR_CUDA(cudaStreamSynchronize(t->stream));
    });
}

tsr_status tsr_tree_copy_permutation(const tsr_tree *t, uint32_t *target) {
    return guarded([&] {
        if (!t || !target) fail(TSR_ERR_INVALID_ARG, "null argument");
        to_host(t->target, t->target.n, target, t->stream);   // one entry per input sample
        TSR_CUDA(cudaStreamSynchronize(t->stream));
    });
}

tsr_status tsr_tree_copy_leaves(const tsr_tree *t, double *scopes, uint32_t *node_index, uint32_t *node_to_leaf,
                                uint32_t *nb_off, uint32_t *nbs) {
    return guarded([&] {
        if (!t) fail(TSR_ERR_INVALID_ARG, "null tree");
        if (scopes) {
            std::string tmp;
            D3 *mins = new D3[t->n_leaves ? t->n_leaves : 1];
            uint32_t *nodes = new uint32_t[t->n_leaves ? t->n_leaves : 1];
            uint8_t *depth = new uint8_t[t->n_nodes];
            try {
                to_host(t->leaf_min, t->n_leaves, mins, t->stream);
                to_host(t->leaf_node, t->n_leaves, nodes, t->stream);
                to_host(t->depth, t->n_nodes, depth, t->stream);
                TSR_CUDA(cudaStreamSynchronize(t->stream));
                for (uint32_t l = 0; l < t->n_leaves; ++l) {
                    scopes[4 * (size_t)l + 0] = mins[l].x;
                    scopes[4 * (size_t)l + 1] = mins[l].y;
                    scopes[4 * (size_t)l + 2] = mins[l].z;
                    scopes[4 * (size_t)l + 3] = size_at(t->root_size, depth[nodes[l]]);
                }
            } catch (...) {
                delete[] mins; delete[] nodes; delete[] depth;
                throw;
            }
            delete[] mins; delete[] nodes; delete[] depth;
        }
        to_host(t->leaf_node, t->n_leaves, node_index, t->stream);
        to_host(t->node_to_leaf, t->n_nodes, node_to_leaf, t->stream);
        to_host(t->nb_off, (size_t)t->n_leaves + 1, nb_off, t->stream);
        to_host(t->nbs, t->n_nb, nbs, t->stream);
        TSR_CUDA(cudaStreamSynchronize(t->stream));
    });
}

tsr_status tsr_tree_copy_dual_cells(const tsr_tree *t, uint32_t *cells8) {
    return guarded([&] {
        if (!t || !cells8) fail(TSR_ERR_INVALID_ARG, "null argument");
        to_host(t->cells, (size_t)t->n_cells * 8, cells8, t->stream);
        TSR_CUDA(cudaStreamSynchronize(t->stream));
    });
}

tsr_status tsr_tree_stage_ms(const tsr_tree *t, float *ms, int n) {
    return guarded([&] {
        if (!t || !ms) fail(TSR_ERR_INVALID_ARG, "null argument");
        for (int i = 0; i < n && i < 8; ++i) ms[i] = t->stage_ms[i];
    });
}

tsr_status tsr_occupancy_compute(const tsr_tree *tree, const tsr_cameras_view *cameras, const tsr_params *params,
                                 int mode, void *cuda_stream, tsr_occupancy **out) {
    if (out) *out = nullptr;
    return guarded([&] {
        if (!tree || !cameras || !out) fail(TSR_ERR_INVALID_ARG, "null argument");
        if (cameras->count && !cameras->positions) fail(TSR_ERR_INVALID_ARG, "null camera positions");
        if (mode != 0) fail(TSR_ERR_INVALID_ARG, "unknown occupancy mode");
        if (tree->n_leaves == 0) fail(TSR_ERR_STATE, "tree has no leaves");
        tsr_params p = tree->params;
        if (params) p = *params;
        check_params(p);
        if (p.max_relative_sampling_distance != tree->params.max_relative_sampling_distance)
            fail(TSR_ERR_INVALID_ARG, "h_SVO must match the tree's");
        tsr_occupancy *o = new tsr_occupancy();
        o->stream = (cudaStream_t)cuda_stream;
        try {
            compute_occupancy(*tree, *cameras, p, mode, *o);
        } catch (...) {
            delete o;
            throw;
        }
        *out = o;
    });
}

tsr_status tsr_occupancy_compute_pruned(const tsr_tree *tree, const tsr_cameras_view *cameras,
                                        const tsr_params *params, const tsr_pruner *pruner, void *cuda_stream,
                                        tsr_occupancy **out) {
    if (out) *out = nullptr;
    return guarded([&] {
        if (!tree || !cameras || !out || !pruner) fail(TSR_ERR_INVALID_ARG, "null argument");
        if (!pruner->weights) fail(TSR_ERR_INVALID_ARG, "null pruner weights");
        if (!(pruner->sign_threshold > 0.0f && pruner->sign_threshold < 0.5f) ||
            !(pruner->band_threshold > 0.0f && pruner->band_threshold < 1.0f))
            fail(TSR_ERR_INVALID_ARG, "pruner thresholds: sign in (0, 0.5), band in (0, 1)");
        if (pruner->dilation > 64) fail(TSR_ERR_INVALID_ARG, "pruner dilation above 64 rings");
        if (pruner->bound_levels > 4) fail(TSR_ERR_INVALID_ARG, "pruner bound_levels above 4");
        if (cameras->count && !cameras->positions) fail(TSR_ERR_INVALID_ARG, "null camera positions");
        if (tree->n_leaves == 0) fail(TSR_ERR_STATE, "tree has no leaves");
        tsr_params p = tree->params;
        if (params) p = *params;
        check_params(p);
        if (p.max_relative_sampling_distance != tree->params.max_relative_sampling_distance)
            fail(TSR_ERR_INVALID_ARG, "h_SVO must match the tree's");
        tsr_occupancy *o = new tsr_occupancy();
        o->stream = (cudaStream_t)cuda_stream;
        try {
            compute_occupancy(*tree, *cameras, p, 0, *o, pruner);
        } catch (...) {
            delete o;
            throw;
        }
        *out = o;
    });
}

tsr_status tsr_occupancy_leaf_features(const tsr_tree *t, const tsr_occupancy *o, float *features) {
    return guarded([&] {
        if (!t || !o || !features) fail(TSR_ERR_INVALID_ARG, "null argument");
        if (o->n_leaves != t->n_leaves) fail(TSR_ERR_INVALID_ARG, "field of another tree");
        DBuf<float> f;
        leaf_features(*t, o->e_sum.p, o->s_sum.p, o->confidence_threshold, f, o->stream);
        TSR_CUDA(cudaMemcpyAsync(features, f.p, (size_t)t->n_leaves * TSR_MLP_FEATURES * sizeof(float),
                                 cudaMemcpyDeviceToHost, o->stream));
        TSR_CUDA(cudaStreamSynchronize(o->stream));
    });
}

tsr_status tsr_mlp_train_batch(const float *x, const float *y, uint32_t n, const float *params, float *grads,
                               float *loss, float pos_weight0, float pos_weight1, void *cuda_stream) {
    return guarded([&] {
        if (!x || !y || !params || !grads || !loss) fail(TSR_ERR_INVALID_ARG, "null argument");
        mlp_train_batch(x, y, n, params, grads, loss, pos_weight0, pos_weight1, (cudaStream_t)cuda_stream);
    });
}

tsr_status tsr_mlp_adam(float *params, const float *grads, float *m, float *v, uint32_t step, float lr,
                        float grad_scale, void *cuda_stream) {
    return guarded([&] {
        if (!params || !grads || !m || !v) fail(TSR_ERR_INVALID_ARG, "null argument");
        if (step == 0) fail(TSR_ERR_INVALID_ARG, "Adam steps count from 1");
        mlp_adam(params, grads, m, v, step, lr, grad_scale, (cudaStream_t)cuda_stream);
    });
}

tsr_status tsr_mlp_forward(const float *x, uint32_t n, const float *params, float *logits, void *cuda_stream) {
    return guarded([&] {
        if (!x || !params || !logits) fail(TSR_ERR_INVALID_ARG, "null argument");
        mlp_forward(x, n, params, logits, (cudaStream_t)cuda_stream);
    });
}

tsr_status tsr_mlp_infer_bf16(const float *x, uint32_t n, const float *params, float *logits,
                              void *cuda_stream) {
    return guarded([&] {
        if (!x || !params || !logits) fail(TSR_ERR_INVALID_ARG, "null argument");
        mlp_infer_bf16(x, n, params, logits, (cudaStream_t)cuda_stream);
    });
}

tsr_status tsr_occupancy_update(tsr_occupancy *o, const tsr_tree *tree, const tsr_cameras_view *cameras,
                                const tsr_params *params, int for_removal, const uint32_t *samples, uint32_t count,
                                void *cuda_stream) {
    return guarded([&] {
        if (!o || !tree || !cameras || (count && !samples)) fail(TSR_ERR_INVALID_ARG, "null argument");
        if (o->n_leaves != tree->n_leaves || o->n_nodes != tree->n_nodes)
            fail(TSR_ERR_INVALID_ARG, "field of another tree");
        if (cameras->count && !cameras->positions) fail(TSR_ERR_INVALID_ARG, "null camera positions");
        for (uint32_t i = 0; i < count; ++i)
            if (samples[i] >= tree->n_samples) fail(TSR_ERR_INVALID_ARG, "sample index out of range");
        tsr_params p = tree->params;
        if (params) p = *params;
        check_params(p);
        o->stream = (cudaStream_t)cuda_stream;
        DBuf<uint32_t> chosen(count, o->stream);
        if (count)
            TSR_CUDA(cudaMemcpyAsync(chosen.p, samples, (size_t)count * 4, cudaMemcpyHostToDevice, o->stream));
        compute_occupancy(*tree, *cameras, p, 0, *o, nullptr, chosen.p, count, for_removal ? -1.0 : 1.0, true);
    });
}

tsr_status tsr_tree_erase_samples(tsr_tree *t, const uint8_t *inliers) {
    return guarded([&] {
        if (!t || !inliers) fail(TSR_ERR_INVALID_ARG, "null argument");
        DBuf<uint8_t> in(t->n_samples, t->stream);
        TSR_CUDA(cudaMemcpyAsync(in.p, inliers, t->n_samples, cudaMemcpyHostToDevice, t->stream));
        erase_tree_samples(*t, in.p);
    });
}

void tsr_occupancy_free(tsr_occupancy *o) { delete o; }

tsr_status tsr_occupancy_get_counts(const tsr_occupancy *o, tsr_occupancy_counts *out) {
    return guarded([&] {
        if (!o || !out) fail(TSR_ERR_INVALID_ARG, "null argument");
        out->links = o->links;
        out->accepted_sampleness = o->accepted[1];
        out->accepted_emptiness = o->accepted[0];
        out->visited_sampleness = o->visits[1];
        out->visited_emptiness = o->visits[0];
        out->visited_priors = o->visits[2];
        out->pruned_leaves = o->pruned;
        out->repaired_leaves = o->repaired;
        out->certified_leaves = o->certified;
    });
}

tsr_status tsr_occupancy_copy(const tsr_occupancy *o, tsr_field field, void *dst) {
    return guarded([&] {
        if (!o || !dst) fail(TSR_ERR_INVALID_ARG, "null argument");
        switch (field) {
            case TSR_FIELD_EMPTINESS_SUM: to_host(o->e_sum, o->n_leaves, dst, o->stream); break;
            case TSR_FIELD_SAMPLENESS_SUM: to_host(o->s_sum, o->n_leaves, dst, o->stream); break;
            case TSR_FIELD_EMPTINESS_LENGTH: to_host(o->e_len, o->n_leaves, dst, o->stream); break;
            case TSR_FIELD_SAMPLENESS_LENGTH: to_host(o->s_len, o->n_leaves, dst, o->stream); break;
            case TSR_FIELD_PRIOR_EMPTINESS: to_host(o->prior, o->n_leaves, dst, o->stream); break;
            case TSR_FIELD_OCCUPANCY: to_host(o->occ, o->n_leaves, dst, o->stream); break;
            case TSR_FIELD_NODE_STATES: to_host(o->states, o->n_nodes, dst, o->stream); break;
            case TSR_FIELD_CONE_COUNT: std::memcpy(dst, &o->cone_count, sizeof(double)); break;
            default: fail(TSR_ERR_INVALID_ARG, "unknown field");
        }
        TSR_CUDA(cudaStreamSynchronize(o->stream));
    });
}

tsr_status tsr_occupancy_stage_ms(const tsr_occupancy *o, float *ms, int n) {
    return guarded([&] {
        if (!o || !ms) fail(TSR_ERR_INVALID_ARG, "null argument");
        for (int i = 0; i < n && i < 8; ++i) ms[i] = o->stage_ms[i];
    });
}

tsr_status tsr_dmc_extract(const tsr_tree *tree, const tsr_occupancy *occ, void *cuda_stream, tsr_mesh **out) {
    if (out) *out = nullptr;
    return guarded([&] {
        if (!tree || !occ || !out) fail(TSR_ERR_INVALID_ARG, "null argument");
        if (occ->n_leaves != tree->n_leaves) fail(TSR_ERR_STATE, "occupancy does not belong to this tree");
        tsr_mesh *m = new tsr_mesh();
        m->stream = (cudaStream_t)cuda_stream;
        try {
            extract_dmc(*tree, *occ, *m);
            TSR_CUDA(cudaStreamSynchronize(m->stream));
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
    });
}

void tsr_mesh_free(tsr_mesh *m) { delete m; }

tsr_status tsr_mesh_get_counts(const tsr_mesh *m, tsr_mesh_counts *out) {
    return guarded([&] {
        if (!m || !out) fail(TSR_ERR_INVALID_ARG, "null argument");
        out->vertices = m->n_verts;
        out->triangles = m->n_tris;
        out->active_cells = m->n_active;
    });
}

tsr_status tsr_mesh_copy(const tsr_mesh *m, uint8_t *cases, double *positions, double *scales, uint32_t *edge_keys,
                         uint32_t *triangles) {
    return guarded([&] {
        if (!m) fail(TSR_ERR_INVALID_ARG, "null mesh");
        to_host(m->cases, m->n_cells, cases, m->stream);
        to_host(m->vpos, 3 * m->n_verts, positions, m->stream);
        to_host(m->vscale, m->n_verts, scales, m->stream);
        to_host(m->vkeys, 2 * m->n_verts, edge_keys, m->stream);
        to_host(m->tris, 3 * m->n_tris, triangles, m->stream);
        TSR_CUDA(cudaStreamSynchronize(m->stream));
    });
}

tsr_status tsr_mesh_postprocess(tsr_mesh *m, uint32_t min_isle_size, tsr_mesh_post_counts *counts) {
    return guarded([&] {
        if (!m) fail(TSR_ERR_INVALID_ARG, "null mesh");
        tsr_mesh_post_counts pc{};
        postprocess_mesh(*m, min_isle_size, pc);
        if (counts) *counts = pc;
    });
}

tsr_status tsr_mesh_copy_normals(const tsr_mesh *m, double *normals) {
    return guarded([&] {
        if (!m || !normals) fail(TSR_ERR_INVALID_ARG, "null argument");
        if (m->vnrm.n != 3 * m->n_verts)
            fail(TSR_ERR_STATE, "normals exist after tsr_mesh_postprocess and for depth-map meshes only");
        to_host(m->vnrm, 3 * m->n_verts, normals, m->stream);
        TSR_CUDA(cudaStreamSynchronize(m->stream));
    });
}

tsr_status tsr_mesh_create(const double *positions, const double *scales, uint64_t vertex_count,
                           const uint32_t *triangles, uint64_t triangle_count, void *cuda_stream, tsr_mesh **out) {
    if (out) *out = nullptr;
    return guarded([&] {
        if (!out || (vertex_count && !positions) || (triangle_count && !triangles))
            fail(TSR_ERR_INVALID_ARG, "null argument");
        if (vertex_count >= INVALID || 3 * triangle_count >= INVALID)
            fail(TSR_ERR_OVERFLOW_U32, "vertex and corner counts must stay below 2^32 - 1");
        for (uint64_t i = 0; i < 3 * triangle_count; ++i)
            if (triangles[i] >= vertex_count)
                fail(TSR_ERR_INVALID_ARG, "triangle index out of range at corner " + std::to_string(i));
        tsr_mesh *m = new tsr_mesh();
        m->stream = (cudaStream_t)cuda_stream;
        try {
            cudaStream_t st = m->stream;
            m->n_verts = vertex_count;
            m->n_tris = triangle_count;
            m->vpos.alloc(3 * vertex_count, st);
            m->vscale.alloc(vertex_count, st);
            m->vkeys.alloc(2 * vertex_count, st);
            m->tris.alloc(3 * triangle_count, st);
            if (vertex_count) {
                TSR_CUDA(cudaMemcpyAsync(m->vpos.p, positions, 24 * vertex_count, cudaMemcpyHostToDevice, st));
                if (scales) TSR_CUDA(cudaMemcpyAsync(m->vscale.p, scales, 8 * vertex_count, cudaMemcpyHostToDevice, st));
                else m->vscale.zero();
                m->vkeys.fill_bytes(0xFF);
            }
            if (triangle_count)
                TSR_CUDA(cudaMemcpyAsync(m->tris.p, triangles, 12 * triangle_count, cudaMemcpyHostToDevice, st));
            TSR_CUDA(cudaStreamSynchronize(st));
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
    });
}

tsr_status tsr_depth_triangulate(const double *depths, uint32_t width, uint32_t height, const double *hps_to_ray_vs,
                                 const double *hps_to_ray_ws, const double *center, const double *colors,
                                 void *cuda_stream, tsr_mesh **out) {
    if (out) *out = nullptr;
    return guarded([&] {
        if (!depths || !hps_to_ray_vs || !hps_to_ray_ws || !center || !out) fail(TSR_ERR_INVALID_ARG, "null argument");
        tsr_mesh *m = new tsr_mesh();
        m->stream = (cudaStream_t)cuda_stream;
        try {
            triangulate_depth(depths, width, height, hps_to_ray_vs, hps_to_ray_ws, center, colors, *m);
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
    });
}

tsr_status tsr_mesh_copy_colors(const tsr_mesh *m, double *colors) {
    return guarded([&] {
        if (!m || !colors) fail(TSR_ERR_INVALID_ARG, "null argument");
        if (m->vcol.n != 3 * m->n_verts) fail(TSR_ERR_STATE, "colours exist for depth-map meshes only");
        to_host(m->vcol, 3 * m->n_verts, colors, m->stream);
        TSR_CUDA(cudaStreamSynchronize(m->stream));
    });
}

tsr_status tsr_mesh_copy_pixel_map(const tsr_mesh *m, uint32_t *pixel_to_vertex) {
    return guarded([&] {
        if (!m || !pixel_to_vertex) fail(TSR_ERR_INVALID_ARG, "null argument");
        const size_t np = (size_t)m->width * m->height;
        if (np == 0 || m->pix2v.n != np) fail(TSR_ERR_STATE, "a pixel map exists for depth-map meshes only");
        to_host(m->pix2v, np, pixel_to_vertex, m->stream);
        TSR_CUDA(cudaStreamSynchronize(m->stream));
    });
}

tsr_status tsr_tree_save(const tsr_tree *tree, const char *path_prefix) {
    return guarded([&] {
        if (!tree || !path_prefix || !*path_prefix) fail(TSR_ERR_INVALID_ARG, "null argument");
        save_tree(*tree, path_prefix);
    });
}

tsr_status tsr_tree_save_samples(const tsr_tree *tree, const double *colors, const char *path) {
    return guarded([&] {
        if (!tree || !path || !*path) fail(TSR_ERR_INVALID_ARG, "null argument");
        save_samples(*tree, colors, path);
    });
}

tsr_status tsr_tree_load(const char *path_prefix, const tsr_samples_view *samples, const double *aabb,
                         const tsr_params *params, void *cuda_stream, tsr_tree **out_tree) {
    if (out_tree) *out_tree = nullptr;
    return guarded([&] {
        if (!path_prefix || !*path_prefix || !samples || !out_tree) fail(TSR_ERR_INVALID_ARG, "null argument");
        check_samples(*samples, false);
        tsr_params p;
        tsr_params_default(&p);
        if (params) p = *params;
        check_params(p);
        tsr_tree *t = new tsr_tree();
        t->stream = (cudaStream_t)cuda_stream;
        t->params = p;
        try {
            load_tree(*t, path_prefix, *samples, aabb);
        } catch (...) {
            delete t;
            throw;
        }
        *out_tree = t;
    });
}

tsr_status tsr_occupancy_save(const tsr_occupancy *occ, const char *path) {
    return guarded([&] {
        if (!occ || !path || !*path) fail(TSR_ERR_INVALID_ARG, "null argument");
        if (occ->pruned)
            fail(TSR_ERR_STATE, "a pruned field holds no prior for its skipped leaves; the file format needs all");
        save_occupancy(*occ, path);
    });
}

tsr_status tsr_occupancy_load(const tsr_tree *tree, const char *path, const tsr_params *params, void *cuda_stream,
                              tsr_occupancy **out) {
    if (out) *out = nullptr;
    return guarded([&] {
        if (!tree || !path || !*path || !out) fail(TSR_ERR_INVALID_ARG, "null argument");
        if (tree->n_leaves == 0) fail(TSR_ERR_STATE, "tree has no leaves");
        tsr_params p = tree->params;
        if (params) p = *params;
        check_params(p);
        tsr_occupancy *o = new tsr_occupancy();
        o->stream = (cudaStream_t)cuda_stream;
        try {
            load_occupancy(*tree, *o, path, p);
        } catch (...) {
            delete o;
            throw;
        }
        *out = o;
    });
}

}  // extern "C"
