// handles.h -- device-resident state behind the opaque C-ABI handles.
#pragma once

#include <vector>

#include "common.cuh"

struct tsr_tree {
    cudaStream_t stream = nullptr;
    tsr_params params{};
    uint32_t n_samples = 0, k = 0;
    double aabb[6] = {0, 0, 0, 0, 0, 0};   // Samples::mAABBWS at the build: min xyz, max xyz
    double root_min[3] = {0, 0, 0};
    double root_size = 0;
    uint32_t n_nodes = 0, n_leaves = 0, max_depth = 0, n_cells = 0;
    uint64_t n_nb = 0;
    uint32_t sampling_rounds = 0, sampling_waves = 0;
    uint64_t sampling_writers = 0;

    // final node arrays (reference order after Nodes::reorder)
    tsr::DBuf<uint32_t> children, parents, counts, starts;
    tsr::DBuf<uint8_t> depth;
    tsr::DBuf<tsr::D3> nmin;
    tsr::DBuf<uint32_t> level_order;   // node indices sorted by depth
    std::vector<uint32_t> level_start; // first position of each depth in level_order (+ end)
    // samples in tree order (reordered like Samples::reorder)
    tsr::DBuf<uint32_t> target;        // old sample index -> new
    tsr::DBuf<tsr::D3> pos, nrm;       // FP64
    tsr::DBuf<double> scale, conf;
    tsr::DBuf<uint32_t> links;         // K per sample
    // leaves
    tsr::DBuf<tsr::D3> leaf_min;
    tsr::DBuf<uint32_t> leaf_node, node_to_leaf, nb_off, nbs;
    // dual cells
    tsr::DBuf<uint32_t> cells;         // 8 per cell
    float stage_ms[8] = {0};
};

struct tsr_occupancy {
    cudaStream_t stream = nullptr;
    uint32_t n_leaves = 0, n_nodes = 0;
    tsr::DBuf<double> e_sum, s_sum, e_len, s_len, prior, occ;
    tsr::DBuf<uint32_t> states;
    double cone_count = 0;
    double confidence_threshold = 0;   // Occupancy::confidenceThreshold of this field
    float stage_ms[8] = {0};
    uint64_t accepted[2] = {0, 0};   // [EMPTINESS, SAMPLENESS]
    uint64_t visits[3] = {0, 0, 0};  // nodes tested: EMPTINESS, SAMPLENESS, priors
    uint64_t links = 0;
    uint64_t pruned = 0;             // leaves whose prior query the pruned field skipped
    uint64_t repaired = 0;           // skipped leaves queried after all (bordering a sign change)
    uint64_t certified = 0;          // skip candidates whose sign the prior bounds proved
};

struct tsr_mesh {
    cudaStream_t stream = nullptr;
    uint64_t n_verts = 0, n_tris = 0, n_active = 0, n_cells = 0;
    tsr::DBuf<uint8_t> cases;
    tsr::DBuf<double> vpos, vscale;
    tsr::DBuf<uint32_t> vkeys, tris;
    tsr::DBuf<double> vnrm;            // 3 per vertex once post-processed; empty before
    tsr::DBuf<double> vcol;            // 3 per vertex, depth-map meshes only
    tsr::DBuf<uint32_t> pix2v;         // vertex of every pixel, depth-map meshes only
    uint32_t width = 0, height = 0;    // depth-map meshes only
};

namespace tsr {
void build_tree(tsr_tree &t, const tsr_samples_view &sv, bool on_device);
void compute_occupancy(const tsr_tree &t, const tsr_cameras_view &cv, const tsr_params &p, int mode,
                       tsr_occupancy &o, const tsr_pruner *pruner = nullptr, const uint32_t *chosen = nullptr,
                       uint32_t nchosen = 0, double sign = 1.0, bool update = false);
void erase_tree_samples(tsr_tree &t, const uint8_t *inliers_dev);
void leaf_features(const tsr_tree &t, const double *esum, const double *ssum, double threshold, DBuf<float> &feat,
                   cudaStream_t st);
void mlp_train_batch(const float *x, const float *y, uint32_t n, const float *params, float *grads, float *loss,
                     float pw0, float pw1, cudaStream_t st);
void mlp_adam(float *p, const float *g, float *m, float *v, uint32_t step, float lr, float gscale,
              cudaStream_t st);
void mlp_forward(const float *x, uint32_t n, const float *params, float *out, cudaStream_t st);
void mlp_infer_bf16(const float *x, uint32_t n, const float *params, float *out, cudaStream_t st);
void pruner_predict(const tsr_tree &t, const tsr_pruner &pr, const double *esum, const double *ssum,
                    double threshold, DBuf<uint8_t> &pred, cudaStream_t st);
void extract_dmc(const tsr_tree &t, const tsr_occupancy &o, tsr_mesh &m);
void postprocess_mesh(tsr_mesh &m, uint32_t min_isle_size, tsr_mesh_post_counts &counts);
void angle_weighted_normals(const uint32_t *tris, uint32_t nt, const double *pos, uint32_t nv, double *nrm,
                            cudaStream_t st);
void triangulate_depth(const double *depths_host, uint32_t width, uint32_t height, const double *hps_to_ray_vs,
                       const double *hps_to_ray_ws, const double *center, const double *colors_host, tsr_mesh &m);
void reserve_pool(size_t want, cudaStream_t st);
void root_scope_noalloc(uint64_t count, const double *positions, const double *scales, double h_svo,
                        double *out_min_xyz_size, cudaStream_t st);
void finalize_field(tsr_occupancy &o, const tsr_params &p);
void save_tree(const tsr_tree &t, const std::string &prefix);
void root_from_aabb(tsr_tree &t);
void load_tree(tsr_tree &t, const std::string &prefix, const tsr_samples_view &sv, const double *aabb);
void save_samples(const tsr_tree &t, const double *colors, const std::string &path);
void save_occupancy(const tsr_occupancy &o, const std::string &path);
void load_occupancy(const tsr_tree &t, tsr_occupancy &o, const std::string &path, const tsr_params &p);
}  // namespace tsr
