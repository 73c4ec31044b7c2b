/*
 * tsr_core.h -- C ABI of the B200 (sm_100a) volumetric core of TSR.
 *
 * Plain pointers, sizes and opaque handles; no C++ or torch types cross this
 * boundary.  Every entry point replaces one call site of the reference's C++
 * scene API (paths relative to SurfaceReconstruction/SurfaceReconstruction/):
 *
 *   tsr_tree_build         Tree::Tree()                       Scene/Tree/Tree.cpp:26-37
 *                          (Nodes::Nodes Nodes.cpp:186-194, Leaves::Leaves
 *                           Leaves.cpp:22-28, DualCells::DualCells DualCells.cpp:21-31)
 *   tsr_tree_copy_*        Tree::getNodes/getLeaves/getDualCells   Scene/Tree/Tree.h:46-57,108-121
 *                          Nodes arrays Nodes.h:144-147, Leaves arrays Leaves.h:90-98,
 *                          DualCells::getIndices DualCells.h:84-87
 *   tsr_tree_copy_permutation  the in-place Samples reorder done by the tree
 *                          (Nodes::reorderSamplesAndFillNodes Nodes.cpp:594-636)
 *   tsr_occupancy_compute  Occupancy::Occupancy(const Tree *)   SurfaceExtraction/Occupancy.cpp:78-127
 *   tsr_occupancy_copy     getOccupancy / getNodeStates / kernel sums, cone lengths,
 *                          priors, cone count   Occupancy.cpp:570-597, Occupancy.h:72-86,192-210
 *   tsr_dmc_extract        DualMarchingCells::DualMarchingCells -> extractMesh
 *                          SurfaceExtraction/DualMarchingCells.cpp:26-169
 *   tsr_mesh_postprocess   its FlexibleMesh post-processing (:31-36): deleteIsolatedGeometry,
 *                          fillHoles, computeNormalsWeightedByAngles (Geometry/FlexibleMesh.cpp,
 *                          Geometry/IslesEraser.cpp, Geometry/Mesh.cpp:145-203)
 *   tsr_occupancy_update   Occupancy::addSamples / eraseSamples (Occupancy.h:167-175)
 *   tsr_tree_erase_samples Tree::eraseSamples (Tree.cpp:50-53) + Samples::compact
 *   tsr_tree_save/_load, tsr_tree_save_samples, tsr_occupancy_save/_load
 *                          Tree::saveToFiles / Tree(filesBeginning), Samples::saveToFile,
 *                          Occupancy::saveToFile / Occupancy(fileName)
 *   tsr_depth_triangulate  DepthImage::triangulate (Image/DepthImage.cpp:186-461), the samples'
 *                          source in Scene::loadDepthMeshes (Scene.cpp:484-525)
 *   tsr_*_free             the owning deletes in Scene (Scene.cpp:627-670)
 *
 * Errors: every call returns a tsr_status; the reference throws
 * FailureHandling::Exception instead (e.g. Nodes.cpp:238,304,405,616).
 * tsr_last_error_message() returns the text of the last failure on the
 * calling thread.
 *
 * Threading: handles are thread-compatible (one thread per handle at a time);
 * every compute call takes the CUDA stream to run on (NULL = legacy default).
 */
#ifndef TSR_CORE_H
#define TSR_CORE_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define TSR_API __attribute__((visibility("default")))
#else
#define TSR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    TSR_OK = 0,
    TSR_ERR_INVALID_ARG = 1,
    TSR_ERR_OVERFLOW_U32 = 2,   /* node / link counts beyond 32-bit indices (Nodes.cpp:399-407, Samples.h:395-402) */
    TSR_ERR_OOM = 3,
    TSR_ERR_CUDA = 4,
    TSR_ERR_DEVICE_ASSERT = 5,  /* a kernel detected a broken invariant and stopped */
    TSR_ERR_TIMEOUT = 6,        /* an iteration limit was reached */
    TSR_ERR_STATE = 7           /* call out of order (e.g. occupancy before a tree) */
} tsr_status;

/* Parameters the reference reads from App.cfg (App.cfg:64-70); the defaults of
 * tsr_params_default() are the shipped App.cfg values. */
typedef struct {
    double max_relative_sampling_distance;  /* Samples::maxRelativeSamplingDistance (h_SVO) = 2   */
    double bandwidth_factor;                /* Occupancy::bandwidthFactor (h_O) = 2               */
    double confidence_threshold;            /* Occupancy::confidenceThreshold = 100               */
    double relative_radius_for_priors;      /* Occupancy::relativeRadiusForPriors = 25            */
    double relative_sample_cone_length;     /* Occupancy::relativeSampleConeLength = 1            */
} tsr_params;

/* Structure-of-arrays view of the reference's Samples (Samples.h:300-312).
 * All pointers are HOST memory; positions/normals are xyz-interleaved. */
typedef struct {
    uint32_t count;
    uint32_t cams_per_sample;          /* K = Samples::getMaxCamerasPerSample */
    const double *positions;           /* 3 * count */
    const double *normals;             /* 3 * count, unit length */
    const double *scales;              /* count, > 0 */
    const double *confidences;         /* count */
    const uint32_t *camera_links;      /* K * count, 0xFFFFFFFF = no camera (Cameras.cpp:29) */
} tsr_samples_view;

/* Camera centres (Cameras::getPositionWS, Cameras.h:161-166), HOST memory. */
typedef struct {
    uint32_t count;
    const double *positions;           /* 3 * count */
} tsr_cameras_view;

typedef struct {
    uint64_t nodes, leaves, dual_cells, neighbor_entries;
    uint32_t max_depth;
    uint32_t sampling_rounds;          /* rounds of the order-exact sampling schedule */
    uint64_t sampling_writers;         /* sample sides that had to create nodes */
    uint32_t sampling_waves;           /* conflict-resolution waves over all rounds */
    uint32_t reserved;
} tsr_tree_counts;

typedef struct {
    uint64_t vertices, triangles, active_cells;
} tsr_mesh_counts;

typedef struct {
    uint64_t links;                    /* camera-to-sample links (N * K) */
    uint64_t accepted_sampleness;      /* (link, leaf) pairs addKernel accepted, SAMPLENESS pass */
    uint64_t accepted_emptiness;       /* ... EMPTINESS pass */
    uint64_t visited_sampleness;       /* tree nodes tested against a cone, SAMPLENESS pass */
    uint64_t visited_emptiness;        /* ... EMPTINESS pass */
    uint64_t visited_priors;           /* tree nodes classified by the prior sphere queries */
    uint64_t pruned_leaves;            /* prior queries the pruned field skipped (0 for the plain field) */
    uint64_t repaired_leaves;          /* skipped positive leaves queried after all: next to a negative leaf, side of EPSILON unproved */
    uint64_t certified_leaves;         /* skip candidates whose sign bounds of their prior proved */
} tsr_occupancy_counts;

/* The learned pruner (no counterpart in the reference).
 * A 10 -> 64 -> 64 -> 2 ReLU MLP over per-leaf features (tsr_occupancy_leaf_features)
 * with two logits: "occupancy > 0" and "near a sign change".  Parameters are
 * FP32, TSR_MLP_PARAMS values in the order W1[10][64], b1[64], W2[64][64],
 * b2[64], W3[64][2], b3[2] (W[in][out]). */
#define TSR_MLP_FEATURES 10
#define TSR_MLP_HIDDEN 64
#define TSR_MLP_OUTPUTS 2
#define TSR_MLP_PARAMS 4994

typedef struct {
    const float *weights;              /* HOST, TSR_MLP_PARAMS values */
    float feature_mean[TSR_MLP_FEATURES];
    float feature_inv_std[TSR_MLP_FEATURES];   /* inputs are (feature - mean) * inv_std */
    float sign_threshold;              /* the sign is taken as known when P(occupancy > 0) is below this
                                          or above 1 - this (0 < sign_threshold < 0.5) */
    float band_threshold;              /* a leaf counts as near a sign change when P(band) >= this */
    uint32_t dilation;                 /* rings of face neighbours added around those leaves */
    uint32_t bound_levels;             /* a skip candidate's sign is certified by a bounds query that
                                          stops at nodes this many levels above the leaf (0 .. 4) */
} tsr_pruner;

typedef struct tsr_tree tsr_tree;
typedef struct tsr_occupancy tsr_occupancy;
typedef struct tsr_mesh tsr_mesh;

/* Fields of tsr_occupancy_copy; scalar fields are double[leaves], node_states
 * is uint32[nodes], cone_count is one double. */
typedef enum {
    TSR_FIELD_EMPTINESS_SUM = 0,   /* mKernelSums[EMPTINESS]  */
    TSR_FIELD_SAMPLENESS_SUM = 1,  /* mKernelSums[SAMPLENESS] */
    TSR_FIELD_EMPTINESS_LENGTH = 2,/* mConeLengths[EMPTINESS] */
    TSR_FIELD_SAMPLENESS_LENGTH = 3,
    TSR_FIELD_PRIOR_EMPTINESS = 4, /* mPriorsForEmptiness */
    TSR_FIELD_OCCUPANCY = 5,       /* getOccupancy(leaf) */
    TSR_FIELD_NODE_STATES = 6,     /* mNodeStates (uint32) */
    TSR_FIELD_CONE_COUNT = 7       /* mConeCount */
} tsr_field;

TSR_API void tsr_params_default(tsr_params *out);
TSR_API const char *tsr_last_error_message(void);
TSR_API const char *tsr_version(void);

TSR_API tsr_status tsr_tree_build(const tsr_samples_view *samples, const tsr_params *params,
                          void *cuda_stream, tsr_tree **out_tree);
/* Same as tsr_tree_build with every pointer of `samples` in DEVICE memory
 * (for callers whose samples already live in HBM). */
TSR_API tsr_status tsr_tree_build_device(const tsr_samples_view *samples, const tsr_params *params,
                                         void *cuda_stream, tsr_tree **out_tree);
TSR_API void tsr_tree_free(tsr_tree *tree);
/* Tree::eraseSamples (Tree.cpp:50-53, Nodes.cpp:644-671) plus Samples::compact
 * (Samples.cpp) of the tree's own samples: `inliers` (HOST, one byte per
 * sample in tree order, nonzero = keep).  Node sample counts and start indices
 * follow the compaction; the topology is unchanged; the permutation maps
 * erased input samples to 0xFFFFFFFF.  Scene::eraseSamples (Scene.cpp:270-307)
 * calls tsr_occupancy_update(..., for_removal = 1, outliers) first. */
TSR_API tsr_status tsr_tree_erase_samples(tsr_tree *tree, const uint8_t *inliers);
TSR_API tsr_status tsr_tree_get_counts(const tsr_tree *tree, tsr_tree_counts *out);
TSR_API tsr_status tsr_tree_root_scope(const tsr_tree *tree, double min_xyz_size[4]);
/* The root scope tsr_tree_build would give these samples (min corner xyz and
 * edge length of the root cube, as tsr_tree_root_scope reports), written to
 * DEVICE memory `out_min_xyz_size[4]` on `cuda_stream`, with DEVICE inputs
 * (`positions` 3 * count xyz-interleaved, `scales` count).  No counterpart in
 * the reference: it exists for callers that must not allocate (their device
 * memory is all handed to their own pool, or their footprint is fixed after
 * start-up).  It allocates no memory; its working memory is a fixed 56,836 B
 * array per device inside the library.  The first call on each device sets
 * that up (address look-up, which may load the library's device code), so
 * make it before any stream capture.  Calls on one device share the array:
 * calls that may overlap in time race, so order them.  count must be
 * 1 .. 2^31 - 1, the tree build's limit (TSR_ERR_OVERFLOW_U32 above); pointers
 * must be 8-byte aligned memory of the current device.  The root cube follows
 * the build's arithmetic for every input, NaN and negative extents included. */
TSR_API tsr_status tsr_samples_root_scope_noalloc(uint64_t count, const double *positions,
                                                  const double *scales, const tsr_params *params,
                                                  double *out_min_xyz_size, void *cuda_stream);
/* Node arrays after the reference's reorder; any pointer may be NULL. */
TSR_API tsr_status tsr_tree_copy_nodes(const tsr_tree *tree, uint32_t *children, uint32_t *parents,
                               uint32_t *sample_counts, uint32_t *sample_starts);
/* The samples in tree order (Samples::reorder, Samples.cpp:825-835), into
 * HOST arrays laid out like tsr_samples_view; any pointer may be NULL. */
TSR_API tsr_status tsr_tree_copy_samples(const tsr_tree *tree, double *positions, double *normals,
                                         double *scales, double *confidences, uint32_t *camera_links);
/* target_indices[old sample index] = new sample index (Nodes.cpp:625-626). */
TSR_API tsr_status tsr_tree_copy_permutation(const tsr_tree *tree, uint32_t *target_indices);
/* scopes: 4 doubles per leaf (min x, y, z, size); node_index per leaf;
 * node_to_leaf per node; CSR neighbour offsets (leaves + 1) and entries. */
TSR_API tsr_status tsr_tree_copy_leaves(const tsr_tree *tree, double *scopes, uint32_t *node_index,
                                uint32_t *node_to_leaf, uint32_t *neighbor_offsets,
                                uint32_t *neighbors);
TSR_API tsr_status tsr_tree_copy_dual_cells(const tsr_tree *tree, uint32_t *cells8);

/* mode 0 = plain field: FP32 kernel values, FP64 per-leaf sums. */
TSR_API tsr_status tsr_occupancy_compute(const tsr_tree *tree, const tsr_cameras_view *cameras,
                                 const tsr_params *params, int mode, void *cuda_stream,
                                 tsr_occupancy **out_occupancy);
TSR_API void tsr_occupancy_free(tsr_occupancy *occ);
/* Occupancy::addSamples / eraseSamples (Occupancy.h:167-175) ->
 * onSamplesChanged (Occupancy.cpp:129-136): the kernels of the links of
 * `samples` (HOST indices in tree order, i.e. the order tsr_tree_copy_samples
 * returns) are added (for_removal = 0) or removed (for_removal = 1) from the
 * field's sums, lengths and cone count (removal keeps node flags, like the
 * reference), then every prior and occupancy value is recomputed
 * (Occupancy::update, Occupancy.h:222-227).  The tree must be the one the
 * field was computed on; the work counters then describe this update. */
TSR_API tsr_status tsr_occupancy_update(tsr_occupancy *occ, const tsr_tree *tree, const tsr_cameras_view *cameras,
                                        const tsr_params *params, int for_removal, const uint32_t *samples,
                                        uint32_t count, void *cuda_stream);
/* Work counters of the last field computation (no counterpart in the
 * reference; instrumentation). */
TSR_API tsr_status tsr_occupancy_get_counts(const tsr_occupancy *occ, tsr_occupancy_counts *out);
TSR_API tsr_status tsr_occupancy_copy(const tsr_occupancy *occ, tsr_field field, void *host_dst);

TSR_API tsr_status tsr_dmc_extract(const tsr_tree *tree, const tsr_occupancy *occ, void *cuda_stream,
                           tsr_mesh **out_mesh);
TSR_API void tsr_mesh_free(tsr_mesh *mesh);
TSR_API tsr_status tsr_mesh_get_counts(const tsr_mesh *mesh, tsr_mesh_counts *out);
/* cases: uint8 per dual cell; positions 3 doubles and scales 1 double per
 * vertex; edge_keys 2 uint32 (min leaf, max leaf) per vertex; triangles 3
 * uint32 per triangle.  Any pointer may be NULL. */
TSR_API tsr_status tsr_mesh_copy(const tsr_mesh *mesh, uint8_t *cases, double *positions, double *scales,
                         uint32_t *edge_keys, uint32_t *triangles);

/* What tsr_mesh_postprocess did. */
typedef struct {
    uint64_t isle_vertices, isle_triangles;   /* deleted with isles below the minimum size */
    uint64_t border_edges;                    /* hole border edges after the isle deletion */
    uint64_t holes;                           /* rings filled */
    uint64_t hole_vertices, hole_triangles;   /* added by the filling */
    uint64_t skipped_rings;                   /* rings of < 3 edges, left open */
} tsr_mesh_post_counts;

/* The post-processing DualMarchingCells::DualMarchingCells runs after
 * extractMesh (DualMarchingCells.cpp:26-39), in place on the mesh's stream:
 *   FlexibleMesh::deleteIsolatedGeometry(min_isle_size) (FlexibleMesh.cpp:
 *   1411-1426, IslesEraser.cpp): isles (vertices connected by edges) of fewer
 *   than min_isle_size vertices are deleted and the rest compacted in order;
 *   then, unless nothing is left, FlexibleMesh::fillHoles (FlexibleMesh.cpp:
 *   1580-1931) and Mesh::computeNormalsWeightedByAngles (Mesh.cpp:145-203).
 * The reference passes Scene::minimumTriangleIsleSize (App.cfg: 1000).
 * Border edges are chained in the order one thread of the reference finds
 * them (its OpenMP loop makes that order timing dependent).  Vertices the
 * filling adds get scale 0 and edge keys {0xFFFFFFFF, 0xFFFFFFFF}; dual-cell
 * cases are unchanged.  An edge shared by three or more triangles returns
 * TSR_ERR_STATE and leaves the mesh unchanged (the reference throws,
 * FlexibleMesh.cpp:1227-1259).  counts may be NULL. */
TSR_API tsr_status tsr_mesh_postprocess(tsr_mesh *mesh, uint32_t min_isle_size, tsr_mesh_post_counts *counts);

/* Vertex normals after tsr_mesh_postprocess or of a depth-map mesh, 3
 * doubles per vertex, HOST memory (zeros when post-processing left no
 * triangles).  Post-processing drops a depth-map mesh's colours and pixel
 * map. */
TSR_API tsr_status tsr_mesh_copy_normals(const tsr_mesh *mesh, double *normals);

/* A mesh from HOST arrays, for tsr_mesh_postprocess of a surface that did
 * not come from tsr_dmc_extract (FlexibleMesh's vertex and index arrays,
 * FlexibleMesh.cpp:1276-1281, 1573-1578).  scales may be NULL (zeros); the
 * mesh has no dual cells and its edge keys are 0xFFFFFFFF.  Triangle
 * indices must be below the vertex count. */
TSR_API tsr_status tsr_mesh_create(const double *positions, const double *scales, uint64_t vertex_count,
                                   const uint32_t *triangles, uint64_t triangle_count, void *cuda_stream,
                                   tsr_mesh **out_mesh);

/* ---- samples from depth maps ---- */
/* DepthImage::triangulate (Image/DepthImage.cpp:186-461): the depth map
 * (width x height doubles, HOST, row major, depth along the pixel ray, <= 0
 * invalid) is triangulated block by block with the reference's depth
 * discontinuity test, vertices are numbered in the reference's order and
 * placed at center + normalize((x, y, 1) * hps_to_ray_ws) * depth, coloured
 * from colors (3 doubles per pixel, HOST) or 0.5 grey, given angle-weighted
 * normals and, as scale, the mean distance to their neighbours
 * (FlexibleMesh::findVertexNeighbors order, Mesh::computeVertexScales).
 * The two row-major 3x3 matrices are the ones the reference computes from
 * its PinholeCamera: hps_to_ray_vs = inverse viewport x inverse projection,
 * hps_to_ray_ws = hps_to_ray_vs x inverse rotation (DepthImage.cpp:189-194);
 * (x, y, 1) * M is a row vector times M.  The mesh's vertices are the
 * samples Samples::addSamplesViaMesh makes (Samples.cpp:262-272): read them
 * with tsr_mesh_copy, tsr_mesh_copy_normals and tsr_mesh_copy_colors. */
TSR_API tsr_status tsr_depth_triangulate(const double *depths, uint32_t width, uint32_t height,
                                         const double hps_to_ray_vs[9], const double hps_to_ray_ws[9],
                                         const double center[3], const double *colors, void *cuda_stream,
                                         tsr_mesh **out_mesh);
/* Vertex colours of a depth-map mesh, 3 doubles per vertex, HOST. */
TSR_API tsr_status tsr_mesh_copy_colors(const tsr_mesh *mesh, double *colors);
/* The vertex of every pixel of a depth-map mesh (width x height, 0xFFFFFFFF
 * for none), HOST; Scene::loadCameraIndices maps per-pixel views with it
 * (Scene.cpp:527-573). */
TSR_API tsr_status tsr_mesh_copy_pixel_map(const tsr_mesh *mesh, uint32_t *pixel_to_vertex);

/* ---- learned pruner (no counterpart in the reference) ---- */
/* The pruner's per-leaf features of a field, leaves x TSR_MLP_FEATURES floats
 * into HOST memory: log1p(samples in the leaf), log(mean sample scale / leaf
 * size), normal spread (1 - |mean normal|), depth / 16, log1p(E), log1p(S),
 * r = S / (E + S) (-1 when both are 0), reliable (E + S >= threshold) as 0/1,
 * and the smallest and largest r among the face neighbours.  Everything is
 * known before the prior queries. */
TSR_API tsr_status tsr_occupancy_leaf_features(const tsr_tree *tree, const tsr_occupancy *occ, float *features);
/* Training on DEVICE arrays: x (n x 10, normalized), y (n x 2 labels in
 * {0,1}), params (TSR_MLP_PARAMS).  Adds the gradient of the summed
 * binary cross-entropy (positive labels of output k weighted by
 * pos_weight[k]) to grads and the summed loss to *loss (both device). */
TSR_API tsr_status tsr_mlp_train_batch(const float *x, const float *y, uint32_t n, const float *params,
                                       float *grads, float *loss, float pos_weight0, float pos_weight1,
                                       void *cuda_stream);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on DEVICE arrays; the
 * gradient is multiplied by grad_scale first; step counts from 1. */
TSR_API tsr_status tsr_mlp_adam(float *params, const float *grads, float *m, float *v, uint32_t step,
                                float lr, float grad_scale, void *cuda_stream);
/* Logits (n x 2, DEVICE) of normalized DEVICE features: FP32 reference, and
 * the BF16 tensor-core path (mma.sync, FP32 accumulation) the pruner uses. */
TSR_API tsr_status tsr_mlp_forward(const float *x, uint32_t n, const float *params, float *logits,
                                   void *cuda_stream);
TSR_API tsr_status tsr_mlp_infer_bf16(const float *x, uint32_t n, const float *params, float *logits,
                                      void *cuda_stream);
/* The pruned field: like tsr_occupancy_compute (both cone passes exact), but
 * the prior query -- the most expensive per-leaf step -- runs only for
 * reliable leaves (E + S >= confidenceThreshold) that the pruner places near
 * a sign change (or within `dilation` rings of face neighbours of one), whose
 * sign it is not sure of, or whose sign cannot be certified; E == 0 or
 * S == 0 fixes the sign without a prior.  Every other reliable leaf gets a
 * cheaper bounds query (the prior's sphere query stopped at nodes
 * `bound_levels` levels above the leaf's depth, their subtrees counted as
 * undecided), and is skipped only when
 * the bounds prove its sign ((1 - p) S > p E for every p in them, or for
 * none); it then takes that sign, with the value 0.5 (S - E) / coneCount
 * when positive (moved to 2 EPSILON or to EPSILON when the bounds prove the
 * exact value above EPSILON or at most EPSILON), and its prior reads NaN.
 * A skipped positive leaf that shares a face with a negative one is queried
 * after all unless that side of EPSILON is proved (a negative leaf's value
 * is -EPSILON with or without its prior, and DMC snaps a vertex to an end
 * within EPSILON of zero).  So every sign is the plain field's and every
 * vertex the plain field's: the DMC mesh equals the plain field's. */
TSR_API tsr_status tsr_occupancy_compute_pruned(const tsr_tree *tree, const tsr_cameras_view *cameras,
                                                const tsr_params *params, const tsr_pruner *pruner,
                                                void *cuda_stream, tsr_occupancy **out_occupancy);

/* Number of this library's kernel launches so far in the process
 * (instrumentation; no counterpart in the reference). */
TSR_API unsigned long long tsr_kernel_launches(void);

/* Iteration bounds of the tree build (no counterpart in the reference, whose
 * loops are unbounded): the conflict waves of one sampling round, a loop that
 * runs on the device inside one cooperative launch and, when it reaches its
 * bound, stops, records the fact and returns; and the host-side rounds of the
 * sampling and balancing passes.  A build that reaches either bound returns
 * TSR_ERR_TIMEOUT and leaves the device usable.  0 restores a default
 * (2^22 waves, 100000 rounds).  Process-wide; not for calls in flight. */
TSR_API void tsr_set_iteration_limits(uint32_t max_sampling_waves, uint32_t max_rounds);

/* Wall-clock-free stage timing: CUDA-event milliseconds of the last call on
 * this handle, per stage (see tsr_stage names in the implementation). */
TSR_API tsr_status tsr_tree_stage_ms(const tsr_tree *tree, float *ms, int n);
TSR_API tsr_status tsr_occupancy_stage_ms(const tsr_occupancy *occ, float *ms, int n);

/* ---------------------------------------------------------------- files
 * The reference's on-disk bodies, little endian, Real = double:
 *   <prefix>.nodes      Nodes::saveToFile (Nodes.cpp:789-807)
 *   <prefix>.leaves     Leaves::saveToFile (Leaves.cpp:261-292)
 *   <prefix>.dualCells  DualCells::saveToFile (DualCells.cpp:378-385)
 *   <path>              Occupancy::saveToFile (Occupancy.cpp:722-766)
 *   <path>              Samples::saveToFile (Samples.cpp:733-765)
 * Each file starts with a 16-byte header in place of the reference's
 * BaseProject File header (that library is not part of the reference tree):
 * "TSRF", u32 format 1, u32 FILE_VERSION 0, u32 kind (1 nodes, 2 leaves,
 * 3 dual cells, 4 occupancy, 5 samples). */

/* Tree::saveToFiles (Tree.cpp:129-134): writes the three tree files. */
TSR_API tsr_status tsr_tree_save(const tsr_tree *tree, const char *path_prefix);

/* Samples::saveToFile(beginning, false, true) (Samples.cpp:733-765): the
 * tree's samples in tree order, <path> = <beginning>.samples, with the AABB
 * the tree was built over (kept through tsr_tree_erase_samples, so that the
 * file reloads the same tree).  colors: HOST, 3 per sample in tree order,
 * or NULL for zeros (colours are not part of tsr_samples_view). */
TSR_API tsr_status tsr_tree_save_samples(const tsr_tree *tree, const double *colors, const char *path);

/* Tree::Tree(filesBeginning) / Tree::loadFromFile (Tree.cpp:39-43, 118-127):
 * reads the three tree files.  The reference takes the samples and their
 * AABB (Samples::mAABBWS, stored in the .samples file) from the Scene
 * singleton; here the caller passes the samples, in tree order (as a
 * .samples file or tsr_tree_copy_samples gives them), host memory, and
 * optionally the AABB {min x, y, z, max x, y, z} of the samples file.  With
 * aabb NULL it is computed from the samples exactly as tsr_tree_build does.
 * The root scope follows from the AABB as in Tree::getRootScope
 * (Tree.cpp:70-101), and every saved leaf scope must equal the one it gives,
 * bit for bit.  A file of another tree or of other samples, a damaged file
 * and any index out of range return TSR_ERR_INVALID_ARG before any device
 * work (the reference throws FileCorruptionException).  The loaded tree's
 * permutation is the identity. */
TSR_API tsr_status tsr_tree_load(const char *path_prefix, const tsr_samples_view *samples, const double *aabb,
                                 const tsr_params *params, void *cuda_stream, tsr_tree **out_tree);

/* Occupancy::saveToFile (Occupancy.cpp:722-766).  A pruned field with
 * skipped prior queries returns TSR_ERR_STATE: the format holds a prior for
 * every leaf. */
TSR_API tsr_status tsr_occupancy_save(const tsr_occupancy *occ, const char *path);

/* Occupancy::Occupancy(fileName) / loadFromFile (Occupancy.cpp:598-603,
 * 663-720): reads sums, cone lengths, priors, node states and cone count
 * for `tree` (counts must match) and computes the occupancy of every leaf
 * with params->confidence_threshold (NULL: the tree's parameters). */
TSR_API tsr_status tsr_occupancy_load(const tsr_tree *tree, const char *path, const tsr_params *params,
                                      void *cuda_stream, tsr_occupancy **out_occupancy);

#ifdef __cplusplus
}
#endif
#endif
