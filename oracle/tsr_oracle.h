/*
 * tsr_oracle.h -- C API of the FP64 CPU oracle for the TSR volumetric core.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker and the timed
 * CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it; the product library (tsr_b200/csrc) never links
 * or calls it.
 *
 * It restates, in plain C++ with Real = double, the reference's hot path:
 *   Scene/Tree/{Tree,Nodes,Leaves,DualCells,NodesIterator,LeavesIterator}.cpp,
 *   SurfaceExtraction/{Occupancy,ConeNodesChecker,SphereNodeStatesChecker,
 *   DualMarchingCells,DualMarchingCell,EdgeVertexIndex}.cpp
 * (paths relative to SurfaceReconstruction/SurfaceReconstruction/ of the
 * reference).  Each function in tsr_oracle.cpp cites the file:line it follows.
 *
 * Parity pinning: the reference has no tests, golden vectors or fixtures for
 * this path, so this restatement is pinned against the reference's own code:
 * `make -C oracle ref` compiles the reference's Scene/Tree and
 * SurfaceExtraction sources unmodified against a project-written shim of the
 * absent BaseProject headers (oracle/ref_shim/), and tests/test_ref_pin.py
 * requires every array of this restatement -- node arrays, permutation,
 * leaves, neighbours, dual cells, the FP64 field, the incremental update and
 * the raw DMC mesh -- to equal the reference's bit for bit, on committed
 * reference-made fixtures (tests/golden/ref_*.npz) and on live runs.  What
 * stays unpinned is BaseProject itself: its geometry helpers
 * (ObliqueCircularCone, intersectAABBWithSphere, intersectAABBWithLineSegment,
 * Plane, EPSILON, REAL_MAX) are restated from their call sites, and the shim
 * uses these same restatements.
 */
#ifndef TSR_ORACLE_H
#define TSR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tsro_scene tsro_scene;

/* params[5] = { Samples::maxRelativeSamplingDistance (h_SVO),
 *               Occupancy::bandwidthFactor (h_O),
 *               Occupancy::confidenceThreshold,
 *               Occupancy::relativeRadiusForPriors,
 *               Occupancy::relativeSampleConeLength } */
tsro_scene *tsro_create(uint32_t n, uint32_t k,
                        const double *pos, const double *nrm,
                        const double *scale, const double *conf,
                        const uint32_t *links, uint32_t ncams,
                        const double *cams, const double *params);
void tsro_free(tsro_scene *s);

/* stop_after: 0 = full build (containment, sampling, balance, reorder,
 * sample reorder, leaves, neighbours, dual cells); 1 = containment only;
 * 2 = + sampling nodes; 3 = + balancing; 4 = full build with the sampling
 * pass run in the round-parallel schedule; 5 = containment + round-parallel
 * sampling only.  For 1, 2, 3 and 5 only the node arrays in creation order
 * are available (no reorder).  Returns 0 on success. */
int tsro_build_tree(tsro_scene *s, int stop_after);

/* counts[10] = { nodes, leaves, dual cells, neighbour entries, dmc vertices,
 *   dmc triangles, writers (sampling), sampling splits, sampling rounds,
 *   deepest unresolved chain in a round } */
void tsro_counts(const tsro_scene *s, uint64_t *counts);
void tsro_root(const tsro_scene *s, double *min_size4);
void tsro_get_nodes(const tsro_scene *s, uint32_t *children, uint32_t *parents,
                    uint32_t *counts, uint32_t *starts);
void tsro_get_permutation(const tsro_scene *s, uint32_t *target_indices);
void tsro_get_leaves(const tsro_scene *s, double *min_size4, uint32_t *node_idx,
                     uint32_t *node_to_leaf, uint32_t *nb_offsets, uint32_t *nbs);
void tsro_get_dual_cells(const tsro_scene *s, uint32_t *cells8);
void tsro_get_sample_depths(const tsro_scene *s, uint32_t *depths);

/* Occupancy::computeOccupancy; nthreads <= 0 uses all OpenMP threads.
 * prune: 1 = conservative cone pruning (default), 0 = visit every leaf up to
 * the depth cap (slow; proves the pruning test cannot change the sums). */
int tsro_occupancy(tsro_scene *s, int nthreads, int prune);
/* Runs only the links [first, first+count) of both passes; used to time a
 * bounded sample of the field computation.  Returns 0 on success. */
int tsro_occupancy_links(tsro_scene *s, int nthreads, uint64_t first, uint64_t count);
/* Occupancy::addSamples / eraseSamples (removal != 0) of samples given by
 * their tree-order indices, after tsro_occupancy (Occupancy.cpp:129-136). */
int tsro_occupancy_update(tsro_scene *s, int nthreads, const uint32_t *samples, uint32_t count, int removal);
void tsro_get_occupancy(const tsro_scene *s, double *e_sum, double *s_sum,
                        double *e_len, double *s_len, double *prior, double *occ,
                        uint32_t *node_states, double *cone_count);

/* Replaces the per-leaf occupancy values DMC reads (to check a GPU mesh
 * against the oracle's DMC on the GPU's own field). */
int tsro_set_occupancy(tsro_scene *s, const double *occ);
int tsro_dmc(tsro_scene *s);
void tsro_get_mesh(const tsro_scene *s, uint8_t *cases, double *vpos, double *vscale,
                   uint32_t *vkeys, uint32_t *tris);

/* seconds spent per stage: 0 containment, 1 sampling, 2 balance, 3 reorder +
 * sample reorder, 4 leaves + neighbours, 5 dual cells, 6 sampleness,
 * 7 emptiness, 8 priors, 9 dmc */
double tsro_stage_seconds(const tsro_scene *s, int stage);

#ifdef __cplusplus
}
#endif
#endif
