// ref_driver.cpp -- runs the reference's own hot path (test infrastructure).
//
// oracle/Makefile (target `ref`) compiles the reference's Scene/Tree and
// SurfaceExtraction sources unmodified, where they lie, against the shim of
// BaseProject in oracle/ref_shim/, and links them with this driver into
// oracle/_ref/libtsr_ref.so.  The driver holds the Scene singleton's samples,
// cameras and tree, runs Tree::Tree() (Tree.cpp:26-37), Occupancy(const Tree
// *) (Occupancy.cpp:78-103) and Occupancy::extractCrust()
// (Occupancy.cpp:523-528) on one OpenMP thread (so that the reference's
// order-dependent steps take their single-thread order), and hands back what
// the reference's own writers save (Nodes/Leaves/DualCells/Occupancy::
// saveToFile, into the shim's in-memory files), the reordered samples and the
// raw DMC mesh.  Only tests and the fixture generator load it.
#include <omp.h>

#include <cstring>
#include <iostream>
#include <string>

#include "Platform/Storage/File.h"
#include "Platform/Utilities/ParametersManager.h"
#include "SurfaceReconstruction/Scene/Camera/Cameras.h"
#include "SurfaceReconstruction/Scene/Samples.h"
#include "SurfaceReconstruction/Scene/Scene.h"
#include "SurfaceReconstruction/Scene/Tree/Leaves.h"
#include "SurfaceReconstruction/Scene/Tree/Tree.h"
#include "SurfaceReconstruction/SurfaceExtraction/DualMarchingCells.h"
#include "SurfaceReconstruction/SurfaceExtraction/Occupancy.h"

using namespace SurfaceReconstruction;

namespace {
Samples g_samples;
Cameras g_cameras;
Tree *g_tree = nullptr;
Occupancy *g_occ = nullptr;
std::string g_error;
std::vector<double> g_occupancy;   // getOccupancy of every leaf
}  // namespace

const uint32 Samples::INVALID_INDEX;
const uint32 Cameras::INVALID_ID;

std::map<std::string, std::vector<char>> &Storage::shim_files() {
    static std::map<std::string, std::vector<char>> files;
    return files;
}

Utilities::ParametersManager &Utilities::ParametersManager::getSingleton() {
    static ParametersManager m;
    return m;
}

Scene &Scene::getSingleton() {
    static Scene s;
    return s;
}
Samples &Scene::getSamples() { return g_samples; }
const Samples &Scene::getSamples() const { return g_samples; }
const Cameras &Scene::getCameras() const { return g_cameras; }
const Tree *Scene::getTree() const { return g_tree; }
uint32 Scene::getMinIsleSize() const { return 0; }

// The reference reports progress on std::cout; the driver discards it.
struct NullBuffer : std::streambuf {
    int overflow(int c) override { return c; }
};
struct QuietCout {
    NullBuffer null;
    std::streambuf *old;
    QuietCout() : old(std::cout.rdbuf(&null)) {}
    ~QuietCout() { std::cout.rdbuf(old); }
};

static void reset() {
    delete g_occ;
    g_occ = nullptr;
    delete g_tree;
    g_tree = nullptr;
    Storage::shim_files().clear();
    g_occupancy.clear();
}

extern "C" {

const char *tsrr_last_error() { return g_error.c_str(); }

// params: h_SVO (maxRelativeSamplingDistance), h_O (Occupancy::bandwidthFactor),
// confidence threshold, relative prior radius, relative sample cone length.
// stage 0: tree; 1: + occupancy field; 2: + DMC mesh.  threads: OpenMP
// threads (1 gives the reference's single-thread order in its order-dependent
// steps; more is for timing).  Returns 0 on success.
int tsrr_run(uint32_t n, uint32_t k, const double *pos, const double *nrm, const double *scale, const double *conf,
             const uint32_t *links, uint32_t ncams, const double *cams, const double *params, int stage,
             int threads) {
    QuietCout quiet;
    try {
        reset();
        omp_set_num_threads(threads > 0 ? threads : 1);
        g_samples = Samples();
        g_samples.mMaxCamsPerSample = k;
        g_samples.mMaxRelativeSamplingDistance = params[0];
        for (uint32_t i = 0; i < n; ++i) {
            g_samples.mPositions.emplace_back(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
            g_samples.mNormals.emplace_back(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
            g_samples.mScales.push_back(scale[i]);
            g_samples.mConfidences.push_back(conf[i]);
        }
        g_samples.mParentCameras.assign(links, links + (size_t)n * k);
        g_samples.computeAABB();
        g_cameras.mPositions.clear();
        for (uint32_t c = 0; c < ncams; ++c) g_cameras.mPositions.emplace_back(cams[3 * c], cams[3 * c + 1], cams[3 * c + 2]);
        Utilities::ParametersManager &pm = Utilities::ParametersManager::getSingleton();
        pm.set("Occupancy::bandwidthFactor", params[1]);
        pm.set("Occupancy::confidenceThreshold", params[2]);
        pm.set("Occupancy::relativeRadiusForPriors", params[3]);
        pm.set("Occupancy::relativeSampleConeLength", params[4]);

        g_tree = new Tree();
        g_tree->saveToFiles(Storage::Path("ref"));
        if (stage >= 1) {
            g_occ = new Occupancy(g_tree);
            g_occ->saveToFile(Storage::Path("ref.occupancy"));
            const uint32 nl = g_tree->getLeaves().getCount();
            g_occupancy.resize(nl);
            for (uint32 l = 0; l < nl; ++l) g_occupancy[l] = g_occ->getOccupancy(l);
        }
        if (stage >= 2) g_occ->extractCrust();
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// Occupancy::eraseSamples (removal != 0) or addSamples (Occupancy.h:167-175)
// of the chosen samples (indices into the reordered samples), then the field
// saved again as "ref.occupancy" and the occupancy of every leaf.
int tsrr_update(const uint32_t *samples, uint32_t count, int removal) {
    QuietCout quiet;
    try {
        if (!g_occ) throw std::runtime_error("no field to update");
        if (removal) g_occ->eraseSamples(samples, count);
        else g_occ->addSamples(samples, count);
        g_occ->saveToFile(Storage::Path("ref.occupancy"));
        for (uint32 l = 0; l < g_occupancy.size(); ++l) g_occupancy[l] = g_occ->getOccupancy(l);
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// Bytes the reference's writer saved under `name` ("ref.nodes", "ref.leaves",
// "ref.dualCells", "ref.occupancy"): the size when dst is null, else copied.
uint64_t tsrr_file(const char *name, void *dst, uint64_t cap) {
    auto &files = Storage::shim_files();
    auto it = files.find(name);
    if (it == files.end()) return 0;
    if (dst) memcpy(dst, it->second.data(), it->second.size() < cap ? it->second.size() : cap);
    return it->second.size();
}

// The samples after the tree build (reordered in place) and the target index
// of every input sample (Nodes.cpp:594-636).
int tsrr_samples(double *pos, double *nrm, double *scale, double *conf, uint32_t *links, uint32_t *targets) {
    const uint32 n = g_samples.getCount(), k = g_samples.mMaxCamsPerSample;
    for (uint32 i = 0; i < n; ++i) {
        const Math::Vector3 &p = g_samples.mPositions[i], &q = g_samples.mNormals[i];
        pos[3 * i] = p.x; pos[3 * i + 1] = p.y; pos[3 * i + 2] = p.z;
        nrm[3 * i] = q.x; nrm[3 * i + 1] = q.y; nrm[3 * i + 2] = q.z;
        scale[i] = g_samples.mScales[i];
        conf[i] = g_samples.mConfidences[i];
    }
    memcpy(links, g_samples.mParentCameras.data(), sizeof(uint32) * (size_t)n * k);
    memcpy(targets, g_samples.mTargets.data(), sizeof(uint32) * g_samples.mTargets.size());
    return 0;
}

// Occupancy::getOccupancy of every leaf (Occupancy.cpp:570-587).
int tsrr_occupancy(double *out) {
    memcpy(out, g_occupancy.data(), sizeof(double) * g_occupancy.size());
    return g_occupancy.empty() ? -1 : 0;
}

// The raw DMC mesh: vertex and triangle counts when the pointers are null.
int tsrr_mesh(uint32_t *counts, double *positions, double *scales, uint32_t *triangles) {
    if (!g_occ || !g_occ->getCrust()) return -1;
    const FlexibleMesh &m = g_occ->getCrust()->getSurface();
    counts[0] = m.getVertexCount();
    counts[1] = m.getIndexCount() / 3;
    if (positions) {
        for (uint32 i = 0; i < counts[0]; ++i) {
            positions[3 * i] = m.mPositions[i].x;
            positions[3 * i + 1] = m.mPositions[i].y;
            positions[3 * i + 2] = m.mPositions[i].z;
            scales[i] = m.mScales[i];
        }
        memcpy(triangles, m.mIndices.data(), sizeof(uint32) * m.mIndices.size());
    }
    return 0;
}

}  // extern "C"
