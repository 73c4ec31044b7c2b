"""Host-side mirror of the reference's scene API over the sm_100a C ABI.

The classes follow the reference's names, argument meaning and error
behaviour (paths relative to SurfaceReconstruction/SurfaceReconstruction/):

* ``Samples``            -- Scene/Samples.h:300-312 (SoA sample store)
* ``Tree``               -- Scene/Tree/Tree.h:26-91; building it reorders the
                            samples in place like Nodes::reorderSamplesAndFillNodes
                            (Nodes.cpp:594-636)
* ``Occupancy``          -- SurfaceExtraction/Occupancy.h:26-149
* ``DualMarchingCells``  -- SurfaceExtraction/DualMarchingCells.h:31-61

Every call goes through include/tsr_core.h in tsr_b200/lib/libtsrcore.so.
There is no CPU path: if the library is missing, importing this module fails.
Failures raise ``TsrError`` (the reference throws FailureHandling::Exception).
"""
from __future__ import annotations

import ctypes
import json
import os
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "lib" / "libtsrcore.so"
if not _LIB_PATH.exists():
    raise ImportError("tsr_b200 CUDA library not built: %s (run python -m tsr_b200.build)" % _LIB_PATH)

_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64


class tsr_params(ctypes.Structure):
    _fields_ = [("max_relative_sampling_distance", ctypes.c_double),
                ("bandwidth_factor", ctypes.c_double),
                ("confidence_threshold", ctypes.c_double),
                ("relative_radius_for_priors", ctypes.c_double),
                ("relative_sample_cone_length", ctypes.c_double)]


class tsr_samples_view(ctypes.Structure):
    _fields_ = [("count", _U32), ("cams_per_sample", _U32), ("positions", _P), ("normals", _P),
                ("scales", _P), ("confidences", _P), ("camera_links", _P)]


class tsr_cameras_view(ctypes.Structure):
    _fields_ = [("count", _U32), ("positions", _P)]


class tsr_tree_counts(ctypes.Structure):
    _fields_ = [("nodes", _U64), ("leaves", _U64), ("dual_cells", _U64), ("neighbor_entries", _U64),
                ("max_depth", _U32), ("sampling_rounds", _U32), ("sampling_writers", _U64),
                ("sampling_waves", _U32), ("reserved", _U32)]


class tsr_mesh_counts(ctypes.Structure):
    _fields_ = [("vertices", _U64), ("triangles", _U64), ("active_cells", _U64)]


class tsr_occupancy_counts(ctypes.Structure):
    _fields_ = [("links", _U64), ("accepted_sampleness", _U64), ("accepted_emptiness", _U64),
                ("visited_sampleness", _U64), ("visited_emptiness", _U64), ("visited_priors", _U64),
                ("pruned_leaves", _U64), ("repaired_leaves", _U64), ("certified_leaves", _U64)]


MLP_FEATURES, MLP_HIDDEN, MLP_OUTPUTS, MLP_PARAMS = 10, 64, 2, 4994


class tsr_mesh_post_counts(ctypes.Structure):
    _fields_ = [("isle_vertices", ctypes.c_uint64), ("isle_triangles", ctypes.c_uint64),
                ("border_edges", ctypes.c_uint64), ("holes", ctypes.c_uint64), ("hole_vertices", ctypes.c_uint64),
                ("hole_triangles", ctypes.c_uint64), ("skipped_rings", ctypes.c_uint64)]


class tsr_pruner(ctypes.Structure):
    _fields_ = [("weights", _P), ("feature_mean", ctypes.c_float * MLP_FEATURES),
                ("feature_inv_std", ctypes.c_float * MLP_FEATURES), ("sign_threshold", ctypes.c_float),
                ("band_threshold", ctypes.c_float), ("dilation", _U32), ("bound_levels", _U32)]


lib = ctypes.CDLL(str(_LIB_PATH))
_sig = {
    "tsr_params_default": (None, [_P]),
    "tsr_last_error_message": (ctypes.c_char_p, []),
    "tsr_version": (ctypes.c_char_p, []),
    "tsr_tree_build": (ctypes.c_int, [_P, _P, _P, _P]),
    "tsr_tree_build_device": (ctypes.c_int, [_P, _P, _P, _P]),
    "tsr_tree_copy_samples": (ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
    "tsr_kernel_launches": (ctypes.c_ulonglong, []),
    "tsr_set_iteration_limits": (None, [ctypes.c_uint32, ctypes.c_uint32]),
    "tsr_tree_free": (None, [_P]),
    "tsr_tree_get_counts": (ctypes.c_int, [_P, _P]),
    "tsr_tree_root_scope": (ctypes.c_int, [_P, _P]),
    "tsr_samples_root_scope_noalloc": (ctypes.c_int, [ctypes.c_uint64, _P, _P, _P, _P, _P]),
    "tsr_tree_copy_nodes": (ctypes.c_int, [_P, _P, _P, _P, _P]),
    "tsr_tree_copy_permutation": (ctypes.c_int, [_P, _P]),
    "tsr_tree_copy_leaves": (ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
    "tsr_tree_copy_dual_cells": (ctypes.c_int, [_P, _P]),
    "tsr_tree_stage_ms": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "tsr_occupancy_compute": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, _P, _P]),
    "tsr_occupancy_free": (None, [_P]),
    "tsr_occupancy_get_counts": (ctypes.c_int, [_P, _P]),
    "tsr_occupancy_copy": (ctypes.c_int, [_P, ctypes.c_int, _P]),
    "tsr_occupancy_stage_ms": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "tsr_dmc_extract": (ctypes.c_int, [_P, _P, _P, _P]),
    "tsr_mesh_free": (None, [_P]),
    "tsr_mesh_get_counts": (ctypes.c_int, [_P, _P]),
    "tsr_mesh_copy": (ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
    "tsr_occupancy_leaf_features": (ctypes.c_int, [_P, _P, _P]),
    "tsr_occupancy_update": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int, _P, ctypes.c_uint32, _P]),
    "tsr_tree_erase_samples": (ctypes.c_int, [_P, _P]),
    "tsr_mlp_train_batch": (ctypes.c_int, [_P, _P, ctypes.c_uint32, _P, _P, _P, ctypes.c_float, ctypes.c_float,
                                           _P]),
    "tsr_mlp_adam": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_uint32, ctypes.c_float, ctypes.c_float, _P]),
    "tsr_mlp_forward": (ctypes.c_int, [_P, ctypes.c_uint32, _P, _P, _P]),
    "tsr_mlp_infer_bf16": (ctypes.c_int, [_P, ctypes.c_uint32, _P, _P, _P]),
    "tsr_occupancy_compute_pruned": (ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
    "tsr_mesh_postprocess": (ctypes.c_int, [_P, ctypes.c_uint32, _P]),
    "tsr_mesh_copy_normals": (ctypes.c_int, [_P, _P]),
    "tsr_mesh_create": (ctypes.c_int, [_P, _P, ctypes.c_uint64, _P, ctypes.c_uint64, _P, _P]),
    "tsr_depth_triangulate": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_uint32, _P, _P, _P, _P, _P, _P]),
    "tsr_mesh_copy_colors": (ctypes.c_int, [_P, _P]),
    "tsr_mesh_copy_pixel_map": (ctypes.c_int, [_P, _P]),
    "tsr_tree_save": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "tsr_tree_save_samples": (ctypes.c_int, [_P, _P, ctypes.c_char_p]),
    "tsr_tree_load": (ctypes.c_int, [ctypes.c_char_p, _P, _P, _P, _P, _P]),
    "tsr_occupancy_save": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "tsr_occupancy_load": (ctypes.c_int, [_P, ctypes.c_char_p, _P, _P, _P]),
}
for _name, (_res, _args) in _sig.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED = tuple(_sig)
STATUS = {0: "TSR_OK", 1: "TSR_ERR_INVALID_ARG", 2: "TSR_ERR_OVERFLOW_U32", 3: "TSR_ERR_OOM",
          4: "TSR_ERR_CUDA", 5: "TSR_ERR_DEVICE_ASSERT", 6: "TSR_ERR_TIMEOUT", 7: "TSR_ERR_STATE"}
FIELDS = {"emptiness_sum": 0, "sampleness_sum": 1, "emptiness_length": 2, "sampleness_length": 3,
          "prior_emptiness": 4, "occupancy": 5, "node_states": 6, "cone_count": 7}
NODE_FLAG_SAMPLENESS = 1
NODE_FLAG_EMPTINESS = 2
INVALID_INDEX = 0xFFFFFFFF


class TsrError(RuntimeError):
    """Raised for a non-OK tsr_status (the reference's FailureHandling::Exception)."""

    def __init__(self, status, message):
        super().__init__("%s: %s" % (STATUS.get(status, status), message))
        self.status = status


def _check(rc):
    if rc != 0:
        raise TsrError(rc, lib.tsr_last_error_message().decode())


def _ptr(a):
    return a.ctypes.data_as(_P) if a is not None else None


def _stream_ptr(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return _P(stream)
    return _P(int(getattr(stream, "cuda_stream", stream)))


def params_default():
    p = tsr_params()
    lib.tsr_params_default(ctypes.byref(p))
    return p


def make_params(h_svo=2.0, h_o=2.0, confidence_threshold=100.0, prior_radius=25.0, rel_cone_length=1.0):
    return tsr_params(h_svo, h_o, confidence_threshold, prior_radius, rel_cone_length)


class Samples:
    """SoA samples (Samples.h:300-312): positions, normals, scales,
    confidences and K camera links per sample."""

    def __init__(self, positions, normals, scales, confidences, camera_links):
        self.positions = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
        self.normals = np.ascontiguousarray(normals, np.float64).reshape(-1, 3)
        self.scales = np.ascontiguousarray(scales, np.float64).reshape(-1)
        self.confidences = np.ascontiguousarray(confidences, np.float64).reshape(-1)
        links = np.ascontiguousarray(camera_links, np.uint32)
        self.camera_links = links.reshape(self.count, -1)

    @classmethod
    def from_scene(cls, scene):
        """Copies the scene's arrays (a Tree reorders its Samples in place)."""
        return cls(scene.pos.copy(), scene.nrm.copy(), scene.scale.copy(), scene.conf.copy(), scene.links.copy())

    @property
    def count(self):
        return int(self.positions.shape[0])

    @property
    def max_cameras_per_sample(self):
        return int(self.camera_links.shape[1])

    def view(self):
        return tsr_samples_view(self.count, self.max_cameras_per_sample, _ptr(self.positions), _ptr(self.normals),
                                _ptr(self.scales), _ptr(self.confidences), _ptr(self.camera_links))

    @classmethod
    def fromDepthMeshes(cls, meshes, camera_indices):
        """Samples::addSamplesViaMeshes (Samples.cpp:224-272): one sample per
        vertex of every DepthMesh, confidence 1, with the mesh's camera links
        -- ``camera_indices[i]`` is either the reference camera's index (the
        reference's fallback without a views image, Scene.cpp:563-570) or a
        (vertices x k) array of camera indices; K is the largest k and shorter
        link lists are padded with 0xFFFFFFFF (Cameras::INVALID_ID)."""
        links = []
        for m, ci in zip(meshes, camera_indices):
            nv = m.positions.shape[0]
            if np.ndim(ci) == 0:
                links.append(np.full((nv, 1), int(ci), np.uint32))
            else:
                a = np.asarray(ci, np.uint32).reshape(nv, -1)
                links.append(a)
        k = max([a.shape[1] for a in links] + [1])
        links = [np.pad(a, ((0, 0), (0, k - a.shape[1])), constant_values=INVALID_INDEX) for a in links]
        pos = np.concatenate([m.positions for m in meshes]) if meshes else np.zeros((0, 3))
        nrm = np.concatenate([m.normals for m in meshes]) if meshes else np.zeros((0, 3))
        sc = np.concatenate([m.scales for m in meshes]) if meshes else np.zeros(0)
        if (sc <= 0).any():   # Samples::check (Samples.cpp:274-288)
            raise ValueError("invalid (non-positive) sample scale detected")
        out = cls(pos, nrm, sc, np.ones(pos.shape[0]), np.concatenate(links) if links else np.zeros((0, k)))
        out.colors = np.concatenate([m.colors for m in meshes]) if meshes else np.zeros((0, 3))
        return out

    def reorder(self, target_indices):
        """Samples::reorder (Samples.cpp:825-835): element i moves to target[i]."""
        t = np.asarray(target_indices, np.int64)
        for name in ("positions", "normals", "scales", "confidences", "camera_links"):
            a = getattr(self, name)
            b = np.empty_like(a)
            b[t] = a
            setattr(self, name, b)


class Cameras:
    """Camera centres (Cameras::getPositionWS, Cameras.h:161-166)."""

    def __init__(self, positions):
        self.positions = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)

    @property
    def count(self):
        return int(self.positions.shape[0])

    def view(self):
        return tsr_cameras_view(self.count, _ptr(self.positions))


class Nodes:
    """Node arrays after the reorder (Nodes.h:144-147)."""

    def __init__(self, children, parents, sample_counts, sample_starts):
        self.children = children
        self.parents = parents
        self.samples_per_node = sample_counts
        self.sample_start_indices = sample_starts

    def getCount(self):
        return int(self.children.shape[0])

    def isLeaf(self, node):
        return node != INVALID_INDEX and self.children[node] == INVALID_INDEX

    def getDepth(self, node):
        d = 0
        p = self.parents[node]
        while p != INVALID_INDEX:
            d += 1
            p = self.parents[p]
        return d


class Leaves:
    """Leaf scopes, node->leaf links and the neighbour CSR (Leaves.h:90-98)."""

    def __init__(self, scopes, node_index, node_to_leaf, offsets, neighbors):
        self.scopes = scopes                # (L, 4): min x, y, z, size
        self.node_index = node_index
        self.node_to_leaf_links = node_to_leaf
        self.neighbors_offsets = offsets
        self.neighbors = neighbors

    def getCount(self):
        return int(self.scopes.shape[0])

    def getNeighbors(self, leaf):
        return self.neighbors[self.neighbors_offsets[leaf]:self.neighbors_offsets[leaf + 1]]

    def getCenterPositions(self):
        return self.scopes[:, :3] + 0.5 * self.scopes[:, 3:4]


class Tree:
    """Tree::Tree() (Tree.cpp:26-37) on the GPU.

    Like the reference, building the tree reorders ``samples`` in place so
    that every node's samples are contiguous.
    """

    def __init__(self, samples: Samples, params=None, stream=None, reorder_samples=True):
        self._h = _P()
        self.params = params or params_default()
        self._stream = stream
        v = samples.view()
        _check(lib.tsr_tree_build(ctypes.byref(v), ctypes.byref(self.params), _stream_ptr(stream),
                                  ctypes.byref(self._h)))
        self._read_counts(samples.count)
        if reorder_samples:
            # the reference reorders Samples in place (Nodes.cpp:630); copy the
            # device-side reordered arrays back instead of permuting on the host
            _check(lib.tsr_tree_copy_samples(self._h, _ptr(samples.positions), _ptr(samples.normals),
                                             _ptr(samples.scales), _ptr(samples.confidences),
                                             _ptr(samples.camera_links)))

    def _read_counts(self, sample_count):
        c = tsr_tree_counts()
        _check(lib.tsr_tree_get_counts(self._h, ctypes.byref(c)))
        self.counts = {k: int(getattr(c, k)) for k, _ in tsr_tree_counts._fields_}
        self.sample_count = sample_count
        self.input_count = sample_count
        self._nodes = self._leaves = self._cells = None

    @classmethod
    def fromFiles(cls, prefix, samples: Samples, aabb=None, params=None, stream=None):
        """Tree::Tree(filesBeginning) (Tree.cpp:39-43): the tree of
        ``prefix``.nodes / .leaves / .dualCells over ``samples`` in tree
        order (the order a built tree leaves them in).  ``aabb``: the
        samples file's AABB (min xyz, max xyz); None computes it from the
        samples."""
        self = cls.__new__(cls)
        self._h = _P()
        self.params = params or params_default()
        self._stream = stream
        v = samples.view()
        bb = None if aabb is None else np.ascontiguousarray(aabb, np.float64).reshape(-1)
        if bb is not None and bb.shape != (6,):
            raise ValueError("AABB: min x, y, z and max x, y, z")
        _check(lib.tsr_tree_load(os.fsencode(prefix), ctypes.byref(v), _ptr(bb) if bb is not None else None,
                                 ctypes.byref(self.params), _stream_ptr(stream), ctypes.byref(self._h)))
        self._read_counts(samples.count)
        return self

    def saveToFiles(self, prefix):
        """Tree::saveToFiles (Tree.cpp:129-134)."""
        _check(lib.tsr_tree_save(self._h, os.fsencode(prefix)))

    def saveSamples(self, path, colors=None):
        """Samples::saveToFile (Samples.cpp:733-765) of the tree's samples in
        tree order with the AABB the tree was built over; ``colors``: 3 per
        sample in tree order, or None for zeros."""
        c = None if colors is None else np.ascontiguousarray(colors, np.float64)
        if c is not None and c.shape != (self.sample_count, 3):
            raise ValueError("one RGB colour per sample expected")
        _check(lib.tsr_tree_save_samples(self._h, _ptr(c) if c is not None else None, os.fsencode(path)))

    def __del__(self):
        if getattr(self, "_h", None) and self._h:
            lib.tsr_tree_free(self._h)
            self._h = _P()

    @property
    def handle(self):
        return self._h

    def getRootScope(self):
        m = np.zeros(4)
        _check(lib.tsr_tree_root_scope(self._h, _ptr(m)))
        return m

    def getRootNodeSize(self):
        return float(self.getRootScope()[3])

    def getCenter(self):
        m = self.getRootScope()
        return m[:3] + 0.5 * m[3]

    def eraseSamples(self, inliers):
        """Tree::eraseSamples (Tree.cpp:50-53) with the samples' compaction;
        ``inliers``: one bool per sample in tree order."""
        keep = np.ascontiguousarray(inliers, np.uint8)
        if keep.shape[0] != self.sample_count:
            raise ValueError("one flag per sample expected")
        _check(lib.tsr_tree_erase_samples(self._h, _ptr(keep)))
        self.sample_count = int(keep.astype(bool).sum())
        self._nodes = None

    def getPermutation(self):
        """Tree-order index of every input sample (0xFFFFFFFF once erased)."""
        t = np.zeros(self.input_count, np.uint32)
        _check(lib.tsr_tree_copy_permutation(self._h, _ptr(t)))
        return t

    def getNodes(self):
        if self._nodes is None:
            n = self.counts["nodes"]
            a = [np.zeros(n, np.uint32) for _ in range(4)]
            _check(lib.tsr_tree_copy_nodes(self._h, *[_ptr(x) for x in a]))
            self._nodes = Nodes(*a)
        return self._nodes

    def getLeaves(self):
        if self._leaves is None:
            L, n, e = self.counts["leaves"], self.counts["nodes"], self.counts["neighbor_entries"]
            scopes = np.zeros((L, 4))
            ni = np.zeros(L, np.uint32)
            n2l = np.zeros(n, np.uint32)
            off = np.zeros(L + 1, np.uint32)
            nbs = np.zeros(e, np.uint32)
            _check(lib.tsr_tree_copy_leaves(self._h, _ptr(scopes), _ptr(ni), _ptr(n2l), _ptr(off), _ptr(nbs)))
            self._leaves = Leaves(scopes, ni, n2l, off, nbs)
        return self._leaves

    def getDualCells(self):
        if self._cells is None:
            nc = self.counts["dual_cells"]
            c = np.zeros((nc, 8), np.uint32)
            if nc:
                _check(lib.tsr_tree_copy_dual_cells(self._h, _ptr(c)))
            self._cells = c
        return self._cells

    def getSampleDepth(self, scale, h_svo=None):
        """Tree::getSampleDepth (Tree.cpp:86-91) for a sample scale."""
        h = self.params.max_relative_sampling_distance if h_svo is None else h_svo
        return np.ceil(np.log2(self.getRootNodeSize() / (np.asarray(scale) * h))).astype(np.uint32)

    def stage_ms(self):
        ms = np.zeros(8, np.float32)
        _check(lib.tsr_tree_stage_ms(self._h, _ptr(ms), 8))
        names = ["containment", "sampling", "balance", "reorder", "neighbors", "dual_cells"]
        return {k: float(v) for k, v in zip(names, ms)}


class Occupancy:
    """Occupancy::Occupancy(const Tree *) (Occupancy.cpp:78-127) on the GPU."""

    EMPTINESS, SAMPLENESS = 0, 1

    def __init__(self, tree: Tree, cameras: Cameras, params=None, mode=0, stream=None, pruner=None):
        """pruner: a ``Pruner`` -- the pruned field (no counterpart in the
        reference); None computes the plain field like the reference."""
        self._h = _P()
        self.tree = tree
        p = params or tree.params
        if pruner is None:
            _check(lib.tsr_occupancy_compute(tree.handle, ctypes.byref(cameras.view()), ctypes.byref(p), mode,
                                             _stream_ptr(stream), ctypes.byref(self._h)))
        else:
            pv = pruner.view()
            _check(lib.tsr_occupancy_compute_pruned(tree.handle, ctypes.byref(cameras.view()), ctypes.byref(p),
                                                    ctypes.byref(pv), _stream_ptr(stream), ctypes.byref(self._h)))
        self._created(stream)

    def _created(self, stream):
        c = tsr_occupancy_counts()
        _check(lib.tsr_occupancy_get_counts(self._h, ctypes.byref(c)))
        self.counts = {k: int(getattr(c, k)) for k, _ in tsr_occupancy_counts._fields_}
        self._cache = {}
        self.mCrust = None
        self._stream = stream

    @classmethod
    def fromFile(cls, tree: Tree, path, params=None, stream=None):
        """Occupancy::Occupancy(fileName) (Occupancy.cpp:598-602) for ``tree``."""
        self = cls.__new__(cls)
        self._h = _P()
        self.tree = tree
        p = params or tree.params
        _check(lib.tsr_occupancy_load(tree.handle, os.fsencode(path), ctypes.byref(p), _stream_ptr(stream),
                                      ctypes.byref(self._h)))
        self._created(stream)
        return self

    def saveToFile(self, path):
        """Occupancy::saveToFile (Occupancy.cpp:722-766)."""
        _check(lib.tsr_occupancy_save(self._h, os.fsencode(path)))

    def __del__(self):
        if getattr(self, "_h", None) and self._h:
            lib.tsr_occupancy_free(self._h)
            self._h = _P()

    @property
    def handle(self):
        return self._h

    def addSamples(self, samples, cameras, params=None):
        """Occupancy::addSamples (Occupancy.h:167-170): tree-order indices."""
        self._on_samples_changed(False, samples, cameras, params)

    def eraseSamples(self, samples, cameras, params=None):
        """Occupancy::eraseSamples (Occupancy.h:172-175): tree-order indices."""
        self._on_samples_changed(True, samples, cameras, params)

    def _on_samples_changed(self, removal, samples, cameras, params):
        ids = np.ascontiguousarray(samples, np.uint32)
        p = params or self.tree.params
        _check(lib.tsr_occupancy_update(self._h, self.tree.handle, ctypes.byref(cameras.view()), ctypes.byref(p),
                                        1 if removal else 0, _ptr(ids), ids.shape[0], _stream_ptr(self._stream)))
        self._cache = {}
        c = tsr_occupancy_counts()
        _check(lib.tsr_occupancy_get_counts(self._h, ctypes.byref(c)))
        self.counts = {k: int(getattr(c, k)) for k, _ in tsr_occupancy_counts._fields_}

    def getLeafFeatures(self):
        """The learned pruner's per-leaf features (leaves x 10 float32)."""
        f = np.zeros((self.tree.counts["leaves"], MLP_FEATURES), np.float32)
        _check(lib.tsr_occupancy_leaf_features(self.tree.handle, self._h, _ptr(f)))
        return f

    def stage_ms(self):
        """CUDA-event milliseconds of the field's stages."""
        ms = np.zeros(8, np.float32)
        _check(lib.tsr_occupancy_stage_ms(self._h, _ptr(ms), 8))
        names = ["sampleness", "flags", "emptiness", "priors", "finalize"]
        return {k: float(v) for k, v in zip(names, ms)}

    def field(self, name):
        if name not in self._cache:
            if name == "cone_count":
                v = np.zeros(1)
            elif name == "node_states":
                v = np.zeros(self.tree.counts["nodes"], np.uint32)
            else:
                v = np.zeros(self.tree.counts["leaves"])
            _check(lib.tsr_occupancy_copy(self._h, FIELDS[name], _ptr(v)))
            self._cache[name] = float(v[0]) if name == "cone_count" else v
        return self._cache[name]

    def getOccupancy(self, leaf=None):
        o = self.field("occupancy")
        return o if leaf is None else float(o[leaf])

    def getNodeStates(self):
        return self.field("node_states")

    def getPriorForEmptiness(self, leaf=None):
        p = self.field("prior_emptiness")
        return p if leaf is None else float(p[leaf])

    def getPriorForSampleness(self, leaf=None):
        p = 1.0 - self.field("prior_emptiness")
        return p if leaf is None else float(p[leaf])

    def getEmptinessCPD(self, leaf=None):
        v = self.field("emptiness_sum") / self.field("cone_count")
        return v if leaf is None else float(v[leaf])

    def getSamplenessCPD(self, leaf=None):
        v = self.field("sampleness_sum") / self.field("cone_count")
        return v if leaf is None else float(v[leaf])

    def extractCrust(self, stream=None, min_isle_size=None):
        """Occupancy::extractCrust (Occupancy.cpp:523-528); the FlexibleMesh
        post-processing runs when ``min_isle_size`` is given (the reference
        always runs it, with Scene::minimumTriangleIsleSize = 1000)."""
        self.mCrust = DualMarchingCells(self, stream=stream if stream is not None else self._stream,
                                        min_isle_size=min_isle_size)
        return self.mCrust

    def getCrust(self):
        return self.mCrust


class DualMarchingCells:
    """DualMarchingCells (DualMarchingCells.cpp:26-169): extractMesh, and
    with ``min_isle_size`` the post-processing of its constructor
    (deleteIsolatedGeometry, fillHoles, computeNormalsWeightedByAngles) on
    the GPU too; the reference passes Scene::minimumTriangleIsleSize = 1000."""

    def __init__(self, occupancy: Occupancy, stream=None, min_isle_size=None):
        self._h = _P()
        _check(lib.tsr_dmc_extract(occupancy.tree.handle, occupancy.handle, _stream_ptr(stream),
                                   ctypes.byref(self._h)))
        self.n_cells = occupancy.tree.counts["dual_cells"]
        self.post_counts = None
        if min_isle_size is not None:
            self._postprocess(min_isle_size)
        self._read()

    @classmethod
    def fromArrays(cls, positions, triangles, scales=None, stream=None, min_isle_size=None):
        """A FlexibleMesh of the given vertices and triangles (for the
        post-processing of a surface from elsewhere)."""
        self = cls.__new__(cls)
        self._h = _P()
        pos = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
        tri = np.ascontiguousarray(triangles, np.uint32).reshape(-1, 3)
        sc = None if scales is None else np.ascontiguousarray(scales, np.float64).reshape(-1)
        if sc is not None and sc.shape[0] != pos.shape[0]:
            raise ValueError("one scale per vertex expected")
        _check(lib.tsr_mesh_create(_ptr(pos), _ptr(sc) if sc is not None else None, pos.shape[0], _ptr(tri),
                                   tri.shape[0], _stream_ptr(stream), ctypes.byref(self._h)))
        self.n_cells = 0
        self.post_counts = None
        if min_isle_size is not None:
            self._postprocess(min_isle_size)
        self._read()
        return self

    def _postprocess(self, min_isle_size):
        pc = tsr_mesh_post_counts()
        _check(lib.tsr_mesh_postprocess(self._h, int(min_isle_size), ctypes.byref(pc)))
        self.post_counts = {k: int(getattr(pc, k)) for k, _ in tsr_mesh_post_counts._fields_}

    def postprocess(self, min_isle_size=1000):
        """The reference constructor's post-processing (DualMarchingCells.cpp:31-36)."""
        self._postprocess(min_isle_size)
        self._read()
        return self.post_counts

    def _read(self):
        c = tsr_mesh_counts()
        _check(lib.tsr_mesh_get_counts(self._h, ctypes.byref(c)))
        self.counts = {k: int(getattr(c, k)) for k, _ in tsr_mesh_counts._fields_}
        nv, nt = self.counts["vertices"], self.counts["triangles"]
        self.cases = np.zeros(self.n_cells, np.uint8)
        self.positions = np.zeros((nv, 3))
        self.scales = np.zeros(nv)
        self.edge_keys = np.zeros((nv, 2), np.uint32)
        self.triangles = np.zeros((nt, 3), np.uint32)
        _check(lib.tsr_mesh_copy(self._h, _ptr(self.cases) if self.n_cells else None, _ptr(self.positions),
                                 _ptr(self.scales), _ptr(self.edge_keys), _ptr(self.triangles)))
        self.normals = None
        if self.post_counts is not None:
            self.normals = np.zeros((nv, 3))
            if nv:
                _check(lib.tsr_mesh_copy_normals(self._h, _ptr(self.normals)))

    def __del__(self):
        if getattr(self, "_h", None) and self._h:
            lib.tsr_mesh_free(self._h)
            self._h = _P()

    def getSurface(self):
        return self.positions, self.triangles


class DepthImage:
    """DepthImage (Image/DepthImage.cpp): a depth map along the pixel rays,
    height x width, values <= 0 invalid."""

    def __init__(self, depths):
        self.depths = np.ascontiguousarray(depths, np.float64)
        if self.depths.ndim != 2:
            raise ValueError("a depth map is height x width")

    def triangulate(self, hps_to_ray_vs, hps_to_ray_ws, center, colors=None, stream=None):
        """DepthImage::triangulate (DepthImage.cpp:186-216) on the GPU.  The
        3x3 matrices are the ones the reference computes from its
        PinholeCamera (inverse viewport x inverse projection, and that x
        inverse rotation), applied to (x, y, 1) as a row vector."""
        return DepthMesh(self, hps_to_ray_vs, hps_to_ray_ws, center, colors, stream)


class DepthMesh:
    """The FlexibleMesh DepthImage::triangulate returns: positions, normals,
    colours, scales, triangles and the vertex of every pixel."""

    def __init__(self, image: DepthImage, hps_to_ray_vs, hps_to_ray_ws, center, colors=None, stream=None):
        H, W = image.depths.shape
        mvs = np.ascontiguousarray(hps_to_ray_vs, np.float64).reshape(9)
        mws = np.ascontiguousarray(hps_to_ray_ws, np.float64).reshape(9)
        c = np.ascontiguousarray(center, np.float64).reshape(3)
        col = None if colors is None else np.ascontiguousarray(colors, np.float64).reshape(H * W * 3)
        h = _P()
        _check(lib.tsr_depth_triangulate(_ptr(image.depths), W, H, _ptr(mvs), _ptr(mws), _ptr(c),
                                         _ptr(col) if col is not None else None, _stream_ptr(stream), ctypes.byref(h)))
        try:
            cnt = tsr_mesh_counts()
            _check(lib.tsr_mesh_get_counts(h, ctypes.byref(cnt)))
            nv, nt = int(cnt.vertices), int(cnt.triangles)
            self.positions, self.normals, self.colors = np.zeros((nv, 3)), np.zeros((nv, 3)), np.zeros((nv, 3))
            self.scales = np.zeros(nv)
            self.triangles = np.zeros((nt, 3), np.uint32)
            self.pixel_to_vertex = np.zeros((H, W), np.uint32)
            _check(lib.tsr_mesh_copy(h, None, _ptr(self.positions), _ptr(self.scales), None, _ptr(self.triangles)))
            if nv:
                _check(lib.tsr_mesh_copy_normals(h, _ptr(self.normals)))
                _check(lib.tsr_mesh_copy_colors(h, _ptr(self.colors)))
            _check(lib.tsr_mesh_copy_pixel_map(h, _ptr(self.pixel_to_vertex)))
        finally:
            lib.tsr_mesh_free(h)


class Pruner:
    """The learned pruner's network and decision thresholds (new; no
    counterpart in the reference).  ``weights``: TSR_MLP_PARAMS float32 values
    (W1[10][64], b1, W2[64][64], b2, W3[64][2], b3); features are normalized
    as (f - mean) * inv_std."""

    def __init__(self, weights, mean, inv_std, sign_threshold, band_threshold, dilation=1, bound_levels=2):
        self.weights = np.ascontiguousarray(weights, np.float32).reshape(-1)
        if self.weights.shape[0] != MLP_PARAMS:
            raise ValueError("expected %d weights" % MLP_PARAMS)
        self.mean = np.asarray(mean, np.float32).reshape(MLP_FEATURES)
        self.inv_std = np.asarray(inv_std, np.float32).reshape(MLP_FEATURES)
        self.sign_threshold = float(sign_threshold)
        self.band_threshold = float(band_threshold)
        self.dilation = int(dilation)
        self.bound_levels = int(bound_levels)

    @classmethod
    def load(cls, path=None):
        path = Path(path) if path else Path(__file__).resolve().parent / "pruner_weights.npz"
        z = np.load(path)
        self = cls(z["weights"], z["mean"], z["inv_std"], float(z["sign_threshold"]), float(z["band_threshold"]),
                   int(z["dilation"]), int(z["bound_levels"]) if "bound_levels" in z.files else 2)
        self.meta = json.loads(str(z["meta"])) if "meta" in z.files else {}
        self.path = str(path)
        return self

    def describe(self):
        """Where the weights came from (the training arguments in their meta)."""
        a = getattr(self, "meta", {}).get("args", {})
        if not a:
            return getattr(self, "path", "in-memory weights")
        n = a.get("samples")
        size = str(n) if n else "%s-%s" % (a.get("samples_min"), a.get("samples_max"))
        return "%s (trained on %s random CSG scenes of %s samples, the last held back for the thresholds)" % (
            Path(getattr(self, "path", "")).name, a.get("scenes"), size)

    def save(self, path, **extra):
        np.savez(path, weights=self.weights, mean=self.mean, inv_std=self.inv_std,
                 sign_threshold=np.float32(self.sign_threshold), band_threshold=np.float32(self.band_threshold),
                 dilation=np.int32(self.dilation), bound_levels=np.int32(self.bound_levels), **extra)

    def view(self):
        v = tsr_pruner()
        v.weights = self.weights.ctypes.data_as(_P)
        for i in range(MLP_FEATURES):
            v.feature_mean[i] = float(self.mean[i])
            v.feature_inv_std[i] = float(self.inv_std[i])
        v.sign_threshold = self.sign_threshold
        v.band_threshold = self.band_threshold
        v.dilation = self.dilation
        v.bound_levels = self.bound_levels
        self._keep = self.weights   # the C side reads the weights during the call
        return v


def version():
    return lib.tsr_version().decode()


def set_iteration_limits(max_sampling_waves=0, max_rounds=0):
    """Bounds of the tree build's conflict waves (device) and rounds (host);
    0 restores the defaults.  A build that reaches one fails with
    TSR_ERR_TIMEOUT."""
    lib.tsr_set_iteration_limits(int(max_sampling_waves), int(max_rounds))


def kernel_launches():
    """This library's kernel launches so far in the process."""
    return int(lib.tsr_kernel_launches())
