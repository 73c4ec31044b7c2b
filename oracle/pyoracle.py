"""ctypes wrapper of the FP64 CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product package never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = _HERE / "lib" / "libtsr_oracle.so"
_lib = None

DEFAULT_PARAMS = (2.0, 2.0, 100.0, 25.0, 1.0)   # App.cfg:64-70


def build():
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not _LIB.exists():
            build()
        L = ctypes.CDLL(str(_LIB))
        P = ctypes.c_void_p
        L.tsro_create.restype = P
        L.tsro_create.argtypes = [ctypes.c_uint32, ctypes.c_uint32, P, P, P, P, P, ctypes.c_uint32, P, P]
        L.tsro_free.argtypes = [P]
        L.tsro_build_tree.argtypes = [P, ctypes.c_int]
        L.tsro_counts.argtypes = [P, P]
        L.tsro_root.argtypes = [P, P]
        L.tsro_get_nodes.argtypes = [P, P, P, P, P]
        L.tsro_get_permutation.argtypes = [P, P]
        L.tsro_get_leaves.argtypes = [P, P, P, P, P, P]
        L.tsro_get_dual_cells.argtypes = [P, P]
        L.tsro_get_sample_depths.argtypes = [P, P]
        L.tsro_occupancy.argtypes = [P, ctypes.c_int, ctypes.c_int]
        L.tsro_occupancy_links.argtypes = [P, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64]
        L.tsro_occupancy_update.argtypes = [P, ctypes.c_int, P, ctypes.c_uint32, ctypes.c_int]
        L.tsro_get_occupancy.argtypes = [P, P, P, P, P, P, P, P, P]
        L.tsro_dmc.argtypes = [P]
        L.tsro_set_occupancy.argtypes = [P, P]
        L.tsro_get_mesh.argtypes = [P, P, P, P, P, P]
        L.tsro_stage_seconds.restype = ctypes.c_double
        L.tsro_stage_seconds.argtypes = [P, ctypes.c_int]
        L.tsro_mesh_postprocess.restype = P
        L.tsro_mesh_postprocess.argtypes = [ctypes.c_uint32, P, P, ctypes.c_uint32, P, ctypes.c_uint32]
        L.tsro_mesh_free.argtypes = [P]
        L.tsro_mesh_counts.argtypes = [P, P]
        L.tsro_mesh_get.argtypes = [P, P, P, P, P]
        L.tsro_depth_triangulate.restype = P
        L.tsro_depth_triangulate.argtypes = [P, ctypes.c_uint32, ctypes.c_uint32, P, P, P, P, P]
        L.tsro_mesh_colors.argtypes = [P, P]
        L.tsro_border_rings.restype = ctypes.c_uint32
        L.tsro_border_rings.argtypes = [ctypes.c_uint32, P, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class Oracle:
    """The reference pipeline on the CPU in FP64 for one scene."""

    def __init__(self, scene, params=DEFAULT_PARAMS):
        L = lib()
        self._keep = [np.ascontiguousarray(scene.pos, np.float64), np.ascontiguousarray(scene.nrm, np.float64),
                      np.ascontiguousarray(scene.scale, np.float64), np.ascontiguousarray(scene.conf, np.float64),
                      np.ascontiguousarray(scene.links, np.uint32), np.ascontiguousarray(scene.cams, np.float64),
                      np.ascontiguousarray(params, np.float64)]
        k = self._keep
        self.n = scene.n
        self.k = scene.k
        self.h = L.tsro_create(self.n, self.k, _p(k[0]), _p(k[1]), _p(k[2]), _p(k[3]), _p(k[4]),
                               k[5].shape[0], _p(k[5]), _p(k[6]))

    def __del__(self):
        if getattr(self, "h", None):
            lib().tsro_free(self.h)
            self.h = None

    def build_tree(self, stop_after=0):
        rc = lib().tsro_build_tree(self.h, stop_after)
        if rc != 0:
            raise RuntimeError("oracle tree build failed")
        return self

    def counts(self):
        c = np.zeros(10, np.uint64)
        lib().tsro_counts(self.h, _p(c))
        keys = ["nodes", "leaves", "cells", "nbs", "verts", "tris", "writers", "sampling_splits",
                "rounds", "max_contagion"]
        return {k: int(v) for k, v in zip(keys, c)}

    def root(self):
        r = np.zeros(4)
        lib().tsro_root(self.h, _p(r))
        return r

    def nodes(self):
        n = self.counts()["nodes"]
        out = [np.zeros(n, np.uint32) for _ in range(4)]
        lib().tsro_get_nodes(self.h, *[_p(a) for a in out])
        return dict(zip(["children", "parents", "counts", "starts"], out))

    def permutation(self):
        t = np.zeros(self.n, np.uint32)
        lib().tsro_get_permutation(self.h, _p(t))
        return t

    def leaves(self):
        c = self.counts()
        L, Nn, E = c["leaves"], c["nodes"], c["nbs"]
        ms = np.zeros((L, 4)); ni = np.zeros(L, np.uint32); n2l = np.zeros(Nn, np.uint32)
        off = np.zeros(L + 1, np.uint32); nbs = np.zeros(E, np.uint32)
        lib().tsro_get_leaves(self.h, _p(ms), _p(ni), _p(n2l), _p(off), _p(nbs))
        return dict(scopes=ms, node_idx=ni, node_to_leaf=n2l, nb_offsets=off, nbs=nbs)

    def dual_cells(self):
        nc = self.counts()["cells"]
        c = np.zeros((nc, 8), np.uint32)
        lib().tsro_get_dual_cells(self.h, _p(c))
        return c

    def sample_depths(self):
        d = np.zeros(self.n, np.uint32)
        lib().tsro_get_sample_depths(self.h, _p(d))
        return d

    def occupancy(self, nthreads=0, prune=True):
        if lib().tsro_occupancy(self.h, nthreads, 1 if prune else 0) != 0:
            raise RuntimeError("oracle occupancy failed")
        return self

    def occupancy_links(self, first, count, nthreads=0):
        if lib().tsro_occupancy_links(self.h, nthreads, first, count) != 0:
            raise RuntimeError("oracle occupancy failed")
        return self

    def update(self, samples, removal, nthreads=1):
        """Occupancy::addSamples / eraseSamples of tree-order sample indices."""
        idx = np.ascontiguousarray(samples, np.uint32)
        if lib().tsro_occupancy_update(self.h, nthreads, _p(idx), idx.shape[0], 1 if removal else 0) != 0:
            raise RuntimeError("oracle update failed")
        return self

    def fields(self):
        c = self.counts()
        L = c["leaves"]
        a = [np.zeros(L) for _ in range(6)]
        st = np.zeros(c["nodes"], np.uint32)
        cc = np.zeros(1)
        lib().tsro_get_occupancy(self.h, *[_p(x) for x in a], _p(st), _p(cc))
        d = dict(zip(["e_sum", "s_sum", "e_len", "s_len", "prior", "occ"], a))
        d["states"] = st
        d["cone_count"] = float(cc[0])
        return d

    def set_occupancy(self, occ):
        occ = np.ascontiguousarray(occ, np.float64)
        assert occ.shape[0] == self.counts()["leaves"]
        lib().tsro_set_occupancy(self.h, _p(occ))
        return self

    def dmc(self):
        if lib().tsro_dmc(self.h) != 0:
            raise RuntimeError("oracle dmc failed")
        c = self.counts()
        cases = np.zeros(c["cells"], np.uint8)
        vpos = np.zeros((c["verts"], 3)); vs = np.zeros(c["verts"]); vk = np.zeros((c["verts"], 2), np.uint32)
        tris = np.zeros((c["tris"], 3), np.uint32)
        lib().tsro_get_mesh(self.h, _p(cases), _p(vpos), _p(vs), _p(vk), _p(tris))
        return dict(cases=cases, vpos=vpos, vscale=vs, vkeys=vk, tris=tris)

    def stage_seconds(self):
        names = ["containment", "sampling", "balance", "reorder", "leaves", "dual_cells",
                 "sampleness", "emptiness", "priors", "dmc"]
        return {n: lib().tsro_stage_seconds(self.h, i) for i, n in enumerate(names)}


MESH_COUNT_KEYS = ("vertices", "triangles", "error", "isle_vertices", "isle_triangles", "border_edges", "holes",
                   "hole_vertices", "hole_triangles", "skipped_rings")


def mesh_postprocess(positions, triangles, scales=None, min_isle_size=1000):
    """The post-processing of DualMarchingCells (isles, holes, normals) on
    the CPU; returns (counts, positions, normals, scales, triangles)."""
    L = lib()
    pos = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
    tri = np.ascontiguousarray(triangles, np.uint32).reshape(-1, 3)
    sc = None if scales is None else np.ascontiguousarray(scales, np.float64)
    h = L.tsro_mesh_postprocess(pos.shape[0], _p(pos), _p(sc), tri.shape[0], _p(tri), min_isle_size)
    try:
        c = np.zeros(len(MESH_COUNT_KEYS), np.uint64)
        L.tsro_mesh_counts(h, _p(c))
        counts = {k: int(v) for k, v in zip(MESH_COUNT_KEYS, c)}
        nv, nt = counts["vertices"], counts["triangles"]
        p, n, s = np.zeros((nv, 3)), np.zeros((nv, 3)), np.zeros(nv)
        t = np.zeros((nt, 3), np.uint32)
        L.tsro_mesh_get(h, _p(p), _p(n), _p(s), _p(t))
    finally:
        L.tsro_mesh_free(h)
    return counts, p, n, s, t


def border_rings(edges):
    """FlexibleMesh::findBorderRings on (tail, head) edges in list order;
    returns the rings as lists of tail vertices."""
    e = np.ascontiguousarray(edges, np.uint32).reshape(-1, 2)
    nb = e.shape[0]
    verts = np.zeros(max(nb, 1), np.uint32)
    lens = np.zeros(max(nb, 1), np.uint32)
    n = lib().tsro_border_rings(nb, _p(e), _p(verts), _p(lens))
    out, k = [], 0
    for r in range(n):
        out.append([int(x) for x in verts[k:k + lens[r]]])
        k += int(lens[r])
    return out


def depth_triangulate(depths, hps_to_ray_vs, hps_to_ray_ws, center, colors=None):
    """DepthImage::triangulate on the CPU: a depth map (H x W, along the
    rays), the two 3x3 matrices (row vector times matrix) and the centre of
    projection.  Returns dict positions, normals, scales, colors, triangles,
    pixel_to_vertex (H x W)."""
    L = lib()
    d = np.ascontiguousarray(depths, np.float64)
    H, W = d.shape
    mvs = np.ascontiguousarray(hps_to_ray_vs, np.float64).reshape(9)
    mws = np.ascontiguousarray(hps_to_ray_ws, np.float64).reshape(9)
    c = np.ascontiguousarray(center, np.float64).reshape(3)
    col = None if colors is None else np.ascontiguousarray(colors, np.float64).reshape(H * W * 3)
    pix = np.zeros((H, W), np.uint32)
    h = L.tsro_depth_triangulate(_p(d), W, H, _p(mvs), _p(mws), _p(c), _p(col), _p(pix))
    try:
        cnt = np.zeros(len(MESH_COUNT_KEYS), np.uint64)
        L.tsro_mesh_counts(h, _p(cnt))
        nv, nt = int(cnt[0]), int(cnt[1])
        p, n, s = np.zeros((nv, 3)), np.zeros((nv, 3)), np.zeros(nv)
        t = np.zeros((nt, 3), np.uint32)
        L.tsro_mesh_get(h, _p(p), _p(n), _p(s), _p(t))
        cols = np.zeros((nv, 3))
        L.tsro_mesh_colors(h, _p(cols))
    finally:
        L.tsro_mesh_free(h)
    return dict(positions=p, normals=n, scales=s, colors=cols, triangles=t, pixel_to_vertex=pix)
