"""The tree, field and samples files in numpy: reader and writer of the
same bodies the library's tsr_tree_save / tsr_occupancy_save /
tsr_tree_save_samples write and tsr_tree_load / tsr_occupancy_load read.

Bodies follow the reference's savers with Real = double, little endian:
Nodes::saveToFile (Nodes.cpp:789-807), Leaves::saveToFile (Leaves.cpp:
261-292), DualCells::saveToFile (DualCells.cpp:378-385),
Occupancy::saveToFile (Occupancy.cpp:722-766) and Samples::saveToFile
(Samples.cpp:733-765); file endings from FileNaming.cpp:21-29.  Each file
starts with a 16-byte header in place of the reference's BaseProject File
header: b"TSRF", u32 format 1, u32 FILE_VERSION 0, u32 kind.
"""
from __future__ import annotations

import os

import numpy as np

MAGIC = b"TSRF"
FORMAT = 1
FILE_VERSION = 0
KIND_NODES, KIND_LEAVES, KIND_DUAL_CELLS, KIND_OCCUPANCY, KIND_SAMPLES = 1, 2, 3, 4, 5
ENDING_NODES, ENDING_LEAVES, ENDING_DUAL_CELLS = ".nodes", ".leaves", ".dualCells"
ENDING_OCCUPANCY, ENDING_OCTREE, ENDING_SAMPLES = ".occupancy", ".octree", ".samples"

# Scope.h:36-38 with Real = double: Vector3 min, Real size, uint32 node,
# padded to 8-byte alignment
SCOPE = np.dtype([("min", "<f8", (3,)), ("size", "<f8"), ("node", "<u4"), ("pad", "<u4")])
assert SCOPE.itemsize == 40


class FileFormatError(ValueError):
    """A file of another kind or version, truncated, or with trailing data
    (the reference throws FileCorruptionException)."""


def _header(kind):
    return MAGIC + np.array([FORMAT, FILE_VERSION, kind], "<u4").tobytes()


class _Reader:
    def __init__(self, path, kind):
        self.path = os.fspath(path)
        with open(self.path, "rb") as f:
            self.buf = f.read()
        self.pos = 0
        if self.take(4, np.uint8).tobytes() != MAGIC or list(self.take(3, "<u4")) != [FORMAT, FILE_VERSION, kind]:
            raise FileFormatError("not a file of the expected kind and version: %s" % self.path)

    def take(self, count, dtype):
        dt = np.dtype(dtype)
        end = self.pos + int(count) * dt.itemsize
        if end > len(self.buf):
            raise FileFormatError("truncated file %s" % self.path)
        a = np.frombuffer(self.buf, dt, int(count), self.pos).copy()
        self.pos = end
        return a

    def done(self):
        if self.pos != len(self.buf):
            raise FileFormatError("trailing data in %s" % self.path)


def _write(path, kind, parts):
    with open(os.fspath(path), "wb") as f:
        f.write(_header(kind))
        for p in parts:
            f.write(np.ascontiguousarray(p).tobytes())


def write_tree(prefix, nodes, leaves, dual_cells):
    """nodes: dict children, parents, counts, starts (uint32 per node);
    leaves: dict scopes (L x 4: min xyz, size), node_idx, node_to_leaf,
    nb_offsets, nbs; dual_cells: (cells x 8) leaf indices."""
    prefix = os.fspath(prefix)
    n = np.asarray(nodes["children"]).shape[0]
    _write(prefix + ENDING_NODES, KIND_NODES,
           [np.array([n], "<u4")] + [np.asarray(nodes[k], "<u4") for k in ("children", "parents", "counts", "starts")])
    sc = np.asarray(leaves["scopes"], np.float64)
    rec = np.zeros(sc.shape[0], SCOPE)
    rec["min"] = sc[:, :3]
    rec["size"] = sc[:, 3]
    rec["node"] = leaves["node_idx"]
    nbs = np.asarray(leaves["nbs"], "<u4")
    _write(prefix + ENDING_LEAVES, KIND_LEAVES,
           [np.array([n, sc.shape[0], nbs.shape[0]], "<u4"), np.asarray(leaves["node_to_leaf"], "<u4"), rec,
            np.asarray(leaves["nb_offsets"], "<u4"), nbs])
    cells = np.asarray(dual_cells, "<u4").reshape(-1)
    _write(prefix + ENDING_DUAL_CELLS, KIND_DUAL_CELLS, [np.array([cells.shape[0]], "<u4"), cells])


def read_tree(prefix):
    """(nodes, leaves, dual_cells) in the layout write_tree takes."""
    prefix = os.fspath(prefix)
    r = _Reader(prefix + ENDING_NODES, KIND_NODES)
    n = int(r.take(1, "<u4")[0])
    nodes = {k: r.take(n, "<u4") for k in ("children", "parents", "counts", "starts")}
    r.done()
    r = _Reader(prefix + ENDING_LEAVES, KIND_LEAVES)
    nn, nl, ne = (int(x) for x in r.take(3, "<u4"))
    if nn != n:
        raise FileFormatError("leaves file of another tree: %s" % r.path)
    n2l = r.take(nn, "<u4")
    rec = r.take(nl, SCOPE)
    off = r.take(nl + 1, "<u4")
    nbs = r.take(ne, "<u4")
    r.done()
    leaves = dict(scopes=np.concatenate([rec["min"], rec["size"][:, None]], 1), node_idx=rec["node"].copy(),
                  node_to_leaf=n2l, nb_offsets=off, nbs=nbs)
    r = _Reader(prefix + ENDING_DUAL_CELLS, KIND_DUAL_CELLS)
    ic = int(r.take(1, "<u4")[0])
    if ic % 8:
        raise FileFormatError("dual cell indices not a multiple of 8 in %s" % r.path)
    cells = r.take(ic, "<u4").reshape(-1, 8)
    r.done()
    return nodes, leaves, cells


OCC_FIELDS = ("e_len", "e_sum", "s_len", "s_sum", "prior")


def write_occupancy(path, fields):
    """fields: dict e_len, e_sum, s_len, s_sum, prior (f64 per leaf), states
    (u32 per node), cone_count."""
    nl = np.asarray(fields["e_sum"]).shape[0]
    st = np.asarray(fields["states"], "<u4")
    _write(path, KIND_OCCUPANCY, [np.array([nl, st.shape[0]], "<u4")] +
           [np.asarray(fields[k], "<f8") for k in OCC_FIELDS] + [st, np.array([fields["cone_count"]], "<f8")])


def read_occupancy(path):
    r = _Reader(path, KIND_OCCUPANCY)
    nl, nn = (int(x) for x in r.take(2, "<u4"))
    d = {k: r.take(nl, "<f8") for k in OCC_FIELDS}
    d["states"] = r.take(nn, "<u4")
    d["cone_count"] = float(r.take(1, "<f8")[0])
    r.done()
    return d


def samples_aabb(positions, scales, h_svo=2.0):
    """Samples::computeAABB (Samples.cpp:290-298, 442-449): min and max of
    every sample's box position +- (scale h_SVO + EPSILON); 2 x 3."""
    p = np.asarray(positions, np.float64)
    r = (np.asarray(scales, np.float64) * h_svo + 1e-6)[:, None]
    return np.stack([(p - r).min(0), (p + r).max(0)])


def write_samples(path, positions, normals, scales, confidences, camera_links, aabb, colors=None):
    """The .samples body; camera_links is (count x K), aabb 2 x 3."""
    n = np.asarray(positions).shape[0]
    links = np.asarray(camera_links, "<u4").reshape(n, -1)
    col = np.zeros((n, 3)) if colors is None else np.asarray(colors, "<f8")
    _write(path, KIND_SAMPLES, [np.array([n, links.shape[1]], "<u4"), np.asarray(aabb, "<f8").reshape(6), col,
                                np.asarray(normals, "<f8"), np.asarray(positions, "<f8"),
                                np.asarray(confidences, "<f8"), np.asarray(scales, "<f8"), links])


def read_samples(path):
    """dict positions, normals, scales, confidences, camera_links (n x K),
    colors, aabb (2 x 3)."""
    r = _Reader(path, KIND_SAMPLES)
    n, k = (int(x) for x in r.take(2, "<u4"))
    d = {"aabb": r.take(6, "<f8").reshape(2, 3)}
    for key in ("colors", "normals", "positions"):
        d[key] = r.take(3 * n, "<f8").reshape(n, 3)
    d["confidences"] = r.take(n, "<f8")
    d["scales"] = r.take(n, "<f8")
    d["camera_links"] = r.take(n * k, "<u4").reshape(n, k)
    r.done()
    return d
