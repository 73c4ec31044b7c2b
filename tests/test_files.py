"""CPU tests of the tree and field files.

The numpy reader/writer (tsr_b200.files) round-trips the golden fixtures'
trees and fields bit for bit and rejects files of another kind, truncated
files and trailing data.  The library's tsr_tree_load validates a file set
completely on the host before it touches the GPU, so its rejections of
damaged files, of other samples and of a wrong AABB run here too (no
GPU call is reached; a valid file set is loaded only in the GPU tests).
"""
import ctypes
import shutil
from pathlib import Path

import numpy as np
import pytest

from tsr_b200 import files

GOLDEN = Path(__file__).resolve().parent / "golden"


def _golden(name):
    return dict(np.load(GOLDEN / (name + ".npz")))


def golden_tree(g):
    nodes = {k: g["nodes_" + k] for k in ("children", "parents", "counts", "starts")}
    leaves = {k: g["leaves_" + k] for k in ("scopes", "node_idx", "node_to_leaf", "nb_offsets", "nbs")}
    return nodes, leaves, g["dual_cells"]


def golden_field(g):
    d = {k: g["field_" + k] for k in ("e_len", "e_sum", "s_len", "s_sum", "prior", "states")}
    d["cone_count"] = float(g["field_cone_count"])
    return d


def tree_order_samples(g):
    """The fixture's input samples in the order the tree leaves them in."""
    from tsr_b200 import core
    perm = g["permutation"].astype(np.int64)
    out = []
    for k in ("in_pos", "in_nrm", "in_scale", "in_conf", "in_links"):
        a = np.empty_like(g[k])
        a[perm] = g[k]
        out.append(a)
    return core.Samples(*out)


@pytest.mark.parametrize("name", ["sphere_small", "csg_3k"])
def test_tree_files_round_trip(name, tmp_path):
    g = _golden(name)
    nodes, leaves, cells = golden_tree(g)
    files.write_tree(tmp_path / "t", nodes, leaves, cells)
    n2, l2, c2 = files.read_tree(tmp_path / "t")
    for k in nodes:
        np.testing.assert_array_equal(n2[k], nodes[k])
    for k in leaves:
        np.testing.assert_array_equal(l2[k], leaves[k])
    np.testing.assert_array_equal(c2, cells)
    # sizes: 16-byte header + the reference's body
    n, nl, ne = nodes["children"].shape[0], leaves["scopes"].shape[0], leaves["nbs"].shape[0]
    assert (tmp_path / "t.nodes").stat().st_size == 16 + 4 + 16 * n
    assert (tmp_path / "t.leaves").stat().st_size == 16 + 12 + 4 * n + 40 * nl + 4 * (nl + 1) + 4 * ne
    assert (tmp_path / "t.dualCells").stat().st_size == 16 + 4 + 32 * cells.shape[0]


@pytest.mark.parametrize("name", ["sphere_small", "csg_3k"])
def test_occupancy_file_round_trip(name, tmp_path):
    g = _golden(name)
    f = golden_field(g)
    files.write_occupancy(tmp_path / "f.occupancy", f)
    f2 = files.read_occupancy(tmp_path / "f.occupancy")
    for k in f:
        np.testing.assert_array_equal(f2[k], f[k])
    nl, nn = f["e_sum"].shape[0], f["states"].shape[0]
    assert (tmp_path / "f.occupancy").stat().st_size == 16 + 8 + 40 * nl + 4 * nn + 8


def test_reader_rejects_damaged_files(tmp_path):
    g = _golden("sphere_small")
    files.write_tree(tmp_path / "t", *golden_tree(g))
    files.write_occupancy(tmp_path / "f", golden_field(g))
    with pytest.raises(files.FileFormatError, match="expected kind"):
        files.read_occupancy(tmp_path / "t.nodes")
    body = (tmp_path / "t.leaves").read_bytes()
    (tmp_path / "t.leaves").write_bytes(body[:-4])
    with pytest.raises(files.FileFormatError, match="truncated"):
        files.read_tree(tmp_path / "t")
    (tmp_path / "t.leaves").write_bytes(body + b"\0")
    with pytest.raises(files.FileFormatError, match="trailing"):
        files.read_tree(tmp_path / "t")
    (tmp_path / "f").write_bytes(b"XSRF" + (tmp_path / "f").read_bytes()[4:])
    with pytest.raises(files.FileFormatError, match="expected kind"):
        files.read_occupancy(tmp_path / "f")


def _load_status(prefix, samples, aabb=None):
    from tsr_b200 import core
    h = ctypes.c_void_p()
    v = samples.view()
    bb = None if aabb is None else np.ascontiguousarray(aabb, np.float64)
    rc = core.lib.tsr_tree_load(str(prefix).encode(), ctypes.byref(v),
                                bb.ctypes.data_as(ctypes.c_void_p) if bb is not None else None, None, None,
                                ctypes.byref(h))
    assert not h.value, "a rejected load returned a tree"
    return core.STATUS[rc], core.lib.tsr_last_error_message().decode()


def _damaged(tmp_path, tag, edit):
    """A copy of the golden file set with one array changed by `edit`."""
    g = _golden("sphere_small")
    nodes, leaves, cells = golden_tree(g)
    nodes = {k: v.copy() for k, v in nodes.items()}
    leaves = {k: v.copy() for k, v in leaves.items()}
    cells = cells.copy()
    edit(nodes, leaves, cells)
    files.write_tree(tmp_path / tag, nodes, leaves, cells)
    return tmp_path / tag


def test_library_rejects_damaged_tree_files(tmp_path):
    g = _golden("sphere_small")
    s = tree_order_samples(g)
    assert _load_status(tmp_path / "missing", s) == ("TSR_ERR_INVALID_ARG", "cannot open " + str(tmp_path / "missing.nodes"))

    def child_out_of_range(n, l, c):
        i = int(np.flatnonzero(n["children"] != 0xFFFFFFFF)[-1])
        n["children"][i] = n["children"].shape[0] - 4

    def wrong_parent(n, l, c):
        n["parents"][9] = 2

    def sample_range(n, l, c):
        i = int(np.flatnonzero(n["counts"])[-1])
        n["starts"][i] = s.count - n["counts"][i] + 1

    def neighbour_range(n, l, c):
        l["nbs"][0] = l["scopes"].shape[0]

    def cell_range(n, l, c):
        c[0, 0] = l["scopes"].shape[0]

    def scope_moved(n, l, c):
        l["scopes"][5, 0] = np.nextafter(l["scopes"][5, 0], np.inf)

    def leaf_link(n, l, c):
        l["node_idx"][3] = l["node_idx"][4]

    cases = [(child_out_of_range, "child block"), (wrong_parent, "parent"), (sample_range, "samples lie outside"),
             (neighbour_range, "neighbour out of range"), (cell_range, "dual cells file"),
             (scope_moved, "scopes do not match"), (leaf_link, "scope and node links")]
    for edit, msg in cases:
        st, text = _load_status(_damaged(tmp_path, edit.__name__, edit), s)
        assert st == "TSR_ERR_INVALID_ARG" and msg in text, (edit.__name__, st, text)

    good = _damaged(tmp_path, "good", lambda n, l, c: None)
    for end in (files.ENDING_NODES, files.ENDING_LEAVES, files.ENDING_DUAL_CELLS):
        p = Path(str(good) + end)
        body = p.read_bytes()
        p.write_bytes(body[:-1])
        assert _load_status(good, s)[0] == "TSR_ERR_INVALID_ARG"
        p.write_bytes(body + b"\0\0\0\0")
        assert "trailing data" in _load_status(good, s)[1]
        p.write_bytes(body)
    # a leaves file read as a nodes file
    shutil.copy(str(good) + files.ENDING_LEAVES, str(tmp_path / "swapped.nodes"))
    for end in (files.ENDING_LEAVES, files.ENDING_DUAL_CELLS):
        shutil.copy(str(good) + end, str(tmp_path / "swapped") + end)
    assert "expected kind" in _load_status(tmp_path / "swapped", s)[1]


def test_library_rejects_other_samples_and_aabbs(tmp_path):
    from tsr_b200 import core
    g = _golden("sphere_small")
    prefix = _damaged(tmp_path, "t", lambda n, l, c: None)
    s = tree_order_samples(g)
    # another sample count
    fewer = core.Samples(s.positions[:-1], s.normals[:-1], s.scales[:-1], s.confidences[:-1], s.camera_links[:-1])
    st, text = _load_status(prefix, fewer)
    assert st == "TSR_ERR_INVALID_ARG" and ("another sample count" in text or "samples lie outside" in text), text
    # samples whose bounds give another root scope
    moved = core.Samples(s.positions.copy(), s.normals, s.scales, s.confidences, s.camera_links)
    moved.positions[0] += 10.0   # outside the others' bounds
    assert "scopes do not match" in _load_status(prefix, moved)[1]
    # an explicit AABB: the samples' own passes every check up to the first
    # device allocation; one ulp off on the largest extent moves the scopes
    bb = files.samples_aabb(s.positions, s.scales)
    ext = bb[1] - bb[0]
    j = int(np.argmax(ext))
    off = bb.copy()
    off[1, j] = np.nextafter(off[1, j], np.inf)
    assert "scopes do not match" in _load_status(prefix, s, off)[1]
    assert "finite" in _load_status(prefix, s, np.array([[0.0, 0.0, np.nan], [1.0, 1.0, 1.0]]))[1]
    assert "min <= max" in _load_status(prefix, s, np.array([[0.0, 0.0, 1.0], [1.0, 1.0, 0.0]]))[1]


def test_library_rejects_bad_arguments(tmp_path):
    from tsr_b200 import core
    h = ctypes.c_void_p()
    assert core.STATUS[core.lib.tsr_tree_load(b"", None, None, None, None, ctypes.byref(h))] == "TSR_ERR_INVALID_ARG"
    assert core.STATUS[core.lib.tsr_tree_save(None, b"x")] == "TSR_ERR_INVALID_ARG"
    assert core.STATUS[core.lib.tsr_occupancy_save(None, b"x")] == "TSR_ERR_INVALID_ARG"
    assert core.STATUS[core.lib.tsr_occupancy_load(None, b"x", None, None, ctypes.byref(h))] == "TSR_ERR_INVALID_ARG"


@pytest.mark.parametrize("name", ["sphere_small", "csg_3k"])
def test_samples_file_round_trip(name, tmp_path):
    g = _golden(name)
    s = tree_order_samples(g)
    bb = files.samples_aabb(s.positions, s.scales)
    # the AABB gives the golden root scope exactly as Tree::getRootScope does
    size = (bb[1] - bb[0]).max()
    np.testing.assert_array_equal(np.append((bb[0] + bb[1]) * 0.5 - size * 0.5, size), g["root"])
    colors = np.random.default_rng(1).random((s.count, 3))
    files.write_samples(tmp_path / "s.samples", s.positions, s.normals, s.scales, s.confidences, s.camera_links,
                        bb, colors)
    d = files.read_samples(tmp_path / "s.samples")
    np.testing.assert_array_equal(d["aabb"], bb)
    np.testing.assert_array_equal(d["colors"], colors)
    for k, v in (("positions", s.positions), ("normals", s.normals), ("scales", s.scales),
                 ("confidences", s.confidences), ("camera_links", s.camera_links)):
        np.testing.assert_array_equal(d[k], v)
    k = s.camera_links.shape[1]
    assert (tmp_path / "s.samples").stat().st_size == 16 + 8 + 48 + s.count * (72 + 16 + 4 * k)


def test_mesh_and_depth_arguments_rejected_on_the_host():
    """tsr_mesh_create and tsr_depth_triangulate check their arguments before
    any device work."""
    import ctypes
    from tsr_b200 import core
    h = ctypes.c_void_p()
    pos = np.zeros((3, 3))
    bad = np.array([[0, 1, 3]], np.uint32)
    rc = core.lib.tsr_mesh_create(core._ptr(pos), None, 3, core._ptr(bad), 1, None, ctypes.byref(h))
    assert core.STATUS[rc] == "TSR_ERR_INVALID_ARG" and "out of range" in core.lib.tsr_last_error_message().decode()
    assert not h.value
    rc = core.lib.tsr_mesh_create(None, None, 3, None, 0, None, ctypes.byref(h))
    assert core.STATUS[rc] == "TSR_ERR_INVALID_ARG"
    m = np.eye(3)
    c = np.zeros(3)
    d = np.ones((1, 5))
    rc = core.lib.tsr_depth_triangulate(core._ptr(d), 5, 1, core._ptr(m), core._ptr(m), core._ptr(c), None, None,
                                        ctypes.byref(h))
    assert core.STATUS[rc] == "TSR_ERR_INVALID_ARG" and "2 x 2" in core.lib.tsr_last_error_message().decode()
    rc = core.lib.tsr_depth_triangulate(None, 5, 5, core._ptr(m), core._ptr(m), core._ptr(c), None, None,
                                        ctypes.byref(h))
    assert core.STATUS[rc] == "TSR_ERR_INVALID_ARG"
    assert core.STATUS[core.lib.tsr_mesh_postprocess(None, 1, None)] == "TSR_ERR_INVALID_ARG"


class _FakeDepthMesh:
    def __init__(self, n, seed):
        rng = np.random.default_rng(seed)
        self.positions = rng.random((n, 3))
        self.normals = rng.random((n, 3))
        self.scales = rng.random(n) + 0.1
        self.colors = rng.random((n, 3))


def test_samples_from_depth_meshes():
    """Samples::addSamplesViaMeshes: concatenation, confidence 1, links of
    the reference camera or per-vertex lists padded to the largest K."""
    from tsr_b200 import core
    a, b = _FakeDepthMesh(4, 0), _FakeDepthMesh(3, 1)
    s = core.Samples.fromDepthMeshes([a, b], [7, np.array([[1, 2], [3, 4], [5, 6]])])
    assert s.count == 7 and s.max_cameras_per_sample == 2
    np.testing.assert_array_equal(s.positions, np.vstack([a.positions, b.positions]))
    np.testing.assert_array_equal(s.colors, np.vstack([a.colors, b.colors]))
    np.testing.assert_array_equal(s.confidences, 1.0)
    np.testing.assert_array_equal(s.camera_links[:4], [[7, 0xFFFFFFFF]] * 4)
    np.testing.assert_array_equal(s.camera_links[4:], [[1, 2], [3, 4], [5, 6]])
    a.scales[2] = 0.0
    with pytest.raises(ValueError, match="non-positive"):
        core.Samples.fromDepthMeshes([a], [0])


@pytest.mark.parametrize("ending", [files.ENDING_NODES, files.ENDING_LEAVES, files.ENDING_DUAL_CELLS])
def test_library_survives_byte_flips(ending, tmp_path):
    """Single flipped bytes anywhere in a file: the load either rejects the
    file set (TSR_ERR_INVALID_ARG) or, when every check still holds (a flip in
    a Scope record's padding, say), gets as far as the first device
    allocation; it never crashes."""
    import ctypes
    from tsr_b200 import core
    g = _golden("sphere_small")
    s = tree_order_samples(g)
    prefix = _damaged(tmp_path, "t", lambda n, l, c: None)
    path = Path(str(prefix) + ending)
    body = path.read_bytes()
    rng = np.random.default_rng(len(ending))
    outcomes = set()
    for pos in rng.integers(0, len(body), 40):
        damaged = bytearray(body)
        damaged[pos] ^= 1 << int(rng.integers(0, 8))
        path.write_bytes(bytes(damaged))
        h = ctypes.c_void_p()
        rc = core.lib.tsr_tree_load(str(prefix).encode(), ctypes.byref(s.view()), None, None, None, ctypes.byref(h))
        if h.value:   # a GPU machine loaded an equivalent tree
            core.lib.tsr_tree_free(h)
        outcomes.add(core.STATUS[rc])
    path.write_bytes(body)
    assert outcomes <= {"TSR_ERR_INVALID_ARG", "TSR_ERR_OOM", "TSR_ERR_CUDA", "TSR_OK"}
    assert "TSR_ERR_INVALID_ARG" in outcomes


def test_numpy_files_round_trip_random_shapes(tmp_path):
    """write/read of every kind with random sizes, including empty arrays."""
    rng = np.random.default_rng(9)
    for trial in range(6):
        nn, nl, ne, nc = (int(x) for x in rng.integers(0, 50, 4))
        nodes = {k: rng.integers(0, 2 ** 32, nn, dtype=np.uint64).astype(np.uint32)
                 for k in ("children", "parents", "counts", "starts")}
        leaves = dict(scopes=rng.standard_normal((nl, 4)), node_idx=rng.integers(0, 99, nl).astype(np.uint32),
                      node_to_leaf=rng.integers(0, 99, nn).astype(np.uint32),
                      nb_offsets=np.sort(rng.integers(0, 99, nl + 1)).astype(np.uint32),
                      nbs=rng.integers(0, 99, ne).astype(np.uint32))
        cells = rng.integers(0, 99, (nc, 8)).astype(np.uint32)
        files.write_tree(tmp_path / ("t%d" % trial), nodes, leaves, cells)
        n2, l2, c2 = files.read_tree(tmp_path / ("t%d" % trial))
        for k in nodes:
            np.testing.assert_array_equal(n2[k], nodes[k])
        for k in leaves:
            np.testing.assert_array_equal(l2[k], leaves[k])
        np.testing.assert_array_equal(c2, cells)
        fld = {k: rng.standard_normal(nl) for k in files.OCC_FIELDS}
        fld["states"] = rng.integers(0, 4, nn).astype(np.uint32)
        fld["cone_count"] = float(rng.random())
        files.write_occupancy(tmp_path / ("f%d" % trial), fld)
        f2 = files.read_occupancy(tmp_path / ("f%d" % trial))
        for k in fld:
            np.testing.assert_array_equal(f2[k], fld[k])
        k = int(rng.integers(1, 5))
        pos, nrm, col = (rng.standard_normal((nl, 3)) for _ in range(3))
        sc, cf = rng.random(nl), rng.random(nl)
        links = rng.integers(0, 2 ** 32, (nl, k), dtype=np.uint64).astype(np.uint32)
        aabb = rng.standard_normal((2, 3))
        files.write_samples(tmp_path / ("s%d" % trial), pos, nrm, sc, cf, links, aabb, col)
        d = files.read_samples(tmp_path / ("s%d" % trial))
        for key, v in (("positions", pos), ("normals", nrm), ("colors", col), ("scales", sc),
                       ("confidences", cf), ("camera_links", links), ("aabb", aabb)):
            np.testing.assert_array_equal(d[key], v)
