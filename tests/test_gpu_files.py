"""Tree, samples and field files through the C ABI on the GPU.

Bit-exact: the files the library writes for a GPU-built tree equal, byte for
byte, the numpy writer's files of the oracle's golden tree and samples; a
tree loaded from files equals the saved one in every array; a field loaded
from a file equals the saved one in every array, occupancy included (the
same kernel on the same inputs), and gives the same mesh.  Tolerance only
where two
different computations meet: a field computed afresh on a loaded tree
against the field of the built tree (FP64 atomic sums in another order:
relative 1e-12), and the GPU occupancy of the oracle's golden field against
the oracle's own (the GPU may fuse a multiply-add: relative 1e-12, signs
identical).
"""
import numpy as np
import pytest

from tsr_b200 import files

from test_files import _golden, golden_field, golden_tree, tree_order_samples

pytestmark = pytest.mark.gpu

SUM_RTOL = 1e-12        # FP64 atomic sums accumulated in another order
OCC_RTOL = 1e-12        # the golden field's occupancy, GPU formula vs oracle


def _samples_from_golden(g):
    from tsr_b200 import core
    return core.Samples(g["in_pos"].copy(), g["in_nrm"].copy(), g["in_scale"].copy(), g["in_conf"].copy(),
                        g["in_links"].copy())


def _tree_arrays(t):
    n, l = t.getNodes(), t.getLeaves()
    return dict(children=n.children, parents=n.parents, counts=n.samples_per_node, starts=n.sample_start_indices,
                scopes=l.scopes, node_idx=l.node_index, node_to_leaf=l.node_to_leaf_links,
                nb_offsets=l.neighbors_offsets, nbs=l.neighbors, cells=t.getDualCells(), root=t.getRootScope())


def _assert_same_tree(a, b):
    a, b = _tree_arrays(a), _tree_arrays(b)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def _assert_same_mesh(m1, m2):
    np.testing.assert_array_equal(m1.cases, m2.cases)
    np.testing.assert_array_equal(m1.edge_keys, m2.edge_keys)
    np.testing.assert_array_equal(m1.positions, m2.positions)
    np.testing.assert_array_equal(m1.triangles, m2.triangles)


FIELD_NAMES = ("emptiness_sum", "sampleness_sum", "emptiness_length", "sampleness_length", "prior_emptiness",
               "occupancy", "node_states")


@pytest.mark.parametrize("name", ["sphere_small", "csg_3k"])
def test_saved_files_equal_golden_files(name, tmp_path):
    """GPU build -> tsr_tree_save / tsr_tree_save_samples give the bytes the
    numpy writer gives for the oracle's tree and tree-ordered samples."""
    from tsr_b200 import core
    g = _golden(name)
    t = core.Tree(_samples_from_golden(g))
    t.saveToFiles(str(tmp_path / "gpu"))
    colors = np.random.default_rng(2).random((t.sample_count, 3))
    t.saveSamples(str(tmp_path / "gpu.samples"), colors)
    files.write_tree(tmp_path / "gold", *golden_tree(g))
    s = tree_order_samples(g)
    files.write_samples(tmp_path / "gold.samples", s.positions, s.normals, s.scales, s.confidences,
                        s.camera_links, files.samples_aabb(s.positions, s.scales), colors)
    for end in (files.ENDING_NODES, files.ENDING_LEAVES, files.ENDING_DUAL_CELLS, files.ENDING_SAMPLES):
        assert (tmp_path / ("gpu" + end)).read_bytes() == (tmp_path / ("gold" + end)).read_bytes(), end


@pytest.mark.parametrize("name", ["sphere_small", "csg_3k"])
def test_golden_files_load_and_give_golden_mesh(name, tmp_path):
    """The oracle's tree and field written by the numpy writer load through
    the C ABI; the loaded field's mesh is the oracle's mesh."""
    from tsr_b200 import core
    g = _golden(name)
    files.write_tree(tmp_path / "gold", *golden_tree(g))
    files.write_occupancy(tmp_path / "gold.occupancy", golden_field(g))
    s = tree_order_samples(g)
    t = core.Tree.fromFiles(str(tmp_path / "gold"), s)
    arr = _tree_arrays(t)
    np.testing.assert_array_equal(arr["root"], g["root"])
    for k in ("children", "parents", "counts", "starts"):
        np.testing.assert_array_equal(arr[k], g["nodes_" + k], err_msg=k)
    for k in ("scopes", "node_idx", "node_to_leaf", "nb_offsets", "nbs"):
        np.testing.assert_array_equal(arr[k], g["leaves_" + k], err_msg=k)
    np.testing.assert_array_equal(arr["cells"], g["dual_cells"])
    np.testing.assert_array_equal(t.getPermutation(), np.arange(s.count, dtype=np.uint32))
    o = core.Occupancy.fromFile(t, str(tmp_path / "gold.occupancy"))
    for name_, key in [("emptiness_sum", "e_sum"), ("sampleness_sum", "s_sum"), ("emptiness_length", "e_len"),
                       ("sampleness_length", "s_len"), ("prior_emptiness", "prior"), ("node_states", "states")]:
        np.testing.assert_array_equal(o.field(name_), g["field_" + key], err_msg=name_)
    occ, gold = o.getOccupancy(), g["field_occ"]
    np.testing.assert_array_equal(occ > 0, gold > 0)
    np.testing.assert_allclose(occ, gold, rtol=OCC_RTOL, atol=0)
    m = o.extractCrust()
    np.testing.assert_array_equal(m.cases, g["mesh_cases"])
    np.testing.assert_array_equal(m.edge_keys, g["mesh_vkeys"])
    np.testing.assert_array_equal(m.triangles, g["mesh_tris"])
    np.testing.assert_allclose(m.positions, g["mesh_vpos"], rtol=0, atol=1e-12 * g["root"][3])


def _samples_from_file(path):
    from tsr_b200 import core
    d = files.read_samples(path)
    return core.Samples(d["positions"], d["normals"], d["scales"], d["confidences"], d["camera_links"]), d["aabb"]


def _round_trip(scene, tmp_path):
    """Save tree, samples and field; resume from the three files alone."""
    from tsr_b200 import core
    s = core.Samples.from_scene(scene)
    t = core.Tree(s)                       # reorders s into tree order
    cams = core.Cameras(scene.cams)
    o = core.Occupancy(t, cams)
    t.saveToFiles(str(tmp_path / "t"))
    t.saveSamples(str(tmp_path / "t.samples"))
    o.saveToFile(str(tmp_path / "t.occupancy"))
    s2, aabb = _samples_from_file(tmp_path / "t.samples")
    np.testing.assert_array_equal(s2.positions, s.positions)
    np.testing.assert_array_equal(s2.camera_links, s.camera_links)
    t2 = core.Tree.fromFiles(str(tmp_path / "t"), s2, aabb=aabb)
    _assert_same_tree(t, t2)
    _assert_same_tree(t, core.Tree.fromFiles(str(tmp_path / "t"), s2))   # AABB recomputed from the samples
    # the saved field, read back: every array identical, the same mesh
    o2 = core.Occupancy.fromFile(t2, str(tmp_path / "t.occupancy"))
    for f in FIELD_NAMES:
        np.testing.assert_array_equal(o2.field(f), o.field(f), err_msg=f)
    assert o2.field("cone_count") == o.field("cone_count")
    _assert_same_mesh(o.extractCrust(), o2.extractCrust())
    # the numpy reader sees the same field
    d = files.read_occupancy(tmp_path / "t.occupancy")
    np.testing.assert_array_equal(d["e_sum"], o.field("emptiness_sum"))
    np.testing.assert_array_equal(d["s_len"], o.field("sampleness_length"))
    np.testing.assert_array_equal(d["states"], o.field("node_states"))
    assert d["cone_count"] == o.field("cone_count")
    # a field computed afresh on the loaded tree
    o3 = core.Occupancy(t2, cams)
    for f in ("emptiness_sum", "sampleness_sum", "emptiness_length", "sampleness_length"):
        a, b = o3.field(f), o.field(f)
        np.testing.assert_allclose(a, b, rtol=SUM_RTOL, atol=SUM_RTOL * np.abs(b).max(), err_msg=f)
    np.testing.assert_array_equal(o3.field("node_states"), o.field("node_states"))
    flips = int(((o3.getOccupancy() > 0) != (o.getOccupancy() > 0)).sum())
    assert flips <= 2, flips
    return t, o


def test_round_trip_csg(csg_small, tmp_path):
    _round_trip(csg_small, tmp_path)


def test_round_trip_one_million_samples(tmp_path):
    """The csg1m workload: save and load are exact at full size too."""
    from tsr_b200 import scenes
    _round_trip(scenes.csg_scene(seed=0, n_target=1_000_000), tmp_path)


def test_round_trip_after_erasing_samples(csg_small, tmp_path):
    """A tree whose samples were erased keeps the build's AABB, which its
    samples file carries; tree and samples files reload the same tree."""
    from tsr_b200 import core
    s = core.Samples.from_scene(csg_small)
    t = core.Tree(s)
    keep = np.random.default_rng(5).random(s.count) > 0.2
    t.eraseSamples(keep)
    t.saveToFiles(str(tmp_path / "e"))
    t.saveSamples(str(tmp_path / "e.samples"))
    s2, aabb = _samples_from_file(tmp_path / "e.samples")
    assert s2.count == int(keep.sum())
    np.testing.assert_array_equal(aabb, files.samples_aabb(s.positions, s.scales))
    t2 = core.Tree.fromFiles(str(tmp_path / "e"), s2, aabb=aabb)
    _assert_same_tree(t, t2)


def test_file_errors(csg_small, tiny_scene, tmp_path):
    from tsr_b200 import core
    s = core.Samples.from_scene(csg_small)
    t = core.Tree(s)
    cams = core.Cameras(csg_small.cams)
    # a pruned field skipped prior queries: the format cannot hold it
    pruned = core.Occupancy(t, cams, pruner=core.Pruner.load())
    if pruned.counts["pruned_leaves"]:
        with pytest.raises(core.TsrError) as e:
            pruned.saveToFile(str(tmp_path / "p.occupancy"))
        assert core.STATUS[e.value.status] == "TSR_ERR_STATE"
    # a field file of another tree
    other = core.Tree(core.Samples.from_scene(tiny_scene))
    core.Occupancy(other, core.Cameras(tiny_scene.cams)).saveToFile(str(tmp_path / "o.occupancy"))
    with pytest.raises(core.TsrError, match="another tree"):
        core.Occupancy.fromFile(t, str(tmp_path / "o.occupancy"))
    # a truncated field file
    o = core.Occupancy(t, cams)
    o.saveToFile(str(tmp_path / "f.occupancy"))
    body = (tmp_path / "f.occupancy").read_bytes()
    (tmp_path / "f.occupancy").write_bytes(body[:-8])
    with pytest.raises(core.TsrError, match="truncated"):
        core.Occupancy.fromFile(t, str(tmp_path / "f.occupancy"))
    # a tree file set loaded over other samples
    t.saveToFiles(str(tmp_path / "t"))
    with pytest.raises(core.TsrError):
        core.Tree.fromFiles(str(tmp_path / "t"), core.Samples.from_scene(tiny_scene))
    # an unwritable path
    with pytest.raises(core.TsrError, match="cannot create"):
        t.saveToFiles(str(tmp_path / "missing_dir" / "t"))
