"""Incremental field updates and sample erasure through the C ABI
(Occupancy::addSamples / eraseSamples, Occupancy.cpp:129-136 and
Occupancy.h:167-175, 222-227; Tree::eraseSamples, Nodes.cpp:644-671).

* Removing a set of samples and adding it back restores the sums, lengths
  and cone count (FP64 accumulation: to 1e-9 of the largest value) and the
  occupancy signs.
* Removing every sample empties the sums, and node flags stay set (removal
  keeps them, like the reference).
* A field updated by removals equals the plain field of the tree's remaining
  links (the removed samples' camera links cut) in everything the node flags
  do not touch: SAMPLENESS sums and lengths, the cone count, and EMPTINESS
  sums and lengths on the leaves the reduced field flags.  Elsewhere the
  updated field keeps EMPTINESS kernels that the kept flags still admit,
  exactly as the reference, whose removal leaves flags set.
* Erasing samples from the tree keeps every node's samples contiguous and
  compacts them in order."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SUM_TOL = 1e-9          # of the largest |value| of the field
E_RTOL = 2e-4           # EMPTINESS sums where FP32 leaf centres may differ
E_OUTLIER_FRAC = 1e-3   # leaves allowed outside E_RTOL


@pytest.fixture(scope="module")
def built():
    from tsr_b200 import core, scenes
    sc = scenes.csg_scene(n_target=30000, width=320, height=240, f=250.0, n_cams=24)
    s = core.Samples.from_scene(sc)
    tree = core.Tree(s)          # reorders s into tree order
    return sc, s, tree, core.Cameras(sc.cams)


FIELDS = ("emptiness_sum", "sampleness_sum", "emptiness_length", "sampleness_length")


def _close(a, b):
    scale = max(np.abs(a).max(), np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() <= SUM_TOL * scale


def test_remove_then_add_restores_the_field(built):
    from tsr_b200 import core
    _, s, tree, cams = built
    occ = core.Occupancy(tree, cams)
    before = {f: occ.field(f).copy() for f in FIELDS}
    cc0, o0 = occ.field("cone_count"), occ.getOccupancy().copy()
    chosen = np.arange(0, s.count, 7, dtype=np.uint32)
    occ.eraseSamples(chosen, cams)
    assert occ.field("cone_count") < cc0
    occ.addSamples(chosen, cams)
    for f in FIELDS:
        assert _close(occ.field(f), before[f]), f
    assert abs(occ.field("cone_count") - cc0) <= SUM_TOL * cc0
    agree = np.mean((occ.getOccupancy() > 0) == (o0 > 0))
    assert agree >= 0.999


def test_removing_every_sample_empties_the_sums(built):
    from tsr_b200 import core
    _, s, tree, cams = built
    occ = core.Occupancy(tree, cams)
    flags = occ.getNodeStates().copy()
    scale = {f: np.abs(occ.field(f)).max() for f in FIELDS}
    occ.eraseSamples(np.arange(s.count, dtype=np.uint32), cams)
    for f in FIELDS:
        assert np.abs(occ.field(f)).max() <= SUM_TOL * scale[f], f
    assert abs(occ.field("cone_count")) <= 1e-9 * s.count
    np.testing.assert_array_equal(occ.getNodeStates(), flags)
    assert np.all(occ.getOccupancy() == -1e-6)


def test_removal_equals_field_without_those_links(built):
    from tsr_b200 import core
    sc, s, tree, cams = built
    chosen = np.arange(3, s.count, 5, dtype=np.uint32)
    occ = core.Occupancy(tree, cams)
    occ.eraseSamples(chosen, cams)
    # the same tree's field with the chosen samples' camera links cut: built
    # from the input order (camera links do not change the tree)
    cut = core.Samples.from_scene(sc)
    inputs = np.nonzero(np.isin(tree.getPermutation(), chosen))[0]
    cut.camera_links[inputs] = 0xFFFFFFFF
    tree2 = core.Tree(cut, reorder_samples=False)
    ref = core.Occupancy(tree2, cams)
    np.testing.assert_array_equal(tree2.getNodes().children, tree.getNodes().children)
    for f in ("sampleness_sum", "sampleness_length"):
        assert _close(occ.field(f), ref.field(f)), f
    # a traversal that meets more flagged siblings reaches a leaf by another
    # route, so its FP32 leaf centre may differ in the last bits: FP32-level
    # tolerance here, with rare flips of kernels sitting on EPSILON allowed
    flagged = (ref.getNodeStates()[tree.getLeaves().node_index] & 1) != 0
    for f in ("emptiness_sum", "emptiness_length"):
        a, b = occ.field(f)[flagged], ref.field(f)[flagged]
        bad = np.abs(a - b) > E_RTOL * np.maximum(np.abs(a), np.abs(b)) + 1e-6 * np.abs(b).max()
        assert bad.mean() <= E_OUTLIER_FRAC, (f, bad.mean())
    assert abs(occ.field("cone_count") - ref.field("cone_count")) <= SUM_TOL * ref.field("cone_count")


def test_tree_erase_samples_compacts(built):
    from tsr_b200 import core
    sc, _, _, cams = built
    s = core.Samples.from_scene(sc)
    tree = core.Tree(s)
    n0 = s.count
    nodes0 = tree.getNodes()
    counts0 = nodes0.samples_per_node.copy()
    inl = np.ones(n0, bool)
    inl[::4] = False
    tree.eraseSamples(inl)
    nodes = tree.getNodes()
    kept = int(inl.sum())
    assert int(nodes.samples_per_node.sum()) == kept
    # per node: count minus the erased samples of its old range
    starts0 = nodes0.sample_start_indices
    erased_before = np.concatenate([[0], np.cumsum(~inl)])
    exp_counts = counts0 - (erased_before[starts0 + counts0] - erased_before[starts0])
    np.testing.assert_array_equal(nodes.samples_per_node, exp_counts)
    np.testing.assert_array_equal(nodes.sample_start_indices, starts0 - erased_before[starts0])
    # the compacted samples are the kept ones, in order
    pos = np.zeros((kept, 3))
    core._check(core.lib.tsr_tree_copy_samples(tree.handle, core._ptr(pos), None, None, None, None))
    np.testing.assert_array_equal(pos, s.positions[inl])
    perm = tree.getPermutation()
    assert perm.shape[0] == n0 and (perm == 0xFFFFFFFF).sum() == n0 - kept
