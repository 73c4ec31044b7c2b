"""The pruned field with the committed trained network, compared with the plain
method on a scene the network never saw (random CSG scene, seed 500).

What the network gains over the method without it: the prior queries of
the leaves it places away from a sign change are skipped (fewer tree nodes
classified), while the mesh stays the plain method's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Every skipped leaf's sign is certified or fixed by E == 0 / S == 0, and every
# skipped leaf on a sign change is queried after all: the mesh is the plain
# field's, case codes and vertices alike.
MIN_CASE_AGREEMENT = 1.0          # DMC case codes equal to the plain field's
MAX_HAUSDORFF_LEAVES = 0.0        # vertex Hausdorff distance, in finest leaf sizes
MIN_PRIOR_WORK_SAVED = 0.4        # fraction of prior-query node visits removed
MIN_EMPTINESS_NEEDED = 0.9        # share of the EMPTINESS kernel sum inside a queried leaf's prior sphere


@pytest.fixture(scope="module")
def heldout():
    from tsr_b200 import core, scenes
    sc = scenes.random_csg_scene(seed=500, n_target=200_000, width=480, height=360, f=400.0)
    tree = core.Tree(core.Samples.from_scene(sc), reorder_samples=False)
    return tree, core.Cameras(sc.cams)


def test_pruned_field_matches_plain_mesh_with_less_work(heldout):
    from tsr_b200 import core, pruner
    tree, cams = heldout
    from fieldcheck import log
    j = pruner.compare_with_plain(tree, cams, core.Pruner.load())
    saved = 1.0 - j["visited"]["visited_priors"][1] / j["visited"]["visited_priors"][0]
    log({"test": "pruner_vs_plain", "prior_work_saved": saved, **j})
    assert j["case_agreement"] >= MIN_CASE_AGREEMENT, j
    assert j["vertex_hausdorff"] <= MAX_HAUSDORFF_LEAVES * j["finest_leaf_size"], j
    assert saved >= MIN_PRIOR_WORK_SAVED, j
    # the cone passes are not pruned: same work as the plain field
    assert j["visited"]["visited_sampleness"][0] == j["visited"]["visited_sampleness"][1]


def test_pruned_field_keeps_exact_values_where_queried(heldout):
    from tsr_b200 import core
    tree, cams = heldout
    plain = core.Occupancy(tree, cams)
    pruned = core.Occupancy(tree, cams, pruner=core.Pruner.load())
    pp, pq = plain.getPriorForEmptiness(), pruned.getPriorForEmptiness()
    queried = ~np.isnan(pq)
    assert queried.sum() > 0 and (~queried).sum() == pruned.counts["pruned_leaves"]
    np.testing.assert_allclose(pq[queried], pp[queried], rtol=0, atol=1e-12)
    oq, op = pruned.getOccupancy(), plain.getOccupancy()
    # the FP64 atomic sums may round differently from run to run
    np.testing.assert_allclose(oq[queried], op[queried], rtol=1e-9, atol=1e-15)
    # the cone passes are the plain field's in the pruned field
    np.testing.assert_allclose(pruned.field("emptiness_sum"), plain.field("emptiness_sum"), rtol=1e-12, atol=0)


def test_pruned_field_is_exact_on_a_cluttered_scene():
    """Outliers and varying confidences make small blobs the network never saw
    in clean training scenes; a sign it gets wrong there is not certified, so
    the leaf is queried, and the mesh stays the plain field's."""
    from fieldcheck import log
    from tsr_b200 import core, pruner, scenes
    sc = scenes.cluttered_scene(seed=4, n_target=150_000, width=384, height=216, f=280.0, n_cams=60)
    tree = core.Tree(core.Samples.from_scene(sc), reorder_samples=False)
    j = pruner.compare_with_plain(tree, core.Cameras(sc.cams), core.Pruner.load())
    log({"test": "pruner_vs_plain_cluttered", **j})
    assert j["sign_agreement"] == 1.0, j
    assert j["case_agreement"] == 1.0, j
    assert j["vertex_hausdorff"] == 0.0, j
    assert j["pruned_leaves"] > 0, j


def test_emptiness_pass_is_needed_by_the_queried_priors(heldout):
    """Why the pruned field keeps the EMPTINESS pass exact: almost every leaf
    that receives EMPTINESS kernels lies inside the prior sphere (25 leaf
    sizes) of a leaf whose prior the pruned field still queries, so its cone
    lengths enter an exact prior -- skipping its cone contributions would
    change a queried leaf's value.  Measured share logged; asserted high."""
    from fieldcheck import log
    from tsr_b200 import core, pruner
    tree, cams = heldout
    plain = core.Occupancy(tree, cams)
    pruned = core.Occupancy(tree, cams, pruner=core.Pruner.load())
    f = pruner.emptiness_needed_fraction(tree, plain, pruned)
    log({"test": "emptiness_needed", **f})
    assert f["kernel_sum"] >= MIN_EMPTINESS_NEEDED, f


def test_network_against_certifying_every_leaf(heldout):
    """What the network adds over the sign certificates alone: the same
    pruned field with the network's band prediction switched off (every
    reliable leaf gets a bounds query).  Both meshes are the plain field's;
    the prior-query work of both is logged beside the plain field's."""
    from fieldcheck import log
    from tsr_b200 import core, pruner
    tree, cams = heldout
    net = core.Pruner.load()
    alone = core.Pruner.load()
    alone.band_threshold = 0.999999
    alone.sign_threshold = 0.4999
    jn = pruner.compare_with_plain(tree, cams, net)
    ja = pruner.compare_with_plain(tree, cams, alone)
    log({"test": "network_vs_certify_all", "network": jn["visited"]["visited_priors"],
         "certify_all": ja["visited"]["visited_priors"], "pruned": [jn["pruned_leaves"], ja["pruned_leaves"]]})
    for j in (jn, ja):
        assert j["case_agreement"] == 1.0 and j["vertex_hausdorff"] == 0.0, j
