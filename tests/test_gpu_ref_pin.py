"""GPU parity against the reference's own outputs (tests/golden/ref_*.npz,
made by the reference's Scene/Tree and SurfaceExtraction sources built
against the BaseProject shim; tests/golden/make_ref_golden.py).

* Tree: node arrays, sample permutation, leaf scopes, node->leaf links,
  neighbour CSR and dual cells bit for bit (K = 1 and K = 3 links with
  invalid and repeated slots, a cluttered capture with outliers).
* Field: the FP32-kernel / FP64-sum field against the reference's FP64 field
  within the tolerances below, every sign flip counted.
* DMC: the reference's own field loaded into the GPU library
  (tsr_occupancy_load) gives the reference's raw mesh bit for bit.

Set TSR_PARITY_LOG to a file name to append the measured errors as JSON lines.
"""
from pathlib import Path

import numpy as np
import pytest
from fieldcheck import OUTLIER_FRAC, field_stats, log

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
FIXTURES = sorted(p.stem for p in GOLDEN.glob("ref_*.npz") if not p.stem.startswith("ref_update"))


def _scene_of(g):
    from tsr_b200 import scenes
    return scenes.Scene(g["in_pos"], g["in_nrm"], g["in_scale"], g["in_conf"], g["in_links"], g["in_cams"], "ref")


def _load(name):
    from tsr_b200 import core
    g = np.load(GOLDEN / (name + ".npz"))
    sc = _scene_of(g)
    t = core.Tree(core.Samples.from_scene(sc))
    return g, sc, t


@pytest.mark.parametrize("name", FIXTURES)
def test_gpu_tree_matches_reference(name):
    g, sc, t = _load(name)
    n = t.getNodes()
    np.testing.assert_array_equal(n.children, g["children"])
    np.testing.assert_array_equal(n.parents, g["parents"])
    np.testing.assert_array_equal(n.samples_per_node, g["counts"])
    np.testing.assert_array_equal(n.sample_start_indices, g["starts"])
    np.testing.assert_array_equal(t.getPermutation(), g["permutation"])
    lv = t.getLeaves()
    np.testing.assert_array_equal(lv.scopes, g["scopes"])
    np.testing.assert_array_equal(lv.node_index, g["node_idx"])
    np.testing.assert_array_equal(lv.node_to_leaf_links, g["node_to_leaf"])
    np.testing.assert_array_equal(lv.neighbors_offsets, g["nb_offsets"])
    np.testing.assert_array_equal(lv.neighbors, g["nbs"])
    np.testing.assert_array_equal(t.getDualCells(), g["dual_cells"])


@pytest.mark.parametrize("name", FIXTURES)
def test_gpu_field_matches_reference(name):
    from tsr_b200 import core
    g, sc, t = _load(name)
    occ = core.Occupancy(t, core.Cameras(sc.cams))
    ref = {k[6:]: g[k] for k in g.files if k.startswith("field_")}
    s = field_stats(ref, occ, t.counts["leaves"])
    log({"test": "field_vs_reference", "fixture": name, **s})
    L = t.counts["leaves"]
    allowed = max(2, int(OUTLIER_FRAC * L))
    for k in ("emptiness_sum", "sampleness_sum", "emptiness_length", "sampleness_length"):
        assert s[k]["outside"] <= allowed, (k, s[k])
    assert s["prior_emptiness"]["outside"] == 0, s["prior_emptiness"]
    assert s["prior_emptiness"]["nan_mismatch"] <= allowed, s["prior_emptiness"]
    assert s["cone_count_rel"] < 1e-12
    assert s["sign_flip_count"] <= allowed, s["sign_flips"]
    assert int((occ.getNodeStates() != g["field_states"]).sum()) <= allowed


@pytest.mark.parametrize("name", FIXTURES)
def test_gpu_dmc_on_reference_field(name, tmp_path):
    """The reference's own FP64 field, loaded into the library, gives the
    reference's raw DMC mesh bit for bit (vertex positions and scales in
    first-use order, triangles)."""
    from tsr_b200 import core, files
    g, sc, t = _load(name)
    fields = {k: g["field_" + k] for k in ("e_len", "e_sum", "s_len", "s_sum", "prior", "states")}
    fields["cone_count"] = float(g["field_cone_count"])
    path = str(tmp_path / "ref.occupancy")
    files.write_occupancy(path, fields)
    occ = core.Occupancy.fromFile(t, path)
    np.testing.assert_array_equal(occ.getOccupancy(), g["field_occ"])
    m = occ.extractCrust()
    np.testing.assert_array_equal(m.positions, g["vpos"])
    np.testing.assert_array_equal(m.scales, g["vscale"])
    np.testing.assert_array_equal(m.triangles, g["tris"])


def test_gpu_update_matches_reference():
    """tsr_occupancy_update against the reference's Occupancy::eraseSamples
    and then addSamples of 10 % of the samples (tree-order indices): the
    updated field within the same tolerances as a fresh one."""
    from tsr_b200 import core
    g = np.load(GOLDEN / "ref_update_csg_3k.npz")
    sc = _scene_of(g)
    t = core.Tree(core.Samples.from_scene(sc))
    cams = core.Cameras(sc.cams)
    occ = core.Occupancy(t, cams)
    allowed = max(2, int(OUTLIER_FRAC * t.counts["leaves"]))
    for step, removal in (("erased", True), ("added", False)):
        if removal:
            occ.eraseSamples(g["chosen"], cams)
        else:
            occ.addSamples(g["chosen"], cams)
        ref = {k[len(step) + 1:]: g[k] for k in g.files if k.startswith(step + "_")}
        s = field_stats(ref, occ, t.counts["leaves"])
        log({"test": "update_vs_reference", "step": step, **s})
        for k in ("emptiness_sum", "sampleness_sum", "emptiness_length", "sampleness_length"):
            assert s[k]["outside"] <= allowed, (step, k, s[k])
        assert s["prior_emptiness"]["outside"] == 0, (step, s["prior_emptiness"])
        assert s["sign_flip_count"] <= allowed, (step, s["sign_flips"])
        assert s["cone_count_rel"] < 1e-12
