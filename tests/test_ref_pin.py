"""The CPU restatement (oracle/) pinned to the reference's own code.

tests/golden/ref_*.npz hold what the reference's Scene/Tree and
SurfaceExtraction sources compute (built unmodified against the BaseProject
shim, run on one thread; tests/golden/make_ref_golden.py).  The restatement
must reproduce every array bit for bit: node arrays (Nodes.cpp:186-636),
the sample permutation, leaf scopes, node->leaf links and the neighbour CSR
(Leaves.cpp:22-180), dual cells (DualCells.cpp:21-357), the FP64 occupancy
field (Occupancy.cpp:105-587) and the raw DMC mesh
(DualMarchingCells.cpp:41-169).  Where the reference build is present
(oracle/_ref), more seeded scenes are compared live.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tsr_b200 import scenes

GOLDEN = Path(__file__).resolve().parent / "golden"
FIXTURES = sorted(p.stem for p in GOLDEN.glob("ref_*.npz") if not p.stem.startswith("ref_update"))
INVALID = 0xFFFFFFFF


def _scene(g):
    return scenes.Scene(g["in_pos"], g["in_nrm"], g["in_scale"], g["in_conf"], g["in_links"], g["in_cams"], "ref")


def restatement(scene):
    o = Oracle(scene).build_tree()
    o.occupancy(nthreads=1)
    m = o.dmc()
    out = dict(o.nodes())
    out["permutation"] = o.permutation()
    out.update(o.leaves())
    out["dual_cells"] = o.dual_cells()
    out.update({"field_" + k: np.asarray(v) for k, v in o.fields().items()})
    out.update(vpos=m["vpos"], vscale=m["vscale"], tris=m["tris"])
    return out


KEYS = ["children", "parents", "counts", "starts", "permutation", "scopes", "node_idx", "node_to_leaf",
        "nb_offsets", "nbs", "dual_cells", "field_e_sum", "field_s_sum", "field_e_len", "field_s_len",
        "field_prior", "field_states", "field_cone_count", "field_occ", "vpos", "vscale", "tris"]


def assert_same(ref, mine, label):
    for k in KEYS:
        a, b = np.asarray(ref[k]), np.asarray(mine[k])
        assert a.shape == b.shape, (label, k, a.shape, b.shape)
        np.testing.assert_array_equal(b, a, err_msg="%s: %s" % (label, k))


@pytest.mark.parametrize("name", FIXTURES)
def test_restatement_matches_reference_fixture(name):
    g = np.load(GOLDEN / (name + ".npz"))
    assert_same(g, restatement(_scene(g)), name)


def test_fixtures_cover_multi_link_and_cluttered_scenes():
    k3 = np.load(GOLDEN / "ref_sphere_k3.npz")
    assert k3["in_links"].shape[1] == 3 and (k3["in_links"] == INVALID).any()
    cl = np.load(GOLDEN / "ref_cluttered_2k.npz")
    assert cl["in_conf"].min() < 0.5 < cl["in_conf"].max()


def test_golden_fixtures_are_the_reference_outputs():
    """The oracle-made golden fixtures of the two small scenes equal the
    reference's outputs on the same inputs."""
    pairs = {"sphere_small": "ref_sphere_small", "csg_3k": "ref_csg_3k"}
    for gold, ref in pairs.items():
        g, r = np.load(GOLDEN / (gold + ".npz")), np.load(GOLDEN / (ref + ".npz"))
        np.testing.assert_array_equal(g["in_pos"], r["in_pos"])
        for gk, rk in [("nodes_children", "children"), ("nodes_parents", "parents"), ("nodes_counts", "counts"),
                       ("nodes_starts", "starts"), ("permutation", "permutation"), ("leaves_scopes", "scopes"),
                       ("leaves_nbs", "nbs"), ("dual_cells", "dual_cells"), ("field_occ", "field_occ"),
                       ("field_prior", "field_prior"), ("mesh_vpos", "vpos"), ("mesh_tris", "tris")]:
            np.testing.assert_array_equal(g[gk], r[rk], err_msg="%s %s" % (gold, gk))


def _live_scenes():
    rng = np.random.default_rng(5)
    sc = scenes.csg_scene(seed=9, n_target=2500, width=200, height=150, f=160.0, n_cams=16)
    n = sc.n
    links = np.stack([sc.links[:, 0], np.where(rng.random(n) < 0.5, (sc.links[:, 0] + 3) % 16, INVALID)], 1)
    k2 = scenes.Scene(sc.pos, sc.nrm, sc.scale, sc.conf, np.ascontiguousarray(links, np.uint32), sc.cams, "k2")
    rc = scenes.random_csg_scene(seed=31, n_target=2500, width=200, height=150, f=160.0)
    return {"csg_k2": k2, "random_csg_31": rc}


@pytest.mark.parametrize("name", ["csg_k2", "random_csg_31"])
def test_restatement_matches_live_reference(name):
    from oracle import refpy
    if not refpy.available():
        pytest.skip("reference build (oracle/_ref) not present")
    sc = _live_scenes()[name]
    r = refpy.run(sc, threads=1)
    ref = {k: v for k, v in r.items() if k != "fields"}
    ref.update({"field_" + k: np.asarray(v) for k, v in r["fields"].items()})
    assert_same(ref, restatement(sc), name)


def test_restatement_update_matches_reference():
    """Occupancy::eraseSamples then addSamples (Occupancy.h:167-175,
    Occupancy.cpp:129-136) of 10 % of the samples: the restatement's update
    reproduces the reference's fields bit for bit after each."""
    g = np.load(GOLDEN / "ref_update_csg_3k.npz")
    o = Oracle(_scene(g)).build_tree()
    o.occupancy(nthreads=1)
    for step, removal in (("erased", True), ("added", False)):
        f = o.update(g["chosen"], removal, nthreads=1).fields()
        for k in ("e_sum", "s_sum", "e_len", "s_len", "prior", "occ", "states", "cone_count"):
            np.testing.assert_array_equal(np.asarray(f[k]), g[step + "_" + k], err_msg="%s %s" % (step, k))
