"""CPU tests of the FP64 oracle: golden fixtures, self-consistency and the
structural invariants the reference's debug checks assert (Nodes.cpp:809-855,
Leaves.cpp:134-137)."""
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tsr_b200 import scenes

GOLDEN = Path(__file__).resolve().parent / "golden"
INVALID = 0xFFFFFFFF


def _scene_from_golden(g):
    return scenes.Scene(g["in_pos"], g["in_nrm"], g["in_scale"], g["in_conf"], g["in_links"], g["in_cams"], "golden")


@pytest.mark.parametrize("name", ["sphere_small", "csg_3k"])
def test_oracle_matches_golden(name):
    sys.path.insert(0, str(GOLDEN))
    from make_golden import oracle_outputs
    g = np.load(GOLDEN / (name + ".npz"))
    out = oracle_outputs(_scene_from_golden(g))
    for k, v in out.items():
        ref = g[k]
        if k.startswith("field_") and k not in ("field_states", "field_cone_count"):
            np.testing.assert_allclose(v, ref, rtol=1e-9, atol=1e-12, equal_nan=True, err_msg=k)
        else:
            np.testing.assert_array_equal(v, ref, err_msg=k)


def test_golden_inputs_regenerate():
    """The fixture scenes are the seeded generators' output."""
    sys.path.insert(0, str(GOLDEN))
    from make_golden import fixture_scenes
    for name, sc in fixture_scenes().items():
        g = np.load(GOLDEN / (name + ".npz"))
        np.testing.assert_array_equal(sc.pos, g["in_pos"])
        np.testing.assert_array_equal(sc.links, g["in_links"])


def test_round_schedule_matches_sequential(tiny_scene):
    """The GPU's round-parallel schedule of the order-dependent sampling pass
    (Nodes.cpp:214-219) reproduces the sequential tree exactly."""
    a = Oracle(tiny_scene).build_tree(0)
    b = Oracle(tiny_scene).build_tree(4)
    na, nb = a.nodes(), b.nodes()
    for k in na:
        np.testing.assert_array_equal(na[k], nb[k])
    np.testing.assert_array_equal(a.permutation(), b.permutation())
    assert b.counts()["rounds"] > 1
    assert a.counts()["writers"] == b.counts()["writers"]


def test_round_schedule_csg(csg_small):
    a = Oracle(csg_small).build_tree(0)
    b = Oracle(csg_small).build_tree(4)
    np.testing.assert_array_equal(a.nodes()["children"], b.nodes()["children"])
    np.testing.assert_array_equal(a.dual_cells(), b.dual_cells())


def test_cone_pruning_cannot_change_sums():
    """addKernel re-tests leaf centres exactly (Occupancy.cpp:288-305), so the
    conservative cone/box pruning must give the same field as visiting every
    leaf under the depth cap."""
    sc = scenes.sphere_scene(stride=6, width=160, height=120, f=125.0)
    a = Oracle(sc).build_tree().occupancy(nthreads=1, prune=True).fields()
    b = Oracle(sc).build_tree().occupancy(nthreads=1, prune=False).fields()
    for k in ("e_sum", "s_sum", "e_len", "s_len", "prior", "occ"):
        np.testing.assert_allclose(a[k], b[k], rtol=1e-12, atol=0, equal_nan=True, err_msg=k)
    np.testing.assert_array_equal(a["states"], b["states"])


def _with_links(sc, links):
    return scenes.Scene(sc.pos, sc.nrm, sc.scale, sc.conf, np.ascontiguousarray(links, np.uint32), sc.cams,
                        sc.name)


def test_multiple_camera_links():
    """K > 1 (MVE captures link up to 5 cameras, Samples.h:311): link l is
    sample l / K, slot l % K (Occupancy.cpp:250-277), invalid slots
    (Cameras::INVALID_ID) add nothing, and a repeated link adds its kernels
    twice."""
    sc = scenes.sphere_scene(stride=8, width=160, height=120, f=125.0)
    one = Oracle(sc).build_tree().occupancy(nthreads=1).fields()
    pad = np.concatenate([sc.links, np.full_like(sc.links, INVALID), np.full_like(sc.links, INVALID)], 1)
    padded = Oracle(_with_links(sc, pad)).build_tree().occupancy(nthreads=1).fields()
    for k in ("e_sum", "s_sum", "e_len", "s_len", "prior", "occ"):
        np.testing.assert_array_equal(padded[k], one[k], err_msg=k)
    assert padded["cone_count"] == one["cone_count"]
    dup = np.concatenate([sc.links, sc.links], 1)
    twice = Oracle(_with_links(sc, dup)).build_tree().occupancy(nthreads=1).fields()
    for k in ("e_sum", "s_sum", "e_len", "s_len"):
        np.testing.assert_allclose(twice[k], 2 * one[k], rtol=1e-12, atol=1e-300, err_msg=k)
    assert twice["cone_count"] == pytest.approx(2 * one["cone_count"], rel=1e-12)
    np.testing.assert_allclose(twice["prior"], one["prior"], rtol=1e-12, equal_nan=True)
    # other cameras' links change the field
    other = np.concatenate([sc.links, (sc.links + 5) % sc.cams.shape[0]], 1)
    more = Oracle(_with_links(sc, other)).build_tree().occupancy(nthreads=1).fields()
    assert np.any(more["e_sum"] != one["e_sum"])


@pytest.fixture(scope="module")
def built(tiny_scene):
    o = Oracle(tiny_scene).build_tree()
    return o


def test_node_links_consistent(built):
    nd = built.nodes()
    ch, pa = nd["children"], nd["parents"]
    assert pa[0] == INVALID
    inner = np.nonzero(ch != INVALID)[0]
    for c in range(8):
        np.testing.assert_array_equal(pa[ch[inner] + c], inner)
    # every non-root node has exactly one parent block entry
    assert (ch != INVALID).sum() * 8 + 1 == ch.shape[0]


def test_block_dfs_layout(built):
    """Nodes::computeTargetIndices (Nodes.cpp:536-554): root 0, each inner
    node's children block allocated in depth-first order."""
    ch = built.nodes()["children"]
    nxt = [1]

    def walk(n):
        if ch[n] == INVALID:
            return
        assert ch[n] == nxt[0]
        nxt[0] += 8
        for c in range(8):
            walk(ch[n] + c)

    sys.setrecursionlimit(10000)
    walk(0)
    assert nxt[0] == ch.shape[0]


def test_samples_in_their_containers(built, tiny_scene):
    """Nodes::checkSamplesOrder (Nodes.cpp:830-855): each reordered sample
    lies in its container's sample range."""
    nd = built.nodes()
    counts, starts = nd["counts"], nd["starts"]
    assert counts.sum() == tiny_scene.n
    np.testing.assert_array_equal(starts, np.concatenate([[0], np.cumsum(counts)[:-1]]))
    perm = built.permutation()
    assert np.array_equal(np.sort(perm), np.arange(tiny_scene.n))


def test_leaf_partition_and_balance(built):
    lv = built.leaves()
    root = built.root()
    sizes = lv["scopes"][:, 3]
    assert np.isclose((sizes ** 3).sum(), root[3] ** 3, rtol=1e-9)
    # 2:1 face balance through the neighbour graph
    depth = np.round(np.log2(root[3] / sizes)).astype(int)
    off, nbs = lv["nb_offsets"], lv["nbs"]
    src = np.repeat(np.arange(len(sizes)), np.diff(off))
    assert np.abs(depth[src] - depth[nbs]).max() <= 1
    # symmetric adjacency
    pairs = set(zip(src.tolist(), nbs.tolist()))
    assert all((b, a) in pairs for a, b in pairs)


def test_dual_cells_reference_leaves(built):
    cells = built.dual_cells()
    L = built.counts()["leaves"]
    assert cells.max() < L
    assert cells.shape[0] > 0


def _mc_tables():
    import re
    src = (Path(__file__).resolve().parents[1] / "tsr_b200" / "csrc" / "mc_tables.h").read_text()

    def grab(name):
        body = re.search(r"#define " + name + r" ([^\n]*)", src.replace("\\\n", "")).group(1)
        return [int(v) for v in re.findall(r"-?\d+", body)]

    reorder = grab("TSR_MC_CORNER_REORDERING_INIT")
    ends = np.array(grab("TSR_MC_EDGE_ENDS_INIT")).reshape(12, 2)
    tri = np.array(grab("TSR_MC_TRIANGLES_INIT")).reshape(256, 16)
    return reorder, ends, tri


def test_mc_tables():
    reorder, ends, tri = _mc_tables()
    assert tri.shape == (256, 16)
    assert tri.max() <= 11 and tri.min() >= -1
    for code in (0, 255):
        assert tri[code, 0] == -1
    # every edge a case's triangles use is cut by that case
    for code in range(256):
        for e in tri[code][tri[code] >= 0]:
            a, b = ends[e]
            assert ((code >> a) ^ (code >> b)) & 1
    assert reorder == [0, 1, 5, 4, 2, 3, 7, 6]


def test_mesh_well_formed(tiny_scene):
    o = Oracle(tiny_scene).build_tree().occupancy(nthreads=2)
    m = o.dmc()
    t = m["tris"]
    assert t.shape[0] > 0
    assert t.max() < m["vpos"].shape[0]
    assert ((t[:, 0] != t[:, 1]) & (t[:, 1] != t[:, 2]) & (t[:, 0] != t[:, 2])).all()
    f = o.fields()
    occ = f["occ"]
    assert np.all((occ == -1e-6) | (occ > 0) | np.isnan(occ))
    pr = f["prior"][np.isfinite(f["prior"])]
    assert pr.min() >= 0 and pr.max() <= 1


def test_mesh_post_golden():
    """The post-processing restatement on the committed damaged mesh (holes,
    isles) reproduces its committed outputs."""
    sys.path.insert(0, str(GOLDEN))
    from make_golden import mesh_post_outputs
    g = dict(np.load(GOLDEN / "mesh_post.npz"))
    out = mesh_post_outputs(g)
    for k, v in out.items():
        if k == "post_nrm":
            np.testing.assert_allclose(v, g[k], rtol=0, atol=1e-12, err_msg=k)
        else:
            np.testing.assert_array_equal(v, g[k], err_msg=k)
    assert int(g["post_holes"]) > 100 and int(g["post_isle_vertices"]) > 0


def test_depth_golden():
    """The depth-map triangulation restatement reproduces its committed outputs."""
    sys.path.insert(0, str(GOLDEN))
    from make_golden import depth_inputs, depth_outputs
    g = dict(np.load(GOLDEN / "depth_small.npz"))
    fresh = depth_inputs()
    for k, v in fresh.items():
        np.testing.assert_array_equal(v, g[k], err_msg=k)
    out = depth_outputs(g)
    for k, v in out.items():
        if k == "depth_normals":
            np.testing.assert_allclose(v, g[k], rtol=0, atol=1e-12, err_msg=k)
        else:
            np.testing.assert_array_equal(v, g[k], err_msg=k)
