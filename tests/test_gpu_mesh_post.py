"""GPU mesh post-processing (tsr_mesh_postprocess) against the CPU restatement.

Bit-exact: element counts, every triangle, every vertex position (kept and
filled: the fill uses the reference's FP64 expression order with correctly
rounded operations on both sides) and every scale.  Tolerance: the vertex
normals, NORMAL_ATOL -- the GPU sums the angle-weighted triangle normals
with atomics in no fixed order and CUDA's acos may differ from the host's
in the last bits -- widened by the sum's condition number where the
weighted normals nearly cancel (check_normals): there the summation order
decides the direction, for the reference's OpenMP atomics as for the GPU.
The CPU restatement itself, fed the same triangles in another order,
differs at 10-17 such vertices of the golden damaged mesh.
"""
import numpy as np
import pytest

from oracle import pyoracle

from test_mesh_oracle import check_normals, uv_sphere

pytestmark = pytest.mark.gpu

NORMAL_ATOL = 1e-12
MIN_ISLE = 1000   # Scene::minimumTriangleIsleSize (App.cfg)


def _compare(mesh, positions, triangles, scales, min_isle):
    c, p, n, s, t = pyoracle.mesh_postprocess(positions, triangles, scales=scales, min_isle_size=min_isle)
    assert c["error"] == 0
    pc = mesh.post_counts
    for k in ("isle_vertices", "isle_triangles", "border_edges", "holes", "hole_vertices", "hole_triangles",
              "skipped_rings"):
        assert pc[k] == c[k], (k, pc[k], c[k])
    assert mesh.positions.shape[0] == c["vertices"] and mesh.triangles.shape[0] == c["triangles"]
    np.testing.assert_array_equal(mesh.triangles, t)
    np.testing.assert_array_equal(mesh.positions, p)
    np.testing.assert_array_equal(mesh.scales, s)
    check_normals(mesh.normals, n, p, t, NORMAL_ATOL)
    return c


@pytest.mark.parametrize("scene_name", ["tiny_scene", "csg_small"])
def test_dmc_crust_matches_oracle(scene_name, request):
    """extractCrust with the reference's post-processing on the field of a
    GPU-built tree, against the restatement run on the same raw mesh."""
    from tsr_b200 import core
    scene = request.getfixturevalue(scene_name)
    t = core.Tree(core.Samples.from_scene(scene))
    occ = core.Occupancy(t, core.Cameras(scene.cams))
    raw = occ.extractCrust()
    crust = occ.extractCrust(min_isle_size=MIN_ISLE)
    c = _compare(crust, raw.positions, raw.triangles, raw.scales, MIN_ISLE)
    np.testing.assert_array_equal(crust.cases, raw.cases)        # cases are not touched
    kept = c["vertices"] - c["hole_vertices"]
    assert np.all(crust.edge_keys[kept:] == 0xFFFFFFFF)


def test_one_million_sample_crust():
    """The csg1m workload: the crust of its field."""
    from tsr_b200 import core, scenes
    scene = scenes.csg_scene(seed=0, n_target=1_000_000)
    t = core.Tree(core.Samples.from_scene(scene))
    occ = core.Occupancy(t, core.Cameras(scene.cams))
    raw = occ.extractCrust()
    crust = occ.extractCrust(min_isle_size=MIN_ISLE)
    _compare(crust, raw.positions, raw.triangles, raw.scales, MIN_ISLE)


@pytest.mark.parametrize("seed", range(6))
def test_damaged_spheres(seed):
    """Random triangle deletions: many holes of every size, bow-tie borders,
    small isles cut loose."""
    from tsr_b200 import core
    rng = np.random.default_rng(seed)
    V, T = uv_sphere(nu=48, nv=40)
    keep = rng.random(T.shape[0]) > (0.02 + 0.05 * (seed % 3))
    T2 = T[keep]
    scales = rng.random(V.shape[0])
    min_isle = int(rng.integers(1, 40))
    mesh = core.DualMarchingCells.fromArrays(V, T2, scales=scales, min_isle_size=min_isle)
    c = _compare(mesh, V, T2, scales, min_isle)
    assert c["holes"] > 0


def test_cap_hole_counts():
    from tsr_b200 import core
    V, T = uv_sphere(nu=37, nv=12)
    mesh = core.DualMarchingCells.fromArrays(V, T[37:], min_isle_size=2)
    c = _compare(mesh, V, T[37:], None, 2)
    assert (c["isle_vertices"], c["holes"]) == (1, 1)


def test_nothing_left_and_nothing_to_do():
    from tsr_b200 import core
    V, T = uv_sphere()
    gone = core.DualMarchingCells.fromArrays(V, T, min_isle_size=10 ** 6)
    assert gone.positions.shape == (0, 3) and gone.triangles.shape == (0, 3)
    assert gone.post_counts["isle_vertices"] == V.shape[0]
    closed = core.DualMarchingCells.fromArrays(V, T, min_isle_size=1)
    _compare(closed, V, T, None, 1)
    np.testing.assert_array_equal(closed.triangles, T)


def test_edge_conflict_leaves_mesh_unchanged():
    from tsr_b200 import core
    V = np.array(np.eye(3).tolist() + [[1.0, 1, 1], [-1.0, -1, -1]])
    T = np.array([[0, 1, 2], [1, 0, 3], [0, 1, 4]], np.uint32)
    mesh = core.DualMarchingCells.fromArrays(V, T)
    with pytest.raises(core.TsrError) as e:
        mesh.postprocess(1)
    assert core.STATUS[e.value.status] == "TSR_ERR_STATE"
    mesh._read()
    np.testing.assert_array_equal(mesh.triangles, T)
    np.testing.assert_array_equal(mesh.positions, V)


def test_create_rejects_bad_indices():
    from tsr_b200 import core
    with pytest.raises(core.TsrError, match="out of range"):
        core.DualMarchingCells.fromArrays(np.zeros((3, 3)), np.array([[0, 1, 3]], np.uint32))


def test_golden_damaged_mesh():
    """The committed fixture (the sphere fixture's DMC mesh with 3 % of its
    triangles removed: about a thousand holes, isles below 50 vertices)."""
    from pathlib import Path
    from tsr_b200 import core
    g = np.load(Path(__file__).resolve().parent / "golden" / "mesh_post.npz")
    mesh = core.DualMarchingCells.fromArrays(g["post_in_pos"], g["post_in_tris"], scales=g["post_in_scale"],
                                             min_isle_size=int(g["post_min_isle"]))
    for k in ("isle_vertices", "isle_triangles", "border_edges", "holes", "hole_vertices", "hole_triangles",
              "skipped_rings"):
        assert mesh.post_counts[k] == int(g["post_" + k]), k
    np.testing.assert_array_equal(mesh.triangles, g["post_tris"])
    np.testing.assert_array_equal(mesh.positions, g["post_pos"])
    np.testing.assert_array_equal(mesh.scales, g["post_scale"])
    check_normals(mesh.normals, g["post_nrm"], g["post_pos"], g["post_tris"], NORMAL_ATOL)
