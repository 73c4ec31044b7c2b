"""GPU depth-map triangulation (tsr_depth_triangulate) against the CPU
restatement, and samples made from depth maps through the whole pipeline.

Bit-exact: triangles, the pixel-to-vertex map, vertex positions, colours and
scales (the neighbour distances are summed in findVertexNeighbors order with
correctly rounded operations on both sides).  Tolerance: normals,
NORMAL_ATOL (FP64 atomic sums in no fixed order, CUDA's acos), widened by
the sum's condition number where the weighted normals nearly cancel
(check_normals).
"""
import numpy as np
import pytest

from oracle import pyoracle
from tsr_b200 import scenes

from test_mesh_oracle import check_normals

pytestmark = pytest.mark.gpu

NORMAL_ATOL = 1e-12


def _check(view, colors=None):
    from tsr_b200 import core
    g = core.DepthImage(view["depths"]).triangulate(view["hps_to_ray_vs"], view["hps_to_ray_ws"], view["center"],
                                                    colors=colors)
    o = pyoracle.depth_triangulate(view["depths"], view["hps_to_ray_vs"], view["hps_to_ray_ws"], view["center"],
                                   colors=colors)
    np.testing.assert_array_equal(g.triangles, o["triangles"])
    np.testing.assert_array_equal(g.pixel_to_vertex, o["pixel_to_vertex"])
    np.testing.assert_array_equal(g.positions, o["positions"])
    np.testing.assert_array_equal(g.colors, o["colors"])
    np.testing.assert_array_equal(g.scales, o["scales"])
    check_normals(g.normals, o["normals"], o["positions"], o["triangles"], NORMAL_ATOL)
    return g


@pytest.mark.parametrize("i", range(6))
def test_views_match_oracle(i):
    views = scenes.sphere_depth_views()
    col = np.random.default_rng(i).random(views[i]["depths"].shape + (3,)) if i % 2 else None
    g = _check(views[i], col)
    assert g.triangles.shape[0] > 1000


def test_full_resolution_view():
    v = scenes.sphere_depth_views(width=640, height=480, f=500.0, n_cams=1)[0]
    _check(v)


def test_holes_and_noise():
    """Random invalid pixels and strong depth noise: many mask cases and
    rejected discontinuities."""
    v = scenes.sphere_depth_views(n_cams=2)[1]
    rng = np.random.default_rng(3)
    d = v["depths"] * (1.0 + 0.05 * rng.standard_normal(v["depths"].shape))
    d[rng.random(d.shape) < 0.15] = -1.0
    _check(dict(v, depths=d))


def test_empty_and_tiny_maps():
    from tsr_b200 import core
    v = scenes.sphere_depth_views(n_cams=1)[0]
    g = _check(dict(v, depths=-np.ones_like(v["depths"])))
    assert g.positions.shape == (0, 3)
    _check(dict(v, depths=np.full((2, 2), 2.0)))
    with pytest.raises(core.TsrError):
        core.DepthImage(np.ones((1, 5))).triangulate(v["hps_to_ray_vs"], v["hps_to_ray_ws"], v["center"])


def test_samples_from_depth_maps_reconstruct_the_sphere():
    """Samples::addSamplesViaMeshes over the depth meshes, then tree, field and
    crust: the crust's vertices lie near the unit sphere or the plate."""
    from tsr_b200 import core
    views = scenes.sphere_depth_views(width=320, height=240, f=250.0, n_cams=8)
    meshes = [core.DepthImage(v["depths"]).triangulate(v["hps_to_ray_vs"], v["hps_to_ray_ws"], v["center"])
              for v in views]
    samples = core.Samples.fromDepthMeshes(meshes, list(range(len(views))))
    assert samples.count == sum(m.positions.shape[0] for m in meshes)
    assert np.all(samples.confidences == 1.0)
    cams = core.Cameras(np.stack([v["center"] for v in views]))
    tree = core.Tree(samples)
    occ = core.Occupancy(tree, cams)
    crust = occ.extractCrust(min_isle_size=1000)
    p = crust.positions
    assert p.shape[0] > 1000
    near_sphere = np.abs(np.linalg.norm(p, axis=1) - 1.0) < 0.05
    near_plate = np.abs(p[:, 2] + 1.5) < 0.1
    assert (near_sphere | near_plate).mean() > 0.8


def test_golden_depth_view():
    """The committed fixture: a 96x72 view with per-pixel colours."""
    from pathlib import Path
    from tsr_b200 import core
    g = np.load(Path(__file__).resolve().parent / "golden" / "depth_small.npz")
    m = core.DepthImage(g["depth_in"]).triangulate(g["depth_in_mvs"], g["depth_in_mws"], g["depth_in_center"],
                                                   colors=g["depth_in_colors"])
    np.testing.assert_array_equal(m.triangles, g["depth_triangles"])
    np.testing.assert_array_equal(m.pixel_to_vertex, g["depth_pixel_to_vertex"])
    np.testing.assert_array_equal(m.positions, g["depth_positions"])
    np.testing.assert_array_equal(m.colors, g["depth_colors"])
    np.testing.assert_array_equal(m.scales, g["depth_scales"])
    check_normals(m.normals, g["depth_normals"], g["depth_positions"], g["depth_triangles"], NORMAL_ATOL)
