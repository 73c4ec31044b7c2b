"""CPU tests of the depth-map triangulation restatement (DepthImage::
triangulate in oracle/mesh_oracle.cpp) on synthetic depth maps of a sphere in
front of a plate: every triangle lies in one 2x2 pixel block and passes the
reference's depth-discontinuity test, vertices are numbered by first use,
lie on their pixel rays and on the sphere, normals face the camera side of
the surface, and each scale is the mean distance to the vertex's mesh
neighbours."""
import numpy as np
import pytest

from oracle import pyoracle
from tsr_b200 import scenes


@pytest.fixture(scope="module")
def views():
    return scenes.sphere_depth_views()


def _pixel_of_vertex(r):
    pix = r["pixel_to_vertex"].ravel()
    used = np.flatnonzero(pix != 0xFFFFFFFF)
    out = np.empty(used.shape[0], np.int64)
    out[pix[used]] = used
    return out


@pytest.mark.parametrize("i", [0, 3])
def test_triangles_stay_in_blocks_and_skip_jumps(views, i):
    v = views[i]
    d = v["depths"]
    H, W = d.shape
    r = pyoracle.depth_triangulate(d, v["hps_to_ray_vs"], v["hps_to_ray_ws"], v["center"])
    pv = _pixel_of_vertex(r)
    tp = pv[r["triangles"].astype(np.int64)]            # triangle corners as pixels
    x, y = tp % W, tp // W
    assert np.all(x.max(1) - x.min(1) == 1) and np.all(y.max(1) - y.min(1) == 1)
    assert np.all(d.ravel()[tp] > 0)
    # no triangle spans the silhouette (sphere at depth ~2-3, plate beyond 3.5)
    dd = d.ravel()[tp]
    assert np.all(dd.max(1) - dd.min(1) < 0.5)
    # first-use numbering: the first corner naming each vertex comes in vertex order
    flat = r["triangles"].ravel()
    seen = np.zeros(pv.shape[0], bool)
    order = []
    for c in flat:
        if not seen[c]:
            seen[c] = True
            order.append(c)
    assert order == list(range(pv.shape[0]))


@pytest.mark.parametrize("i", [1, 4])
def test_vertices_rays_normals_scales(views, i):
    v = views[i]
    d = v["depths"]
    H, W = d.shape
    col = np.random.default_rng(i).random((H, W, 3))
    r = pyoracle.depth_triangulate(d, v["hps_to_ray_vs"], v["hps_to_ray_ws"], v["center"], colors=col)
    pv = _pixel_of_vertex(r)
    xs, ys = pv % W, pv // W
    ray = np.stack([xs, ys, np.ones_like(xs)], 1) @ v["hps_to_ray_ws"]
    ray /= np.linalg.norm(ray, axis=1, keepdims=True)
    np.testing.assert_allclose(r["positions"], v["center"] + ray * d.ravel()[pv][:, None], rtol=0, atol=1e-12)
    np.testing.assert_array_equal(r["colors"], col.reshape(-1, 3)[pv])
    rad = np.linalg.norm(r["positions"], axis=1)
    on_sphere = rad < 1.05
    assert on_sphere.sum() > 1000
    np.testing.assert_allclose(np.linalg.norm(r["normals"], axis=1), 1.0, atol=1e-12)
    assert float((r["normals"][on_sphere] * r["positions"][on_sphere]).sum(1).mean()) > 0.99
    # scale = mean distance to the mesh neighbours
    t = r["triangles"].astype(np.int64)
    nb = [set() for _ in range(pv.shape[0])]
    for a, b, c in t:
        nb[a] |= {b, c}; nb[b] |= {a, c}; nb[c] |= {a, b}
    p = r["positions"]
    want = np.array([np.mean([np.linalg.norm(p[q] - p[k]) for q in nb[k]]) for k in range(len(nb))])
    np.testing.assert_allclose(r["scales"], want, rtol=1e-12)


def test_no_valid_pixels():
    v = scenes.sphere_depth_views(n_cams=1)[0]
    r = pyoracle.depth_triangulate(-np.ones_like(v["depths"]), v["hps_to_ray_vs"], v["hps_to_ray_ws"], v["center"])
    assert r["positions"].shape == (0, 3) and r["triangles"].shape == (0, 3)
    assert np.all(r["pixel_to_vertex"] == 0xFFFFFFFF)
