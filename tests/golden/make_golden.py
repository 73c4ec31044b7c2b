"""Generates the golden fixtures of tests/golden from the FP64 oracle.

The reference ships no tests or golden vectors for this path, so these
fixtures pin the oracle's own outputs on two small seeded scenes (a sparse
unit-sphere capture and a small CSG capture) against regressions, and give
the GPU tests a committed answer to compare with.  Two more pin the mesh
post-processing (the sphere fixture's DMC mesh with triangles removed) and
the depth-map triangulation (one small sphere-and-plate view).

Usage: python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.pyoracle import Oracle  # noqa: E402
from tsr_b200 import scenes  # noqa: E402

GOLDEN = Path(__file__).resolve().parent


def fixture_scenes():
    return {
        "sphere_small": scenes.sphere_scene(stride=6, width=160, height=120, f=125.0),
        "csg_3k": scenes.csg_scene(seed=3, n_target=3000, width=160, height=120, f=125.0, n_cams=12),
    }


def oracle_outputs(scene):
    o = Oracle(scene).build_tree()
    out = {}
    out["root"] = o.root()
    out.update({"nodes_" + k: v for k, v in o.nodes().items()})
    out["permutation"] = o.permutation()
    for k, v in o.leaves().items():
        out["leaves_" + k] = v
    out["dual_cells"] = o.dual_cells()
    o.occupancy(nthreads=1)
    for k, v in o.fields().items():
        out["field_" + k] = np.asarray(v)
    for k, v in o.dmc().items():
        out["mesh_" + k] = v
    return out


def mesh_post_inputs():
    """The sphere_small fixture's DMC mesh with 3 % of its triangles removed
    (seed 11): holes of many sizes and small isles cut loose."""
    g = np.load(GOLDEN / "sphere_small.npz")
    keep = np.random.default_rng(11).random(g["mesh_tris"].shape[0]) > 0.03
    return dict(post_in_pos=g["mesh_vpos"], post_in_scale=g["mesh_vscale"], post_in_tris=g["mesh_tris"][keep],
                post_min_isle=np.uint32(50))


def mesh_post_outputs(inp):
    from oracle.pyoracle import mesh_postprocess
    c, p, n, s, t = mesh_postprocess(inp["post_in_pos"], inp["post_in_tris"], inp["post_in_scale"],
                                     int(inp["post_min_isle"]))
    out = {"post_" + k: np.uint64(v) for k, v in c.items()}
    out.update(post_pos=p, post_nrm=n, post_scale=s, post_tris=t)
    return out


def depth_inputs():
    v = scenes.sphere_depth_views(seed=5, width=96, height=72, f=75.0, n_cams=2)[1]
    col = np.random.default_rng(5).random(v["depths"].shape + (3,))
    return dict(depth_in=v["depths"], depth_in_mvs=v["hps_to_ray_vs"], depth_in_mws=v["hps_to_ray_ws"],
                depth_in_center=v["center"], depth_in_colors=col)


def depth_outputs(inp):
    from oracle.pyoracle import depth_triangulate
    r = depth_triangulate(inp["depth_in"], inp["depth_in_mvs"], inp["depth_in_mws"], inp["depth_in_center"],
                          colors=inp["depth_in_colors"])
    return {"depth_" + k: v for k, v in r.items()}


def main():
    for name, sc in fixture_scenes().items():
        out = oracle_outputs(sc)
        inputs = dict(in_pos=sc.pos, in_nrm=sc.nrm, in_scale=sc.scale, in_conf=sc.conf, in_links=sc.links,
                      in_cams=sc.cams)
        np.savez_compressed(GOLDEN / (name + ".npz"), **inputs, **out)
        print(name, sc.n, "samples,", out["nodes_children"].shape[0], "nodes,", out["mesh_tris"].shape[0], "triangles")
    inp = mesh_post_inputs()
    out = mesh_post_outputs(inp)
    np.savez_compressed(GOLDEN / "mesh_post.npz", **inp, **out)
    print("mesh_post", {k: int(v) for k, v in out.items() if v.ndim == 0})
    inp = depth_inputs()
    out = depth_outputs(inp)
    np.savez_compressed(GOLDEN / "depth_small.npz", **inp, **out)
    print("depth_small", out["depth_positions"].shape[0], "vertices,", out["depth_triangles"].shape[0], "triangles")


if __name__ == "__main__":
    main()
