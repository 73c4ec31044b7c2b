"""Generates the golden fixtures of tests/golden from the FP64 oracle.

The reference ships no tests or golden vectors for this path, so these
fixtures pin the oracle's own outputs on two small seeded scenes (a sparse
unit-sphere capture and a small CSG capture) against regressions, and give
the GPU tests a committed answer to compare with.

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


def main():
    for name, sc in fixture_scenes().items():
        out = oracle_outputs(sc)
        inputs = dict(in_pos=sc.pos, in_nrm=sc.nrm, in_scale=sc.scale, in_conf=sc.conf, in_links=sc.links,
                      in_cams=sc.cams)
        np.savez_compressed(GOLDEN / (name + ".npz"), **inputs, **out)
        print(name, sc.n, "samples,", out["nodes_children"].shape[0], "nodes,", out["mesh_tris"].shape[0], "triangles")


if __name__ == "__main__":
    main()
