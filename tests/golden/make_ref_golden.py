"""Generates the reference-pinned fixtures tests/golden/ref_*.npz from the
reference's own hot path (its Scene/Tree and SurfaceExtraction sources built
unmodified against the project's BaseProject shim: `make -C oracle ref`,
oracle/refpy.py), run on one thread.

Each fixture holds a seeded scene's samples and cameras and what the
reference computes for them: the node arrays, the sample permutation, leaf
scopes, node->leaf links, the neighbour CSR, dual cells, the occupancy field
(kernel sums, cone lengths, priors, node states, cone count, occupancy of
every leaf) and the raw DMC mesh.  Scenes: the two golden scenes of
make_golden.py, a K = 3 capture with invalid and repeated camera links, a
small cluttered capture (outliers, confidences in [0.2, 1]) and the
degenerate inputs of edge_scenes() (ref_edge_*).
ref_update_csg_3k.npz holds the incremental update of the CSG fixture's
field: Occupancy::eraseSamples of 10 % of the samples (tree-order indices,
seed 4), then Occupancy::addSamples of the same samples.

Usage: python tests/golden/make_ref_golden.py [fixture names]   (needs the reference sources)
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import refpy  # noqa: E402
from tsr_b200 import scenes  # noqa: E402

GOLDEN = Path(__file__).resolve().parent
INVALID = 0xFFFFFFFF


def k3_scene():
    """The sparse sphere capture with K = 3 links per sample: its own camera,
    then a random other camera or an invalid slot, then a repeat of the first
    link or an invalid slot."""
    sc = scenes.sphere_scene(stride=8, width=160, height=120, f=125.0)
    rng = np.random.default_rng(21)
    n, nc = sc.n, sc.cams.shape[0]
    other = (sc.links[:, 0] + rng.integers(1, nc, n)) % nc
    s1 = np.where(rng.random(n) < 0.6, other, INVALID).astype(np.uint32)
    s2 = np.where(rng.random(n) < 0.3, sc.links[:, 0], INVALID).astype(np.uint32)
    links = np.stack([sc.links[:, 0], s1, s2], 1).astype(np.uint32)
    return scenes.Scene(sc.pos, sc.nrm, sc.scale, sc.conf, np.ascontiguousarray(links), sc.cams, "sphere_k3")


def edge_scenes():
    """Degenerate inputs: one sample, two samples, every sample three times
    at the same position, a flat patch (zero extent along z) seen by two
    cameras, and samples whose every link is invalid (no cones at all)."""
    base = scenes.sphere_scene(stride=16)

    def sub(idx, name, links=None):
        return scenes.Scene(base.pos[idx], base.nrm[idx], base.scale[idx], base.conf[idx],
                            np.ascontiguousarray(base.links[idx] if links is None else links, np.uint32), base.cams,
                            name)

    rng = np.random.default_rng(1)
    xy = rng.uniform(-1.0, 1.0, (3000, 2))
    plane = scenes.Scene(np.c_[xy, np.zeros(3000)], np.tile([0.0, 0.0, 1.0], (3000, 1)), np.full(3000, 0.02),
                         np.ones(3000), (np.arange(3000, dtype=np.uint32) % 2)[:, None].copy(),
                         np.array([[0.0, 0.0, 3.0], [1.0, 1.0, 2.0]]), "plane")
    every = np.arange(0, base.n, 8)
    return {
        "ref_edge_single": sub(np.arange(1), "single"),
        "ref_edge_two": sub(np.arange(2), "two"),
        "ref_edge_duplicates": sub(np.repeat(np.arange(200), 3), "duplicates"),
        "ref_edge_plane": plane,
        "ref_edge_no_links": sub(every, "no_links", np.full((every.shape[0], 1), INVALID, np.uint32)),
    }


def fixture_scenes():
    return {
        "ref_sphere_small": scenes.sphere_scene(stride=6, width=160, height=120, f=125.0),
        "ref_csg_3k": scenes.csg_scene(seed=3, n_target=3000, width=160, height=120, f=125.0, n_cams=12),
        "ref_sphere_k3": k3_scene(),
        "ref_cluttered_2k": scenes.cluttered_scene(seed=2, n_target=2000),
        **edge_scenes(),
    }


def main(names=None):
    """All fixtures, or only those named on the command line."""
    for name, sc in fixture_scenes().items():
        if names and name not in names:
            continue
        r = refpy.run(sc, threads=1)
        out = {k: v for k, v in r.items() if k != "fields" and not k.startswith("samples_")}
        out.update({"field_" + k: np.asarray(v) for k, v in r["fields"].items()})
        inputs = dict(in_pos=sc.pos, in_nrm=sc.nrm, in_scale=sc.scale, in_conf=sc.conf, in_links=sc.links,
                      in_cams=sc.cams)
        np.savez_compressed(GOLDEN / (name + ".npz"), **inputs, **out)
        print(name, sc.n, "samples, K =", sc.k, ",", out["children"].shape[0], "nodes,", out["tris"].shape[0],
              "triangles")
    if not names or "ref_update_csg_3k" in names:
        update_fixture()


def update_fixture():
    sc = fixture_scenes()["ref_csg_3k"]
    refpy.run(sc, threads=1)
    chosen = np.sort(np.random.default_rng(4).choice(sc.n, size=sc.n // 10, replace=False)).astype(np.uint32)
    erased = refpy.update(chosen, True)
    added = refpy.update(chosen, False)
    out = {"chosen": chosen}
    out.update({"erased_" + k: np.asarray(v) for k, v in erased.items()})
    out.update({"added_" + k: np.asarray(v) for k, v in added.items()})
    inputs = dict(in_pos=sc.pos, in_nrm=sc.nrm, in_scale=sc.scale, in_conf=sc.conf, in_links=sc.links,
                  in_cams=sc.cams)
    np.savez_compressed(GOLDEN / "ref_update_csg_3k.npz", **inputs, **out)
    print("ref_update_csg_3k", chosen.shape[0], "samples erased and added again")


if __name__ == "__main__":
    main(sys.argv[1:])
