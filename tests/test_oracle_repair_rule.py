"""The rule the pruned field's repair rests on, checked on the oracle's own
DMC (DualMarchingCells.cpp:41-169; the oracle is bit-exact with the
reference build): the raw mesh depends on the occupancy only through the
signs and, at the positive end of each sign change between face
neighbours, through whether the value exceeds EPSILON.

A negative leaf's value is -EPSILON with or without its prior
(Occupancy.cpp:570-587), and the vertex interpolation snaps to an end whose
value is within EPSILON of zero, so every vertex of a sign change lies at
its negative end unless the positive end's value is at most EPSILON.  A
skipped leaf of the pruned field keeps its sign, and its value only needs
to fall on the same side of EPSILON as the plain field's.
"""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tsr_b200 import scenes

EPS = 1e-6


def _positive_ends(occ, nb_offsets, nbs):
    """Positive leaves that share a face with a non-positive one (the
    neighbour CSR lists face neighbours, Leaves.cpp:82-134)."""
    pos = occ > 0.0
    keep = np.zeros(occ.shape[0], bool)
    owner = np.repeat(np.arange(occ.shape[0]), np.diff(nb_offsets))
    cross = pos[owner] != pos[nbs]
    keep[owner[cross & pos[owner]]] = True
    keep[nbs[cross & pos[nbs]]] = True
    return keep


def _field(make):
    o = Oracle(make()).build_tree()
    o.occupancy(nthreads=1)
    occ = o.fields()["occ"].copy()
    lv = o.leaves()
    return o, occ, _positive_ends(occ, lv["nb_offsets"], lv["nbs"])


SCENES = [lambda: scenes.sphere_scene(stride=16),
          lambda: scenes.csg_scene(seed=3, n_target=3000, width=160, height=120, f=125.0, n_cams=12)]


@pytest.mark.parametrize("make", SCENES, ids=["sphere", "csg"])
def test_mesh_depends_on_positive_values_only_through_epsilon(make):
    o, occ, ends = _field(make)
    m0 = o.dmc()
    assert ends.any() and (occ[ends] > EPS).any()
    rng = np.random.default_rng(7)
    changed = occ.copy()
    high = occ > EPS                      # every positive value above EPSILON, ends included
    changed[high] = rng.uniform(2 * EPS, 1e3, int(high.sum()))
    m1 = o.set_occupancy(changed).dmc()
    for k in ("cases", "vpos", "vscale", "tris"):
        np.testing.assert_array_equal(m1[k], m0[k], err_msg=k)


def test_side_of_epsilon_at_a_positive_end_matters():
    """The converse, so the rule above is not vacuous: a positive end whose
    value drops to EPSILON moves its vertices to the positive end."""
    o, occ, ends = _field(SCENES[0])
    m0 = o.dmc()
    changed = occ.copy()
    changed[ends & (occ > EPS)] = EPS
    m1 = o.set_occupancy(changed).dmc()
    np.testing.assert_array_equal(m1["tris"], m0["tris"])
    assert np.abs(m1["vpos"] - m0["vpos"]).max() > 0.0
