"""CPU tests of the mesh post-processing restatement (oracle/mesh_oracle.cpp).

Checks on meshes with known answers: a closed surface stays as it is apart
from its normals; a removed cap is closed by the concentric fill with the
vertex and triangle counts the reference's recursion gives; small isles
are deleted with the kept elements in their old order; filled meshes have no
border edge left; bow-tie borders (two holes sharing a vertex) and odd ring
sizes work.  The ring search is also replayed the way the GPU kernel does it
(an index of the edges by tail, the candidate at the smallest current list
position) and must give the literal scan's rings on shuffled edge lists.
"""
import numpy as np
import pytest

from oracle import pyoracle


def uv_sphere(nu=16, nv=10):
    """Closed, consistently wound UV sphere."""
    verts = [[0.0, 0.0, 1.0]]
    for i in range(1, nv):
        th = np.pi * i / nv
        for j in range(nu):
            ph = 2 * np.pi * j / nu
            verts.append([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
    verts.append([0.0, 0.0, -1.0])
    V = np.array(verts)
    S = len(V) - 1
    tris = []
    for j in range(nu):
        tris.append([0, 1 + j, 1 + (j + 1) % nu])
    for i in range(nv - 2):
        for j in range(nu):
            a = 1 + i * nu + j
            b = 1 + i * nu + (j + 1) % nu
            tris.append([a, a + nu, b])
            tris.append([b, a + nu, b + nu])
    for j in range(nu):
        tris.append([S, 1 + (nv - 2) * nu + (j + 1) % nu, 1 + (nv - 2) * nu + j])
    return V, np.array(tris, np.uint32)


def edge_uses(T):
    e = np.concatenate([T[:, [0, 1]], T[:, [1, 2]], T[:, [2, 0]]])
    _, c = np.unique(np.sort(e, 1), axis=0, return_counts=True)
    return c


def normal_sums(positions, triangles, order=None):
    """Per vertex: the sum of angle-weighted unit triangle normals (what
    Mesh::computeNormalsWeightedByAngles normalises) and the sum of the
    weights (the corner angles), in numpy; ``order`` permutes the triangles'
    accumulation."""
    p = np.asarray(positions, np.float64)
    t = np.asarray(triangles, np.int64)
    if order is not None:
        t = t[order]
    vec = np.zeros_like(p)
    wsum = np.zeros(p.shape[0])
    if t.shape[0] == 0:
        return vec, wsum
    v0, v1, v2 = p[t[:, 0]], p[t[:, 1]], p[t[:, 2]]

    def unit(a):
        n = np.linalg.norm(a, axis=1, keepdims=True)
        return np.divide(a, n, out=np.zeros_like(a), where=n > 0)

    d0, d1, d2 = unit(v1 - v0), unit(v2 - v1), unit(v2 - v0)
    n = unit(np.cross(v1 - v0, v2 - v0))
    cos = [np.einsum("ij,ij->i", d0, d2), -np.einsum("ij,ij->i", d0, d1), np.einsum("ij,ij->i", d1, d2)]
    for k in range(3):
        ang = np.arccos(np.clip(cos[k], -1.0, 1.0))
        np.add.at(vec, t[:, k], n * ang[:, None])
        np.add.at(wsum, t[:, k], ang)
    return vec, wsum


# Rounding in the weighted sum is a few units in the last place of the
# weights' total W; after normalising by the sum's length |s| that becomes a
# direction error of about 1e-16 W / |s|.  Vertices whose weighted normals
# (nearly) cancel are ill-conditioned: the summation order -- the reference's
# OpenMP atomics or the GPU's -- decides their direction, so the tolerance
# grows with W / |s| (and is unbounded where s = 0).
NORMAL_COND_FACTOR = 1e-13


def check_normals(got, want, positions, triangles, atol):
    got, want = np.asarray(got), np.asarray(want)
    if len(want) == 0:
        return
    diff = np.abs(got - want).max(1)
    bad = diff > atol
    if not bad.any():
        return
    vec, wsum = normal_sums(positions, triangles)
    mag = np.linalg.norm(vec, axis=1)[bad]
    tol = atol + NORMAL_COND_FACTOR * np.divide(wsum[bad], mag, out=np.full(mag.shape, np.inf), where=mag > 0)
    assert np.all(diff[bad] <= tol), (int(bad.sum()), diff[bad][diff[bad] > tol][:5], mag[diff[bad] > tol][:5])


def fill_counts(n):
    """New vertices and triangles the reference's recursion adds to a ring."""
    va = ta = 0
    while n > 5:
        a = n // 2
        va += a
        ta += n + a
        n = a
    return va, ta + n - 2


def test_closed_surface_only_gets_normals():
    V, T = uv_sphere()
    c, p, n, s, t = pyoracle.mesh_postprocess(V, T, min_isle_size=1)
    assert (c["vertices"], c["triangles"], c["border_edges"], c["holes"]) == (V.shape[0], T.shape[0], 0, 0)
    np.testing.assert_array_equal(p, V)
    np.testing.assert_array_equal(t, T)
    np.testing.assert_allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-12)
    assert float((n * V).sum(1).min()) > 0.9   # outward on the unit sphere


@pytest.mark.parametrize("nu", [16, 13, 7])
def test_cap_hole_is_filled(nu):
    V, T = uv_sphere(nu=nu)
    T2 = T[nu:]                       # the top cap; its apex becomes a one-vertex isle
    c, p, n, s, t = pyoracle.mesh_postprocess(V, T2, scales=np.ones(V.shape[0]), min_isle_size=2)
    va, ta = fill_counts(nu)
    assert c["isle_vertices"] == 1 and c["isle_triangles"] == 0
    assert (c["border_edges"], c["holes"], c["hole_vertices"], c["hole_triangles"]) == (nu, 1, va, ta)
    assert (c["vertices"], c["triangles"]) == (V.shape[0] - 1 + va, T2.shape[0] + ta)
    # kept vertices compacted in order, indices shifted past the deleted apex
    np.testing.assert_array_equal(p[:V.shape[0] - 1], V[1:])
    np.testing.assert_array_equal(t[:T2.shape[0]], T2 - 1)
    np.testing.assert_array_equal(s[V.shape[0] - 1:], 0.0)   # filled vertices get scale 0
    assert np.all(edge_uses(t) == 2)                         # closed again
    np.testing.assert_allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-12)


def test_two_holes_and_an_isle():
    V, T = uv_sphere()
    far = np.array([[5.0, 5, 5], [6, 5, 5], [5, 6, 5]])
    V3 = np.vstack([V, far])
    T3 = np.vstack([T[16:100], T[110:], [[V.shape[0], V.shape[0] + 1, V.shape[0] + 2]]]).astype(np.uint32)
    c, p, n, s, t = pyoracle.mesh_postprocess(V3, T3, min_isle_size=5)
    assert c["isle_vertices"] == 4 and c["isle_triangles"] == 1   # the apex and the far triangle
    assert c["holes"] == 2
    assert np.all(edge_uses(t) == 2)


def test_bow_tie_border():
    """Two triangular holes meeting at one vertex, which starts two border
    edges: the greedy search runs through it into the second hole, so one
    ring of 6 edges (a figure eight) is filled, and the surface closes."""
    V, T = uv_sphere(nu=12, nv=8)
    # two triangles of the band that share only vertex 1 + 12 + 5
    v = 1 + 12 + 5
    share = [i for i, tr in enumerate(T) if v in tr]
    a = share[0]
    b = next(i for i in share[1:] if len(set(T[i]) & set(T[a])) == 1)
    T2 = np.delete(T, [a, b], axis=0)
    c, p, n, s, t = pyoracle.mesh_postprocess(V, T2, min_isle_size=1)
    assert (c["border_edges"], c["holes"], c["hole_vertices"], c["hole_triangles"]) == (6,) + (1,) + fill_counts(6)
    assert np.all(edge_uses(t) == 2)


def test_everything_deleted():
    V, T = uv_sphere()
    c, p, n, s, t = pyoracle.mesh_postprocess(V, T, min_isle_size=10 ** 6)
    assert (c["vertices"], c["triangles"], c["isle_vertices"], c["isle_triangles"]) == (0, 0, V.shape[0], T.shape[0])


def test_edge_conflict_reported():
    V = np.eye(3).tolist() + [[1.0, 1, 1], [-1.0, -1, -1]]
    T = np.array([[0, 1, 2], [1, 0, 3], [0, 1, 4]], np.uint32)   # edge (0, 1) in three triangles
    c, *_ = pyoracle.mesh_postprocess(np.array(V), T, min_isle_size=1)
    assert c["error"] == 1


def replay_indexed(edges):
    """The GPU ring search (meshpost.cu k_rings) in Python: a tail-sorted
    index, the unused candidate at the smallest current position, a swap
    behind the ring; an unclosed set stays whole."""
    nb = len(edges)
    tail = [e[0] for e in edges]
    head = [e[1] for e in edges]
    by_tail = {}
    for j in sorted(range(nb), key=lambda j: (tail[j], j)):
        by_tail.setdefault(tail[j], []).append(j)
    order = list(range(nb))
    pos = list(range(nb))
    used = [False] * nb
    rings, s0 = [], 0
    while s0 < nb:
        start = tail[order[s0]]
        used[order[s0]] = True
        r, closed = s0 + 1, False
        while r < nb:
            end = head[order[r - 1]]
            cands = [pos[j] for j in by_tail.get(end, []) if not used[j]]
            if not cands:
                break
            best = min(cands)
            jd, other = order[best], order[r]
            order[r], pos[jd] = jd, r
            order[best], pos[other] = other, best
            used[jd] = True
            r += 1
            if head[jd] == start:
                closed = True
                break
        stop = r if closed else nb
        rings.append([tail[order[p]] for p in range(s0, stop)])
        s0 = stop
    return rings


@pytest.mark.parametrize("seed", range(12))
def test_indexed_ring_replay_matches_literal_scan(seed):
    rng = np.random.default_rng(seed)
    edges = []
    base = 0
    for _ in range(rng.integers(1, 6)):                      # disjoint cycles
        n = int(rng.integers(3, 14))
        vs = list(range(base, base + n))
        edges += [(vs[i], vs[(i + 1) % n]) for i in range(n)]
        base += n
    # bow-ties: cycles through one shared vertex
    hub = base
    for _ in range(rng.integers(0, 3)):
        n = int(rng.integers(3, 8))
        vs = [hub] + list(range(base + 1, base + n))
        edges += [(vs[i], vs[(i + 1) % n]) for i in range(n)]
        base += n
    if seed % 4 == 3:                                          # an open chain: a ring that cannot close
        edges += [(base + 1, base + 2), (base + 2, base + 3)]
    order = rng.permutation(len(edges))
    edges = [edges[i] for i in order]
    assert replay_indexed(edges) == pyoracle.border_rings(edges)


def test_normal_tolerance_covers_reordered_sums():
    """The restatement fed the golden damaged mesh's triangles in other orders
    (what FP64 atomics do): its normals move only where check_normals'
    condition-number tolerance allows."""
    from pathlib import Path
    g = np.load(Path(__file__).resolve().parent / "golden" / "mesh_post.npz")
    p, t, n = g["post_pos"], g["post_tris"], g["post_nrm"]
    rng = np.random.default_rng(0)
    moved = 0
    for _ in range(3):
        perm = rng.permutation(t.shape[0])
        c, _, n2, _, _ = pyoracle.mesh_postprocess(p, t[perm], min_isle_size=1)
        assert c["holes"] == 0 and c["isle_vertices"] == 0
        moved += int((np.abs(n2 - n).max(1) > 1e-12).sum())
        check_normals(n2, n, p, t, 1e-12)
    assert moved > 0   # the phenomenon is real on this mesh
