"""Seeded synthetic scenes: analytic ray casting of camera depth maps into
oriented, scaled point samples linked to the camera that saw them.

The reference builds its samples from Embree-rendered depth maps
(SyntheticScene.cpp:45-336) and real MVE captures; neither can run here, so
these generators stand in for them with the shapes, sizes and value
distributions of the benchmark configurations:

* ``sphere_scene``   -- unit sphere, 24 cameras on a ring of radius 3 at
  elevations +-20 deg, 640x480, f = 500 px (about 250k samples).
* ``csg_scene``      -- 2 mm plate, cylinder r = 0.3, torus R = 0.5 / r = 0.1,
  120 cameras at distances uniform in [1.5, 12] (about 4M samples).
* ``random_csg_scene`` -- 3-8 random spheres / boxes / cylinders / thin plates,
  64-160 cameras (training scenes and the 16M-sample held-out scene).

Every sample has: position (FP64), unit normal (true normal jittered uniformly
inside a cone), scale = 2 * depth / f, confidence, and K = 1 camera link.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Scene:
    pos: np.ndarray        # (N, 3) float64
    nrm: np.ndarray        # (N, 3) float64
    scale: np.ndarray      # (N,) float64
    conf: np.ndarray       # (N,) float64
    links: np.ndarray      # (N, K) uint32
    cams: np.ndarray       # (C, 3) float64
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    @property
    def k(self) -> int:
        return int(self.links.shape[1])

    def subset(self, idx) -> "Scene":
        return Scene(self.pos[idx].copy(), self.nrm[idx].copy(), self.scale[idx].copy(),
                     self.conf[idx].copy(), self.links[idx].copy(), self.cams.copy(), self.name)


# ----------------------------------------------------------------- primitives
class Sphere:
    def __init__(self, c, r):
        self.c = np.asarray(c, float); self.r = float(r)

    def hit(self, o, d):
        oc = o - self.c
        b = d @ oc if d.ndim == 1 else np.einsum("ij,j->i", d, oc)
        cc = oc @ oc - self.r * self.r
        disc = b * b - cc
        t = np.full(d.shape[0], np.inf)
        ok = disc >= 0
        sq = np.sqrt(np.where(ok, disc, 0))
        t0 = -b - sq
        t1 = -b + sq
        tt = np.where(t0 > 1e-9, t0, np.where(t1 > 1e-9, t1, np.inf))
        t[ok] = tt[ok]
        return t

    def normal(self, p):
        n = p - self.c
        return n / np.linalg.norm(n, axis=1, keepdims=True)


class Box:
    def __init__(self, lo, hi):
        self.lo = np.asarray(lo, float); self.hi = np.asarray(hi, float)

    def hit(self, o, d):
        with np.errstate(divide="ignore", invalid="ignore"):
            inv = 1.0 / d
            ta = (self.lo - o) * inv
            tb = (self.hi - o) * inv
        tmin = np.nanmax(np.minimum(ta, tb), axis=1)
        tmax = np.nanmin(np.maximum(ta, tb), axis=1)
        t = np.where((tmax >= tmin) & (tmax > 1e-9), np.where(tmin > 1e-9, tmin, tmax), np.inf)
        return t

    def normal(self, p):
        c = 0.5 * (self.lo + self.hi)
        h = 0.5 * (self.hi - self.lo)
        q = (p - c) / h
        ax = np.argmax(np.abs(q), axis=1)
        n = np.zeros_like(p)
        n[np.arange(p.shape[0]), ax] = np.sign(q[np.arange(p.shape[0]), ax])
        return n


class Cylinder:
    """Finite cylinder with caps, axis along z."""

    def __init__(self, cx, cy, r, z0, z1):
        self.cx, self.cy, self.r, self.z0, self.z1 = float(cx), float(cy), float(r), float(z0), float(z1)

    def hit(self, o, d):
        ox, oy = o[0] - self.cx, o[1] - self.cy
        a = d[:, 0] ** 2 + d[:, 1] ** 2
        b = 2 * (ox * d[:, 0] + oy * d[:, 1])
        c = ox * ox + oy * oy - self.r * self.r
        disc = b * b - 4 * a * c
        t = np.full(d.shape[0], np.inf)
        with np.errstate(divide="ignore", invalid="ignore"):
            sq = np.sqrt(np.maximum(disc, 0))
            for tt in ((-b - sq) / (2 * a), (-b + sq) / (2 * a)):
                z = o[2] + tt * d[:, 2]
                ok = (disc >= 0) & (a > 1e-15) & (tt > 1e-9) & (z >= self.z0) & (z <= self.z1)
                t = np.where(ok & (tt < t), tt, t)
            for zc in (self.z0, self.z1):
                tt = (zc - o[2]) / d[:, 2]
                x = o[0] + tt * d[:, 0] - self.cx
                y = o[1] + tt * d[:, 1] - self.cy
                ok = (tt > 1e-9) & (x * x + y * y <= self.r * self.r)
                t = np.where(ok & (tt < t), tt, t)
        return t

    def normal(self, p):
        n = np.zeros_like(p)
        side = (p[:, 2] > self.z0 + 1e-9) & (p[:, 2] < self.z1 - 1e-9)
        n[:, 0] = np.where(side, p[:, 0] - self.cx, 0)
        n[:, 1] = np.where(side, p[:, 1] - self.cy, 0)
        n[:, 2] = np.where(side, 0, np.where(p[:, 2] >= 0.5 * (self.z0 + self.z1), 1.0, -1.0))
        return n / np.linalg.norm(n, axis=1, keepdims=True)


class Torus:
    """Torus around the z axis through c, sphere-traced then Newton-refined."""

    def __init__(self, c, R, r):
        self.c = np.asarray(c, float); self.R = float(R); self.r = float(r)

    def _sdf(self, p):
        q = np.sqrt(p[:, 0] ** 2 + p[:, 1] ** 2) - self.R
        return np.sqrt(q * q + p[:, 2] ** 2) - self.r

    def hit(self, o, d):
        oc = o - self.c
        # bounding sphere
        b = np.einsum("ij,j->i", d, oc)
        cc = oc @ oc - (self.R + self.r) ** 2
        disc = b * b - cc
        t = np.where(disc >= 0, np.maximum(-b - np.sqrt(np.maximum(disc, 0)), 0.0), np.inf)
        tfar = np.where(disc >= 0, -b + np.sqrt(np.maximum(disc, 0)), -np.inf)
        active = np.isfinite(t)
        out = np.full(d.shape[0], np.inf)
        idx = np.nonzero(active)[0]
        tt = t[idx]
        dd = d[idx]
        for _ in range(400):
            if idx.size == 0:
                break
            p = oc + dd * tt[:, None]
            s = self._sdf(p)
            hit = s < 1e-9
            miss = tt > tfar[idx]
            done = hit | miss
            out[idx[hit]] = tt[hit]
            keep = ~done
            idx, tt, dd = idx[keep], tt[keep] + s[keep], dd[keep]
        return out

    def normal(self, p):
        q = p - self.c
        rho = np.sqrt(q[:, 0] ** 2 + q[:, 1] ** 2)
        k = (rho - self.R) / np.maximum(rho, 1e-12)
        n = np.stack([q[:, 0] * k, q[:, 1] * k, q[:, 2]], axis=1)
        return n / np.linalg.norm(n, axis=1, keepdims=True)


# -------------------------------------------------------------------- cameras
def look_at_basis(cam, target):
    fwd = target - cam
    fwd = fwd / np.linalg.norm(fwd)
    up = np.array([0.0, 0.0, 1.0])
    if abs(fwd @ up) > 0.99:
        up = np.array([0.0, 1.0, 0.0])
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    down = np.cross(fwd, right)
    return right, down, fwd


def _jitter_normals(n, deg, rng):
    if deg <= 0:
        return n
    m = n.shape[0]
    cos_max = math.cos(math.radians(deg))
    cz = rng.uniform(cos_max, 1.0, m)
    phi = rng.uniform(0, 2 * math.pi, m)
    sz = np.sqrt(np.maximum(0, 1 - cz * cz))
    a = np.where(np.abs(n[:, 0:1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0, 1.0, 0]]))
    u = np.cross(n, a)
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    v = np.cross(n, u)
    out = n * cz[:, None] + u * (sz * np.cos(phi))[:, None] + v * (sz * np.sin(phi))[:, None]
    return out / np.linalg.norm(out, axis=1, keepdims=True)


def render(prims, cams, width, height, f, noise_rel, jitter_deg, rng, stride=1,
           target=None, conf_range=(1.0, 1.0), outlier_frac=0.0, name="", bound_radius=2.5):
    """Ray-cast every camera's depth map against the union of `prims`, which
    must lie inside the sphere of radius `bound_radius` around the origin."""
    cams = np.asarray(cams, float)
    ys, xs = np.mgrid[0:height:stride, 0:width:stride]
    px = (xs.ravel() + 0.5 - 0.5 * width) / f
    py = (ys.ravel() + 0.5 - 0.5 * height) / f
    P, Nn, S, L = [], [], [], []
    for ci, cam in enumerate(cams):
        right, down, fwd = look_at_basis(cam, np.zeros(3))
        d = fwd[None, :] + px[:, None] * right[None, :] + py[:, None] * down[None, :]
        zlen = np.linalg.norm(d, axis=1)
        d = d / zlen[:, None]
        # only rays that meet the scene's bounding sphere can hit a primitive
        b = d @ cam
        near = b * b - (cam @ cam - bound_radius * bound_radius) >= 0
        d, zlen = d[near], zlen[near]
        best = np.full(d.shape[0], np.inf)
        who = np.full(d.shape[0], -1)
        for pi, pr in enumerate(prims):
            t = pr.hit(cam, d)
            upd = t < best
            best = np.where(upd, t, best)
            who = np.where(upd, pi, who)
        ok = np.isfinite(best)
        if not ok.any():
            continue
        t = best[ok]
        dd = d[ok]
        w = who[ok]
        p = cam + dd * t[:, None]
        nrm = np.zeros_like(p)
        for pi, pr in enumerate(prims):
            m = w == pi
            if m.any():
                nrm[m] = pr.normal(p[m])
        flip = np.einsum("ij,ij->i", nrm, dd) > 0
        nrm[flip] *= -1
        depth = t / zlen[ok]          # z-depth
        tn = t + rng.normal(0.0, 1.0, t.shape) * noise_rel * depth
        p = cam + dd * tn[:, None]
        P.append(p); Nn.append(nrm); S.append(2.0 * depth / f)
        L.append(np.full(p.shape[0], ci, np.uint32))
    pos = np.concatenate(P); nrm = np.concatenate(Nn); scale = np.concatenate(S); links = np.concatenate(L)
    if target is not None and pos.shape[0] > target:
        keep = np.sort(rng.choice(pos.shape[0], size=target, replace=False))
        pos, nrm, scale, links = pos[keep], nrm[keep], scale[keep], links[keep]
    nrm = _jitter_normals(nrm, jitter_deg, rng)
    if outlier_frac > 0:
        m = int(outlier_frac * pos.shape[0])
        sel = rng.choice(pos.shape[0], size=m, replace=False)
        lo, hi = pos.min(0), pos.max(0)
        pos[sel] = rng.uniform(lo, hi, (m, 3))
        v = rng.normal(size=(m, 3))
        nrm[sel] = v / np.linalg.norm(v, axis=1, keepdims=True)
    lo, hi = conf_range
    conf = np.full(pos.shape[0], lo) if lo == hi else rng.uniform(lo, hi, pos.shape[0])
    return Scene(np.ascontiguousarray(pos), np.ascontiguousarray(nrm), np.ascontiguousarray(scale),
                 np.ascontiguousarray(conf), np.ascontiguousarray(links.reshape(-1, 1)), cams, name)


def sphere_scene(seed=0, stride=3, width=640, height=480, f=500.0):
    """Unit sphere, 24 cameras (12 azimuths x elevations +-20 deg) at radius 3."""
    rng = np.random.default_rng(seed)
    cams = []
    for el in (20.0, -20.0):
        for k in range(12):
            az = 2 * math.pi * k / 12 + (0.0 if el > 0 else math.pi / 12)
            e = math.radians(el)
            cams.append([3 * math.cos(e) * math.cos(az), 3 * math.cos(e) * math.sin(az), 3 * math.sin(e)])
    return render([Sphere([0, 0, 0], 1.0)], cams, width, height, f, 0.003, 5.0, rng, stride=stride,
                  name="sphere")


def _random_cams(rng, n, dmin, dmax):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    v[:, 2] = np.abs(v[:, 2]) * 0.8 + 0.05
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v * rng.uniform(dmin, dmax, n)[:, None]


def csg_scene(seed=0, n_target=4_000_000, width=1280, height=960, f=600.0, n_cams=120):
    """2 mm plate, cylinder r = 0.3, torus R = 0.5 / r = 0.1 in the box [-1, 1]^3."""
    rng = np.random.default_rng(seed)
    prims = [Box([-0.9, -0.9, -0.601], [0.9, 0.9, -0.599]),
             Cylinder(0.35, -0.3, 0.3, -0.6, 0.2),
             Torus([-0.3, 0.35, 0.0], 0.5, 0.1)]
    cams = _random_cams(rng, n_cams, 1.5, 12.0)
    return render(prims, cams, width, height, f, 0.005, 8.0, rng, target=n_target, name="csg")


def random_csg_scene(seed, n_target=3_000_000, width=800, height=600, f=600.0, n_cams=None,
                     n_prims=None):
    """3-8 random spheres / boxes / cylinders / thin plates in [-1, 1]^3."""
    rng = np.random.default_rng(1000 + seed)
    n_prims = n_prims or int(rng.integers(3, 9))
    prims = []
    for _ in range(n_prims):
        kind = rng.integers(0, 4)
        c = rng.uniform(-0.6, 0.6, 3)
        if kind == 0:
            prims.append(Sphere(c, rng.uniform(0.1, 0.4)))
        elif kind == 1:
            h = rng.uniform(0.05, 0.3, 3)
            prims.append(Box(c - h, c + h))
        elif kind == 2:
            z0 = c[2] - rng.uniform(0.1, 0.4)
            prims.append(Cylinder(c[0], c[1], rng.uniform(0.05, 0.3), z0, z0 + rng.uniform(0.2, 0.8)))
        else:
            h = np.array([rng.uniform(0.2, 0.6), rng.uniform(0.2, 0.6), 0.001])
            prims.append(Box(c - h, c + h))
    n_cams = n_cams or int(rng.integers(64, 161))
    cams = _random_cams(rng, n_cams, 1.5, 8.0)
    return render(prims, cams, width, height, f, 0.005, 8.0, rng, target=n_target,
                  name="random_csg_%d" % seed)


def tiny_scene(seed=0, stride=16):
    """A few thousand samples of the sphere scene, for fast tests."""
    return sphere_scene(seed=seed, stride=stride)


def depth_views(prims, cams, width, height, f, noise_rel, rng, bound_radius=2.5):
    """Per camera a depth map along the pixel rays (height x width, -1 where
    nothing is hit) with the two matrices DepthImage::triangulate takes:
    (x, y, 1) times ``hps_to_ray_vs`` is the pixel's view-space ray
    ((x + 0.5 - w/2) / f, (y + 0.5 - h/2) / f, 1); times ``hps_to_ray_ws`` its
    world-space ray (right, down, forward basis of the camera looking at the
    origin).  The stand-in for the reference's rendered or captured depth
    maps (SyntheticScene.cpp:45-336)."""
    views = []
    A = np.array([[1.0 / f, 0.0, 0.0], [0.0, 1.0 / f, 0.0],
                  [(0.5 - 0.5 * width) / f, (0.5 - 0.5 * height) / f, 1.0]])
    ys, xs = np.mgrid[0:height, 0:width]
    hps = np.stack([xs.ravel().astype(float), ys.ravel().astype(float), np.ones(xs.size)], 1)
    for cam in np.asarray(cams, float):
        right, down, fwd = look_at_basis(cam, np.zeros(3))
        B = np.stack([right, down, fwd])
        Mws = A @ B
        d = hps @ Mws
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        best = np.full(d.shape[0], np.inf)
        b = d @ cam
        near = b * b - (cam @ cam - bound_radius * bound_radius) >= 0
        for pr in prims:
            t = np.full(d.shape[0], np.inf)
            if near.any():
                t[near] = pr.hit(cam, d[near])
            best = np.minimum(best, t)
        ok = np.isfinite(best)
        depth = np.where(ok, best * (1.0 + rng.normal(0.0, noise_rel, best.shape)), -1.0)
        views.append(dict(depths=depth.reshape(height, width), hps_to_ray_vs=A, hps_to_ray_ws=Mws,
                          center=cam.copy()))
    return views


def sphere_depth_views(seed=0, width=160, height=120, f=125.0, n_cams=6):
    """Depth maps of the unit sphere in front of a plate (a depth jump at the
    silhouette) from cameras on a ring of radius 3."""
    rng = np.random.default_rng(seed)
    cams = [[3 * math.cos(2 * math.pi * k / n_cams), 3 * math.sin(2 * math.pi * k / n_cams), 0.4]
            for k in range(n_cams)]
    prims = [Sphere([0, 0, 0], 1.0), Box([-2.2, -2.2, -1.6], [2.2, 2.2, -1.5])]
    return depth_views(prims, cams, width, height, f, 0.001, rng)
