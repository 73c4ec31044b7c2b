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
* ``cluttered_scene`` -- many random primitives on a ground plate, 400 cameras
  at 1920x1080, f = 1400, 5 % outliers uniform in the bounding box, depth
  noise 1 %, confidences uniform in [0.2, 1] (60M samples).
* ``vase_scene_device`` -- a thin-walled vase (1 mm wall) on a ground plane,
  1000 cameras at distances 0.3-300 (log-uniform), so sample scales span
  ~1000x (100M samples).

``render`` casts rays with numpy on the host; ``render_device`` casts the same
rays with torch on a CUDA device (seconds instead of minutes for the 16M-100M
sample scenes) and returns a ``DeviceScene`` whose arrays stay in device
memory.  The two draw their noise from different generators, so a device
scene has the host scene's geometry and cameras but other noise draws.

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

    def hit_t(self, o, d):
        import torch
        oc = o - _tt(self.c, d)
        b = (d * oc).sum(dim=1)
        disc = b * b - ((oc * oc).sum(dim=1) - self.r * self.r)
        sq = torch.sqrt(torch.clamp(disc, min=0.0))
        t0, t1 = -b - sq, -b + sq
        tt = torch.where(t0 > 1e-9, t0, torch.where(t1 > 1e-9, t1, torch.full_like(t0, math.inf)))
        return torch.where(disc >= 0, tt, torch.full_like(tt, math.inf))

    def normal_t(self, p):
        n = p - _tt(self.c, p)
        return n / n.norm(dim=1, keepdim=True)


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

    def hit_t(self, o, d):
        import torch
        inv = 1.0 / d
        ta = (_tt(self.lo, d) - o) * inv
        tb = (_tt(self.hi, d) - o) * inv
        inf = math.inf
        tmin = torch.nan_to_num(torch.minimum(ta, tb), nan=-inf, posinf=inf, neginf=-inf).amax(dim=1)
        tmax = torch.nan_to_num(torch.maximum(ta, tb), nan=inf, posinf=inf, neginf=-inf).amin(dim=1)
        t = torch.where(tmin > 1e-9, tmin, tmax)
        return torch.where((tmax >= tmin) & (tmax > 1e-9), t, torch.full_like(t, inf))

    def normal_t(self, p):
        import torch
        c = _tt(0.5 * (self.lo + self.hi), p)
        h = _tt(0.5 * (self.hi - self.lo), p)
        q = (p - c) / h
        ax = q.abs().argmax(dim=1)
        n = torch.zeros_like(p)
        r = torch.arange(p.shape[0], device=p.device)
        n[r, ax] = torch.sign(q[r, ax])
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

    def hit_t(self, o, d):
        import torch
        ox, oy, oz = o[:, 0] - self.cx, o[:, 1] - self.cy, o[:, 2]
        a = d[:, 0] ** 2 + d[:, 1] ** 2
        b = 2 * (ox * d[:, 0] + oy * d[:, 1])
        c = ox * ox + oy * oy - self.r * self.r
        disc = b * b - 4 * a * c
        t = torch.full_like(a, math.inf)
        sq = torch.sqrt(torch.clamp(disc, min=0.0))
        for tt in ((-b - sq) / (2 * a), (-b + sq) / (2 * a)):
            z = oz + tt * d[:, 2]
            ok = (disc >= 0) & (a > 1e-15) & (tt > 1e-9) & (z >= self.z0) & (z <= self.z1)
            t = torch.where(ok & (tt < t), tt, t)
        for zc in (self.z0, self.z1):
            tt = (zc - oz) / d[:, 2]
            x = ox + tt * d[:, 0]
            y = oy + tt * d[:, 1]
            ok = (tt > 1e-9) & (x * x + y * y <= self.r * self.r)
            t = torch.where(ok & (tt < t), tt, t)
        return t

    def normal_t(self, p):
        import torch
        side = (p[:, 2] > self.z0 + 1e-9) & (p[:, 2] < self.z1 - 1e-9)
        zero = torch.zeros_like(p[:, 0])
        cap = torch.where(p[:, 2] >= 0.5 * (self.z0 + self.z1), zero + 1.0, zero - 1.0)
        n = torch.stack([torch.where(side, p[:, 0] - self.cx, zero), torch.where(side, p[:, 1] - self.cy, zero),
                         torch.where(side, zero, cap)], dim=1)
        return n / n.norm(dim=1, keepdim=True)


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

    def _sdf_t(self, p):
        import torch
        q = torch.sqrt(p[:, 0] ** 2 + p[:, 1] ** 2) - self.R
        return torch.sqrt(q * q + p[:, 2] ** 2) - self.r

    def hit_t(self, o, d):
        return _sphere_trace(self._sdf_t, o - _tt(self.c, d), d, self.R + self.r, 400, 1e-9)

    def normal_t(self, p):
        import torch
        q = p - _tt(self.c, p)
        rho = torch.sqrt(q[:, 0] ** 2 + q[:, 1] ** 2)
        k = (rho - self.R) / torch.clamp(rho, min=1e-12)
        n = torch.stack([q[:, 0] * k, q[:, 1] * k, q[:, 2]], dim=1)
        return n / n.norm(dim=1, keepdim=True)


class Vase:
    """Thin-walled vase: the wall {z0 <= z <= z1, |rho - r(z)| <= wall / 2}
    around the vertical axis through (cx, cy), profile r(z) = r0 + a sin(w (z -
    z0) + phi), closed by a base disc of the same thickness.  Device rendering
    only: sphere tracing on a distance bound (the wall's |rho - r(z)| divided
    by the profile's Lipschitz factor)."""

    def __init__(self, cx, cy, z0, z1, r0, a, w, phi, wall):
        self.cx, self.cy, self.z0, self.z1 = float(cx), float(cy), float(z0), float(z1)
        self.r0, self.a, self.w, self.phi, self.wall = float(r0), float(a), float(w), float(phi), float(wall)
        self.lip = math.sqrt(1.0 + (self.a * self.w) ** 2)
        self.bound = math.sqrt((self.r0 + abs(self.a) + wall) ** 2 + (0.5 * (z1 - z0) + wall) ** 2)

    def radius_t(self, z):
        import torch
        return self.r0 + self.a * torch.sin(self.w * (z - self.z0) + self.phi)

    def _sdf_t(self, p):   # p relative to (cx, cy, zmid)
        import torch
        zmid = 0.5 * (self.z0 + self.z1)
        z = p[:, 2] + zmid
        rho = torch.sqrt(p[:, 0] ** 2 + p[:, 1] ** 2)
        rz = self.radius_t(torch.clamp(z, self.z0, self.z1))
        dwall = torch.maximum(((rho - rz).abs() - 0.5 * self.wall) / self.lip,
                              torch.maximum(self.z0 - z, z - self.z1))
        r_base = self.r0 + self.a * math.sin(self.phi)
        dbase = torch.maximum(rho - r_base, torch.maximum(self.z0 - z, z - (self.z0 + self.wall)))
        return torch.minimum(dwall, dbase)

    def _origin(self, like):
        return _tt([self.cx, self.cy, 0.5 * (self.z0 + self.z1)], like)

    def hit_t(self, o, d):
        return _sphere_trace(self._sdf_t, o - self._origin(d), d, self.bound, 3000, 2e-8)

    def normal_t(self, p):
        import torch
        q = p - self._origin(p)
        h = 1e-7
        g = []
        for ax in range(3):
            e = torch.zeros_like(q)
            e[:, ax] = h
            g.append(self._sdf_t(q + e) - self._sdf_t(q - e))
        n = torch.stack(g, dim=1)
        return n / torch.clamp(n.norm(dim=1, keepdim=True), min=1e-30)


# -------------------------------------------------------------------- cameras
def look_at_basis(cam, target):
    fwd = np.asarray(target, float) - cam
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
    prims = _random_csg_prims(rng, n_prims)
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


# ------------------------------------------------------------ device rendering
def _tt(x, like):
    """A float64 tensor on the device of `like`."""
    import torch
    return torch.as_tensor(np.asarray(x, float), dtype=torch.float64, device=like.device)


def _sphere_trace(sdf, oc, d, bound_r, iters, eps):
    """First t > 0 with sdf(oc + t d) < eps, marching by the distance bound,
    for rays (origins oc relative to the shape, unit directions d) that meet
    the shape's bounding sphere of radius bound_r; inf elsewhere."""
    import torch
    b = (d * oc).sum(dim=1)
    disc = b * b - ((oc * oc).sum(dim=1) - bound_r * bound_r)
    sq = torch.sqrt(torch.clamp(disc, min=0.0))
    out = torch.full_like(b, math.inf)
    idx = torch.nonzero((disc >= 0) & (-b + sq > 0)).squeeze(1)
    tt = torch.clamp(-b - sq, min=0.0)[idx]
    tf = (-b + sq)[idx]
    oo, dd = oc[idx], d[idx]
    for it in range(iters):
        if idx.numel() == 0:
            break
        s = sdf(oo + dd * tt[:, None])
        hit = s < eps
        out[idx[hit]] = tt[hit]
        keep = ~(hit | (tt > tf))
        idx, tt, tf, oo, dd = idx[keep], tt[keep] + s[keep], tf[keep], oo[keep], dd[keep]
        if it >= 256 and idx.numel() * 1_000_000 < d.shape[0]:
            break   # the last grazing rays (under 1e-6 of them) count as misses
    return out


@dataclasses.dataclass
class DeviceScene:
    """A scene whose sample arrays are torch tensors in device memory."""
    pos: object            # (N, 3) float64
    nrm: object            # (N, 3) float64
    scale: object          # (N,) float64
    conf: object           # (N,) float64
    links: object          # (N, K) int32 (uint32 bit patterns)
    cams: np.ndarray       # (C, 3) float64
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    @property
    def k(self) -> int:
        return int(self.links.shape[1])

    def host(self) -> Scene:
        return Scene(self.pos.cpu().numpy(), self.nrm.cpu().numpy(), self.scale.cpu().numpy(),
                     self.conf.cpu().numpy(), self.links.cpu().numpy().view(np.uint32), self.cams.copy(), self.name)


def _jitter_normals_t(n, deg, gen):
    import torch
    if deg <= 0:
        return n
    m = n.shape[0]
    cos_max = math.cos(math.radians(deg))
    cz = cos_max + (1.0 - cos_max) * torch.rand(m, generator=gen, device=n.device, dtype=torch.float64)
    phi = 2 * math.pi * torch.rand(m, generator=gen, device=n.device, dtype=torch.float64)
    sz = torch.sqrt(torch.clamp(1 - cz * cz, min=0.0))
    ax = torch.zeros_like(n)
    small = n[:, 0].abs() < 0.9
    ax[:, 0] = small.double()
    ax[:, 1] = (~small).double()
    u = torch.linalg.cross(n, ax)
    u = u / u.norm(dim=1, keepdim=True)
    v = torch.linalg.cross(n, u)
    out = n * cz[:, None] + u * (sz * torch.cos(phi))[:, None] + v * (sz * torch.sin(phi))[:, None]
    return out / out.norm(dim=1, keepdim=True)


def _cast(prims, o, d):
    """Nearest hit over `prims`: distance (inf for a miss) and primitive index."""
    import torch
    best = torch.full((d.shape[0],), math.inf, dtype=torch.float64, device=d.device)
    who = torch.full((d.shape[0],), -1, dtype=torch.int64, device=d.device)
    for pi, pr in enumerate(prims):
        t = pr.hit_t(o, d)
        upd = t < best
        best = torch.where(upd, t, best)
        who = torch.where(upd, torch.full_like(who, pi), who)
    return best, who


def render_device(prims, cams, width, height, f, noise_rel, jitter_deg, seed, target=None,
                  conf_range=(1.0, 1.0), outlier_frac=0.0, name="", bound_radius=2.5, looks=None,
                  device="cuda", rays_per_batch=1 << 23):
    """``render`` on a device with torch.  Cameras are cast in batches of
    about `rays_per_batch` rays.  With a `target` sample count, a coarse pass
    (every 8th pixel in each direction) estimates the hits and each pixel is
    kept with the probability that leaves about 1.2x the target before the
    cast -- the same distribution as casting every pixel and subsampling --
    and the hits are then subsampled to exactly `target` (fewer if the scene
    gives fewer).  `looks` are the cameras' look-at points (origin by
    default)."""
    import torch
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    cams = np.asarray(cams, float)
    nc = cams.shape[0]
    looks = np.zeros((nc, 3)) if looks is None else np.asarray(looks, float)
    bases = [look_at_basis(cams[i], looks[i]) for i in range(nc)]
    R = torch.as_tensor(np.stack([b[0] for b in bases]), device=device)
    D = torch.as_tensor(np.stack([b[1] for b in bases]), device=device)
    F = torch.as_tensor(np.stack([b[2] for b in bases]), device=device)
    C = torch.as_tensor(cams, device=device)

    def rays(ci, sel, stride):
        # pixel ids `sel` (row-major over the strided grid) of cameras `ci`
        w = (width + stride - 1) // stride
        ys = (sel // w) * stride
        xs = (sel % w) * stride
        px = (xs.double() + 0.5 - 0.5 * width) / f
        py = (ys.double() + 0.5 - 0.5 * height) / f
        d = F[ci] + px[:, None] * R[ci] + py[:, None] * D[ci]
        zlen = d.norm(dim=1)
        d = d / zlen[:, None]
        o = C[ci]
        b = (d * o).sum(dim=1)
        near = b * b - ((o * o).sum(dim=1) - bound_radius * bound_radius) >= 0
        return o[near], d[near], zlen[near], ci[near]

    def cams_per_batch(npx):
        return max(1, min(nc, rays_per_batch // max(1, npx)))

    keep_p = 1.0
    if target is not None:
        st = 8
        npx = ((width + st - 1) // st) * ((height + st - 1) // st)
        hits = 0
        cb = cams_per_batch(npx)
        for c0 in range(0, nc, cb):
            c1 = min(nc, c0 + cb)
            ci = torch.arange(c0, c1, device=device).repeat_interleave(npx)
            sel = torch.arange(npx, device=device).repeat(c1 - c0)
            o, d, _, _ = rays(ci, sel, st)
            best, _ = _cast(prims, o, d)
            hits += int(torch.isfinite(best).sum())
        est = hits * (width * height) / npx
        keep_p = min(1.0, 1.2 * target / max(est, 1.0))
    npx = width * height
    P, Nn, S, L = [], [], [], []
    cb = cams_per_batch(int(npx * keep_p) + 1)
    for c0 in range(0, nc, cb):
        c1 = min(nc, c0 + cb)
        if keep_p < 1.0:
            m = torch.rand((c1 - c0) * npx, generator=gen, device=device) < keep_p
            flat = torch.nonzero(m).squeeze(1)
            ci = (flat // npx) + c0
            sel = flat % npx
        else:
            ci = torch.arange(c0, c1, device=device).repeat_interleave(npx)
            sel = torch.arange(npx, device=device).repeat(c1 - c0)
        o, d, zlen, ci = rays(ci, sel, 1)
        best, who = _cast(prims, o, d)
        ok = torch.isfinite(best)
        t, o, d, zlen, ci, who = best[ok], o[ok], d[ok], zlen[ok], ci[ok], who[ok]
        p = o + d * t[:, None]
        nrm = torch.zeros_like(p)
        for pi, pr in enumerate(prims):
            mm = who == pi
            if bool(mm.any()):
                nrm[mm] = pr.normal_t(p[mm])
        flip = (nrm * d).sum(dim=1) > 0
        nrm[flip] *= -1
        depth = t / zlen
        tn = t + torch.randn(t.shape, generator=gen, device=device, dtype=torch.float64) * noise_rel * depth
        P.append(o + d * tn[:, None]); Nn.append(nrm); S.append(2.0 * depth / f); L.append(ci.to(torch.int32))
    pos = torch.cat(P); nrm = torch.cat(Nn); scale = torch.cat(S); links = torch.cat(L)
    del P, Nn, S, L
    if target is not None and pos.shape[0] > target:
        keep = torch.randperm(pos.shape[0], generator=gen, device=device)[:target].sort().values
        pos, nrm, scale, links = pos[keep], nrm[keep], scale[keep], links[keep]
    nrm = _jitter_normals_t(nrm, jitter_deg, gen)
    n = pos.shape[0]
    if outlier_frac > 0:
        m = int(outlier_frac * n)
        sel = torch.randperm(n, generator=gen, device=device)[:m]
        lo, hi = pos.min(dim=0).values, pos.max(dim=0).values
        pos[sel] = lo + (hi - lo) * torch.rand((m, 3), generator=gen, device=device, dtype=torch.float64)
        v = torch.randn((m, 3), generator=gen, device=device, dtype=torch.float64)
        nrm[sel] = v / v.norm(dim=1, keepdim=True)
    lo, hi = conf_range
    if lo == hi:
        conf = torch.full((n,), float(lo), dtype=torch.float64, device=device)
    else:
        conf = lo + (hi - lo) * torch.rand(n, generator=gen, device=device, dtype=torch.float64)
    return DeviceScene(pos.contiguous(), nrm.contiguous(), scale.contiguous(), conf, links.reshape(-1, 1).contiguous(),
                       cams, name)


def _random_csg_prims(rng, n_prims):
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
    return prims


def random_csg_scene_device(seed, n_target, width, height, f, device="cuda", outlier_frac=0.0,
                            conf_range=(1.0, 1.0)):
    """``random_csg_scene`` rendered on the device: the same primitives and
    cameras (drawn from the same numpy generator), other noise draws;
    optionally with outliers and varying confidences."""
    rng = np.random.default_rng(1000 + seed)
    n_prims = int(rng.integers(3, 9))
    prims = _random_csg_prims(rng, n_prims)
    n_cams = int(rng.integers(64, 161))
    cams = _random_cams(rng, n_cams, 1.5, 8.0)
    return render_device(prims, cams, width, height, f, 0.005, 8.0, seed=7919 * (seed + 1), target=n_target,
                         name="random_csg_%d" % seed, device=device, outlier_frac=outlier_frac,
                         conf_range=conf_range)


def csg_scene_device(seed=0, n_target=4_000_000, width=1280, height=960, f=600.0, n_cams=120, device="cuda"):
    """``csg_scene`` rendered on the device (same primitives and cameras)."""
    rng = np.random.default_rng(seed)
    prims = [Box([-0.9, -0.9, -0.601], [0.9, 0.9, -0.599]),
             Cylinder(0.35, -0.3, 0.3, -0.6, 0.2),
             Torus([-0.3, 0.35, 0.0], 0.5, 0.1)]
    cams = _random_cams(rng, n_cams, 1.5, 12.0)
    return render_device(prims, cams, width, height, f, 0.005, 8.0, seed=104729 + seed, target=n_target,
                         name="csg", device=device)


def _cluttered_setup(seed, n_prims, n_cams):
    rng = np.random.default_rng(5000 + seed)
    prims = [Box([-1.2, -1.2, -0.75], [1.2, 1.2, -0.7])]   # ground plate
    prims += _random_csg_prims(rng, n_prims)
    cams = _random_cams(rng, n_cams, 1.5, 8.0)
    return prims, cams


def cluttered_scene(seed=0, n_target=60_000, width=192, height=108, f=140.0, n_cams=40, n_prims=24):
    """The cluttered scene on the host (small versions for tests and the CPU
    oracle): `n_prims` random primitives on a ground plate, 5 % outliers
    uniform in the samples' bounding box, depth noise 1 %, confidences
    uniform in [0.2, 1]."""
    prims, cams = _cluttered_setup(seed, n_prims, n_cams)
    rng = np.random.default_rng(6000 + seed)
    return render(prims, cams, width, height, f, 0.01, 8.0, rng, target=n_target, conf_range=(0.2, 1.0),
                  outlier_frac=0.05, name="cluttered")


def cluttered_scene_device(seed=0, n_target=60_000_000, width=1920, height=1080, f=1400.0, n_cams=400,
                           n_prims=24, device="cuda"):
    """The 60M-sample cluttered scene: 400 cameras at 1920x1080, f = 1400,
    5 % outliers, depth noise 1 %, confidences uniform in [0.2, 1]."""
    prims, cams = _cluttered_setup(seed, n_prims, n_cams)
    return render_device(prims, cams, width, height, f, 0.01, 8.0, seed=15485863 + seed, target=n_target,
                         conf_range=(0.2, 1.0), outlier_frac=0.05, name="cluttered", device=device)


def _vase_setup(seed, n_cams, dmin, dmax):
    rng = np.random.default_rng(9000 + seed)
    vase = Vase(0.0, 0.0, 0.0, 1.0, 0.3, 0.12, 5.0, 0.4, 0.001)
    plane = Box([-4.0, -4.0, -0.002], [4.0, 4.0, 0.0])
    cams, looks = [], []
    while len(cams) < n_cams:
        zt = rng.uniform(0.05, 0.95)
        th = rng.uniform(0, 2 * math.pi)
        rt = vase.r0 + vase.a * math.sin(vase.w * zt + vase.phi)
        look = np.array([rt * math.cos(th), rt * math.sin(th), zt])
        el = rng.uniform(-0.3, 1.2)
        az = th + rng.uniform(-0.6, 0.6)
        dirv = np.array([math.cos(el) * math.cos(az), math.cos(el) * math.sin(az), math.sin(el)])
        dist = math.exp(rng.uniform(math.log(dmin), math.log(dmax)))
        cam = look + dist * dirv
        rho = math.hypot(cam[0], cam[1])
        rz = vase.r0 + vase.a * math.sin(vase.w * min(max(cam[2], 0.0), 1.0) + vase.phi)
        if cam[2] < 0.02 or (cam[2] < 1.0 and rho < rz + 0.01):
            continue   # under the plane or inside the vase
        cams.append(cam)
        looks.append(look)
    return [vase, plane], np.array(cams), np.array(looks)


def vase_scene_device(seed=0, n_target=100_000_000, width=1024, height=768, f=900.0, n_cams=1000, device="cuda"):
    """The density-stress scene: a vase 1 m tall with a 1 mm wall on a ground
    plane, 1000 cameras aimed at points of the vase from distances
    log-uniform in [0.3, 300], so sample scales span ~1000x."""
    prims, cams, looks = _vase_setup(seed, n_cams, 0.3, 300.0)
    return render_device(prims, cams, width, height, f, 0.005, 8.0, seed=32452843 + seed, target=n_target,
                         name="vase", bound_radius=6.0, looks=looks, device=device)
