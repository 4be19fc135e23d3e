"""Seeded synthetic point clouds standing in for the reference's datasets.

The reference evaluates on ShapeNet / Matterport / D-FAUST scans, none of which
are available here; these generators produce oriented point clouds with the
shapes, sizes and noise levels of the benchmark workloads:

* ``torus``          -- 10k points, area-uniform on a torus (R=0.35, r=0.15), exact normals
* ``superquadrics``  -- points on a union of random superquadrics, with optional noise
* ``learned_problem``-- one noisy superquadric with query points and an analytic target field
* ``room``           -- large indoor scene: walls, floor, ceiling and boxes / cylinders
* ``serving_stream`` -- request sizes, depths and Poisson arrival times for the serving loop
"""
from __future__ import annotations

import math

import numpy as np


def torus(n=10000, R=0.35, r=0.15, seed=0):
    """Area-uniform torus about z, centred at the origin; exact unit normals."""
    rng = np.random.default_rng(seed)
    pts_u, pts_v = [], []
    need = n
    while need > 0:
        u = rng.uniform(0, 2 * math.pi, 4 * need)
        v = rng.uniform(0, 2 * math.pi, 4 * need)
        keep = rng.uniform(0, R + r, 4 * need) < (R + r * np.cos(v))
        pts_u.append(u[keep])
        pts_v.append(v[keep])
        need -= int(keep.sum())
    u = np.concatenate(pts_u)[:n]
    v = np.concatenate(pts_v)[:n]
    xyz = np.stack([(R + r * np.cos(v)) * np.cos(u), (R + r * np.cos(v)) * np.sin(u), r * np.sin(v)], 1)
    nrm = np.stack([np.cos(v) * np.cos(u), np.cos(v) * np.sin(u), np.sin(v)], 1)
    return xyz.astype(np.float32), nrm.astype(np.float32)


def _rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _spow(x, e):
    return np.sign(x) * np.abs(x) ** e


class Superquadric:
    """Superquadric with scales ``a``, exponents ``e1, e2``, rotation ``rot`` and centre ``c``."""

    def __init__(self, a, e1, e2, rot, c):
        self.a, self.e1, self.e2, self.rot, self.c = np.asarray(a), e1, e2, rot, np.asarray(c)

    def param(self, eta, om):
        a, e1, e2 = self.a, self.e1, self.e2
        p = np.stack([a[0] * _spow(np.cos(eta), e1) * _spow(np.cos(om), e2),
                      a[1] * _spow(np.cos(eta), e1) * _spow(np.sin(om), e2),
                      a[2] * _spow(np.sin(eta), e1)], -1)
        return p

    def inside_outside(self, x):
        """F(x) - 1 in the local frame: < 0 inside, > 0 outside (the analytic SDF proxy)."""
        loc = (x - self.c) @ self.rot
        a, e1, e2 = self.a, self.e1, self.e2
        t = (np.abs(loc[:, 0] / a[0]) ** (2 / e2) + np.abs(loc[:, 1] / a[1]) ** (2 / e2)) ** (e2 / e1)
        return t + np.abs(loc[:, 2] / a[2]) ** (2 / e1) - 1.0

    def gradient(self, x):
        loc = (x - self.c) @ self.rot
        a, e1, e2 = self.a, self.e1, self.e2
        ax = np.abs(loc[:, 0] / a[0]) + 1e-30
        ay = np.abs(loc[:, 1] / a[1]) + 1e-30
        az = np.abs(loc[:, 2] / a[2]) + 1e-30
        s = ax ** (2 / e2) + ay ** (2 / e2)
        gx = (2 / e1) * s ** (e2 / e1 - 1) * ax ** (2 / e2 - 1) * np.sign(loc[:, 0]) / a[0]
        gy = (2 / e1) * s ** (e2 / e1 - 1) * ay ** (2 / e2 - 1) * np.sign(loc[:, 1]) / a[1]
        gz = (2 / e1) * az ** (2 / e1 - 1) * np.sign(loc[:, 2]) / a[2]
        g = np.stack([gx, gy, gz], 1) @ self.rot.T
        return g

    def sample(self, n, rng):
        """Area-weighted samples: dense parametric grid, area element by finite differences."""
        m = max(4 * n, 20000)
        eta = rng.uniform(-math.pi / 2, math.pi / 2, m)
        om = rng.uniform(-math.pi, math.pi, m)
        h = 1e-4
        p = self.param(eta, om)
        de = (self.param(eta + h, om) - self.param(eta - h, om)) / (2 * h)
        do = (self.param(eta, om + h) - self.param(eta, om - h)) / (2 * h)
        area = np.linalg.norm(np.cross(de, do), axis=1)
        area = np.nan_to_num(area, nan=0.0, posinf=0.0)
        prob = area / area.sum()
        idx = rng.choice(m, size=n, replace=True, p=prob)
        world = p[idx] @ self.rot.T + self.c
        g = self.gradient(world)
        nrm = g / (np.linalg.norm(g, axis=1, keepdims=True) + 1e-30)
        return world, nrm, float(area.mean() * 2 * math.pi * math.pi)


def random_superquadrics(k, rng, scale=(0.1, 0.3), exps=(0.3, 2.0), box=0.5):
    shapes = []
    for _ in range(k):
        a = rng.uniform(*scale, size=3)
        e1, e2 = rng.uniform(*exps, size=2)
        c = rng.uniform(-box + a.max(), box - a.max(), size=3)
        shapes.append(Superquadric(a, e1, e2, _rotation(rng), c))
    return shapes


def superquadrics(n=300000, k=4, seed=0, normal_noise=0.02, pos_noise=0.002):
    """Union of ``k`` random superquadrics in [-0.5, 0.5]^3; points split by surface area."""
    rng = np.random.default_rng(seed)
    shapes = random_superquadrics(k, rng)
    areas = []
    for s in shapes:
        _, _, a = s.sample(2000, np.random.default_rng(seed + 1))
        areas.append(a)
    areas = np.asarray(areas)
    counts = np.floor(n * areas / areas.sum()).astype(int)
    counts[0] += n - counts.sum()
    xs, ns = [], []
    for s, c in zip(shapes, counts):
        x, nn, _ = s.sample(int(c), rng)
        xs.append(x)
        ns.append(nn)
    xyz = np.concatenate(xs)
    nrm = np.concatenate(ns)
    if normal_noise > 0:
        nrm = nrm + rng.normal(0, normal_noise, nrm.shape)
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    if pos_noise > 0:
        xyz = xyz + rng.normal(0, pos_noise, xyz.shape)
    return xyz.astype(np.float32), nrm.astype(np.float32), shapes


def learned_problem(n=3000, n_query=20000, seed=0, pos_noise=0.005, band=0.01):
    """One random superquadric for the learned-basis (Neural Galerkin) training form.

    Returns points (position noise ``pos_noise``), exact unit normals, query points scattered
    around the surface (N(0, band)) and the analytic target field at the queries,
    ``-0.1 * tanh(F(q) / 0.2)`` of the inside-outside function F (positive inside, 0 on the surface).
    """
    rng = np.random.default_rng(seed)
    shape = random_superquadrics(1, rng)[0]
    xyz, nrm, _ = shape.sample(n, rng)
    xyz = xyz + rng.normal(0, pos_noise, xyz.shape)
    q, _, _ = shape.sample(n_query, rng)
    q = q + rng.normal(0, band, q.shape)
    target = -0.1 * np.tanh(shape.inside_outside(q) / 0.2)
    return xyz.astype(np.float32), nrm.astype(np.float32), q.astype(np.float32), target.astype(np.float32)


def room(n=5_000_000, seed=0, size=(8.0, 8.0, 3.0), n_objects=40, noise=0.005):
    """Synthetic room: 4 walls, floor, ceiling and axis-aligned boxes / cylinders (metres)."""
    rng = np.random.default_rng(seed)
    W, D, H = size
    quads = []   # (origin, u, v, normal)
    quads += [((0, 0, 0), (W, 0, 0), (0, D, 0), (0, 0, 1)), ((0, 0, H), (W, 0, 0), (0, D, 0), (0, 0, -1)),
              ((0, 0, 0), (W, 0, 0), (0, 0, H), (0, 1, 0)), ((0, D, 0), (W, 0, 0), (0, 0, H), (0, -1, 0)),
              ((0, 0, 0), (0, D, 0), (0, 0, H), (1, 0, 0)), ((W, 0, 0), (0, D, 0), (0, 0, H), (-1, 0, 0))]
    cyl = []
    for _ in range(n_objects):
        sz = rng.uniform(0.2, 1.5, 3)
        sz[2] = min(sz[2], H - 0.1)
        o = np.array([rng.uniform(0.1, W - sz[0] - 0.1), rng.uniform(0.1, D - sz[1] - 0.1), 0.0])
        if rng.uniform() < 0.5:
            x0, y0, z0 = o
            sx, sy, sz_ = sz
            quads += [((x0, y0, sz_), (sx, 0, 0), (0, sy, 0), (0, 0, 1)),
                      ((x0, y0, 0), (sx, 0, 0), (0, 0, sz_), (0, -1, 0)),
                      ((x0, y0 + sy, 0), (sx, 0, 0), (0, 0, sz_), (0, 1, 0)),
                      ((x0, y0, 0), (0, sy, 0), (0, 0, sz_), (-1, 0, 0)),
                      ((x0 + sx, y0, 0), (0, sy, 0), (0, 0, sz_), (1, 0, 0))]
        else:
            rad = min(sz[0], sz[1]) / 2
            cyl.append((o[0] + rad, o[1] + rad, rad, sz[2]))
    areas = [np.linalg.norm(np.cross(u, v)) for _, u, v, _ in quads] + \
            [2 * math.pi * r * h + math.pi * r * r for _, _, r, h in cyl]
    areas = np.asarray(areas)
    counts = rng.multinomial(n, areas / areas.sum())
    xs, ns = [], []
    for (o, u, v, nn), c in zip(quads, counts[:len(quads)]):
        s, t = rng.uniform(size=(2, c))
        xs.append(np.asarray(o) + s[:, None] * np.asarray(u) + t[:, None] * np.asarray(v))
        ns.append(np.broadcast_to(np.asarray(nn, dtype=np.float64), (c, 3)))
    for (cx, cy, r, h), c in zip(cyl, counts[len(quads):]):
        side = rng.uniform(size=c) < (2 * math.pi * r * h) / (2 * math.pi * r * h + math.pi * r * r)
        th = rng.uniform(0, 2 * math.pi, c)
        z = np.where(side, rng.uniform(0, h, c), h)
        rr = np.where(side, r, r * np.sqrt(rng.uniform(size=c)))
        xs.append(np.stack([cx + rr * np.cos(th), cy + rr * np.sin(th), z], 1))
        ns.append(np.where(side[:, None], np.stack([np.cos(th), np.sin(th), 0 * th], 1), [0, 0, 1]))
    xyz = np.concatenate(xs) + rng.normal(0, noise, (n, 3))
    nrm = np.concatenate(ns)
    return xyz.astype(np.float32), nrm.astype(np.float32)


def serving_stream(n_requests=1024, seed=0, rate=200.0, n_range=(1e3, 5e5), depth_range=(6, 9)):
    """Request descriptors: (arrival_s, n_points, finest_depth, shape_seed)."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    npts = np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]), n_requests)).astype(int)
    depth = rng.integers(depth_range[0], depth_range[1] + 1, n_requests)
    return [dict(arrival=float(a), n=int(p), finest_depth=int(d), seed=int(seed * 100003 + i))
            for i, (a, p, d) in enumerate(zip(arrivals, npts, depth))]


def serving_request(req):
    """Points of one serving request: superquadric/torus union, N(0, 0.003) noise."""
    rng = np.random.default_rng(req["seed"])
    n = req["n"]
    k = int(rng.integers(1, 4))
    xyz, nrm, _ = superquadrics(n - n // 4, k=k, seed=req["seed"], normal_noise=0.0, pos_noise=0.003)
    tx, tn = torus(n // 4, R=rng.uniform(0.15, 0.3), r=rng.uniform(0.05, 0.1), seed=req["seed"] + 7)
    tx = tx + np.float32(0.003) * rng.normal(size=tx.shape).astype(np.float32)
    return np.concatenate([xyz, tx]).astype(np.float32), np.concatenate([nrm, tn]).astype(np.float32)


# ----------------------------------------------------------------------------- serving requests on the GPU
def _spow_t(x, e):
    import torch
    return torch.sign(x) * torch.abs(x) ** e


def serving_request_device(req, device):
    """``serving_request``'s distribution generated on the GPU (seeded torch generator), so that a
    stream of a thousand requests of up to 500k points is produced in seconds: a union of 1-3 random
    superquadrics (area-weighted parametric samples) and a torus (a quarter of the points), exact
    normals, positions with N(0, 0.003) noise.  Returns float32 (xyz, nrm) on ``device``."""
    import torch
    rng = np.random.default_rng(req["seed"])
    n = int(req["n"])
    k = int(rng.integers(1, 4))
    shapes = random_superquadrics(k, rng)
    g = torch.Generator(device=device)
    g.manual_seed(int(req["seed"]))
    f64 = dict(dtype=torch.float64, device=device)
    n_t = n // 4
    n_sq = n - n_t
    # areas of the shapes from a coarse parametric grid
    xs, ns = [], []
    areas, samplers = [], []
    for sh in shapes:
        a = torch.tensor(sh.a, **f64)
        rot = torch.tensor(sh.rot, **f64)
        c = torch.tensor(sh.c, **f64)
        e1, e2 = float(sh.e1), float(sh.e2)

        def param(eta, om, a=a, e1=e1, e2=e2):
            ce, se = _spow_t(torch.cos(eta), e1), _spow_t(torch.sin(eta), e1)
            return torch.stack([a[0] * ce * _spow_t(torch.cos(om), e2), a[1] * ce * _spow_t(torch.sin(om), e2),
                                a[2] * se], -1)

        def area(eta, om, param=param):
            h = 1e-4
            de = (param(eta + h, om) - param(eta - h, om)) / (2 * h)
            do = (param(eta, om + h) - param(eta, om - h)) / (2 * h)
            return torch.nan_to_num(torch.linalg.norm(torch.cross(de, do, dim=-1), dim=-1), nan=0.0, posinf=0.0)
        eta = (torch.rand(20000, generator=g, **f64) - 0.5) * math.pi
        om = (torch.rand(20000, generator=g, **f64) - 0.5) * 2 * math.pi
        areas.append(float(area(eta, om).mean()))
        samplers.append((param, area, rot, c, sh))
    areas = np.asarray(areas)
    counts = np.floor(n_sq * areas / areas.sum()).astype(int)
    counts[0] += n_sq - counts.sum()
    for (param, area, rot, c, sh), m in zip(samplers, counts):
        if m <= 0:
            continue
        cand = max(4 * int(m), 20000)
        eta = (torch.rand(cand, generator=g, **f64) - 0.5) * math.pi
        om = (torch.rand(cand, generator=g, **f64) - 0.5) * 2 * math.pi
        w = area(eta, om)
        cdf = torch.cumsum(w, 0)
        idx = torch.searchsorted(cdf, torch.rand(int(m), generator=g, **f64) * cdf[-1]).clamp_(max=cand - 1)
        p = param(eta[idx], om[idx]) @ rot.T + c
        # outward normal: gradient of the inside-outside function
        loc = (p - c) @ rot
        e1, e2 = float(sh.e1), float(sh.e2)
        a = torch.tensor(sh.a, **f64)
        ax = torch.abs(loc[:, 0] / a[0]) + 1e-30
        ay = torch.abs(loc[:, 1] / a[1]) + 1e-30
        az = torch.abs(loc[:, 2] / a[2]) + 1e-30
        sxy = ax ** (2 / e2) + ay ** (2 / e2)
        gx = (2 / e1) * sxy ** (e2 / e1 - 1) * ax ** (2 / e2 - 1) * torch.sign(loc[:, 0]) / a[0]
        gy = (2 / e1) * sxy ** (e2 / e1 - 1) * ay ** (2 / e2 - 1) * torch.sign(loc[:, 1]) / a[1]
        gz = (2 / e1) * az ** (2 / e1 - 1) * torch.sign(loc[:, 2]) / a[2]
        gn = torch.stack([gx, gy, gz], 1) @ rot.T
        xs.append(p)
        ns.append(gn / (torch.linalg.norm(gn, dim=1, keepdim=True) + 1e-30))
    # torus (area-uniform by rejection on R + r cos v)
    R, r = float(rng.uniform(0.15, 0.3)), float(rng.uniform(0.05, 0.1))
    cand = 3 * n_t + 64
    u = torch.rand(cand, generator=g, **f64) * 2 * math.pi
    v = torch.rand(cand, generator=g, **f64) * 2 * math.pi
    keep = torch.rand(cand, generator=g, **f64) * (R + r) < (R + r * torch.cos(v))
    u, v = u[keep][:n_t], v[keep][:n_t]
    xs.append(torch.stack([(R + r * torch.cos(v)) * torch.cos(u), (R + r * torch.cos(v)) * torch.sin(u),
                           r * torch.sin(v)], 1))
    ns.append(torch.stack([torch.cos(v) * torch.cos(u), torch.cos(v) * torch.sin(u), torch.sin(v)], 1))
    xyz = torch.cat(xs)
    nrm = torch.cat(ns)
    xyz = xyz + 0.003 * torch.randn(xyz.shape, generator=g, **f64)
    return xyz.float().contiguous(), nrm.float().contiguous()
