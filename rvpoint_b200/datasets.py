"""Seeded synthetic point clouds with the shapes of the five benchmark workloads.

No public dataset is involved: every cloud is drawn from numpy's PCG64 with a
fixed seed, in float64, and rounded once to float32. The shapes are:

* ``room_cloud``       100,000 pts: floor + two walls (70%), a sphere (28%),
                       uniform outliers (2%), sigma = 2 mm.
* ``lidar_frame``      one 64-beam x 2048-azimuth spinning-LiDAR sweep cast
                       against a ground plane and 40 boxes, sigma = 2 cm range
                       noise, 5% dropped returns.
* ``lidar_batch``      many such frames, each thinned to a log-uniform size in
                       [20k, 131k] points.
* ``precision_room``   2,000,000 pts: 8x6x3 m room + 200 spheres/cylinders,
                       sigma = 1 mm, translated by (1e4, 1e4, 0).
* ``plane_scenes``     scenes of 1-6 planes in a 10 m cube with 30-70%
                       uniform outliers, sigma = 5 mm.

Clouds are returned as ``Cloud`` (three contiguous float32 arrays, SoA), the
layout the library consumes.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

SEED_BASE = 1000  # workload i uses seed SEED_BASE + i


@dataclasses.dataclass
class Cloud:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    @staticmethod
    def from_xyz(p: np.ndarray) -> "Cloud":
        p = np.asarray(p, dtype=np.float32)
        return Cloud(np.ascontiguousarray(p[:, 0]), np.ascontiguousarray(p[:, 1]),
                     np.ascontiguousarray(p[:, 2]))

    def aos(self) -> np.ndarray:
        return np.ascontiguousarray(np.stack([self.x, self.y, self.z], axis=1))

    def subset(self, idx) -> "Cloud":
        return Cloud(np.ascontiguousarray(self.x[idx]), np.ascontiguousarray(self.y[idx]),
                     np.ascontiguousarray(self.z[idx]))


@dataclasses.dataclass
class Batch:
    """Frames concatenated SoA; frame f owns points offsets[f]:offsets[f+1]."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    offsets: np.ndarray  # int64, n_frames + 1

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    @property
    def n_frames(self) -> int:
        return int(self.offsets.shape[0] - 1)

    def frame(self, f: int) -> Cloud:
        a, b = int(self.offsets[f]), int(self.offsets[f + 1])
        return Cloud(self.x[a:b], self.y[a:b], self.z[a:b])

    @staticmethod
    def from_frames(frames) -> "Batch":
        """Concatenate clouds into one batch, in the given order."""
        offs = np.zeros(len(frames) + 1, np.int64)
        offs[1:] = np.cumsum([f.n for f in frames])
        cat = lambda a: np.ascontiguousarray(np.concatenate(a), np.float32)  # noqa: E731
        return Batch(cat([f.x for f in frames]), cat([f.y for f in frames]),
                     cat([f.z for f in frames]), offs)


def _f32(p: np.ndarray) -> Cloud:
    return Cloud.from_xyz(p.astype(np.float32))


# --------------------------------------------------------------------------
# Indoor room (workload 0)
# --------------------------------------------------------------------------
def room_cloud(n: int = 100_000, seed: int = SEED_BASE + 0) -> Cloud:
    rng = np.random.Generator(np.random.PCG64(seed))
    n_planes = int(round(0.70 * n))
    n_sphere = int(round(0.28 * n))
    n_out = n - n_planes - n_sphere
    # floor (16 m^2) and two 4x3 walls (12 m^2 each), chosen by area
    which = rng.choice(3, size=n_planes, p=np.array([16.0, 12.0, 12.0]) / 40.0)
    u = rng.uniform(0.0, 1.0, size=(n_planes, 2))
    pts = np.empty((n_planes, 3))
    f = which == 0
    pts[f] = np.stack([4 * u[f, 0], 4 * u[f, 1], np.zeros(f.sum())], 1)
    w = which == 1  # wall x = 0
    pts[w] = np.stack([np.zeros(w.sum()), 4 * u[w, 0], 3 * u[w, 1]], 1)
    w = which == 2  # wall y = 0
    pts[w] = np.stack([4 * u[w, 0], np.zeros(w.sum()), 3 * u[w, 1]], 1)
    d = rng.normal(size=(n_sphere, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    sph = np.array([2.0, 2.0, 1.0]) + 0.5 * d
    surf = np.concatenate([pts, sph], 0)
    surf += rng.normal(0.0, 0.002, size=surf.shape)
    out = rng.uniform(0.0, 1.0, size=(n_out, 3)) * np.array([4.0, 4.0, 3.0])
    allp = np.concatenate([surf, out], 0)
    allp = allp[rng.permutation(allp.shape[0])]
    return _f32(allp)


# --------------------------------------------------------------------------
# Spinning LiDAR (workloads 1 and 2)
# --------------------------------------------------------------------------
GROUND_Z = -1.7
MAX_RANGE = 120.0


def _boxes(rng, n_boxes=40, radius=60.0):
    lo = np.empty((n_boxes, 3))
    hi = np.empty((n_boxes, 3))
    b = 0
    while b < n_boxes:
        side = rng.uniform(1.0, 5.0, size=3)
        r = radius * math.sqrt(rng.uniform())
        th = rng.uniform(0.0, 2 * math.pi)
        cx, cy = r * math.cos(th), r * math.sin(th)
        # keep the sensor outside every box, with a margin
        if math.hypot(cx, cy) < 3.0 + 0.75 * math.hypot(side[0], side[1]):
            continue
        lo[b] = (cx - side[0] / 2, cy - side[1] / 2, GROUND_Z)
        hi[b] = (cx + side[0] / 2, cy + side[1] / 2, GROUND_Z + side[2])
        b += 1
    return lo, hi


def lidar_frame(seed: int = SEED_BASE + 1, beams: int = 64, azimuths: int = 2048,
                drop: float = 0.05, sigma: float = 0.02) -> Cloud:
    rng = np.random.Generator(np.random.PCG64(seed))
    lo, hi = _boxes(rng)
    elev = np.deg2rad(np.linspace(-25.0, 3.0, beams))
    az = (np.arange(azimuths) + rng.uniform()) * (2 * math.pi / azimuths)
    ce, se = np.cos(elev)[:, None], np.sin(elev)[:, None]
    dx = (ce * np.cos(az)[None, :]).ravel()
    dy = (ce * np.sin(az)[None, :]).ravel()
    dz = np.broadcast_to(se, (beams, azimuths)).ravel()
    d = np.stack([dx, dy, dz], 1)
    t = np.full(d.shape[0], np.inf)
    down = dz < 0
    t[down] = GROUND_Z / dz[down]
    inv = 1.0 / np.where(d == 0.0, 1e-30, d)
    cols = np.arange(beams)[:, None] * azimuths
    step = 2 * math.pi / azimuths
    for b in range(lo.shape[0]):
        # only azimuth columns inside the box's angular span can hit it (the
        # sensor is outside every box, so the span is below pi)
        cx = np.array([lo[b, 0], hi[b, 0], lo[b, 0], hi[b, 0]])
        cy = np.array([lo[b, 1], lo[b, 1], hi[b, 1], hi[b, 1]])
        ang = np.arctan2(cy, cx)
        ref = ang[0]
        rel = (ang - ref + math.pi) % (2 * math.pi) - math.pi
        a0, a1 = ref + rel.min(), ref + rel.max()
        j0 = int(math.floor(a0 / step)) - 2
        j1 = int(math.ceil(a1 / step)) + 2
        js = np.arange(j0, j1 + 1) % azimuths
        r = (cols + js[None, :]).ravel()
        t0 = lo[b][None, :] * inv[r]
        t1 = hi[b][None, :] * inv[r]
        tmin = np.minimum(t0, t1).max(axis=1)
        tmax = np.maximum(t0, t1).min(axis=1)
        hit = (tmin <= tmax) & (tmin > 0.0) & (tmin < t[r])
        t[r[hit]] = tmin[hit]
    keep = np.isfinite(t) & (t < MAX_RANGE)
    keep &= rng.uniform(size=t.shape[0]) >= drop
    t = t + rng.normal(0.0, sigma, size=t.shape[0])
    p = d[keep] * t[keep, None]
    return _f32(p)


def lidar_batch(n_frames: int = 256, seed: int = SEED_BASE + 2, min_pts: int = 20_000,
                max_pts: int = 131_072) -> Batch:
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = np.exp(rng.uniform(math.log(min_pts), math.log(max_pts), size=n_frames))
    xs, ys, zs, offs = [], [], [], [0]
    for f in range(n_frames):
        fr = lidar_frame(seed=seed * 100_003 + f)
        m = min(int(sizes[f]), fr.n)
        sel = np.sort(rng.choice(fr.n, size=m, replace=False))
        xs.append(fr.x[sel]); ys.append(fr.y[sel]); zs.append(fr.z[sel])
        offs.append(offs[-1] + m)
    return Batch(np.concatenate(xs), np.concatenate(ys), np.concatenate(zs),
                 np.asarray(offs, dtype=np.int64))


# --------------------------------------------------------------------------
# Precision stress room (workload 3)
# --------------------------------------------------------------------------
def precision_room(n: int = 2_000_000, seed: int = SEED_BASE + 3, n_objects: int = 200,
                   shift=(1.0e4, 1.0e4, 0.0), sigma: float = 0.001) -> Cloud:
    rng = np.random.Generator(np.random.PCG64(seed))
    L, W, H = 8.0, 6.0, 3.0
    # six room planes: (area, sampler)
    planes = [
        (L * W, lambda u: np.stack([L * u[:, 0], W * u[:, 1], 0 * u[:, 0]], 1)),
        (L * W, lambda u: np.stack([L * u[:, 0], W * u[:, 1], H + 0 * u[:, 0]], 1)),
        (L * H, lambda u: np.stack([L * u[:, 0], 0 * u[:, 0], H * u[:, 1]], 1)),
        (L * H, lambda u: np.stack([L * u[:, 0], W + 0 * u[:, 0], H * u[:, 1]], 1)),
        (W * H, lambda u: np.stack([0 * u[:, 0], W * u[:, 0], H * u[:, 1]], 1)),
        (W * H, lambda u: np.stack([L + 0 * u[:, 0], W * u[:, 0], H * u[:, 1]], 1)),
    ]
    objs = []
    for _ in range(n_objects):
        r = rng.uniform(0.05, 0.5)
        kind = int(rng.integers(0, 2))
        c = np.array([rng.uniform(r + 0.1, L - r - 0.1), rng.uniform(r + 0.1, W - r - 0.1),
                      rng.uniform(r + 0.1, H - r - 0.1)])
        if kind == 0:
            objs.append(("sphere", 4 * math.pi * r * r, c, r, 0.0))
        else:
            h = rng.uniform(0.2, min(2.0, H - 0.2))
            c[2] = rng.uniform(0.05, H - h - 0.05)
            objs.append(("cyl", 2 * math.pi * r * h, c, r, h))
    n_room = int(0.6 * n)
    n_obj = n - n_room
    pa = np.array([a for a, _ in planes])
    cnt = rng.multinomial(n_room, pa / pa.sum())
    parts = [s(rng.uniform(size=(m, 2))) for (_, s), m in zip(planes, cnt)]
    oa = np.array([o[1] for o in objs])
    ocnt = rng.multinomial(n_obj, oa / oa.sum())
    for (kind, _, c, r, h), m in zip(objs, ocnt):
        if kind == "sphere":
            d = rng.normal(size=(m, 3))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            parts.append(c + r * d)
        else:
            th = rng.uniform(0, 2 * math.pi, size=m)
            zz = rng.uniform(0, h, size=m)
            parts.append(np.stack([c[0] + r * np.cos(th), c[1] + r * np.sin(th), c[2] + zz], 1))
    p = np.concatenate(parts, 0)
    p += rng.normal(0.0, sigma, size=p.shape)
    p = p[rng.permutation(p.shape[0])]
    p = p + np.asarray(shift)[None, :]
    return _f32(p)


# --------------------------------------------------------------------------
# Plane scenes for the learned proposal (workload 4)
# --------------------------------------------------------------------------
def plane_scene(seed: int, n: int = 50_000, size: float = 10.0, sigma: float = 0.005):
    """One scene; returns (Cloud, plane_label) with label -1 for outliers."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n_planes = int(rng.integers(1, 7))
    out_frac = rng.uniform(0.3, 0.7)
    n_out = int(round(out_frac * n))
    n_in = n - n_out
    w = rng.dirichlet(np.ones(n_planes) * 2.0)
    cnt = rng.multinomial(n_in, w)
    pts, lab = [], []
    for k in range(n_planes):
        nrm = rng.normal(size=3)
        nrm /= np.linalg.norm(nrm)
        anchor = rng.uniform(0.2 * size, 0.8 * size, size=3)
        got = np.empty((0, 3))
        while got.shape[0] < cnt[k]:
            q = rng.uniform(0, size, size=(max(4 * (cnt[k] - got.shape[0]), 64), 3))
            q = q - ((q - anchor) @ nrm)[:, None] * nrm[None, :]
            ok = np.all((q >= 0) & (q <= size), axis=1)
            got = np.concatenate([got, q[ok]], 0)
        got = got[: cnt[k]] + rng.normal(0, sigma, size=(cnt[k], 1)) * nrm[None, :]
        pts.append(got)
        lab.append(np.full(cnt[k], k))
    pts.append(rng.uniform(0, size, size=(n_out, 3)))
    lab.append(np.full(n_out, -1))
    p = np.concatenate(pts, 0)
    lab = np.concatenate(lab)
    perm = rng.permutation(n)
    return _f32(p[perm]), lab[perm]


def plane_scenes(n_scenes: int = 512, n: int = 50_000, seed: int = SEED_BASE + 4):
    return [plane_scene(seed * 100_003 + s, n=n) for s in range(n_scenes)]


def plane_batch(n_scenes: int = 512, n: int = 50_000, seed: int = SEED_BASE + 4) -> Batch:
    """plane_scenes concatenated into one Batch (scene s = frame s)."""
    sc = plane_scenes(n_scenes=n_scenes, n=n, seed=seed)
    offs = np.zeros(n_scenes + 1, np.int64)
    offs[1:] = np.cumsum([c.n for c, _ in sc])
    return Batch(np.concatenate([c.x for c, _ in sc]), np.concatenate([c.y for c, _ in sc]),
                 np.concatenate([c.z for c, _ in sc]), offs)
