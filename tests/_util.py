"""Shared helpers of the test suite: seeded ray sets and image statistics."""
from __future__ import annotations

import numpy as np

FLT_MAX = np.float32(3.4028234663852886e38)


def scene_bounds(sc):
    pts = [sc["tri_vertices"].reshape(-1, 3)]
    if sc["spheres"].size:
        s = sc["spheres"]
        pts.append(s[:, :3] - s[:, 3:4])
        pts.append(s[:, :3] + s[:, 3:4])
    p = np.concatenate(pts, 0)
    return p.min(0), p.max(0)


def seeded_rays(sc, n, seed=0):
    """Mixed closest-hit query set: camera-origin rays, rays from random interior points and
    rays leaving surface points (tMin 1e-3, the continuation convention)."""
    rng = np.random.default_rng(seed)
    lo, hi = scene_bounds(sc)
    cam = sc["camera"][:3]
    n1, n2 = n // 3, n // 3
    n3 = n - n1 - n2
    tgt = rng.uniform(lo, hi, (n1, 3))
    d1 = tgt - cam
    o1 = np.tile(cam, (n1, 1))
    o2 = rng.uniform(lo, hi, (n2, 3))
    d2 = rng.normal(0, 1, (n2, 3))
    tv = sc["tri_vertices"].reshape(-1, 3, 3)
    ti = rng.integers(0, tv.shape[0], n3)
    u = rng.uniform(0, 1, n3)
    v = rng.uniform(0, 1, n3)
    flip = u + v > 1
    u[flip], v[flip] = 1 - u[flip], 1 - v[flip]
    p = tv[ti, 0] * (1 - u - v)[:, None] + tv[ti, 1] * u[:, None] + tv[ti, 2] * v[:, None]
    d3 = rng.normal(0, 1, (n3, 3))
    o = np.concatenate([o1, o2, p], 0).astype(np.float32)
    d = np.concatenate([d1, d2, d3], 0).astype(np.float32)
    tmin = np.concatenate([np.zeros(n1), np.full(n2, 1e-4), np.full(n3, 1e-3)]).astype(np.float32)
    tmax = np.full(n, FLT_MAX, np.float32)
    return o, d, tmin, tmax


def pixel_subset(w, h, n, seed=0):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(w * h, size=min(n, w * h), replace=False)).astype(np.int32)


def three_se_pass(mean_a, se_a, mean_b, se_b, floor=1e-6):
    """Fraction of pixel channels with |a - b| <= 3 sqrt(se_a^2 + se_b^2) (+ floor)."""
    tol = 3.0 * np.sqrt(se_a ** 2 + se_b ** 2) + floor
    return float(np.mean(np.abs(mean_a - mean_b) <= tol))


def rel_mse(img, ref):
    """relMSE = mean[(I - I_ref)^2 / (I_ref^2 + 1e-2)]."""
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))
