"""Seeded synthetic point clouds with the shapes, sizes and distributions of
the benchmark workloads.  No public dataset is involved; every cloud is drawn
here from a fixed seed.

* `sphere`         — the unit-sphere cloud of the reference README (README.md:62-72):
                     z ~ U(-1, 1), theta ~ U(0, 2 pi) drawn in that order, normals = points.
* `torus`          — area-uniform samples on a torus (major R, minor r) with Gaussian
                     position noise and outward normals scaled by a confidence U(lo, hi).
* `sphere_union`   — samples on the outer surface of a union of random spheres.
* `ellipsoid`      — area-weighted samples on a random ellipsoid.
* `batch_clouds`   — many clouds of uneven size and depth (ellipsoids and tori).
* `serving_stream` — Poisson arrivals of requests with log-normal sizes.
"""

from __future__ import annotations

import numpy as np


def sphere(count: int = 2000, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    rng = np.random.default_rng(seed)
    z = rng.uniform(-1.0, 1.0, count)
    theta = rng.uniform(0.0, 2.0 * np.pi, count)
    r = np.sqrt(1.0 - z * z)
    pts = np.ascontiguousarray(np.column_stack((r * np.cos(theta), r * np.sin(theta), z)))
    return pts, pts.copy()


def torus(count: int = 1_000_000, seed: int = 1, major: float = 0.6, minor: float = 0.25,
          noise: float = 0.002, confidence: tuple[float, float] | None = (0.5, 1.5),
          rng: np.random.Generator | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Area-uniform torus samples: the tube angle phi is drawn by rejection with
    acceptance (R + r cos phi) / (R + r), the angle around the axis uniformly."""
    rng = np.random.default_rng(seed) if rng is None else rng
    phis = np.empty(0)
    while phis.size < count:
        want = int((count - phis.size) * 1.4) + 16
        phi = rng.uniform(0.0, 2.0 * np.pi, want)
        keep = rng.uniform(0.0, 1.0, want) < (major + minor * np.cos(phi)) / (major + minor)
        phis = np.concatenate([phis, phi[keep]])
    phi = phis[:count]
    theta = rng.uniform(0.0, 2.0 * np.pi, count)
    ring = major + minor * np.cos(phi)
    pts = np.column_stack((ring * np.cos(theta), ring * np.sin(theta), minor * np.sin(phi)))
    nrm = np.column_stack((np.cos(phi) * np.cos(theta), np.cos(phi) * np.sin(theta), np.sin(phi)))
    if noise > 0:
        pts = pts + rng.normal(0.0, noise, size=pts.shape)
    if confidence is not None:
        nrm = nrm * rng.uniform(confidence[0], confidence[1], size=(count, 1))
    return np.ascontiguousarray(pts), np.ascontiguousarray(nrm)


def _unit_vectors(rng: np.random.Generator, count: int) -> np.ndarray:
    v = rng.normal(size=(count, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def sphere_union(count: int = 20_000_000, spheres: int = 64, seed: int = 2,
                 noise: float = 0.0005) -> tuple[np.ndarray, np.ndarray]:
    """Samples on the boundary of a union of spheres (centres U(-0.7, 0.7)^3,
    radii U(0.05, 0.25)); samples per sphere proportional to r^2; samples that
    fall strictly inside another sphere are dropped and topped up."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-0.7, 0.7, size=(spheres, 3))
    radii = rng.uniform(0.05, 0.25, size=spheres)
    share = radii**2 / np.sum(radii**2)
    out_p, out_n, have = [], [], 0
    while have < count:
        want = int((count - have) * 1.3) + 64
        which = rng.choice(spheres, size=want, p=share)
        u = _unit_vectors(rng, want)
        p = centres[which] + u * radii[which, None]
        inside = np.zeros(want, dtype=bool)
        for s in range(spheres):
            d2 = np.sum((p - centres[s]) ** 2, axis=1)
            inside |= (d2 < radii[s] ** 2 * (1 - 1e-12)) & (which != s)
        p, u = p[~inside], u[~inside]
        out_p.append(p)
        out_n.append(u)
        have += len(p)
    pts = np.concatenate(out_p)[:count]
    nrm = np.concatenate(out_n)[:count]
    if noise > 0:
        pts = pts + rng.normal(0.0, noise, size=pts.shape)
    return np.ascontiguousarray(pts), np.ascontiguousarray(nrm)


def ellipsoid(count: int, rng: np.random.Generator, axes=None) -> tuple[np.ndarray, np.ndarray]:
    """Random ellipsoid (semi-axes U(0.2, 0.9)); area-weighted by rejection on
    the surface-element ratio; outward normals."""
    axes = rng.uniform(0.2, 0.9, size=3) if axes is None else np.asarray(axes, np.float64)
    pts_all, nrm_all, have = [], [], 0
    while have < count:
        want = int((count - have) * 2.2) + 16
        u = _unit_vectors(rng, want)
        g = u / axes  # gradient direction of x^2/a^2 at p = a*u, up to scale
        element = np.linalg.norm(u * axes[[1, 2, 0]] * axes[[2, 0, 1]], axis=1)
        keep = rng.uniform(0.0, element.max(), want) < element
        p = (u * axes)[keep]
        n = g[keep] / np.linalg.norm(g[keep], axis=1, keepdims=True)
        pts_all.append(p)
        nrm_all.append(n)
        have += len(p)
    return (np.ascontiguousarray(np.concatenate(pts_all)[:count]),
            np.ascontiguousarray(np.concatenate(nrm_all)[:count]))


def batch_clouds(clouds: int = 256, seed: int = 3, min_points: int = 1_000,
                 max_points: int = 200_000, depths=(5, 6, 7, 8)):
    """Uneven batch: sizes log-uniform in [min, max], depths uniform over
    `depths`, shapes random ellipsoids or tori.  Yields (points, normals, depth)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(clouds):
        size = int(np.exp(rng.uniform(np.log(min_points), np.log(max_points))))
        depth = int(rng.choice(depths))
        if rng.uniform() < 0.5:
            p, n = ellipsoid(size, rng)
        else:
            major = rng.uniform(0.4, 0.7)
            p, n = torus(size, major=major, minor=rng.uniform(0.1, 0.35) * major, noise=0.0,
                         confidence=None, rng=rng)
        out.append((p, n, depth))
    return out


def serving_stream(rate: float = 200.0, duration: float = 60.0, seed: int = 4,
                   median: int = 50_000, sigma: float = 1.0, min_points: int = 1_000,
                   max_points: int = 2_000_000, depths=(6, 7, 8, 9)):
    """Poisson arrivals: returns a list of (arrival_s, size, depth, shape) tuples;
    the cloud itself is drawn when the request is built (`request_cloud`)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        size = int(np.clip(np.exp(rng.normal(np.log(median), sigma)), min_points, max_points))
        depth = int(rng.choice(depths))
        shape = ("ellipsoid", "torus", "sphere_union")[int(rng.integers(3))]
        out.append((t, size, depth, shape, int(rng.integers(2**31))))
    return out


def request_cloud(size: int, shape: str, seed: int) -> tuple[np.ndarray, np.ndarray]:
    rng = np.random.default_rng(seed)
    if shape == "ellipsoid":
        return ellipsoid(size, rng)
    if shape == "torus":
        return torus(size, noise=0.0, confidence=None, rng=rng)
    return sphere_union(size, spheres=8, seed=seed, noise=0.0)
