"""Seeded synthetic workloads with the shapes the benchmarks are quoted on.

No public dataset backs these benchmarks; protein-like packing is stood in for by a
jittered cubic lattice:

* ``lattice_balls(n, seed)`` -- 2.9 A lattice, uniform +/-0.4 A jitter per axis
  (numpy ``default_rng(seed)``), cropped to the n points nearest the origin (kept in
  lattice order, which keeps neighbouring balls close in memory).  Radii are i.i.d.
  C 1.75 (p=.62), N 1.55 (p=.17), O 1.52 (p=.19), S 1.80 (p=.02).  Probe 1.4.
* ``periodic_box_balls(n, density, radius, seed)`` -- n balls uniform in a cube of side
  (n / density)^(1/3), all with the same radius; returns the balls and the cube side.
* ``batch_sizes(count, lo, hi, seed)`` -- log-uniform structure sizes.
"""
from __future__ import annotations

import numpy as np

RADII = np.array([1.75, 1.55, 1.52, 1.80])
RADII_P = np.array([0.62, 0.17, 0.19, 0.02])
SPACING = 2.9
JITTER = 0.4
PROBE = 1.4


def lattice_balls(n: int, seed: int = 0) -> np.ndarray:
    """(n, 4) float64 array of x, y, z, r."""
    if n <= 0:
        return np.zeros((0, 4), np.float64)
    rng = np.random.default_rng(seed)
    # side of the lattice cube that holds the sphere of n points with margin
    k = int(np.ceil((n * 6.0 / np.pi) ** (1.0 / 3.0))) + 3
    half = k // 2
    g = np.arange(-half, k - half, dtype=np.float64) * SPACING
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    pts = pts + rng.uniform(-JITTER, JITTER, size=pts.shape)
    d2 = np.einsum("ij,ij->i", pts, pts)
    keep = np.sort(np.argpartition(d2, n - 1)[:n]) if n < len(d2) else np.arange(len(d2))
    radii = rng.choice(RADII, size=len(keep), p=RADII_P)
    return np.ascontiguousarray(np.column_stack([pts[keep], radii]))


def periodic_box_balls(n: int, density: float = 0.033, radius: float = 1.52, seed: int = 0):
    """(balls (n, 4), side) for n balls uniform in a cube at the given number density."""
    side = (n / density) ** (1.0 / 3.0)
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, side, size=(n, 3))
    balls = np.column_stack([pos, np.full(n, radius)])
    return np.ascontiguousarray(balls), side


def batch_sizes(count: int = 4096, lo: int = 300, hi: int = 20000, seed: int = 7) -> np.ndarray:
    """Log-uniform integer sizes in [lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=count)).astype(np.int64)


def x_sign_groups(balls: np.ndarray) -> np.ndarray:
    """Groups 0 for x < 0 and 1 otherwise (the inter-group contacts-only workload)."""
    return np.where(np.asarray(balls)[:, 0] < 0.0, 0, 1).astype(np.int32)
