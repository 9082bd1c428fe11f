"""Shared fixtures and helpers for the test-suite."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

RING_17 = [  # the C++ API example ring (src/tessellation.rs:743-761)
    (0.0, 0.0, 2.0, 1.0), (0.0, 1.0, 0.0, 0.5), (0.382683, 0.92388, 0.0, 0.5),
    (0.707107, 0.707107, 0.0, 0.5), (0.92388, 0.382683, 0.0, 0.5), (1.0, 0.0, 0.0, 0.5),
    (0.92388, -0.382683, 0.0, 0.5), (0.707107, -0.707107, 0.0, 0.5), (0.382683, -0.92388, 0.0, 0.5),
    (0.0, -1.0, 0.0, 0.5), (-0.382683, -0.92388, 0.0, 0.5), (-0.707107, -0.707107, 0.0, 0.5),
    (-0.92388, -0.382683, 0.0, 0.5), (-1.0, 0.0, 0.0, 0.5), (-0.92388, 0.382683, 0.0, 0.5),
    (-0.707107, 0.707107, 0.0, 0.5), (-0.382683, 0.92388, 0.0, 0.5),
]
CENTRAL_POINTS = [[0.0, 0.0, 0.0], [2.5, 0.0, 0.0], [1.25, 2.0, 0.0], [1.25, 0.8, 2.0],
                  [0.0, 2.5, 1.0], [2.5, 2.5, 1.0], [1.25, -1.5, 1.0], [3.5, 1.25, 1.0]]
THREE_LINE = [(0.0, 0.0, 0.0, 1.0), (2.0, 0.0, 0.0, 1.0), (4.0, 0.0, 0.0, 1.0)]


def goldens():
    with open(os.path.join(GOLDEN, "goldens.json")) as f:
        return json.load(f)


def load_balls(name):
    return np.load(os.path.join(GOLDEN, f"balls_{name}.npy"))


def central_golden():
    return np.load(os.path.join(GOLDEN, "central_golden.npy"))


def contact_lookup(res_a, res_b, a, b):
    idx = np.where((np.asarray(res_a) == a) & (np.asarray(res_b) == b))[0]
    return int(idx[0]) if len(idx) else None


def sunflower(k, R=4.0, d=5.0, rr=1.0, rho=3.6):
    """Two large balls whose contact is cut by k small balls on a ring around it: the
    contact's contour has k points (touching small balls) or 2k (arcs between them), more
    than a warp holds for k > 32, which exercises the serial contour fallback."""
    balls = [(0.0, 0.0, 0.0, R), (d, 0.0, 0.0, R)]
    for i in range(k):
        t = 2 * np.pi * i / k
        balls.append((d / 2, rho * np.cos(t), rho * np.sin(t), rr))
    return np.array(balls, float)


def big_ball_in_lattice(big_r=10.0, spacing=2.5, half=14.0, small_r=1.6, seed=0):
    """A ball of radius big_r at the origin inside a jittered lattice of small balls: the
    big ball has several hundred neighbour candidates (more than a warp sorts at once)."""
    rng = np.random.default_rng(seed)
    g = np.arange(-half, half + 1e-9, spacing)
    pts = np.array(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1).T
    pts = pts + rng.uniform(-0.3, 0.3, pts.shape)
    small = np.column_stack([pts, np.full(len(pts), small_r)])
    return np.vstack([[0.0, 0.0, 0.0, big_r], small])
