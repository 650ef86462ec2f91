"""Seeded dense SDF inputs of the adaptive-tree fixtures (float32, C order), shared by the fixture
generator and the tests: unions of spheres and boxes on ragged grids, one grid smaller than a root
block and one whose shape is a multiple of 8."""
from __future__ import annotations

import numpy as np

CASES = {
    "spheres_37x41x29": dict(shape=(37, 41, 29), n_spheres=6, n_boxes=0, seed=1),
    "mixed_70x64x53": dict(shape=(70, 64, 53), n_spheres=5, n_boxes=5, seed=2),
    "boxes_64x64x64": dict(shape=(64, 64, 64), n_spheres=0, n_boxes=8, seed=3),
    "tiny_5x9x12": dict(shape=(5, 9, 12), n_spheres=2, n_boxes=1, seed=4),
}


def dense_case(shape, n_spheres, n_boxes, seed):
    """(float32 dense SDF, pitch): union of random spheres and axis-aligned boxes in the unit
    cube, sampled at the vertices i * pitch of a grid with pitch 1 / max(shape)."""
    rng = np.random.default_rng(seed)
    pitch = 1.0 / max(shape)
    grid = np.meshgrid(*[np.arange(n, dtype=np.float64) * pitch for n in shape], indexing="ij")
    x, y, z = grid
    d = np.full(shape, 1.0e3)
    for _ in range(n_spheres):
        c = rng.uniform(0.15, 0.85, 3)
        r = rng.uniform(0.05, 0.2)
        d = np.minimum(d, np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) - r)
    for _ in range(n_boxes):
        c = rng.uniform(0.15, 0.85, 3)
        h = rng.uniform(0.03, 0.15, 3)
        q = np.stack([np.abs(x - c[0]) - h[0], np.abs(y - c[1]) - h[1], np.abs(z - c[2]) - h[2]])
        outside = np.sqrt(np.sum(np.maximum(q, 0.0) ** 2, axis=0))
        inside = np.minimum(np.max(q, axis=0), 0.0)
        d = np.minimum(d, outside + inside)
    return d.astype(np.float32), pitch
