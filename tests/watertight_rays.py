"""Rays aimed at points of shared mesh edges, for the watertight-mode tests.

Directions are within a few degrees of straight down, so a height field
never shows a silhouette along them: every such ray meets the surface, and a
miss can only be a crack between the two triangles of the edge it was aimed
at (with the reference's Shirley test, 1.8 to 2.6 % of them on the seeded
height fields)."""
from __future__ import annotations

from collections import defaultdict

import numpy as np


def shared_edge_rays(pos, idx, n, seed, spread=0.05):
    cnt = defaultdict(int)
    for t in np.asarray(idx):
        for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
            cnt[(min(a, b), max(a, b))] += 1
    shared = np.array([k for k, v in cnt.items() if v == 2])
    rng = np.random.default_rng(seed)
    e = shared[rng.integers(0, len(shared), n)]
    s = rng.random(n).astype(np.float32)
    pa, pb = pos[e[:, 0]].astype(np.float32), pos[e[:, 1]].astype(np.float32)
    p = (pa + (pb - pa) * s[:, None]).astype(np.float32)
    d = np.c_[rng.normal(size=(n, 2)) * spread, -np.ones(n)]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = (p - d * 2.0).astype(np.float32)
    o4 = np.c_[o, np.zeros(n)].astype(np.float32)
    d4 = np.c_[d, np.full(n, 1e30)].astype(np.float32)
    return o4, d4
