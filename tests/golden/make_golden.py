"""Generate the golden ray-query fixtures from the reference's own code.

Runs the reference's BasicSpace -> KDTreeMesh and -> BVHMesh closest-hit and
any-hit queries (compiled from the reference tree by oracle/Makefile into
oracle/_ref/libilref.so) on small seeded heightfields and writes their outputs
next to the inputs. The GPU never reads the reference tree; the tests read
these files.

    python tests/golden/make_golden.py     # needs oracle/_ref/libilref.so
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from illuminaprt_b200 import scenes  # noqa: E402
from oracle.bindings import RefLib, build  # noqa: E402

CASES = {
    # name: (nx, ny, amplitude, seed, n_coherent_side, n_incoherent)
    "heightfield_64x32": (64, 32, 0.2, 1, 48, 2304),
    "heightfield_16x8_flat": (16, 8, 0.0, 3, 24, 576),
}


def shadow_segments(pos, idx, n, seed):
    """Segments between random points above the surface (visibility queries)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    a = rng.random((n, 3)) * np.array([1.0, 1.0, 0.3])
    b = rng.random((n, 3)) * np.array([1.0, 1.0, 0.3])
    o4 = np.empty((n, 4), np.float32)
    d4 = np.empty((n, 4), np.float32)
    o4[:, :3] = a
    o4[:, 3] = 1e-4
    d4[:, :3] = b - a
    d4[:, 3] = 1.0 - 1e-4
    return o4, d4


def main():
    build(ref=True)
    ref = RefLib()
    for name, (nx, ny, amp, seed, side, ninc) in CASES.items():
        pos, idx = scenes.heightfield(nx, ny, amp, seed)
        co, cd = scenes.pinhole_rays(side, side, (0.5, -0.6, 0.8), (0.5, 0.5, 0.0), (0, 0, 1), 60.0)
        io, idr = scenes.incoherent_rays(pos, idx, ninc, seed + 1)
        so, sd = shadow_segments(pos, idx, 1024, seed + 2)
        o4 = np.concatenate([co, io]).astype(np.float32)
        d4 = np.concatenate([cd, idr]).astype(np.float32)
        out = dict(pos=pos, idx=idx, o4=o4, d4=d4, so=so, sd=sd)
        for kind in ("kd", "bvh"):
            m = ref.mesh(pos, idx, kind)
            p, t, u, v = m.intersect(o4, d4, nthreads=1)
            out[f"{kind}_prim"], out[f"{kind}_t"], out[f"{kind}_u"], out[f"{kind}_v"] = p, t, u, v
            out[f"{kind}_occ"] = m.occluded(so, sd, nthreads=1)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path), "bytes;", "hits", int((out["kd_prim"] >= 0).sum()), "/", len(o4))


if __name__ == "__main__":
    main()
