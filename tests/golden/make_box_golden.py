"""Render the box scene with the reference's own PathIntegrator (compiled from
its sources into oracle/_ref/libilref.so) and store the image as the
path-tracing parity fixture.

    python tests/golden/make_box_golden.py [spp] [seed]

Default: 256 x 256 at 4096 samples per pixel, seed 1 (about 7 minutes on 8
cores). The GPU path tracer's converged image must match it within
relMSE 1e-3 (tests/test_render_gpu.py).
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from illuminaprt_b200.scenes import box_scene  # noqa: E402
from oracle.bindings import RefLib, build  # noqa: E402


def main():
    spp = int(sys.argv[1]) if len(sys.argv) > 1 else 4096
    seed = int(sys.argv[2]) if len(sys.argv) > 2 else 1
    build(ref=True)
    scene = box_scene()
    t0 = time.time()
    img = RefLib().render_box(scene, 256, 256, spp, seed)
    dt = time.time() - t0
    path = os.path.join(HERE, f"box_256_{spp}spp_seed{seed}.npz")
    np.savez_compressed(path, image=img, spp=spp, seed=seed, seconds=dt, threads=os.cpu_count())
    print(path, f"{dt:.1f} s", img.mean(axis=(0, 1)))


if __name__ == "__main__":
    main()
