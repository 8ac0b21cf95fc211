"""Render the box scene with the reference's own PathIntegrator (compiled from
its sources into oracle/_ref/libilref.so) and store the image as the
path-tracing parity fixture.

    python tests/golden/make_box_golden.py [spp] [seed] [specular] [size]

Default: 256 x 256 at 4096 samples per pixel, seed 1 (about 7 minutes on 8
cores). The GPU path tracer's converged image must match it within
relMSE 1e-3 (tests/test_render_gpu.py). With `specular` = 1 the scene's
short box is a mirror and its tall box glass (scenes.box_scene(True)); the
fixture is named box_specular_<size>_<spp>spp_seed<seed>.npz.
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
    specular = len(sys.argv) > 3 and sys.argv[3] == "1"
    size = int(sys.argv[4]) if len(sys.argv) > 4 else 256
    build(ref=True)
    scene = box_scene(specular)
    t0 = time.time()
    img = RefLib().render_box(scene, size, size, spp, seed)
    dt = time.time() - t0
    name = f"box_specular_{size}" if specular else f"box_{size}"
    path = os.path.join(HERE, f"{name}_{spp}spp_seed{seed}.npz")
    np.savez_compressed(path, image=img, spp=spp, seed=seed, seconds=dt, threads=os.cpu_count())
    print(path, f"{dt:.1f} s", img.mean(axis=(0, 1)))


if __name__ == "__main__":
    main()
