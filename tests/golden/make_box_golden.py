"""Render the box scene with the reference's own PathIntegrator (compiled from
its sources into oracle/_ref/libilref.so) and store the image as the
path-tracing parity fixture.

    python tests/golden/make_box_golden.py [spp] [seed] [variant] [size]

Default: 256 x 256 at 4096 samples per pixel, seed 1 (about 7 minutes on 8
cores). The GPU path tracer's converged image must match it within
relMSE 1e-3 (tests/test_render_gpu.py). Variants (scenes.box_scene):
  0 / plain   the box scene: box_<size>_<spp>spp_seed<seed>.npz
  1 / specular  short box a mirror, tall box glass: box_specular_...
  meshlight   the ceiling light a 6-triangle mesh of unequal triangles
              (DiffuseAreaLight on a triangle mesh): box_meshlight_...
  infinite    the specular box plus an InfiniteAreaLight of intensity
              (0.5, 0.6, 0.8), camera at 60 deg so border pixels see past
              the box: box_infinite_...
The mesh-light and infinite-light fixtures also hold the RadianceContext's
Direct ("direct").
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


VARIANTS = {
    "plain": ("box", lambda: box_scene()),
    "specular": ("box_specular", lambda: box_scene(True)),
    "meshlight": ("box_meshlight", lambda: box_scene(light="mesh")),
    "infinite": ("box_infinite", lambda: box_scene(True, infinite=(0.5, 0.6, 0.8), fov=60.0)),
}


def main():
    spp = int(sys.argv[1]) if len(sys.argv) > 1 else 4096
    seed = int(sys.argv[2]) if len(sys.argv) > 2 else 1
    variant = sys.argv[3] if len(sys.argv) > 3 else "plain"
    variant = {"0": "plain", "1": "specular"}.get(variant, variant)
    size = int(sys.argv[4]) if len(sys.argv) > 4 else 256
    build(ref=True)
    prefix, make = VARIANTS[variant]
    scene = make()
    t0 = time.time()
    extra = {}
    if variant in ("plain", "specular"):
        img = RefLib().render_box(scene, size, size, spp, seed)
    else:
        img, direct, _ = RefLib().render_box_lights(scene, size, size, spp, seed)
        extra["direct"] = direct
    dt = time.time() - t0
    path = os.path.join(HERE, f"{prefix}_{size}_{spp}spp_seed{seed}.npz")
    np.savez_compressed(path, image=img, spp=spp, seed=seed, seconds=dt, threads=os.cpu_count(), **extra)
    print(path, f"{dt:.1f} s", img.mean(axis=(0, 1)))


if __name__ == "__main__":
    main()
