"""Autotuner for batched rendering: sweeps the wavefront size and the block
shape of the extend / shade / shadow kernels on the actual batch and keeps the
fastest setting (device-synchronised wall time of one ilg_render_batch call)."""
from __future__ import annotations

import json
import time


def tune_batch(runner, items, waves=(1 << 20, 1 << 21, 1 << 22, 1 << 23), blocks=(64, 128, 256), repeats=1,
               profile_path=None):
    results = []
    runner.render_batch(items, paths_per_wave=waves[0], block=blocks[0])  # allocation, first-touch
    for w in waves:
        for b in blocks:
            best = float("inf")
            for _ in range(repeats):
                t0 = time.perf_counter()
                runner.render_batch(items, paths_per_wave=w, block=b)
                best = min(best, time.perf_counter() - t0)
            results.append({"paths_per_wave": w, "block": b, "seconds": best})
    results.sort(key=lambda r: r["seconds"])
    choice = results[0]
    if profile_path:
        with open(profile_path, "w") as f:
            json.dump({"choice": choice, "sweep": results}, f, indent=1)
    return choice, results
