"""Autotuner for batched rendering: sweeps the schedule (the wavefront, with
its wave size and the block shape of the extend / shade / shadow kernels, or
the one-launch persistent renderer) on the actual batch and keeps the fastest
setting (device-synchronised wall time of one ilg_render_batch call, after
one untimed call of the same setting has captured its CUDA graph)."""
from __future__ import annotations

import json
import time


def tune_batch(runner, items, waves=(1 << 20, 1 << 21, 1 << 22, 1 << 23), blocks=(64, 128, 256), repeats=1,
               profile_path=None, one_launch=True):
    results = []
    runner.render_batch(items, paths_per_wave=waves[0], block=blocks[0])  # allocation, first-touch
    settings = [{"paths_per_wave": w, "block": b, "one_launch": False} for w in waves for b in blocks]
    if one_launch:
        runner.render_batch(items, one_launch=True)  # its graph, first-touch
        settings.append({"paths_per_wave": 0, "block": 128, "one_launch": True})
    for st in settings:
        runner.render_batch(items, **st)  # captures this setting's graph
        best = float("inf")
        for _ in range(repeats):
            t0 = time.perf_counter()
            runner.render_batch(items, **st)
            best = min(best, time.perf_counter() - t0)
        results.append(dict(st, seconds=best))
    results.sort(key=lambda r: r["seconds"])
    choice = results[0]
    if profile_path:
        with open(profile_path, "w") as f:
            json.dump({"choice": choice, "sweep": results}, f, indent=1)
    return choice, results
