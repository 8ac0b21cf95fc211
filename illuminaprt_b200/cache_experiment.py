"""Equal-time comparison of the radiance-cached path tracer with plain path
tracing, both against a high-sample plain render as ground truth.

    relMSE(x, gt) = mean over pixels and channels of (x - gt)^2 / (gt^2 + 0.01)

The cached run renders `frames` frames of `spp_per_frame` samples each: every
frame stops its rendering paths into the cache at vertex `cache_depth` and
then trains the cache on the records of its training paths (one in
`train_every`); frames after `warmup` are averaged. The plain run renders
frames of the same size until it has used as much wall time as the whole
cached run (its warm-up and training included), and averages them all.
"""
from __future__ import annotations

import time

import numpy as np


def rel_mse(x, gt, eps=1e-2):
    x = np.asarray(x, np.float64)
    gt = np.asarray(gt, np.float64)
    return float(np.mean((x - gt) ** 2 / (gt ** 2 + eps)))


def equal_time(space, scene, width, height, gt, frames=64, warmup=8, spp_per_frame=1, cache_depth=1,
               train_every=16, train_steps=4, train_batch=16384, max_depth=12, seed=100, lr=1e-2,
               ablate_training=False, train_tail=0, device_accumulate=False, train_epochs=1, hash_cache=False):
    """device_accumulate: frames are rendered into a device tensor and summed
    on the device (as a progressive renderer's accumulation buffer would be),
    with a synchronisation after every frame in both runs; otherwise each
    frame comes back to the host and is summed there."""
    cam = dict(scene["camera"], aspect=width / height)
    sky = scene.get("sky", (0.0, 0.0, 0.0))
    kw = dict(max_depth=max_depth, sky=sky)
    out = acc_dev = None
    if device_accumulate:
        import torch
        out = torch.empty((height, width, 3), dtype=torch.float32, device=f"cuda:{space.device}")
        acc_dev = torch.zeros((height, width, 3), dtype=torch.float64, device=out.device)

    def frame(**args):
        """One frame, summed into the accumulator when `keep`."""
        keep = args.pop("keep")
        if device_accumulate:
            space.render(cam, width, height, spp_per_frame, out=out, **args, **kw)
            if keep:
                acc_dev.add_(out)
            space.sync()
            return None
        img = space.render(cam, width, height, spp_per_frame, **args, **kw)
        return img if keep else None

    def reset():
        if device_accumulate:
            acc_dev.zero_()
        return np.zeros((height, width, 3))

    def result(acc, n):
        total = acc_dev.cpu().numpy() if device_accumulate else acc
        return total / max(1, n)

    cache_kw = dict(cache_depth=cache_depth, train_every=train_every,
                    train_steps=0 if ablate_training else train_steps, train_batch=train_batch,
                    train_tail=train_tail, train_epochs=train_epochs, hash_cache=hash_cache)
    reset_cache = space.hash_cache_reset if hash_cache else (lambda: space.mlp_init(seed=seed, lr=lr))
    reset_cache()
    # untimed: first call allocates the wavefront and cache buffers
    frame(seed=seed + 99991, keep=False, **cache_kw)
    reset_cache()
    acc = reset()
    n_acc = 0
    t0 = time.perf_counter()
    for f in range(frames):
        img = frame(seed=seed + f, keep=f >= warmup, **cache_kw)
        if f >= warmup:
            if img is not None:
                acc += img
            n_acc += 1
    t_cache = time.perf_counter() - t0
    cached = result(acc, n_acc)
    # plain path tracing for the same wall time
    frame(seed=seed + 77777, keep=False)
    acc = reset()
    n_plain = 0
    t0 = time.perf_counter()
    while True:
        img = frame(seed=seed + 500000 + n_plain, keep=True)
        if img is not None:
            acc += img
        n_plain += 1
        if time.perf_counter() - t0 >= t_cache:
            break
    t_plain = time.perf_counter() - t0
    plain = result(acc, n_plain)
    e_plain, e_cache = rel_mse(plain, gt), rel_mse(cached, gt)
    return {
        "relmse_plain": e_plain,
        "relmse_cached": e_cache,
        "gain": e_plain / e_cache if e_cache > 0 else float("inf"),
        "bias_cached": (cached.mean((0, 1)) / gt.mean((0, 1)) - 1.0).tolist(),
        "bias_plain": (plain.mean((0, 1)) / gt.mean((0, 1)) - 1.0).tolist(),
        "seconds_cached": t_cache, "seconds_plain": t_plain,
        "frames_cached": frames, "frames_plain": n_plain, "spp_per_frame": spp_per_frame,
        "plain_spp_total": n_plain * spp_per_frame, "cached_spp_averaged": n_acc * spp_per_frame,
        "cached_image": cached, "plain_image": plain,
    }


# The wavefront's default size (ilg_render_opts::paths_per_wave = 0): a plain
# call of at least this many paths keeps the device at full throughput.
FULL_WAVE_PATHS = 1 << 22


def plain_at_budget(space, scene, width, height, budget_s, seed=500000, max_depth=12, spp_per_call=None):
    """Plain path tracing given `budget_s` seconds of wall time: calls of
    `spp_per_call` samples per pixel (default: enough to fill a wave), summed
    on the device, until the budget is spent (the last call may end past
    it). Returns (image, seconds, total spp)."""
    import torch
    cam = dict(scene["camera"], aspect=width / height)
    kw = dict(max_depth=max_depth, sky=scene.get("sky", (0.0, 0.0, 0.0)))
    spp = spp_per_call or max(1, -(-FULL_WAVE_PATHS // (width * height)))
    out = torch.empty((height, width, 3), dtype=torch.float32, device=f"cuda:{space.device}")
    acc = torch.zeros((height, width, 3), dtype=torch.float64, device=out.device)
    space.render(cam, width, height, spp, seed=seed - 1, out=out, **kw)  # untimed: allocations
    space.sync()
    calls = 0
    t0 = time.perf_counter()
    while True:
        space.render(cam, width, height, spp, seed=seed + calls, out=out, **kw)
        acc.add_(out)
        calls += 1
        space.sync()
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    return (acc / calls).cpu().numpy(), dt, calls * spp


def cached_at_budget(space, scene, width, height, budget_s, warmup=8, seed=100, max_depth=12, spp_per_frame=1,
                     cache_depth=1, train_every=16, train_steps=4, train_batch=16384, train_tail=0, train_epochs=1,
                     lr=1e-2, encoding="hashgrid", hash_cache=False):
    """The radiance-cached path tracer given `budget_s` seconds of wall time
    (a fresh cache; its training included): frames of `spp_per_frame`
    samples, each trained on by the cache right after it, until the budget
    is spent; frames after the first `warmup` are averaged on the device.
    Returns (image, seconds, frames, averaged frames, training records
    dropped by the hash-grid cache, records)."""
    import torch
    cam = dict(scene["camera"], aspect=width / height)
    kw = dict(max_depth=max_depth, sky=scene.get("sky", (0.0, 0.0, 0.0)), cache_depth=cache_depth,
              train_every=train_every, train_steps=train_steps, train_batch=train_batch, train_tail=train_tail,
              train_epochs=train_epochs, hash_cache=hash_cache)
    reset = space.hash_cache_reset if hash_cache else (lambda: space.mlp_init(seed=seed, lr=lr, encoding=encoding))
    out = torch.empty((height, width, 3), dtype=torch.float32, device=f"cuda:{space.device}")
    acc = torch.zeros((height, width, 3), dtype=torch.float64, device=out.device)
    reset()
    space.render(cam, width, height, spp_per_frame, seed=seed + 99991, out=out, **kw)  # untimed: allocations
    reset()
    space.sync()
    frames = kept = dropped = records = 0
    t0 = time.perf_counter()
    while True:
        space.render(cam, width, height, spp_per_frame, seed=seed + frames, out=out, **kw)
        if frames >= warmup:
            acc.add_(out)
            kept += 1
        frames += 1
        space.sync()
        if hash_cache:
            r, d = space.last_train_stats()
            records, dropped = records + r, dropped + d
        if time.perf_counter() - t0 >= budget_s and kept > 0:
            break
    dt = time.perf_counter() - t0
    return (acc / kept).cpu().numpy(), dt, frames, kept, dropped, records


def gain_versus_budget(space, scene, width, height, gt, budgets=(0.5, 2.0, 8.0), arms=None):
    """relMSE against `gt` of plain path tracing and of each cached arm at
    every wall-time budget, with the gain (plain relMSE / cached relMSE) and
    the cached image's mean bias per channel. arms: {name: cached_at_budget
    keyword arguments}."""
    res = {"budgets_s": list(budgets), "plain": [], "arms": {k: [] for k in arms}}
    for b in budgets:
        img, dt, spp = plain_at_budget(space, scene, width, height, b)
        e_plain = rel_mse(img, gt)
        res["plain"].append({"relmse": round(e_plain, 6), "seconds": round(dt, 3), "spp": spp,
                             "bias": [round(x, 5) for x in (img.mean((0, 1)) / gt.mean((0, 1)) - 1.0).tolist()]})
        for name, kw in arms.items():
            img, dt, frames, kept, dropped, records = cached_at_budget(space, scene, width, height, b, **kw)
            e = rel_mse(img, gt)
            entry = {"relmse": round(e, 6), "gain": round(e_plain / e, 3), "seconds": round(dt, 3),
                     "frames": frames, "frames_averaged": kept,
                     "bias": [round(x, 5) for x in (img.mean((0, 1)) / gt.mean((0, 1)) - 1.0).tolist()]}
            if kw.get("hash_cache"):
                entry["hash_records_dropped"] = dropped
                entry["hash_records"] = records
            res["arms"][name].append(entry)
    return res


# The three cache designs compared at equal time: the network exactly as the
# 1080p workload specifies it (12-band frequency encoding of position,
# direction, normal, roughness and albedo; 1 path in 16 traced to full depth
# as the training target; Adam at 1e-2 every frame), this project's
# hash-grid network with self-training tails, and the non-learned hash-grid
# cache in the network's place.
ARMS = {
    "spec_freq12_full_depth_cache_depth_1": dict(encoding="freq12", cache_depth=1, train_tail=0),
    "spec_freq12_full_depth_cache_depth_2": dict(encoding="freq12", cache_depth=2, train_tail=0),
    "hashgrid_self_training": dict(encoding="hashgrid", cache_depth=1, train_tail=1, train_epochs=2),
    "hashgrid_self_training_8_steps": dict(encoding="hashgrid", cache_depth=1, train_tail=1, train_epochs=2,
                                           train_steps=8),
    "hash_grid_cache": dict(hash_cache=True, cache_depth=1, train_tail=1),
}
