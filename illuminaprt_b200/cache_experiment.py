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
