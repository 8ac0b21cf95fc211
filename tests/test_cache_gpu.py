"""The radiance-cached path tracer: online training on the path tracer's own
tails, and its error at equal wall time against plain path tracing."""
import numpy as np
import pytest

from illuminaprt_b200 import scenes
from illuminaprt_b200.cache_experiment import equal_time, rel_mse

pytestmark = pytest.mark.gpu

W, H = 192, 108


@pytest.fixture(scope="module")
def field():
    from illuminaprt_b200.ilg import GpuSpace
    s = scenes.sphere_field(4, 4, seed=5, width=W, height=H)
    sp = GpuSpace()
    scenes.load_sphere_field(sp, s)
    gt = sp.render(dict(s["camera"], aspect=W / H), W, H, 16384, max_depth=12, seed=424242, sky=s["sky"])
    return sp, s, gt


def test_plain_render_unchanged_by_cache_support(field):
    sp, s, _ = field
    a = sp.render(s["camera"], 64, 36, 4, max_depth=12, seed=3, sky=s["sky"])
    b = sp.render(s["camera"], 64, 36, 4, max_depth=12, seed=3, sky=s["sky"], cache_depth=0)
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6)


def test_cache_trains_online(field):
    sp, s, gt = field
    sp.mlp_init(seed=1, lr=1e-2)
    cam = dict(s["camera"], aspect=W / H)
    errs = []
    for f in range(40):
        img = sp.render(cam, W, H, 1, max_depth=12, seed=1000 + f, sky=s["sky"], cache_depth=1)
        assert np.isfinite(img).all()
        # how well does the cache alone (no noise averaging) match the truth?
        if f in (0, 39):
            errs.append(rel_mse(sp.render(cam, W, H, 64, max_depth=12, seed=77 + f, sky=s["sky"], cache_depth=1,
                                          train_steps=0), gt))
    print(f"cached 64-spp relMSE before / after 40 training frames: {errs[0]:.4f} / {errs[1]:.4f}")
    assert errs[1] < errs[0]


def test_self_training_tails(field):
    # training paths stop into the cache two vertices after the query vertex;
    # the cache's answer there completes their records' targets. The cache
    # still learns online, the frame ends at depth 3 (cheaper than tracing
    # the training paths to depth 12), and a training-free frame is unchanged
    sp, s, gt = field
    cam = dict(s["camera"], aspect=W / H)
    sp.mlp_init(seed=2, lr=1e-2)
    frozen = lambda f: sp.render(cam, W, H, 64, max_depth=12, seed=77 + f, sky=s["sky"], cache_depth=1,
                                 train_steps=0, train_tail=2)
    before = rel_mse(frozen(0), gt)
    for f in range(40):
        img = sp.render(cam, W, H, 1, max_depth=12, seed=2000 + f, sky=s["sky"], cache_depth=1, train_tail=2)
        assert np.isfinite(img).all()
    after = rel_mse(frozen(1), gt)
    print(f"self-trained cache, 64-spp relMSE before / after 40 frames: {before:.4f} / {after:.4f}")
    assert after < before
    # a frozen cache (no training) renders the same image with or without tails:
    # tails only change what the training records receive
    a = sp.render(cam, W, H, 4, max_depth=12, seed=5, sky=s["sky"], cache_depth=1, train_steps=0, train_tail=2)
    b = sp.render(cam, W, H, 4, max_depth=12, seed=5, sky=s["sky"], cache_depth=1, train_steps=0, train_tail=0)
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6)


def test_hash_grid_cache_baseline(field):
    # the non-learned baseline: an empty hash-grid cache answers 0 (the image
    # lacks everything past the cache vertex); filled by the training paths
    # of 40 frames it approaches the truth, and it needs no network
    from illuminaprt_b200.ilg import IlgError
    sp, s, gt = field
    cam = dict(s["camera"], aspect=W / H)
    kw = dict(max_depth=12, sky=s["sky"], cache_depth=1, hash_cache=True)
    sp.hash_cache_reset()
    empty = sp.render(cam, W, H, 64, seed=7, **kw)
    dropped = records = 0
    for f in range(40):
        img = sp.render(cam, W, H, 1, seed=3000 + f, train_tail=2, **kw)
        assert np.isfinite(img).all()
        r, d = sp.last_train_stats()
        records, dropped = records + r, dropped + d
    # every record found a cell: none was lost to a full probe window
    assert records > 0 and dropped <= records // 10000
    filled = sp.render(cam, W, H, 64, seed=8, **kw)
    e0, e1 = rel_mse(empty, gt), rel_mse(filled, gt)
    print(f"hash-grid cache, 64-spp relMSE empty / after 40 frames: {e0:.4f} / {e1:.4f}")
    assert e1 < 0.5 * e0
    assert np.allclose(filled.mean((0, 1)), gt.mean((0, 1)), rtol=0.1)
    with pytest.raises(IlgError):
        sp.render(cam, W, H, 1, seed=1, max_depth=12, sky=s["sky"], hash_cache=True)  # needs cache_depth


def test_cache_in_regions(field):
    # a frozen cache (train_steps 0): region calls query the same network, so
    # tiles reproduce the whole image's paths; the whole image as one region
    # equals ilg_render's cached image; Direct does not depend on the cache
    sp, s, _ = field
    sp.mlp_init(seed=3, lr=1e-2)
    cam = dict(s["camera"], aspect=W / H)
    frame = sp.camera_frame(cam, W, H)
    kw = dict(max_depth=12, seed=9, sky=s["sky"])
    whole = sp.render(cam, W, H, 8, cache_depth=1, train_steps=0, **kw)
    one, direct, _ = sp.render_region(frame, W, H, 8, (0, 0, W, H), cache_depth=1, train_steps=0, **kw)
    assert np.allclose(one, whole, rtol=1e-5, atol=1e-6)
    tiled = np.zeros_like(whole)
    for y in range(0, H, 40):
        for x in range(0, W, 64):
            w, h = min(64, W - x), min(40, H - y)
            tiled[y:y + h, x:x + w] = sp.render_region(frame, W, H, 8, (x, y, w, h), cache_depth=1, train_steps=0,
                                                       aux=False, **kw)[0]
    assert np.allclose(tiled, whole, rtol=1e-5, atol=1e-6)
    plain, plain_direct, _ = sp.render_region(frame, W, H, 8, (0, 0, W, H), **kw)
    assert not np.allclose(one, plain, rtol=1e-3, atol=1e-4)  # the cache answered the tails
    assert np.allclose(direct, plain_direct, rtol=1e-5, atol=1e-6)
    # training after a region call changes the next call's image
    sp.render_region(frame, W, H, 1, (0, 0, W, H), cache_depth=1, train_steps=4, aux=False, **kw)
    after = sp.render_region(frame, W, H, 8, (0, 0, W, H), cache_depth=1, train_steps=0, **kw)[0]
    assert not np.allclose(after, one, rtol=1e-4, atol=1e-5)


def test_training_is_what_helps(field):
    """Ablation: the same cached renderer with a network that never trains."""
    sp, s, gt = field
    trained = equal_time(sp, s, W, H, gt, frames=48, warmup=16, cache_depth=1)
    frozen = equal_time(sp, s, W, H, gt, frames=48, warmup=16, cache_depth=1, ablate_training=True)
    print(f"relMSE trained {trained['relmse_cached']:.5f} vs untrained {frozen['relmse_cached']:.5f}")
    assert trained["relmse_cached"] < frozen["relmse_cached"] / 2


def test_gain_at_equal_time_under_the_fair_protocol():
    """The full 64-icosphere field (20,971,530 triangles) at 960 x 540 and a
    0.25 s budget: plain path tracing renders its budget in calls that fill a
    wave (no per-frame synchronisation), and the self-training hash-grid
    cache must still beat it by a set factor, against a 4096-spp ground
    truth. (On cheap scenes, where plain path tracing converges within the
    budget, the cache's approximation error floor makes it lose; that is the
    expected crossover, not a failure.)"""
    from illuminaprt_b200.ilg import GpuSpace
    from illuminaprt_b200.cache_experiment import ARMS, gain_versus_budget
    w, h = 960, 540
    s = scenes.sphere_field(8, 7, seed=3, width=w, height=h)
    sp = GpuSpace()
    scenes.load_sphere_field(sp, s)
    gt = sp.render(dict(s["camera"], aspect=w / h), w, h, 4096, max_depth=12, seed=424242, sky=s["sky"])
    arms = {k: ARMS[k] for k in ("hashgrid_self_training", "spec_freq12_full_depth_cache_depth_1")}
    r = gain_versus_budget(sp, s, w, h, gt, budgets=(0.25,), arms=arms)
    print(r)
    best = r["arms"]["hashgrid_self_training"][0]
    assert best["gain"] >= 2.5  # 3.6x measured on a B200
    assert max(abs(b) for b in best["bias"]) < 0.02
