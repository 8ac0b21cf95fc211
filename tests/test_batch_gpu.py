"""Batched rendering of independent scenes in one wavefront."""
import numpy as np
import pytest

from illuminaprt_b200 import scenes

pytestmark = pytest.mark.gpu


def _spaces(items):
    from illuminaprt_b200.ilg import GpuSpace
    out = []
    for s in items:
        sp = GpuSpace()
        scenes.load_sphere_field(sp, s)
        out.append(sp)
    return out


def test_batch_equals_individual_renders():
    from illuminaprt_b200.ilg import GpuSpace
    items = scenes.batch_workload(5, seed=21, tri_range=(2_000, 50_000), side_range=(24, 80))
    spaces = _spaces(items)
    runner = GpuSpace()
    batch = [{"space": sp, "camera": s["camera"], "width": s["width"], "height": s["height"], "spp": s["spp"],
              "max_depth": s["max_depth"], "seed": 40 + i, "sky": s["sky"]} for i, (sp, s) in enumerate(zip(spaces, items))]
    imgs = runner.render_batch(batch, paths_per_wave=1 << 14, block=64)
    for it, img in zip(batch, imgs):
        single = it["space"].render(it["camera"], it["width"], it["height"], it["spp"], max_depth=it["max_depth"],
                                    seed=it["seed"], sky=it["sky"])
        assert np.allclose(img, single, rtol=1e-5, atol=1e-6)
    # a different wave size and block shape changes nothing but the schedule
    imgs2 = runner.render_batch(batch, paths_per_wave=1 << 20, block=256)
    for a, b in zip(imgs, imgs2):
        assert np.allclose(a, b, rtol=1e-5, atol=1e-6)


def test_autotuner_picks_a_measured_setting(tmp_path):
    from illuminaprt_b200.ilg import GpuSpace
    from illuminaprt_b200.autotune import tune_batch
    items = scenes.batch_workload(4, seed=22, tri_range=(2_000, 20_000), side_range=(32, 64))
    spaces = _spaces(items)
    runner = GpuSpace()
    batch = [{"space": sp, "camera": s["camera"], "width": s["width"], "height": s["height"], "spp": 4,
              "max_depth": s["max_depth"], "sky": s["sky"]} for sp, s in zip(spaces, items)]
    choice, sweep = tune_batch(runner, batch, waves=(1 << 12, 1 << 16), blocks=(64, 256),
                               profile_path=str(tmp_path / "tune.json"))
    assert choice == min(sweep, key=lambda r: r["seconds"])
    assert len(sweep) == 5 and any(r["one_launch"] for r in sweep)
    assert (tmp_path / "tune.json").exists()


def test_one_launch_renders_the_wavefront_paths():
    # the persistent one-launch renderer (ILG_RENDER_PERSISTENT) traces the
    # wavefront's paths: same sample sequence, shading and traversal, so the
    # images agree up to the order of the float additions into each pixel
    from illuminaprt_b200.ilg import GpuSpace
    items = scenes.batch_workload(5, seed=23, tri_range=(2_000, 50_000), side_range=(24, 80))
    spaces = _spaces(items)
    runner = GpuSpace()
    batch = [{"space": sp, "camera": s["camera"], "width": s["width"], "height": s["height"], "spp": s["spp"],
              "max_depth": s["max_depth"], "seed": 70 + i, "sky": s["sky"]} for i, (sp, s) in enumerate(zip(spaces, items))]
    wave = runner.render_batch(batch, paths_per_wave=1 << 16, block=128)
    one = runner.render_batch(batch, one_launch=True)
    for a, b in zip(wave, one):
        assert np.isfinite(b).all()
        assert np.allclose(a, b, rtol=1e-4, atol=1e-5)
    # again: the captured graph is replayed
    one2 = runner.render_batch(batch, one_launch=True)
    for a, b in zip(one, one2):
        assert np.allclose(a, b, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("kw", [dict(), dict(specular=True), dict(light="mesh"),
                                dict(specular=True, infinite=(0.5, 0.6, 0.8), fov=60.0)],
                         ids=["box", "specular", "meshlight", "infinite"])
def test_one_launch_renders_every_material_and_light(kw):
    from illuminaprt_b200.ilg import GpuSpace, IlgError
    sp = GpuSpace()
    scene = scenes.load_box_scene(sp, scenes.box_scene(**kw))
    a = sp.render(scene["camera"], 96, 96, 64, seed=5)
    b = sp.render(scene["camera"], 96, 96, 64, seed=5, one_launch=True)
    assert np.allclose(a, b, rtol=1e-4, atol=1e-5)
    with pytest.raises(IlgError):  # plain renders only
        sp.render(scene["camera"], 32, 32, 1, seed=5, one_launch=True, count=True)
