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
    assert (tmp_path / "tune.json").exists()
