"""Scene import onto the device: a scene script loaded by the reference's own
loader (Environment::Load -> EnvironmentLoader -> WavefrontSceneLoader,
Core/Scene/*.cpp) with the plug-in's "GPU" space and renderer factories
registered, so the OBJ mesh (one primitive with a MaterialGroup), the Quad
light and the camera all arrive through the engine's objects."""
from __future__ import annotations

import os

import numpy as np
import pytest

from illuminaprt_b200 import build as pkg_build
from illuminaprt_b200 import scenes
from oracle import bindings
from tests.test_scene_script import GOLDEN, SPECULAR, coarse_expectation, rel_mse

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.exists(pkg_build.PLUGIN) and bindings.ref_available()),
                                 reason="plug-in or reference engine library not built")]


def test_script_scene_on_the_gpu_renderer_matches_the_reference_image(tmp_path):
    script = scenes.write_box_script(tmp_path, width=256, height=256, spp=1024)
    final, direct, albedo, info = bindings.RefLib().render_script(script, 256, 256, plugin=pkg_build.PLUGIN)
    assert "space=GpuSpace" in info and "renderer=GpuRenderer" in info, info
    ref_img = np.load(GOLDEN)["image"]
    err = rel_mse(final, ref_img)
    print(f"relMSE(script scene on GpuRenderer 1024 spp, reference 4096 spp) = {err:.2e}")
    assert np.isfinite(final).all()
    assert err < 1e-3
    assert np.allclose(final.mean((0, 1)), ref_img.mean((0, 1)), rtol=1e-2)
    assert (direct <= final + 1e-4).all() and albedo.mean() > 0.2


def test_reference_renderer_over_the_loaded_gpu_space_matches_basic_space(tmp_path):
    # BasicRenderer + PathIntegrator with the scene's fixed-seed sampler: the
    # same sample sequence over either space, so paths differ only where a
    # near tie picks the other of two coincident surfaces
    w, spp = 32, 2
    ref = bindings.RefLib()
    basic = ref.render_script(scenes.write_box_script(tmp_path / "basic", width=w, height=w, spp=spp, space="Basic",
                                                      renderer="Basic"), w, w)
    gpu = ref.render_script(scenes.write_box_script(tmp_path / "gpu", width=w, height=w, spp=spp, space="GPU",
                                                    renderer="Basic"), w, w, plugin=pkg_build.PLUGIN)
    assert "space=GpuSpace" in gpu[3], gpu[3]
    same = np.all(basic[0] == gpu[0], axis=2)
    assert same.mean() >= 0.98, f"{int((~same).sum())} of {same.size} pixels differ"


@pytest.mark.parametrize("container", ["KDTreeMesh", "BasicMesh"])
def test_every_mesh_container_gives_the_same_device_image(tmp_path, container):
    # GpuSpace flattens any ITriangleMesh in its triangle order, so the device
    # scene, and with the counter-based samples the image, do not depend on
    # the container the script chose
    w, spp = 48, 8
    ref = bindings.RefLib()
    a = ref.render_script(scenes.write_box_script(tmp_path / "bvh", width=w, height=w, spp=spp), w, w,
                          plugin=pkg_build.PLUGIN)
    b = ref.render_script(scenes.write_box_script(tmp_path / container, width=w, height=w, spp=spp,
                                                  container=container), w, w, plugin=pkg_build.PLUGIN)
    for x, y in zip(a[:3], b[:3]):  # float atomics may sum a pixel's samples in another order
        assert np.allclose(x, y, rtol=1e-5, atol=1e-6)


def test_script_scene_regions_tile_the_frame(tmp_path):
    script = scenes.write_box_script(tmp_path, width=100, height=72, spp=4)
    ref = bindings.RefLib()
    whole = ref.render_script(script, 100, 72, plugin=pkg_build.PLUGIN)
    tiled = ref.render_script(script, 100, 72, plugin=pkg_build.PLUGIN, tile=32)
    for a, b in zip(whole[:3], tiled[:3]):
        assert np.allclose(a, b, rtol=1e-5, atol=1e-6)


def test_gpu_integrator_with_the_radiance_cache(tmp_path):
    # Integrator { Type = GPU  Cache = MLP }: the device renderer stops paths
    # into the learned cache at their first bounce vertex and trains it after
    # every region; the image stays near the reference's and differs from the
    # uncached render of the same samples
    ref = bindings.RefLib()
    w, spp = 128, 64
    cached = ref.render_script(scenes.write_box_script(tmp_path / "mlp", width=w, height=w, spp=spp, integrator="GPU",
                                                       integrator_args={"Cache": "MLP", "CacheDepth": 1,
                                                                        "TrainSteps": 8}),
                               w, w, plugin=pkg_build.PLUGIN, tile=32)
    plain = ref.render_script(scenes.write_box_script(tmp_path / "pt", width=w, height=w, spp=spp, integrator="GPU"),
                              w, w, plugin=pkg_build.PLUGIN, tile=32)
    assert "GpuRenderer" in cached[3]
    assert np.isfinite(cached[0]).all()
    assert not np.allclose(cached[0], plain[0], rtol=1e-3, atol=1e-4)
    # Direct and Albedo come from the first vertex, before the cache
    assert np.allclose(cached[1], plain[1], rtol=1e-5, atol=1e-6)
    assert np.allclose(cached[2], plain[2], rtol=1e-5, atol=1e-6)
    expected = coarse_expectation(np.load(GOLDEN)["image"], w)
    e_cached, e_plain = rel_mse(cached[0], expected), rel_mse(plain[0], expected)
    print(f"relMSE at {spp} spp: cached {e_cached:.2e}, plain {e_plain:.2e}")
    assert e_cached < 0.1
    assert np.allclose(cached[0].mean((0, 1)), expected.mean((0, 1)), rtol=0.15)


def test_specular_script_scene_on_the_gpu_renderer(tmp_path):
    # the script's mirror (MTL illum 5) and glass (script Glass material)
    # reach the device through GpuSpace / GpuRenderer
    ref = np.load(SPECULAR.format(4096, 1))["image"]
    floor = rel_mse(np.load(SPECULAR.format(1024, 2))["image"], ref)
    script = scenes.write_box_script(tmp_path, scene=scenes.box_scene(specular=True), width=128, height=128,
                                     spp=8192)
    final, direct, albedo, info = bindings.RefLib().render_script(script, 128, 128, plugin=pkg_build.PLUGIN)
    assert "space=GpuSpace" in info and "primitives=3" in info, info
    err = rel_mse(final, ref)
    print(f"relMSE(specular script on GpuRenderer 8192 spp, reference 4096 spp) = {err:.2e}; floor {floor:.2e}")
    assert np.isfinite(final).all()
    # independent noise alone gives (1/8192 + 1/4096) / (1/1024 + 1/4096) = 0.3 of the floor
    assert err < 0.5 * floor
    assert np.allclose(final.mean((0, 1)), ref.mean((0, 1)), rtol=1e-2)
