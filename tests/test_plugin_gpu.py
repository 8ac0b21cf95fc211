"""The reference engine over GpuSpace (the engine plug-in) against the same
engine over its own BasicSpace, on the box scene (walls, two boxes, a quad
light): every field of every Intersection record, the any-hit answers, the
p_pExclude overloads, and whole images from the reference's own
PathIntegrator, which never sees anything but ISpace."""
from __future__ import annotations

import os

import numpy as np
import pytest

from illuminaprt_b200 import build as pkg_build
from illuminaprt_b200 import scenes
from oracle import bindings

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.exists(pkg_build.PLUGIN) and bindings.ref_available()),
                                 reason="plug-in or reference engine library not built")]

TIE_WINDOW = 1e-5
SHAPE_BIT = 2048


def _rays(scene, n, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-0.95, 0.95, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    cam = scene["camera"]
    co, cd = scenes.pinhole_rays(32, 32, cam["eye"], cam["target"], cam["up"], cam["fov"])
    o4 = np.concatenate([np.c_[o, np.zeros(n)].astype(np.float32), co])
    d4 = np.concatenate([np.c_[d, np.full(n, 3.0e38)].astype(np.float32), cd])
    return o4, d4


def _check_closest(hit, t, diff=None):
    assert np.array_equal(hit[:, 0], hit[:, 1]), f"hit flags differ on {int((hit[:, 0] != hit[:, 1]).sum())} rays"
    both = (hit[:, 0] == 1) & (hit[:, 1] == 1)
    differ = both & (t[:, 0].view(np.uint32) != t[:, 1].view(np.uint32))
    if diff is not None:
        differ |= both & (diff != 0)
    # of two hits less than 1e-5 apart the first one visited wins: BasicSpace
    # visits primitives in list order, the device BVH in tree order
    gap = np.where(both, np.abs(t[:, 0] - np.where(both, t[:, 1], 0)), np.inf)
    tie = differ & (gap < TIE_WINDOW)
    bad = differ & ~tie
    assert not bad.any(), f"{int(bad.sum())} rays differ outside the tie window; first {np.nonzero(bad)[0][:5]}"
    return int(both.sum()), int(tie.sum())


def test_gpu_space_intersection_records_match_basic_space():
    scene = scenes.box_scene()
    o4, d4 = _rays(scene, 4096, 3)
    n = o4.shape[0]
    rng = np.random.default_rng(4)
    n_prims = scene["albedo"].shape[0]
    exclude = rng.integers(-1, n_prims, n).astype(np.int32)
    r = bindings.RefLib().compare_spaces(pkg_build.PLUGIN, scene, o4, d4, exclude=exclude)
    both, ties = _check_closest(r["hit"], r["t"], r["diff"])
    assert both > 0.7 * n  # the box is open at z = +1, so some rays leave it
    # the inner boxes stand on the floor: rays starting inside one and going
    # down meet its bottom face and the floor at the same distance
    assert ties <= n // 50, ties
    # every other hit record equals BasicSpace's in all twelve fields, bit
    # for bit (_check_closest); ties are the only records that differ
    hit = r["hit"][:, 0] == 1
    assert int((r["diff"][hit] != 0).sum()) <= ties
    # any hit is an order-free predicate: exact
    assert np.array_equal(r["occ"][:, 0], r["occ"][:, 1])
    ex = exclude >= 0
    _check_closest(r["xhit"][ex], r["xt"][ex])
    assert np.array_equal(r["xocc"][ex, 0], r["xocc"][ex, 1])
    # excluding the struck primitive changes the answer somewhere
    assert (r["xhit"][ex, 0] != r["hit"][ex, 0]).any() or (r["xt"][ex, 0] != r["t"][ex, 0]).any()


def test_reference_path_integrator_over_gpu_space():
    scene = scenes.box_scene()
    w, h, spp = 32, 24, 2
    ref = bindings.RefLib()
    img_basic = ref.render_box(scene, w, h, spp, seed=5, nthreads=1)
    img_gpu = ref.render_box_plugin(pkg_build.PLUGIN, scene, w, h, spp, seed=5, nthreads=1)
    assert np.isfinite(img_gpu).all()
    same = np.all(img_basic == img_gpu, axis=2)
    # a path diverges only where a near tie picked the other of two coincident
    # surfaces (shared edges of the box walls)
    assert same.mean() >= 0.99, f"{int((~same).sum())} of {same.size} pixels differ"


def _rel_mse(x, ref, eps=1e-2):
    return float(np.mean((x.astype(np.float64) - ref) ** 2 / (ref.astype(np.float64) ** 2 + eps)))


def test_gpu_renderer_through_the_engine_matches_the_reference_image():
    # the engine's Scene / camera / PathIntegrator / filter / RadianceBuffer
    # driving the plug-in's GpuRenderer over its GpuSpace, against the
    # reference's own 4096-spp render of the same scene
    import glob
    paths = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "box_256_4096spp_seed*.npz")))
    if not paths:
        pytest.skip("no reference image")
    ref_img = np.load(paths[0])["image"]
    scene = scenes.box_scene()
    final, direct, albedo = bindings.RefLib().render_box_renderer(pkg_build.PLUGIN, scene, 256, 256, 1024)
    err = _rel_mse(final, ref_img)
    print(f"relMSE(GpuRenderer 1024 spp, reference 4096 spp) = {err:.2e}")
    assert np.isfinite(final).all()
    assert err < 1e-3
    assert np.allclose(final.mean((0, 1)), ref_img.mean((0, 1)), rtol=1e-2)
    assert (direct <= final + 1e-4).all() and albedo.mean() > 0.2


def test_gpu_renderer_regions_tile_the_frame():
    scene = scenes.box_scene()
    ref = bindings.RefLib()
    whole = ref.render_box_renderer(pkg_build.PLUGIN, scene, 100, 72, 4)
    tiled = ref.render_box_renderer(pkg_build.PLUGIN, scene, 100, 72, 4, tile=32)
    for a, b in zip(whole, tiled):  # same paths; float atomics may sum them in another order
        assert np.allclose(a, b, rtol=1e-5, atol=1e-6)


def test_gpu_renderer_renders_mirror_and_glass_like_the_reference():
    # MirrorMaterial and GlassMaterial reach the device through the engine's
    # objects: GpuRenderer reads their reflectivity, transmittance and indices
    p4096 = os.path.join(os.path.dirname(__file__), "golden", "box_specular_128_4096spp_seed1.npz")
    if not os.path.exists(p4096):
        pytest.skip("no reference image")
    ref_img = np.load(p4096)["image"]
    floor = _rel_mse(np.load(p4096.replace("4096spp_seed1", "1024spp_seed2"))["image"], ref_img)
    scene = scenes.box_scene(specular=True)
    final, direct, albedo = bindings.RefLib().render_box_renderer(pkg_build.PLUGIN, scene, 128, 128, 8192)
    err = _rel_mse(final, ref_img)
    print(f"relMSE(GpuRenderer 8192 spp, reference 4096 spp) = {err:.2e}; reference floor {floor:.2e}")
    assert np.isfinite(final).all()
    # independent noise alone gives (1/8192 + 1/4096) / (1/1024 + 1/4096) = 0.3 of the floor
    assert err < 0.5 * floor
    assert np.allclose(final.mean((0, 1)), ref_img.mean((0, 1)), rtol=1e-2)


@pytest.mark.parametrize("prefix,kw", [("box_meshlight", dict(light="mesh")),
                                       ("box_infinite", dict(specular=True, infinite=(0.5, 0.6, 0.8), fov=60.0))])
def test_gpu_renderer_renders_mesh_and_infinite_lights_like_the_reference(prefix, kw):
    # a DiffuseAreaLight on a triangle mesh and an InfiniteAreaLight reach the
    # device through the engine's LightList (PrepareDeviceScene)
    p4096 = os.path.join(os.path.dirname(__file__), "golden", f"{prefix}_128_4096spp_seed1.npz")
    if not os.path.exists(p4096):
        pytest.skip("no reference image")
    ref_img = np.load(p4096)["image"]
    floor = _rel_mse(np.load(p4096.replace("4096spp_seed1", "1024spp_seed2"))["image"], ref_img)
    scene = scenes.box_scene(**kw)
    final, direct, albedo = bindings.RefLib().render_box_engine(pkg_build.PLUGIN, scene, 128, 128, 8192)
    err = _rel_mse(final, ref_img)
    print(f"{prefix}: relMSE(GpuRenderer 8192 spp, reference 4096 spp) = {err:.2e}; reference floor {floor:.2e}")
    assert np.isfinite(final).all()
    assert err < 0.5 * floor
    assert np.allclose(final.mean((0, 1)), ref_img.mean((0, 1)), rtol=1e-2)


@pytest.mark.parametrize("kw", [dict(), dict(light="mesh"), dict(specular=True, infinite=(0.5, 0.6, 0.8), fov=60.0)],
                         ids=["quad", "meshlight", "infinite"])
def test_reference_renderer_over_the_device_integrator(kw):
    # the reference's BasicRenderer calling GpuPathIntegrator::Radiance once
    # per pixel sample: every path runs on the device (ilg_radiance), none on
    # the CPU. Its image against the reference's own PathIntegrator at 4096
    # spp: no further from it than a 64-spp reference render is
    scene = scenes.box_scene(**kw)
    w = h = 32
    ref = bindings.RefLib()
    truth = ref.render_box_lights(scene, w, h, 4096, seed=1)[0]
    noisy = ref.render_box_lights(scene, w, h, 64, seed=2)[0]
    floor = _rel_mse(noisy, truth)
    final, direct, albedo = ref.render_box_engine(pkg_build.PLUGIN, scene, w, h, 64, renderer="", integrator="GPU")
    err = _rel_mse(final, truth)
    print(f"{kw}: relMSE(BasicRenderer + device Radiance 64 spp, reference 4096 spp) = {err:.2e}; "
          f"reference 64 spp: {floor:.2e}")
    assert np.isfinite(final).all()
    assert err < 1.5 * floor
    assert np.allclose(final.mean((0, 1)), truth.mean((0, 1)), rtol=3e-2)
    # Direct is part of Final, and the first hit's albedo is filled
    assert (direct <= final + 1e-4).all() and albedo.mean() > 0.1


def test_device_integrator_refuses_what_it_cannot_run():
    # no CPU fallback: the learned cache under a per-sample renderer is
    # refused with the reason (it would never train there)
    scene = scenes.box_scene()
    ref = bindings.RefLib()
    with pytest.raises(RuntimeError, match="Cache = MLP"):
        ref.render_box_engine(pkg_build.PLUGIN, scene, 8, 8, 1, renderer="", integrator="GPU",
                              integrator_args={"Cache": "MLP"})
