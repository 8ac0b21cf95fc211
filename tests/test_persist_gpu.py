"""Persistent scenes (ilg_save / ilg_load): a loaded scene answers every
query exactly as the built one, renders the same image, and malformed or
corrupted files are refused."""
import numpy as np
import pytest

from illuminaprt_b200 import scenes

pytestmark = pytest.mark.gpu


def test_loaded_scene_answers_queries_like_the_built_one(tmp_path):
    from illuminaprt_b200.ilg import GpuSpace
    pos, idx = scenes.heightfield(97, 61, 0.2, 8)
    a = GpuSpace()
    a.initialise(pos, idx)
    a.build()
    path = tmp_path / "hf.ilgbvh"
    a.save(path)
    b = GpuSpace()
    b.load(path)
    assert b.stats()["n_nodes"] == a.stats()["n_nodes"]
    co, cd = scenes.pinhole_rays(128, 128, (0.5, -0.6, 0.8), (0.5, 0.5, 0.0), (0, 0, 1), 60.0)
    io, idr = scenes.incoherent_rays(pos, idx, 32768, 9)
    o4, d4 = np.concatenate([co, io]), np.concatenate([cd, idr])
    for wt in (False, True):
        ra, rb = a.intersects(o4, d4, watertight=wt), b.intersects(o4, d4, watertight=wt)
        for x, y in zip(ra, rb):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    assert np.array_equal(a.occluded(o4, d4), b.occluded(o4, d4))


def test_loaded_scene_renders_like_the_built_one(tmp_path):
    from illuminaprt_b200.ilg import GpuSpace
    a = GpuSpace()
    box = scenes.load_box_scene(a)
    path = tmp_path / "box.ilgbvh"
    a.save(path)
    b = GpuSpace()
    b.load(path)
    # materials and lights are not part of the file
    b.set_materials([{"albedo": tuple(x)} for x in box["albedo"]])
    first = int(np.nonzero(box["prim_of_tri"] == box["light_prim"])[0][0])
    b.set_quad_lights([{"v": box["light_quad"], "emit": box["light_emit"], "first_tri": first}])
    ia = a.render(box["camera"], 64, 64, 8, seed=4)
    ib = b.render(box["camera"], 64, 64, 8, seed=4)
    assert np.allclose(ia, ib, rtol=1e-5, atol=1e-6)


def test_bad_files_are_refused(tmp_path):
    from illuminaprt_b200.ilg import GpuSpace, IlgError
    pos, idx = scenes.heightfield(16, 8, 0.2, 3)
    a = GpuSpace()
    a.initialise(pos, idx)
    a.build()
    good = tmp_path / "g.ilgbvh"
    a.save(good)
    raw = good.read_bytes()
    cases = {
        "flipped.ilgbvh": raw[:200] + bytes([raw[200] ^ 0x40]) + raw[201:],   # checksum
        "short.ilgbvh": raw[:len(raw) - 100],                                  # truncated
        "magic.ilgbvh": b"NOTABVH\0" + raw[8:],                                # not a scene file
        "empty.ilgbvh": b"",
    }
    for name, data in cases.items():
        p = tmp_path / name
        p.write_bytes(data)
        with pytest.raises(IlgError):
            GpuSpace().load(p)
    with pytest.raises(IlgError):
        GpuSpace().load(tmp_path / "missing.ilgbvh")
    with pytest.raises(IlgError):
        GpuSpace().save(tmp_path / "unbuilt.ilgbvh")  # nothing built yet
