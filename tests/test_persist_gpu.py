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


def _read_scene_file(path):
    raw = open(path, "rb").read()
    head = np.frombuffer(raw[:64], np.uint32)
    assert raw[:7] == b"ILGBVH8"
    n_verts, n_tris, n_nodes, n_leaf, _, has_mat, node_bytes, tri_bytes = (int(x) for x in head[4:12])
    assert node_bytes == 80 and tri_bytes == 48
    off = 64
    def take(count, dtype, shape):
        nonlocal off
        nb = count * np.dtype(dtype).itemsize
        a = np.frombuffer(raw[off:off + nb], dtype).reshape(shape)
        off += nb
        return a
    pos = take(3 * n_verts, np.float32, (n_verts, 3))
    idx = take(3 * n_tris, np.uint32, (n_tris, 3))
    if has_mat:
        take(n_tris, np.uint32, (n_tris,))
    nodes = take(20 * n_nodes, np.uint32, (n_nodes, 20))
    tris = take(12 * n_leaf, np.float32, (n_leaf, 12))
    prim = take(n_leaf, np.uint32, (n_leaf,))
    return pos, idx, nodes, tris, prim


@pytest.mark.parametrize("case", ["heightfield", "spheres", "duplicates", "two"])
def test_built_tree_is_well_formed(tmp_path, case):
    # the 8-wide tree the build writes (treelet-restructured binary tree,
    # collapsed by the SAH costs): every node reached once from the root,
    # every triangle record once, the records the mesh's own triangles, and
    # every quantised child box around what it holds
    from illuminaprt_b200.ilg import GpuSpace
    if case == "heightfield":
        pos, idx = scenes.heightfield(128, 64, 0.2, 7)
    elif case == "spheres":
        f = scenes.sphere_field(3, 3, seed=2)
        pos, idx = f["pos"], f["idx"]
    elif case == "duplicates":
        pos, idx = scenes.heightfield(32, 16, 0.1, 3)
        idx = np.concatenate([idx, idx, idx[:5]])
    else:
        pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
        idx = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    sp = GpuSpace()
    sp.initialise(pos, idx)
    sp.build()
    path = str(tmp_path / "scene.ilg")
    sp.save(path)
    fpos, fidx, nodes, tris, prim = _read_scene_file(path)
    n = idx.shape[0]
    assert np.array_equal(np.sort(prim), np.arange(n))
    seen_nodes = np.zeros(nodes.shape[0], np.int32)
    seen_tris = np.zeros(n, np.int32)
    inf = np.full(3, np.inf)
    stack = [(0, -inf, inf)]  # node, the intersection of its ancestors' slot boxes
    while stack:
        x, acc_lo, acc_hi = stack.pop()
        seen_nodes[x] += 1
        q = nodes[x]
        org = q[0:3].view(np.float32).astype(np.float64)
        w = int(q[3])
        scale = np.array([2.0 ** (((w >> (8 * a)) & 0xFF) - 127) for a in range(3)])
        imask, cb, tb = w >> 24, int(q[4]), int(q[5])
        meta = [(int(q[6 + s // 4]) >> (8 * (s % 4))) & 0xFF for s in range(8)]
        planes = q[8:20].view(np.uint8).reshape(3, 4, 4)  # axis, (lo 0-3, lo 4-7, hi 0-3, hi 4-7), byte
        for s in range(8):
            if meta[s] == 0:
                continue
            lo = np.array([planes[a, s // 4, s % 4] for a in range(3)], np.float64) * scale + org
            hi = np.array([planes[a, 2 + s // 4, s % 4] for a in range(3)], np.float64) * scale + org
            lo, hi = np.maximum(lo, acc_lo), np.minimum(hi, acc_hi)
            if meta[s] == 0x80:
                assert imask >> s & 1
                stack.append((cb + bin(imask & ((1 << s) - 1)).count("1"), lo, hi))
            else:
                cnt, toff = meta[s] >> 5, meta[s] & 31
                for j in range(tb + toff, tb + toff + cnt):
                    seen_tris[j] += 1
                    p = prim[j]
                    a, b, cc = fpos[fidx[p]]
                    assert np.array_equal(tris[j, 0:3], a)
                    assert np.array_equal(tris[j, 4:7], (b - a).astype(np.float32))
                    assert np.array_equal(tris[j, 8:11], (cc - a).astype(np.float32))
                    for vtx in (a, b, cc):
                        assert np.all(vtx >= lo) and np.all(vtx <= hi), (x, s, vtx, lo, hi)
    assert np.all(seen_nodes == 1)
    assert np.all(seen_tris == 1)
