"""Parity of the sm_100a closest-hit / any-hit kernels (through the C ABI)."""
import glob
import os

import numpy as np
import pytest

from illuminaprt_b200 import scenes
from tests.parity import classify

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "heightfield_*.npz")))


def space_for(pos, idx):
    from illuminaprt_b200.ilg import GpuSpace
    s = GpuSpace()
    s.initialise(pos, idx)
    s.build()
    return s


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_closest_hit_matches_reference_golden(path, oracle):
    g = np.load(path)
    pos, idx, o4, d4 = g["pos"], g["idx"], g["o4"], g["d4"]
    got = space_for(pos, idx).intersects(o4, d4)
    for tree in ("kd", "bvh"):
        ref = (g[f"{tree}_prim"], g[f"{tree}_t"], g[f"{tree}_u"], g[f"{tree}_v"])
        n_same, ties, bad, bits_ok = classify(pos, idx, o4, d4, got, ref, oracle)
        assert bad == [], f"{tree}: non-tie mismatches at {bad[:10]}"
        assert bits_ok, f"{tree}: t/u/v bits differ on matching hits"
        assert ties <= max(2, len(o4) // 1000)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_any_hit_matches_reference_golden(path):
    g = np.load(path)
    occ = space_for(g["pos"], g["idx"]).occluded(g["so"], g["sd"])
    assert np.array_equal(occ, g["kd_occ"])


@pytest.mark.parametrize("nx,ny", [(256, 128), (97, 61)])
def test_closest_hit_matches_oracle_seeded(nx, ny, oracle):
    pos, idx = scenes.heightfield(nx, ny, 0.2, 7)
    co, cd = scenes.pinhole_rays(256, 256, (0.5, -0.6, 0.8), (0.5, 0.5, 0.0), (0, 0, 1), 60.0)
    io, idr = scenes.incoherent_rays(pos, idx, 65536, 8)
    o4 = np.concatenate([co, io])
    d4 = np.concatenate([cd, idr])
    got = space_for(pos, idx).intersects(o4, d4)
    ref = oracle.bvh(pos, idx).intersect(o4, d4)
    n_same, ties, bad, bits_ok = classify(pos, idx, o4, d4, got, ref, oracle)
    assert bad == [] and bits_ok
    assert ties <= len(o4) // 10000 + 2
    occ = space_for(pos, idx).occluded(o4, d4)
    assert np.array_equal(occ.astype(bool), ref[0] >= 0)


def test_full_size_heightfield_sample(oracle):
    """The 1,048,576-triangle heightfield; a seeded sample of both ray sets."""
    pos, idx = scenes.heightfield(1024, 512, 0.2, 1)
    co, cd = scenes.coherent_rays(2048)
    io, idr = scenes.incoherent_rays(pos, idx, 1 << 20, 2)
    rng = np.random.default_rng(5)
    pick = rng.choice(co.shape[0], 1 << 17, replace=False)
    o4 = np.concatenate([co[pick], io[: 1 << 17]])
    d4 = np.concatenate([cd[pick], idr[: 1 << 17]])
    sp = space_for(pos, idx)
    st = sp.stats()
    assert st["n_leaf_tris"] == idx.shape[0]
    got = sp.intersects(o4, d4)
    ref = oracle.bvh(pos, idx).intersect(o4, d4)
    n_same, ties, bad, bits_ok = classify(pos, idx, o4, d4, got, ref, oracle)
    assert bad == [] and bits_ok
    # near ties (two valid hits < 1e-5 apart, decided by visit order) came to
    # 1.5e-5 of the full 8,388,608-ray workload against the reference's BVH;
    # the reference's own KD-tree and BVH disagree at 1.3e-5
    assert ties / len(o4) < 5e-5
    # size-independent property on the whole incoherent set: a ray that hits
    # reports a t inside its window and barycentrics inside the triangle
    p, t, u, v = sp.intersects(io, idr)
    h = p >= 0
    assert (t[h] >= 1e-5).all() and (u[h] >= 0).all() and (v[h] >= 0).all() and ((u + v)[h] <= 1.0).all()
    # determinism
    p2, t2, _, _ = sp.intersects(io, idr)
    assert np.array_equal(p, p2) and np.array_equal(t.view(np.uint32), t2.view(np.uint32))


@pytest.mark.parametrize("ntris", [1, 2, 3, 4, 9])
def test_tiny_scenes(ntris, oracle):
    rng = np.random.default_rng(ntris)
    pos = rng.random((3 * ntris, 3)).astype(np.float32)
    idx = np.arange(3 * ntris, dtype=np.uint32).reshape(-1, 3)
    o4 = np.zeros((4096, 4), np.float32)
    d4 = np.zeros((4096, 4), np.float32)
    o4[:, :3] = rng.random((4096, 3)) * 2 - 0.5
    dd = rng.normal(size=(4096, 3))
    d4[:, :3] = dd / np.linalg.norm(dd, axis=1, keepdims=True)
    d4[:, 3] = 3.4e38
    got = space_for(pos, idx).intersects(o4, d4)
    ref = oracle.intersect_brute(pos, idx, o4, d4)
    n_same, ties, bad, bits_ok = classify(pos, idx, o4, d4, got, ref, oracle)
    assert bad == [] and bits_ok


def test_degenerate_and_duplicate_triangles(oracle):
    pos, idx = scenes.heightfield(32, 16, 0.1, 3)
    # duplicate every triangle and add zero-area ones: identical centroids stress the build
    idx = np.concatenate([idx, idx, np.array([[0, 0, 0], [1, 1, 2]], np.uint32)])
    co, cd = scenes.pinhole_rays(64, 64, (0.5, -0.6, 0.8), (0.5, 0.5, 0.0), (0, 0, 1), 60.0)
    got = space_for(pos, idx).intersects(co, cd)
    ref = oracle.intersect_brute(pos, idx, co, cd)
    n_same, ties, bad, bits_ok = classify(pos, idx, co, cd, got, ref, oracle)
    assert bad == [] and bits_ok


def test_device_pointer_path_and_errors():
    import torch
    from illuminaprt_b200.ilg import GpuSpace, IlgError, ILG_ESTATE, ILG_EINVAL
    pos, idx = scenes.heightfield(64, 32, 0.2, 1)
    co, cd = scenes.pinhole_rays(64, 64, (0.5, -0.6, 0.8), (0.5, 0.5, 0.0), (0, 0, 1), 60.0)
    s = GpuSpace()
    with pytest.raises(IlgError) as e:
        s.intersects(co, cd)
    assert e.value.code == ILG_ESTATE
    with pytest.raises(IlgError) as e:
        s.initialise(pos, np.array([[0, 1, 10 ** 7]], np.uint32))
    assert e.value.code == ILG_EINVAL
    s.initialise(pos, idx)
    s.build()
    host = s.intersects(co, cd)
    o = torch.from_numpy(co).cuda()
    d = torch.from_numpy(cd).cuda()
    n = co.shape[0]
    prim = torch.empty(n, dtype=torch.int32, device="cuda")
    t, u, v = (torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(3))
    torch.cuda.synchronize()
    s.intersects_into(o, d, prim, t, u, v, device_ptrs=True)
    s.sync()
    assert np.array_equal(prim.cpu().numpy(), host[0])
    assert np.array_equal(t.cpu().numpy().view(np.uint32), host[1].view(np.uint32))
    # zero rays is a no-op
    s.intersects(co[:0], cd[:0])


@pytest.mark.parametrize("first,count", [(0, 1), (1000, 2048), (5000, 3000)])
def test_excluding_queries_match_oracle_without_the_range(first, count, oracle):
    # the p_pExclude overloads: the oracle sees the mesh with the range removed
    pos, idx = scenes.heightfield(64, 64, 0.2, 11)
    n_tris = idx.shape[0]
    co, cd = scenes.pinhole_rays(64, 64, (0.5, -0.6, 0.8), (0.5, 0.5, 0.0), (0, 0, 1), 60.0)
    io, idr = scenes.incoherent_rays(pos, idx, 8192, 12)
    o4, d4 = np.concatenate([co, io]), np.concatenate([cd, idr])
    sp = space_for(pos, idx)
    got = sp.intersects_excluding(o4, d4, first, count)
    keep = np.r_[0:first, first + count:n_tris]
    rp, rt, ru, rv = oracle.bvh(pos, idx[keep]).intersect(o4, d4)
    rp = np.where(rp >= 0, keep[np.maximum(rp, 0)], rp).astype(np.int32)
    n_same, ties, bad, bits_ok = classify(pos, idx, o4, d4, got, (rp, rt, ru, rv), oracle)
    assert bad == [] and bits_ok
    assert not np.isin(got[0], np.arange(first, first + count)).any()
    occ = sp.occluded_excluding(o4, d4, first, count)
    assert np.array_equal(occ.astype(bool), rp >= 0)
    # an empty range is the plain query
    assert np.array_equal(sp.intersects_excluding(o4, d4, 0, 0)[0], sp.intersects(o4, d4)[0])


def _wt_genuine(oracle, pos, idx, o4, d4, i, p):
    # is triangle p a hit of the watertight test for ray i?
    r = oracle.watertight_brute(pos, idx[p:p + 1], o4[i:i + 1], d4[i:i + 1])
    return r[0][0] == 0, r[1][0]


@pytest.mark.parametrize("nx,ny", [(64, 32), (97, 61)])
def test_watertight_mode_matches_its_oracle(nx, ny, oracle):
    from tests.watertight_rays import shared_edge_rays
    pos, idx = scenes.heightfield(nx, ny, 0.2, 5)
    idx = idx.astype(np.uint32)
    co, cd = scenes.pinhole_rays(128, 128, (0.5, -0.6, 0.8), (0.5, 0.5, 0.0), (0, 0, 1), 60.0)
    io, idr = scenes.incoherent_rays(pos, idx, 8192, 6)
    eo, ed = shared_edge_rays(pos, idx, 8192, 7)
    o4, d4 = np.concatenate([co, io, eo]), np.concatenate([cd, idr, ed])
    sp = space_for(pos, idx)
    gp, gt, gu, gv = sp.intersects(o4, d4, watertight=True)
    rp, rt, ru, rv, rocc = oracle.watertight_brute(pos, idx, o4, d4)
    same = gp == rp
    hit = same & (gp >= 0)
    # the device evaluates the test operation for operation as the oracle does
    assert np.array_equal(gt[hit].view(np.uint32), rt[hit].view(np.uint32))
    assert np.array_equal(gu[hit].view(np.uint32), ru[hit].view(np.uint32))
    assert np.array_equal(gv[hit].view(np.uint32), rv[hit].view(np.uint32))
    # other differences: two genuine hits within the tie window, found in another order
    bad = []
    for i in np.nonzero(~same)[0]:
        ok = gp[i] >= 0 and rp[i] >= 0 and abs(float(gt[i]) - float(rt[i])) < 1e-5
        ok = ok and _wt_genuine(oracle, pos, idx, o4, d4, i, gp[i])[0]
        if not ok:
            bad.append(int(i))
    assert bad == [], bad[:10]
    assert (~same).sum() <= len(o4) // 5000 + 2
    # no edge rays fall through, and any hit is the same predicate
    assert (gp[len(co) + len(io):] >= 0).all()
    assert np.array_equal(sp.occluded(o4, d4, watertight=True), rocc)


def test_watertight_mode_closes_the_reference_edge_cracks(oracle):
    from tests.watertight_rays import shared_edge_rays
    pos, idx = scenes.heightfield(64, 32, 0.2, 3)
    o4, d4 = shared_edge_rays(pos, idx, 65536, 9)
    sp = space_for(pos, idx)
    ref_mode = sp.intersects(o4, d4)[0]
    wt_mode = sp.intersects(o4, d4, watertight=True)[0]
    brute = oracle.intersect_brute(pos, idx.astype(np.uint32), o4, d4)[0]
    assert np.array_equal(ref_mode < 0, brute < 0)  # the reference test's cracks, reproduced
    assert (ref_mode < 0).sum() > 100
    assert (wt_mode < 0).sum() == 0


def test_pageable_host_buffers_give_the_pinned_results():
    """Host rays and hits in pageable memory (plain numpy) go through the
    context's three page-locked slots in chunks (here eight of 337,536 rays);
    the answers must equal those from page-locked buffers, for both queries
    and both triangle tests, on a ragged batch that uses every slot more
    than once."""
    import torch
    from illuminaprt_b200.ilg import GpuSpace
    pos, idx = scenes.heightfield(256, 128, 0.2, 4)
    sp = GpuSpace()
    sp.initialise(pos, idx)
    sp.build()
    o4, d4 = scenes.incoherent_rays(pos, idx, 2_700_001, 6)
    po, pd = torch.from_numpy(o4).pin_memory(), torch.from_numpy(d4).pin_memory()
    n = o4.shape[0]
    for wt in (False, True):
        pinned = (torch.empty(n, dtype=torch.int32).pin_memory(), *(torch.empty(n).pin_memory() for _ in range(3)))
        sp.intersects_into(po, pd, *pinned, device_ptrs=False, watertight=wt)
        got = sp.intersects(o4, d4, watertight=wt)
        for a, b in zip(got, pinned):
            assert np.array_equal(np.asarray(a).view(np.uint32), b.numpy().view(np.uint32))
        occ = sp.occluded(o4, d4, watertight=wt)
        assert np.array_equal(occ.astype(bool), pinned[0].numpy() >= 0)
    sp.close()


def test_fast_build_answers_the_same_queries_with_more_work(oracle):
    # ILG_BUILD_FAST keeps the Morton tree (no treelet restructuring): the same
    # hits up to near ties, and more node and triangle visits a ray than the
    # default SAH-restructured tree
    import torch
    from illuminaprt_b200.ilg import GpuSpace
    pos, idx = scenes.heightfield(256, 128, 0.2, 7)
    io, idr = scenes.incoherent_rays(pos, idx, 65536, 9)
    spaces = {}
    for fast in (False, True):
        sp = GpuSpace(fast_build=fast)
        sp.initialise(pos, idx)
        sp.build()
        spaces[fast] = sp
    best, fast = spaces[False].intersects(io, idr), spaces[True].intersects(io, idr)
    n_same, ties, bad, bits_ok = classify(pos, idx, io, idr, best, fast, oracle)
    assert bad == [] and bits_ok and ties <= len(io) // 10000 + 2
    O, D = torch.from_numpy(io).cuda(), torch.from_numpy(idr).cuda()
    work = {k: sum(sp.traversal_counts(O, D)) for k, sp in spaces.items()}
    assert work[False] < 0.95 * work[True], work


def test_ray_interval_edges_match_oracle(oracle):
    # the ray's [Min, Max] interval: Max before the first hit, Min before it,
    # Min past Max. The reference's triangle test ignores Min (it rejects
    # t < 1e-5 instead, IndexedTriangle.cpp:115); only its trees' box tests
    # use Min, so a hit before Min is reported or not as the tree's boxes
    # decide. Rays whose Min lies past their first hit are therefore checked
    # apart: whatever the device reports must be a genuine hit of the
    # reference's test, and a ray the device misses must have its first hit
    # before Min.
    pos, idx = scenes.heightfield(64, 32, 0.2, 5)
    co, cd = scenes.pinhole_rays(64, 64, (0.5, -0.6, 0.8), (0.5, 0.5, 0.0), (0, 0, 1), 60.0)
    n = co.shape[0]
    rng = np.random.default_rng(3)
    o4, d4 = co.copy(), cd.copy()
    full = space_for(pos, idx).intersects(co, cd)
    t_hit = np.where(full[0] >= 0, full[1], 2.0).astype(np.float32)
    kind = rng.integers(0, 4, n)
    o4[kind == 0, 3] = 0.5 * t_hit[kind == 0]          # Min before the hit
    o4[kind == 1, 3] = 1.5 * t_hit[kind == 1]          # Min past the hit
    d4[kind == 2, 3] = 0.5 * t_hit[kind == 2]          # Max before the hit
    o4[kind == 3, 3] = 1.0
    d4[kind == 3, 3] = 0.5                              # Min > Max
    got = space_for(pos, idx).intersects(o4, d4)
    ref = oracle.intersect_brute(pos, idx, o4, d4)
    keep = kind != 1
    sub = lambda r: tuple(x[keep] for x in r)
    n_same, ties, bad, bits_ok = classify(pos, idx, o4[keep], d4[keep], sub(got), sub(ref), oracle)
    assert bad == [] and bits_ok
    assert (got[0][kind == 2] == -1).all()
    for i in np.nonzero(kind == 1)[0]:
        if got[0][i] >= 0:
            acc, t, _, _ = oracle.shirley(pos, idx.reshape(-1), got[0][i], o4[i], d4[i], d4[i, 3])
            assert acc and np.float32(t).view(np.uint32) == got[1][i].view(np.uint32)
        else:
            assert full[0][i] == -1 or full[1][i] < o4[i, 3]


def test_large_host_batch_in_many_chunks():
    # a host-buffer call of 5,000,003 rays runs in 9 chunks of about 512 K
    # over three streams, the last one short; its hits equal the
    # device-pointer call's
    import torch
    from illuminaprt_b200.ilg import GpuSpace
    pos, idx = scenes.heightfield(256, 128, 0.2, 2)
    io, idr = scenes.incoherent_rays(pos, idx, 5_000_003, 4)
    sp = GpuSpace()
    sp.initialise(pos, idx)
    sp.build()
    n = io.shape[0]
    host = (torch.empty(n, dtype=torch.int32).pin_memory(), *(torch.empty(n).pin_memory() for _ in range(3)))
    sp.intersects_into(torch.from_numpy(io).pin_memory(), torch.from_numpy(idr).pin_memory(), *host,
                       device_ptrs=False)
    O, D = torch.from_numpy(io).cuda(), torch.from_numpy(idr).cuda()
    dev = (torch.empty(n, dtype=torch.int32, device="cuda"), *(torch.empty(n, device="cuda") for _ in range(3)))
    sp.intersects_into(O, D, *dev, device_ptrs=True)
    sp.sync()
    for a, b in zip(host, dev):
        assert torch.equal(a, b.cpu())
