"""ilg_intersect_noalloc: the closest-hit query for callers that cannot
allocate device memory when they query.

A renderer that issues its ray queries inside a frame whose device memory was
budgeted and handed out up front, or a process whose device memory belongs to
another allocator, must not have the library call cudaMalloc behind its back.
ilg_intersect may do exactly that (it grows its staging buffers on demand);
ilg_intersect_noalloc stages through one fixed device array instead and so
accepts at most ILG_NOALLOC_MAX_RAYS rays per call.

These tests call the entry point through the C ABI and require its hits to be
the ones ilg_intersect returns for the same rays, bit for bit (the tolerance
every closest-hit test here uses), on two calls in a row, the second smaller
than the first so the array still holds the first call's data.

This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from illuminaprt_b200 import scenes

pytestmark = pytest.mark.gpu


def _noalloc(sp, o4, d4):
    o4 = np.ascontiguousarray(o4, np.float32)
    d4 = np.ascontiguousarray(d4, np.float32)
    n = o4.shape[0]
    prim = np.full(n, -7, np.int32)
    t, u, v = (np.full(n, np.nan, np.float32) for _ in range(3))
    rc = sp.L.ilg_intersect_noalloc(sp.h, o4.ctypes.data, d4.ctypes.data, n, prim.ctypes.data, t.ctypes.data,
                                    u.ctypes.data, v.ctypes.data)
    return rc, (prim, t, u, v)


def _same(a, b):
    return (np.array_equal(a[0], b[0]) and
            all(np.array_equal(x.view(np.uint32), y.view(np.uint32)) for x, y in zip(a[1:], b[1:])))


def test_noalloc_matches_intersect_on_two_calls_in_a_row():
    from illuminaprt_b200.ilg import GpuSpace, ILG_OK
    pos, idx = scenes.heightfield(256, 128, 0.2, 5)
    sp = GpuSpace()
    sp.initialise(pos, idx)
    sp.build()
    io, idr = scenes.incoherent_rays(pos, idx, 1 << 17, 6)
    co, cd = scenes.pinhole_rays(256, 256, (0.5, -0.6, 0.8), (0.5, 0.5, 0.0), (0, 0, 1), 60.0)
    calls = [(io, idr), (co[:50000], cd[:50000])]
    for o4, d4 in calls:
        rc, got = _noalloc(sp, o4, d4)
        assert rc == ILG_OK, sp.L.ilg_last_error(sp.h)
        want = sp.intersects(o4, d4)
        assert _same(got, want)
        assert (got[0] >= 0).any()
    sp.close()


def test_noalloc_allocates_no_device_memory():
    """The property the entry point exists for: once a context exists, a call
    leaves the device's free memory unchanged (ilg_create made the fixed array
    resident and loaded the traversal kernel). Checked on a fresh context
    before any ilg_intersect call, which would grow the context's staging."""
    import torch
    from illuminaprt_b200.ilg import GpuSpace, ILG_OK
    pos, idx = scenes.heightfield(128, 64, 0.2, 9)
    sp = GpuSpace()
    sp.initialise(pos, idx)
    sp.build()
    io, idr = scenes.incoherent_rays(pos, idx, 1 << 16, 3)
    rc, first = _noalloc(sp, io[:1000], idr[:1000])
    assert rc == ILG_OK, sp.L.ilg_last_error(sp.h)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(0)[0]
    rc, second = _noalloc(sp, io, idr)
    assert rc == ILG_OK, sp.L.ilg_last_error(sp.h)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free_before
    assert _same(second, sp.intersects(io, idr))
    sp.close()


def test_noalloc_rejects_batches_over_the_limit():
    from illuminaprt_b200.ilg import GpuSpace, ILG_EINVAL, ILG_NOALLOC_MAX_RAYS
    pos, idx = scenes.heightfield(16, 8, 0.2, 5)
    sp = GpuSpace()
    sp.initialise(pos, idx)
    sp.build()
    one = np.zeros((1, 4), np.float32)
    out = np.zeros(1, np.float32)
    rc = sp.L.ilg_intersect_noalloc(sp.h, one.ctypes.data, one.ctypes.data, ILG_NOALLOC_MAX_RAYS + 1,
                                    out.ctypes.data, out.ctypes.data, out.ctypes.data, out.ctypes.data)
    assert rc == ILG_EINVAL
    assert b"exceed the maximum" in sp.L.ilg_last_error(sp.h)
    # the largest allowed batch goes through and still agrees with ilg_intersect
    o4 = np.tile(np.array([[0.5, 0.5, 1.0, 0.0]], np.float32), (ILG_NOALLOC_MAX_RAYS, 1))
    d4 = np.tile(np.array([[0.0, 0.0, -1.0, 3.4e38]], np.float32), (ILG_NOALLOC_MAX_RAYS, 1))
    rc, got = _noalloc(sp, o4, d4)
    assert rc == 0
    assert _same(got, sp.intersects(o4, d4))
    sp.close()
