"""Device post-processing (ilg_accumulate, ilg_tonemap) against the
reference's own AccumulationBuffer, GlobalTone, AutoTone and DragoTone
(Core/Postproc/*.h, compiled from the reference tree)."""
import numpy as np
import pytest

from oracle import bindings

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not bindings.ref_available(), reason="reference engine library not built")]


def _frames(n, h, w, seed):
    rng = np.random.default_rng(seed)
    # HDR-like values: mostly below 1, a tail up to ~50
    return (rng.random((n, h, w, 3)) ** 4 * 50).astype(np.float32)


@pytest.fixture(scope="module")
def space():
    from illuminaprt_b200.ilg import GpuSpace
    return GpuSpace()


def test_accumulation_is_the_reference_bit_for_bit(space):
    ref = bindings.RefLib()
    fr = _frames(7, 23, 37, 1)  # odd sizes
    space.accumulate_reset()
    for k in range(fr.shape[0]):
        out = space.accumulate(fr[k])
        assert np.array_equal(out.view(np.uint32), ref.postprocess("accumulate", fr[:k + 1]).view(np.uint32)), k
    # reset starts over; a new size starts over too
    space.accumulate_reset()
    assert np.array_equal(space.accumulate(fr[3]), fr[3])
    small = _frames(1, 5, 4, 2)[0]
    assert np.array_equal(space.accumulate(small), small)


@pytest.mark.parametrize("op", ["global", "auto"])
def test_tone_operators_are_the_reference_bit_for_bit(space, op):
    ref = bindings.RefLib()
    img = _frames(1, 61, 97, 3)[0]
    got = space.tonemap(img, op)
    want = ref.postprocess(op, img)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_drago_matches_the_reference(space):
    ref = bindings.RefLib()
    img = _frames(1, 61, 97, 4)[0]
    got = space.tonemap(img, "drago")
    want = ref.postprocess("drago", img)
    ulps = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
    print(f"drago: {np.mean(ulps == 0):.4f} of values bit-equal, max {ulps.max()} ulp")
    # measured on a B200: every value bit-equal (double log10/log/pow, rounded to float)
    assert ulps.max() <= 1
    assert np.mean(ulps == 0) > 0.99


def test_progressive_frames_stay_on_the_device(space):
    # render -> accumulate -> tone map on the device; one copy back at the end
    import torch
    from illuminaprt_b200 import scenes
    from illuminaprt_b200.ilg import GpuSpace
    sp = GpuSpace()
    box = scenes.load_box_scene(sp)
    W = H = 64
    frame = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    avg = torch.empty_like(frame)
    shown = torch.empty_like(frame)
    host_frames = []
    sp.accumulate_reset()
    for f in range(6):
        sp.render(box["camera"], W, H, 4, seed=50 + f, out=frame)
        sp.accumulate(frame, out=avg)
        sp.tonemap(avg, "global", out=shown)
        sp.sync()
        host_frames.append(frame.cpu().numpy())
    ref = bindings.RefLib()
    want_avg = ref.postprocess("accumulate", np.stack(host_frames))
    assert np.array_equal(avg.cpu().numpy(), want_avg)
    assert np.array_equal(shown.cpu().numpy(), ref.postprocess("global", want_avg))
