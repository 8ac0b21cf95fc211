"""The BF16 tensor-core MLP kernels against the float64 CPU oracle."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


GRID = np.random.default_rng(17).uniform(-0.3, 0.3, mo.GRID_PARAMS).astype(np.float32)


@pytest.fixture(scope="module")
def net():
    from illuminaprt_b200.ilg import GpuSpace
    sp = GpuSpace()
    sp.mlp_init(seed=7, lr=1e-2)
    sp.mlp_set_grid(GRID)  # features large enough that the encoding matters
    return sp


def test_forward_matches_oracle(net):
    raw, _ = mo.random_batch(5000, seed=1)  # not a multiple of 16: ragged last tile
    p = net.mlp_params()
    y_gpu = net.mlp_infer(raw)
    y_ref, _, _ = mo.forward(p, raw, net.mlp_grid(), bf=True)
    scale = np.abs(y_ref).max()
    err = np.abs(y_gpu - y_ref).max() / scale
    print(f"forward: max |gpu - oracle| / max|y| = {err:.2e}")
    assert err < 1e-2
    assert np.mean(np.abs(y_gpu - y_ref)) / np.mean(np.abs(y_ref)) < 2e-3


@pytest.mark.parametrize("n", [16, 1000, 20000])
def test_gradients_match_oracle(net, n):
    raw, tgt = mo.random_batch(n, seed=n)
    p = net.mlp_params()
    grid = net.mlp_grid()
    loss_g, g_gpu = net.mlp_grads(raw, tgt)
    gg_gpu = net.mlp_grid_grads()
    loss_r, g_ref, gg_ref = mo.loss_and_grads(p, raw, tgt, grid, bf=True)
    loss_x, g_exact, _ = mo.loss_and_grads(p, raw, tgt, grid, bf=False)
    rel = np.linalg.norm(g_gpu - g_ref) / np.linalg.norm(g_ref)
    cos_exact = g_gpu @ g_exact / (np.linalg.norm(g_gpu) * np.linalg.norm(g_exact))
    print(f"n={n}: loss gpu {loss_g:.6f} oracle {loss_r:.6f}; grad rel err vs bf16 oracle {rel:.2e}; "
          f"cosine vs exact float64 {cos_exact:.5f}")
    assert abs(loss_g - loss_r) <= 1e-3 * abs(loss_r) + 1e-6
    assert rel < 3e-2
    assert cos_exact > 0.995
    # the hash-grid part: every touched entry, against the bf16 oracle
    rel_g = np.linalg.norm(gg_gpu - gg_ref) / np.linalg.norm(gg_ref)
    print(f"n={n}: grid grad rel err {rel_g:.2e}, {np.count_nonzero(gg_ref)} entries touched")
    assert rel_g < 3e-2
    assert np.array_equal(gg_gpu != 0, gg_ref != 0) or n >= 1000
    # per layer, too
    for l in range(mo.LAYERS):
        a, b = g_gpu[mo.OFFS[l]:mo.OFFS[l + 1]], g_ref[mo.OFFS[l]:mo.OFFS[l + 1]]
        assert np.linalg.norm(a - b) <= 5e-2 * np.linalg.norm(b) + 1e-9, l


def test_set_get_params_round_trip(net):
    p = mo.init_params(seed=3)
    net.mlp_set_params(p)
    assert np.array_equal(net.mlp_params(), p)
    net.mlp_set_grid(GRID)
    assert np.array_equal(net.mlp_grid(), GRID)
    raw, _ = mo.random_batch(333, seed=9)
    y_ref, _, _ = mo.forward(p, raw, GRID, bf=True)
    assert np.abs(net.mlp_infer(raw) - y_ref).max() < 1e-2 * np.abs(y_ref).max()


def test_training_fits_a_smooth_field():
    from illuminaprt_b200.ilg import GpuSpace
    sp = GpuSpace()
    sp.mlp_init(seed=11, lr=1e-2)
    raw, tgt = mo.random_batch(1 << 15, seed=12)
    losses = [sp.mlp_train_step(raw[i % 4::4], tgt[i % 4::4]) for i in range(400)]
    test_raw, test_tgt = mo.random_batch(4096, seed=13)
    y = sp.mlp_infer(test_raw)
    rel = np.mean((y - test_tgt) ** 2 / (test_tgt ** 2 + 0.01))
    print(f"training: loss {losses[0]:.4f} -> {losses[-1]:.5f}; held-out relative L2 {rel:.5f}")
    assert losses[-1] < losses[0] / 20
    # measured 0.008 - 0.028 across runs: the fine grid levels see few points
    # per entry and float atomics change the summation order from run to run
    assert rel < 0.05


@pytest.mark.parametrize("n", [1, 127, 128, 129, 70000])
def test_tcgen05_inference_matches_warp_mma(net, n):
    """The tcgen05 (TMEM-accumulating) inference kernel against the warp-level
    mma.sync kernel and the oracle, on ragged row counts."""
    raw, tgt = mo.random_batch(max(n, 1), seed=n + 5)
    for _ in range(3):  # move the weights away from their initial values
        net.mlp_train_step(raw[:4096], tgt[:4096])
    y_tc = net.mlp_infer(raw)
    y_warp = net.mlp_infer(raw, warp_mma=True)
    y_ref, _, _ = mo.forward(net.mlp_params(), raw, net.mlp_grid(), bf=True)
    scale = np.abs(y_ref).max() + 1e-6
    d_warp = np.abs(y_tc - y_warp).max() / scale
    d_ref = np.abs(y_tc - y_ref).max() / scale
    print(f"n={n}: tcgen05 vs mma.sync {d_warp:.2e}, vs oracle {d_ref:.2e}")
    assert d_warp < 1e-2 and d_ref < 1e-2
    assert np.mean(np.abs(y_tc - y_warp)) / (np.mean(np.abs(y_warp)) + 1e-9) < 2e-3


@pytest.mark.parametrize("n", [16, 5000])
def test_frequency_encoding_matches_oracle(n):
    """The frequency-only encoding (12 bands of position + raw direction,
    normal, roughness, albedo): forward and gradients against the oracle."""
    from illuminaprt_b200.ilg import GpuSpace
    sp = GpuSpace()
    sp.mlp_init(seed=5, lr=1e-2, encoding="freq12")
    raw, tgt = mo.random_batch(n, seed=n + 1)
    for _ in range(2):  # move the weights away from their initial values
        sp.mlp_train_step(raw, tgt)
    p = sp.mlp_params()
    y_ref, _, _ = mo.forward(p, raw, None, bf=True, encoding="freq12")
    y = sp.mlp_infer(raw)
    y_warp = sp.mlp_infer(raw, warp_mma=True)
    scale = np.abs(y_ref).max()
    assert np.abs(y - y_ref).max() / scale < 1e-2 and np.abs(y_warp - y_ref).max() / scale < 1e-2
    loss_g, g_gpu = sp.mlp_grads(raw, tgt)
    loss_r, g_ref, gg_ref = mo.loss_and_grads(p, raw, tgt, None, bf=True, encoding="freq12")
    _, g_exact, _ = mo.loss_and_grads(p, raw, tgt, None, bf=False, encoding="freq12")
    rel = np.linalg.norm(g_gpu - g_ref) / np.linalg.norm(g_ref)
    cos_exact = g_gpu @ g_exact / (np.linalg.norm(g_gpu) * np.linalg.norm(g_exact))
    print(f"freq12 n={n}: loss {loss_g:.6f} / {loss_r:.6f}; grad rel err {rel:.2e}; cosine vs exact {cos_exact:.5f}")
    assert abs(loss_g - loss_r) <= 1e-3 * abs(loss_r) + 1e-6
    assert rel < 3e-2 and cos_exact > 0.995
    assert not gg_ref.any()
    sp.close()


@pytest.mark.parametrize("encoding", ["hashgrid", "freq12"])
def test_tcgen05_training_matches_warp_mma_training(encoding):
    """Training's forward, loss, backward and weight gradients on tcgen05
    (the default) against the warp-level mma.sync kernels on the same batch:
    the same BF16 rounding points, FP32 accumulation in another order."""
    from illuminaprt_b200.ilg import GpuSpace
    sp = GpuSpace()
    sp.mlp_init(seed=13, lr=1e-2, encoding=encoding)
    if encoding == "hashgrid":
        sp.mlp_set_grid(GRID)
    raw, tgt = mo.random_batch(3000, seed=21)  # 23.4 tiles of 128 rows: ragged last tile
    for _ in range(2):
        sp.mlp_train_step(raw, tgt)
    l_tc, g_tc = sp.mlp_grads(raw, tgt)
    l_mma, g_mma = sp.mlp_grads(raw, tgt, warp_mma=True)
    rel = np.linalg.norm(g_tc - g_mma) / np.linalg.norm(g_mma)
    print(f"{encoding}: loss tcgen05 {l_tc:.6f} mma.sync {l_mma:.6f}; grad rel diff {rel:.2e}")
    assert abs(l_tc - l_mma) <= 1e-3 * abs(l_mma) + 1e-7
    assert rel < 1e-2
    for l in range(mo.LAYERS):
        a, b = g_tc[mo.OFFS[l]:mo.OFFS[l + 1]], g_mma[mo.OFFS[l]:mo.OFFS[l + 1]]
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-9, l
    sp.close()
