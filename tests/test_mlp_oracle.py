"""The MLP oracle's hand-written backward pass against torch float64 autograd
and finite differences (no GPU)."""
import numpy as np

from oracle import mlp_oracle as mo


def test_backward_matches_autograd():
    import torch
    raw, tgt = mo.random_batch(64, seed=3)
    p = mo.init_params(seed=1).astype(np.float64)
    grid = np.random.default_rng(5).uniform(-0.5, 0.5, mo.GRID_PARAMS).astype(np.float32)
    loss, g, gg = mo.loss_and_grads(p, raw, tgt, grid, bf=False)
    pt = torch.tensor(p, dtype=torch.float64, requires_grad=True)
    gt = torch.tensor(grid, dtype=torch.float64, requires_grad=True)
    x = torch.tensor(mo.encode(raw, grid), dtype=torch.float64)
    # grid columns: the oracle's float32 values, differentiated through the
    # trilinear interpolation (linear in the grid)
    pos = raw[:, 0:3]
    cols = []
    gv = gt.reshape(mo.GRID_LEVELS, mo.GRID_SIZE, mo.GRID_FEAT)
    for l in range(mo.GRID_LEVELS):
        idx, w = mo.grid_corners(pos, l)
        lin = sum(torch.tensor(w[:, c:c + 1], dtype=torch.float64) * gv[l, torch.tensor(idx[:, c])]
                  for c in range(8))
        cols.append(lin - lin.detach())
    x = x + torch.nn.functional.pad(torch.cat(cols, 1), (0, mo.IN - 2 * mo.GRID_LEVELS))
    h = x
    for l in range(mo.LAYERS):
        w = pt[mo.OFFS[l]:mo.OFFS[l + 1]].reshape(mo.DIMS[l])
        h = h @ w
        if l < mo.LAYERS - 1:
            h = torch.relu(h)
    y = h[:, :3]
    t = torch.tensor(tgt, dtype=torch.float64)
    tl = (((y - t) ** 2) / (y.detach() ** 2 + 0.01)).mean()
    tl.backward()
    ga = pt.grad.numpy().copy()
    ga[mo.OFFS[5]:].reshape(mo.HID, mo.OUTP)[:, 3:] = 0.0
    assert abs(tl.item() - loss) < 1e-12
    assert np.allclose(g, ga, rtol=1e-9, atol=1e-12)
    assert np.allclose(gg, gt.grad.numpy(), rtol=1e-9, atol=1e-14)
    assert np.count_nonzero(gg) > 1000


def test_backward_matches_finite_differences():
    raw, tgt = mo.random_batch(32, seed=4)
    p = mo.init_params(seed=2).astype(np.float64)
    grid = mo.init_grid(seed=2)
    _, g, _ = mo.loss_and_grads(p, raw, tgt, grid, bf=False)

    def f(q):
        y, _, _ = mo.forward(q, raw, grid, bf=False)
        # the loss treats its denominator as a constant, evaluated at p
        y0, _, _ = mo.forward(p, raw, grid, bf=False)
        return np.sum((y - tgt) ** 2 / (y0 * y0 + 0.01)) / (3 * y.shape[0])

    rng = np.random.default_rng(0)
    for i in rng.choice(mo.OFFS[5] + 3, 12, replace=False):
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (f(p + e) - f(p - e)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    # bf16 keeps 7 fraction bits: the spacing above 1 is 2^-7
    x = np.array([1.0, 1.00390625, 1.001953125, 1.005859375, -3.14159, 0.0, 1.01171875])
    r = mo.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0          # 1 + 2^-8: a tie, rounds to the even neighbour
    assert r[2] == 1.0          # below the midpoint
    assert r[3] == 1.0078125    # above the midpoint
    assert r[6] == 1.015625     # 1 + 3 * 2^-8: a tie, rounds to even (1 + 2^-6)
    assert abs(r[4] + 3.140625) < 1e-12


def test_grid_indexing():
    # dense levels cover every corner without collisions; hashed ones stay in range
    assert mo.GRID_RES[0] == 16 and mo.GRID_RES[-1] == 2048
    pos = np.random.default_rng(1).random((4096, 3)).astype(np.float32)
    for l in range(mo.GRID_LEVELS):
        idx, w = mo.grid_corners(pos, l)
        assert idx.min() >= 0 and idx.max() < mo.GRID_SIZE
        assert np.allclose(w.sum(1), 1.0, atol=1e-6)
        if (mo.GRID_RES[l] + 1) ** 3 <= mo.GRID_SIZE:
            assert len(np.unique(idx[0])) == 8
    # a constant grid encodes to that constant everywhere
    g = np.full(mo.GRID_PARAMS, 0.25, np.float32)
    assert np.allclose(mo.grid_features(g, pos), 0.25, atol=1e-6)


def test_frequency_encoding_backward_matches_autograd():
    import torch
    raw, tgt = mo.random_batch(48, seed=8)
    x = mo.encode(raw, None, "freq12")
    # columns as documented: band 11 of axis 2, then the raw features and the constant
    # band 11 of axis 2, three doublings after the band-8 anchor: a few ulp from the exact value
    assert np.allclose(x[:, 24 * 2 + 22], np.sin(np.pi * raw[:, 2].astype(np.float64) * 2048), rtol=0, atol=2e-6)
    assert np.array_equal(x[:, 72:82], raw[:, 3:13].astype(np.float64)) and (x[:, 82] == 1).all()
    assert not x[:, 83:].any()
    p = mo.init_params(seed=2).astype(np.float64)
    loss, g, gg = mo.loss_and_grads(p, raw, tgt, None, bf=False, encoding="freq12")
    pt = torch.tensor(p, dtype=torch.float64, requires_grad=True)
    h = torch.tensor(x, dtype=torch.float64)
    for l in range(mo.LAYERS):
        w = pt[mo.OFFS[l]:mo.OFFS[l + 1]].reshape(mo.DIMS[l])
        h = h @ w
        if l < mo.LAYERS - 1:
            h = torch.relu(h)
    y = h[:, :3]
    t = torch.tensor(tgt, dtype=torch.float64)
    lt = ((y - t) ** 2 / (y.detach() ** 2 + 0.01)).mean()
    lt.backward()
    gref = pt.grad.numpy().copy()
    gref[mo.OFFS[5]:].reshape(mo.HID, mo.OUTP)[:, 3:] = 0.0
    assert abs(loss - lt.item()) < 1e-12
    assert np.allclose(g, gref, rtol=1e-9, atol=1e-12)
    assert not gg.any()
