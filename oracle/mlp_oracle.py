"""CPU oracle of the radiance-cache MLP - TEST INFRASTRUCTURE ONLY.

Restates, in float64 numpy, what the device network computes (the reference
has no learned component, so this is this project's own oracle):

* encoding: 16 raw floats per query -> 96 columns. Columns 0..31: a
  multiresolution hash grid over the normalised position (Mueller et al.
  2022): level l < 16 has resolution N_l = floor(16 * 2^(7 l / 15)) and a
  table of 2^15 entries of 2 features, indexed densely when (N_l + 1)^3
  corners fit and otherwise by (x ^ 2654435761 y ^ 805459861 z) mod 2^15;
  column 2l + f is feature f of level l, trilinearly interpolated from the
  cell's eight corners in float32 exactly as the device does it (corner
  order x, y, z bits; every product and sum rounded). Columns 32..55: for
  axis a and band b in 0..3, column 32 + 8a + 2b = sin(2^b pi x_a), the next
  cos; 56..71 the 16 real spherical harmonics of degree < 4 of the outgoing
  direction; 72..74 normal, 75 roughness, 76..78 albedo, 79 constant 1,
  80..95 zero.
* encoding "freq12" (the frequency-only one): for axis a and band b < 12,
  column 24a + 2b = sin(2^b pi x_a), the next cos, with bands 0, 4, 8 from
  the sine and cosine (float64, rounded to float32) and the three bands
  after each by float32 double-angle steps (sin 2a = (2 sin a) cos a,
  cos 2a = (cos a - sin a)(cos a + sin a)), as the device computes them;
  72..74 outgoing
  direction, 75..77 normal, 78 roughness, 79..81 albedo, 82 constant 1,
  83..95 zero; no grid.
* network: 96 -> 64 -> 64 -> 64 -> 64 -> 64 -> 8 (3 used), ReLU after every
  hidden layer, no biases, weights per layer row-major [in][out] in one flat
  vector of 23,040 floats.
* loss: mean over rows and the 3 channels of (y - t)^2 / (y^2 + 0.01), the
  denominator treated as a constant.

`bf16=True` rounds to bfloat16 at the points the device does (weights,
encoded input, hidden activations, dL/dy and every dZ); `bf16=False` is the
exact float64 function, whose gradient is also checked against torch
autograd in the tests.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUTP, LAYERS, RAW = 96, 64, 8, 6, 16
GRID_LEVELS, GRID_FEAT, GRID_SIZE = 16, 2, 1 << 15
GRID_PARAMS = GRID_LEVELS * GRID_SIZE * GRID_FEAT
GRID_RES = [int(np.floor(16.0 * 2.0 ** (7.0 * l / 15.0))) for l in range(GRID_LEVELS)]
DIMS = [(IN, HID)] + [(HID, HID)] * 4 + [(HID, OUTP)]
OFFS = np.cumsum([0] + [i * o for i, o in DIMS]).tolist()
N_PARAMS = OFFS[-1]


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    return np.where(np.isfinite(f), out, f.astype(np.float64))


def grid_corners(pos, l):
    """Entry indices (n, 8) and float32 trilinear weights (n, 8) of level l."""
    res = GRID_RES[l]
    p = np.clip(np.asarray(pos, np.float32), np.float32(0), np.float32(1)) * np.float32(res)
    i = np.minimum(np.floor(p).astype(np.int64), res - 1)
    f = (p - i.astype(np.float32)).astype(np.float32)
    one = np.float32(1)
    side = res + 1
    idx = np.zeros((p.shape[0], 8), np.int64)
    w = np.zeros((p.shape[0], 8), np.float32)
    for c in range(8):
        b = [(c >> k) & 1 for k in range(3)]
        cx, cy, cz = (i[:, k] + b[k] for k in range(3))
        if side ** 3 <= GRID_SIZE:
            idx[:, c] = cx + side * (cy + side * cz)
        else:
            h = (cx.astype(np.uint32) ^ (cy.astype(np.uint32) * np.uint32(2654435761))
                 ^ (cz.astype(np.uint32) * np.uint32(805459861))) & np.uint32(GRID_SIZE - 1)
            idx[:, c] = h.astype(np.int64)
        wx, wy, wz = (f[:, k] if b[k] else (one - f[:, k]) for k in range(3))
        w[:, c] = (wx * wy) * wz
    return idx, w


def grid_features(grid, pos):
    """(n, 32) float32 grid columns."""
    g = np.asarray(grid, np.float32).reshape(GRID_LEVELS, GRID_SIZE, GRID_FEAT)
    out = np.zeros((pos.shape[0], 2 * GRID_LEVELS), np.float32)
    for l in range(GRID_LEVELS):
        idx, w = grid_corners(pos, l)
        a = np.zeros((pos.shape[0], GRID_FEAT), np.float32)
        for c in range(8):
            a = a + w[:, c:c + 1] * g[l, idx[:, c]]
        out[:, 2 * l:2 * l + 2] = a
    return out


def sh16(d):
    """Real spherical harmonics, degree < 4, of unit vectors d (n, 3)."""
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    xx, yy, zz = x * x, y * y, z * z
    return np.stack([
        np.full_like(x, 0.28209479177387814), -0.48860251190291987 * y, 0.48860251190291987 * z,
        -0.48860251190291987 * x, 1.0925484305920792 * x * y, -1.0925484305920792 * y * z,
        0.94617469575755997 * zz - 0.31539156525251999, -1.0925484305920792 * x * z,
        0.54627421529603959 * (xx - yy), 0.59004358992664352 * y * (3 * xx - yy),
        2.8906114426405538 * x * y * z, 0.45704579946446572 * y * (5 * zz - 1),
        0.3731763325901154 * z * (5 * zz - 3), 0.45704579946446572 * x * (5 * zz - 1),
        1.4453057213202769 * z * (xx - yy), 0.59004358992664352 * x * (xx - 3 * yy)], 1)


def init_grid(seed=0):
    rng = np.random.default_rng(seed + 7)
    return rng.uniform(-1e-4, 1e-4, GRID_PARAMS).astype(np.float32)


def encode_freq12(raw):
    r = np.asarray(raw, np.float32).astype(np.float64)
    x = np.zeros((r.shape[0], IN))
    two = np.float32(2)
    for a in range(3):
        for j in range(3):
            arg = np.pi * r[:, a] * (2.0 ** (4 * j))
            s, c = np.sin(arg).astype(np.float32), np.cos(arg).astype(np.float32)
            for k in range(4):
                if k:
                    s, c = (two * s) * c, (c - s) * (c + s)
                b = 4 * j + k
                x[:, 24 * a + 2 * b] = s
                x[:, 24 * a + 2 * b + 1] = c
    x[:, 72:82] = r[:, 3:13]
    x[:, 82] = 1.0
    return x


def encode(raw, grid, encoding="hashgrid"):
    if encoding == "freq12":
        return encode_freq12(raw)
    raw = np.asarray(raw, np.float32)
    n = raw.shape[0]
    x = np.zeros((n, IN))
    x[:, 0:32] = grid_features(grid, raw[:, 0:3])
    r = raw.astype(np.float64)
    for a in range(3):
        for b in range(4):
            arg = np.pi * r[:, a] * (2.0 ** b)
            x[:, 32 + 8 * a + 2 * b] = np.sin(arg)
            x[:, 32 + 8 * a + 2 * b + 1] = np.cos(arg)
    x[:, 56:72] = sh16(r[:, 3:6])
    x[:, 72:75] = r[:, 6:9]
    x[:, 75] = r[:, 9]
    x[:, 76:79] = r[:, 10:13]
    x[:, 79] = 1.0
    return x


def unflatten(params):
    p = np.asarray(params, np.float64)
    return [p[OFFS[l]:OFFS[l + 1]].reshape(DIMS[l]) for l in range(LAYERS)]


def forward(params, raw, grid, bf=True, encoding="hashgrid"):
    r = bf16 if bf else (lambda v: v)
    W = [r(w) for w in unflatten(params)]
    h = r(encode(raw, grid, encoding))
    acts = [h]
    for l in range(LAYERS - 1):
        h = r(np.maximum(h @ W[l], 0.0))
        acts.append(h)
    y = h @ W[-1]
    return y[:, :3], acts, W


def loss_and_grads(params, raw, target, grid, bf=True, encoding="hashgrid"):
    """(loss, weight gradient, grid gradient; zero without a grid)."""
    r = bf16 if bf else (lambda v: v)
    y, acts, W = forward(params, raw, grid, bf, encoding)
    t = np.asarray(target, np.float64)
    n = y.shape[0]
    den = y * y + 0.01
    loss = float(np.sum((y - t) ** 2 / den) / (3 * n))
    dy = np.zeros((n, OUTP))
    dy[:, :3] = 2 * (y - t) / den / (3 * n)
    dz = r(dy)
    grads = [None] * LAYERS
    for l in range(LAYERS - 1, -1, -1):
        grads[l] = acts[l].T @ dz
        if l > 0:
            dh = dz @ W[l].T
            dz = r(np.where(acts[l] > 0, dh, 0.0))
    g = np.concatenate([gl.reshape(-1) for gl in grads])
    g[OFFS[5]:].reshape(HID, OUTP)[:, 3:] = 0.0
    # through the encoding: dX of the grid columns, scattered to the corners
    gg = np.zeros((GRID_LEVELS, GRID_SIZE, GRID_FEAT))
    if encoding != "hashgrid":
        return loss, g, gg.reshape(-1)
    dx = dz @ W[0].T
    pos = np.asarray(raw, np.float32)[:, 0:3]
    for l in range(GRID_LEVELS):
        idx, w = grid_corners(pos, l)
        for c in range(8):
            for f in range(GRID_FEAT):
                np.add.at(gg[l, :, f], idx[:, c], w[:, c].astype(np.float64) * dx[:, 2 * l + f])
    return loss, g, gg.reshape(-1)


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    ps = []
    for l, (i, o) in enumerate(DIMS):
        fan_out = 3 if l == LAYERS - 1 else o
        bound = np.sqrt(6.0 / (i + fan_out))
        w = rng.uniform(-bound, bound, (i, o))
        if l == LAYERS - 1:
            w[:, 3:] = 0.0
        ps.append(w.reshape(-1))
    return np.concatenate(ps).astype(np.float32)


def random_batch(n, seed=0):
    """Seeded queries and a smooth target field, for tests."""
    rng = np.random.default_rng(seed)
    raw = np.zeros((n, RAW), np.float32)
    raw[:, 0:3] = rng.random((n, 3))
    d = rng.normal(size=(n, 3))
    raw[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    nn = rng.normal(size=(n, 3))
    raw[:, 6:9] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    raw[:, 9] = rng.random(n)
    raw[:, 10:13] = rng.random((n, 3))
    p = raw[:, 0:3].astype(np.float64)
    target = np.stack([1.0 + np.sin(3 * p[:, 0]) * np.cos(2 * p[:, 1]),
                       0.5 + 0.5 * p[:, 2] ** 2,
                       0.2 + np.abs(np.sin(5 * p[:, 0] + p[:, 1]))], 1).astype(np.float32)
    return raw, target
