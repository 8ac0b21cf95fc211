"""CPU oracle of the radiance-cache MLP - TEST INFRASTRUCTURE ONLY.

Restates, in float64 numpy, what the device network computes (the reference
has no learned component, so this is this project's own oracle):

* encoding: 16 raw floats per query -> 96 columns. For axis a in 0..2 and
  band b in 0..11, column 24a + 2b = sin(2^b pi x_a), 24a + 2b + 1 =
  cos(2^b pi x_a); 72..74 direction, 75..77 normal, 78 roughness, 79..81
  albedo, 82 constant 1, 83..95 zero.
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


def encode(raw):
    raw = np.asarray(raw, np.float64)
    n = raw.shape[0]
    x = np.zeros((n, IN))
    for a in range(3):
        for b in range(12):
            arg = np.pi * raw[:, a] * (2.0 ** b)
            x[:, 24 * a + 2 * b] = np.sin(arg)
            x[:, 24 * a + 2 * b + 1] = np.cos(arg)
    x[:, 72:75] = raw[:, 3:6]
    x[:, 75:78] = raw[:, 6:9]
    x[:, 78] = raw[:, 9]
    x[:, 79:82] = raw[:, 10:13]
    x[:, 82] = 1.0
    return x


def unflatten(params):
    p = np.asarray(params, np.float64)
    return [p[OFFS[l]:OFFS[l + 1]].reshape(DIMS[l]) for l in range(LAYERS)]


def forward(params, raw, bf=True):
    r = bf16 if bf else (lambda v: v)
    W = [r(w) for w in unflatten(params)]
    h = r(encode(raw))
    acts = [h]
    for l in range(LAYERS - 1):
        h = r(np.maximum(h @ W[l], 0.0))
        acts.append(h)
    y = h @ W[-1]
    return y[:, :3], acts, W


def loss_and_grads(params, raw, target, bf=True):
    r = bf16 if bf else (lambda v: v)
    y, acts, W = forward(params, raw, bf)
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
    return loss, g


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
