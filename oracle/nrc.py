"""ORACLE (test infrastructure only): CPU restatement of the learned radiance cache's
network -- hash encoding, MLP forward, relative-L2 loss and its backward pass -- used by
the tests to check the CUDA kernels (vork_b200/csrc/vkb_nrc.cuh).  The product never
imports this module.

The reference renderer has no learned component, so there is no reference file to cite;
the network follows the published methods it is built on:
  * multiresolution hash encoding: Mueller, Evans, Schied, Keller 2022, "Instant Neural
    Graphics Primitives with a Multiresolution Hash Encoding" (levels, spatial hash with
    primes 1, 2654435761, 805459861, trilinear interpolation);
  * neural radiance caching: Mueller, Rousselle, Novak, Keller 2021, "Real-time Neural
    Radiance Caching for Path Tracing" (inputs, relative L2 loss, online training);
  * real spherical harmonics bands 0..3 (standard Cartesian forms).

`emulate=True` rounds exactly where the GPU rounds (network inputs, weights, hidden
activations and backward deltas to BF16; hash table to FP16) and accumulates in float64,
so the remaining difference is only the GPU's FP32 accumulation order.  `emulate=False`
is plain float64 throughout (used for finite-difference checks of this oracle itself).
"""
from __future__ import annotations

import numpy as np

WIDTH, OUT_ROWS, LAYERS = 64, 16, 5
LEVELS, FEATURES, LOG2_T = 16, 2, 19
T = 1 << LOG2_T
BASE_RES, MAX_RES = 16.0, 2048.0
MLP_PARAMS = 4 * WIDTH * WIDTH + OUT_ROWS * WIDTH
HASH_PARAMS = LEVELS * T * FEATURES
LOSS_EPS = 0.01
PRIMES = (1, 2654435761, 805459861)


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def fp16(x):
    return np.asarray(x, np.float32).astype(np.float16).astype(np.float64)


def level_scale(level: int) -> float:
    """floor(16 * (2048/16)^(l/15)) evaluated in double (the kernel's constant table)."""
    return float(np.floor(BASE_RES * (MAX_RES / BASE_RES) ** (level / (LEVELS - 1)) + 1e-9))


def grid_index(x, y, z, res: int):
    side = res + 1
    if side ** 3 <= T:
        return (x + side * (y + side * z)).astype(np.int64)
    h = (x.astype(np.uint64) * PRIMES[0]) ^ (y.astype(np.uint64) * PRIMES[1] & 0xFFFFFFFF) ^ (z.astype(np.uint64) * PRIMES[2] & 0xFFFFFFFF)
    return (h & (T - 1)).astype(np.int64)


def sh16(d):
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    xx, yy, zz = x * x, y * y, z * z
    return np.stack([
        np.full_like(x, 0.28209479177387814), -0.48860251190291987 * y, 0.48860251190291987 * z, -0.48860251190291987 * x,
        1.0925484305920792 * x * y, -1.0925484305920792 * y * z, 0.94617469575755997 * zz - 0.31539156525251999,
        -1.0925484305920792 * x * z, 0.54627421529603959 * (xx - yy), 0.59004358992664352 * y * (-3 * xx + yy),
        2.8906114426405538 * x * y * z, 0.45704579946446572 * y * (1 - 5 * zz), 0.3731763325901154 * z * (5 * zz - 3),
        0.45704579946446572 * x * (1 - 5 * zz), 1.4453057213202769 * z * (xx - yy), 0.59004358992664352 * x * (-xx + 3 * yy)], 1)


def corners(pos):
    """Per level: (indices (n, 8), weights (n, 8)) of the trilinear corners."""
    out = []
    p = np.clip(np.asarray(pos, np.float64), 0.0, 1.0)
    for level in range(LEVELS):
        s = level_scale(level)
        res = int(s)
        q = p * s
        c = np.minimum(q.astype(np.int64), res - 1)
        f = q - c
        idx, w = [], []
        for k in range(8):
            dx, dy, dz = k & 1, (k >> 1) & 1, (k >> 2) & 1
            idx.append(grid_index(c[:, 0] + dx, c[:, 1] + dy, c[:, 2] + dz, res))
            w.append((f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) * (f[:, 2] if dz else 1 - f[:, 2]))
        out.append((np.stack(idx, 1), np.stack(w, 1)))
    return out


def encode(records, table, emulate=True):
    """records (n, 16) -> network inputs (n, 64).  table: (LEVELS, T, 2) float."""
    r = np.asarray(records, np.float64)
    tab = (fp16(table) if emulate else np.asarray(table, np.float64)).reshape(LEVELS, T, FEATURES)
    n = r.shape[0]
    x = np.zeros((n, WIDTH))
    for level, (idx, w) in enumerate(corners(r[:, 0:3])):
        x[:, 2 * level] = (w * tab[level, idx, 0]).sum(1)
        x[:, 2 * level + 1] = (w * tab[level, idx, 1]).sum(1)
    x[:, 32:48] = sh16(r[:, 3:6])
    x[:, 48:51] = r[:, 6:9] * 0.5 + 0.5
    x[:, 51] = r[:, 9]
    x[:, 52:55] = r[:, 11:14]
    x[:, 55] = r[:, 10]
    x[:, 56] = 1.0
    return bf16(x) if emulate else x


def layers(mlp):
    m = np.asarray(mlp, np.float64)
    ws = [m[l * WIDTH * WIDTH:(l + 1) * WIDTH * WIDTH].reshape(WIDTH, WIDTH) for l in range(4)]
    ws.append(m[4 * WIDTH * WIDTH:].reshape(OUT_ROWS, WIDTH))
    return ws


def forward(x, mlp, emulate=True):
    """Returns (y (n, 3), layer inputs [x, h1..h4])."""
    ws = [bf16(w) if emulate else w for w in layers(mlp)]
    a = [np.asarray(x, np.float64)]
    h = a[0]
    for l in range(4):
        h = np.maximum(h @ ws[l].T, 0.0)
        if emulate:
            h = bf16(h)
        a.append(h)
    y = h @ ws[4].T
    return y[:, :3], a


def loss_and_grad_y(y, target):
    n = y.shape[0]
    d = y - target
    den = y * y + LOSS_EPS
    loss = float((d * d / den).sum() / (3 * n))
    gy = 2 * d / den / (3 * n)       # sg(y) in the denominator: no derivative through it
    return loss, gy


def backward(x_records, mlp, table, target, emulate=True, x=None):
    """Loss, MLP gradient (MLP_PARAMS) and hash gradient ((LEVELS, T, 2)) for the records.
    `x`, when given, overrides the encoded inputs (the GPU's own, to isolate the MLP)."""
    r = np.asarray(x_records, np.float64)
    if x is None:
        x = encode(r, table, emulate)
    y, a = forward(x, mlp, emulate)
    loss, gy = loss_and_grad_y(y, np.asarray(target, np.float64))
    ws = [bf16(w) if emulate else w for w in layers(mlp)]
    n = r.shape[0]
    delta = np.zeros((n, OUT_ROWS))
    delta[:, :3] = gy
    if emulate:
        delta = bf16(delta)
    grads = [None] * LAYERS
    for l in range(LAYERS - 1, -1, -1):
        grads[l] = delta.T @ a[l]
        nxt = delta @ ws[l]
        if l > 0:
            delta = np.where(a[l] > 0, nxt, 0.0)
            if emulate:
                delta = bf16(delta)
        else:
            dx = nxt
    grads[4][3:] = 0.0
    mlp_grad = np.concatenate([g.reshape(-1) for g in grads])
    hash_grad = np.zeros((LEVELS, T, FEATURES))
    for level, (idx, w) in enumerate(corners(r[:, 0:3])):
        for f in range(FEATURES):
            np.add.at(hash_grad[level, :, f], idx.reshape(-1), (w * dx[:, 2 * level + f][:, None]).reshape(-1))
    return loss, mlp_grad, hash_grad, y


def random_records(n, seed=0):
    """Seeded records: positions in [0,1]^3, unit directions/normals, materials."""
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 16), np.float32)
    r[:, 0:3] = rng.uniform(0, 1, (n, 3))
    d = rng.normal(size=(n, 3)); r[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    m = rng.normal(size=(n, 3)); r[:, 6:9] = m / np.linalg.norm(m, axis=1, keepdims=True)
    r[:, 9] = rng.uniform(0.05, 1.0, n)
    r[:, 10] = (rng.uniform(size=n) < 0.3).astype(np.float32)
    r[:, 11:14] = rng.uniform(0.1, 0.9, (n, 3))
    return r


def random_params(seed=0, hash_scale=0.5):
    rng = np.random.default_rng(seed)
    mlp = np.zeros(MLP_PARAMS, np.float32)
    for l in range(LAYERS):
        rows = 3 if l == LAYERS - 1 else WIDTH
        a = np.sqrt(6.0 / (WIDTH + rows))
        blk = rng.uniform(-a, a, (rows, WIDTH)).astype(np.float32)
        if l == LAYERS - 1:
            full = np.zeros((OUT_ROWS, WIDTH), np.float32); full[:3] = blk; blk = full
        mlp[l * WIDTH * WIDTH: l * WIDTH * WIDTH + blk.size] = blk.reshape(-1)
    table = rng.uniform(-hash_scale, hash_scale, HASH_PARAMS).astype(np.float32)
    return mlp, table
