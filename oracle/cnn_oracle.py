"""CPU oracle of the warm-start network (test infrastructure only).

FP64 numpy restatement of the 3D residual CNN that the GPU trains and runs
for the learned warm start: forward pass, weighted squared-error loss and
the gradient of the loss with respect to every parameter. The network has no
counterpart in the reference (it is one of the components the GPU build adds
on top of icd_iteration.cpp); the oracle is pinned instead by central finite
differences and an adjoint identity in the CPU tests.

Layout (identical to the GPU's flat parameter array):
    W_in[27][C], b_in[C],
    per block l: W1[27][C][C] (tap, in, out), b1[C], W2[27][C][C], b2[C],
    W_out[27][C], b_out[1],
tap t = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1) reading the input at
(x + dx, y + dy, z + dz), zero outside the volume. Volumes are [nz][ny][nx]
(channels last for the hidden activations).

    a_0     = relu(conv_in(s_in * x) + b_in)
    h_l     = relu(conv(a_l; W1_l) + b1_l)
    a_{l+1} = a_l + conv(h_l; W2_l) + b2_l
    out     = conv_out(a_B) + b_out
    loss    = sum w (out - (xc - x) s_out)^2 / sum w

Only tests/ may import this module.
"""
from __future__ import annotations

import numpy as np

C = 32
TAPS = 27


def offsets():
    return [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(TAPS)]  # (dz, dy, dx)


def num_params(blocks: int) -> int:
    return TAPS * C + C + blocks * 2 * (TAPS * C * C + C) + TAPS * C + 1


def unpack(p: np.ndarray, blocks: int) -> dict:
    p = np.asarray(p, dtype=np.float64)
    assert p.size == num_params(blocks)
    o = 0

    def take(*shape):
        nonlocal o
        n = int(np.prod(shape))
        a = p[o:o + n].reshape(shape)
        o += n
        return a

    d = {"W_in": take(TAPS, C), "b_in": take(C), "W": [], "b": []}
    for _ in range(2 * blocks):
        d["W"].append(take(TAPS, C, C))
        d["b"].append(take(C))
    d["W_out"] = take(TAPS, C)
    d["b_out"] = take(1)
    return d


def pack(d: dict) -> np.ndarray:
    parts = [d["W_in"].ravel(), d["b_in"].ravel()]
    for W, b in zip(d["W"], d["b"]):
        parts += [W.ravel(), b.ravel()]
    parts += [d["W_out"].ravel(), d["b_out"].ravel()]
    return np.concatenate(parts)


def shift(a: np.ndarray, dz: int, dy: int, dx: int) -> np.ndarray:
    """out[z, y, x] = a[z + dz, y + dy, x + dx], zero outside (leading 3 axes)."""
    out = np.zeros_like(a)
    nz, ny, nx = a.shape[:3]

    def rng(d, n):
        return (max(0, -d), min(n, n - d))

    (z0, z1), (y0, y1), (x0, x1) = rng(dz, nz), rng(dy, ny), rng(dx, nx)
    if z1 > z0 and y1 > y0 and x1 > x0:
        out[z0:z1, y0:y1, x0:x1] = a[z0 + dz:z1 + dz, y0 + dy:y1 + dy, x0 + dx:x1 + dx]
    return out


def conv(a: np.ndarray, W: np.ndarray) -> np.ndarray:
    """a [nz,ny,nx,Cin] (or [nz,ny,nx] for Cin = 1), W [27][Cin][Cout] (or [27][Cout])."""
    if a.ndim == 3:
        a = a[..., None]
        W = W[:, None, :]
    out = 0.0
    for t, (dz, dy, dx) in enumerate(offsets()):
        out = out + shift(a, dz, dy, dx) @ W[t]
    return out


def conv_data_grad(g: np.ndarray, W: np.ndarray) -> np.ndarray:
    """Gradient w.r.t. the input of conv(., W) given the output gradient g."""
    out = 0.0
    for t, (dz, dy, dx) in enumerate(offsets()):
        out = out + shift(g @ W[t].T, -dz, -dy, -dx)
    return out


def conv_weight_grad(a: np.ndarray, g: np.ndarray) -> np.ndarray:
    """dW[t] = sum_v a[v + off(t)] (x) g[v]."""
    if a.ndim == 3:
        a = a[..., None]
    cin, cout = a.shape[-1], g.shape[-1]
    dW = np.zeros((TAPS, cin, cout))
    for t, (dz, dy, dx) in enumerate(offsets()):
        dW[t] = shift(a, dz, dy, dx).reshape(-1, cin).T @ g.reshape(-1, cout)
    return dW


def forward(p: np.ndarray, x: np.ndarray, blocks: int, s_in: float = 1.0):
    d = unpack(p, blocks)
    x = np.asarray(x, dtype=np.float64)
    a = [np.maximum(conv(s_in * x, d["W_in"]) + d["b_in"], 0.0)]
    h = []
    for l in range(blocks):
        h.append(np.maximum(conv(a[l], d["W"][2 * l]) + d["b"][2 * l], 0.0))
        a.append(a[l] + conv(h[l], d["W"][2 * l + 1]) + d["b"][2 * l + 1])
    out = conv(a[blocks], d["W_out"][:, :, None])[..., 0] + d["b_out"][0]
    return out, {"a": a, "h": h, "d": d}


def loss_and_grad(p: np.ndarray, x: np.ndarray, xc: np.ndarray, blocks: int, s_in: float = 1.0,
                  s_out: float = 1.0, w: np.ndarray | None = None):
    x = np.asarray(x, dtype=np.float64)
    xc = np.asarray(xc, dtype=np.float64)
    w = np.ones_like(x) if w is None else np.asarray(w, dtype=np.float64)
    out, cache = forward(p, x, blocks, s_in)
    a, h, d = cache["a"], cache["h"], cache["d"]
    r = out - (xc - x) * s_out
    loss = float(np.sum(w * r * r) / np.sum(w))
    dout = 2.0 * w * r / np.sum(w)
    g = {"W": [None] * (2 * blocks), "b": [None] * (2 * blocks)}
    g["W_out"] = conv_weight_grad(a[blocks], dout[..., None])[:, :, 0]
    g["b_out"] = np.array([dout.sum()])
    ga = conv_data_grad(dout[..., None], d["W_out"][:, :, None])
    for l in range(blocks - 1, -1, -1):
        g["W"][2 * l + 1] = conv_weight_grad(h[l], ga)
        g["b"][2 * l + 1] = ga.reshape(-1, C).sum(0)
        du = conv_data_grad(ga, d["W"][2 * l + 1]) * (h[l] > 0)
        g["W"][2 * l] = conv_weight_grad(a[l], du)
        g["b"][2 * l] = du.reshape(-1, C).sum(0)
        ga = ga + conv_data_grad(du, d["W"][2 * l])
    du0 = ga * (a[0] > 0)
    g["W_in"] = conv_weight_grad(s_in * x, du0)[:, 0, :]
    g["b_in"] = du0.reshape(-1, C).sum(0)
    return loss, pack(g), out


def init_params(blocks: int, seed: int, scale: float = 1.0) -> np.ndarray:
    """Random parameters for tests (not the GPU's initialisation)."""
    rng = np.random.default_rng(seed)
    d = {"W_in": rng.uniform(-1, 1, (TAPS, C)) * np.sqrt(6 / TAPS) * scale,
         "b_in": rng.uniform(-0.1, 0.1, C), "W": [], "b": []}
    for i in range(2 * blocks):
        d["W"].append(rng.uniform(-1, 1, (TAPS, C, C)) * np.sqrt(6 / (TAPS * C)) * scale)
        d["b"].append(rng.uniform(-0.1, 0.1, C))
    d["W_out"] = rng.uniform(-1, 1, (TAPS, C)) * np.sqrt(6 / (TAPS * C)) * scale
    d["b_out"] = rng.uniform(-0.1, 0.1, 1)
    return pack(d)
