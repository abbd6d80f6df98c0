"""CPU oracle of the learned warm start's network (test infrastructure only: the product
path never imports this module).

A NumPy FP64 restatement of the 3-level 3-D convolutional encoder-decoder that
ettention_b200/csrc/etcu_learned.cu runs on the tensor cores, its loss and the gradient
of the loss with respect to every parameter.  The reference has no learned component, so
nothing in it pins this network; the oracle is checked against central finite differences
of its own FP64 loss (tests/test_warmstart_oracle.py) and the CUDA path against the
oracle.

With ``bf16=True`` the oracle rounds weights and every stored activation and gradient
tensor to bfloat16 (round to nearest even) at the points where the CUDA path stores them
in BF16, so the two differ only by FP32-versus-FP64 accumulation; with ``bf16=False`` it
is the exact FP64 network.

Layout: volumes (B, Z, Y, X); feature maps (B, C, Z, Y, X).  Parameters: one vector,
per layer W[27][cout][cin] (tap t = dz*9 + dy*3 + dx reads voxel (x+dx-1, y+dy-1,
z+dz-1)), then b[cout].
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

# (real input channels of source 0, channels of source 1, output channels)
LAYERS: List[Tuple[int, int, int]] = [
    (1, 0, 16), (16, 0, 16), (16, 0, 32), (32, 0, 32), (32, 0, 64), (64, 0, 64),
    (64, 32, 32), (32, 0, 32), (32, 16, 16), (16, 0, 16), (16, 0, 1),
]


def layer_offsets() -> List[Tuple[int, int]]:
    """(W offset, b offset) of every layer in the parameter vector."""
    out, off = [], 0
    for c0, c1, co in LAYERS:
        out.append((off, off + 27 * co * (c0 + c1)))
        off += 27 * co * (c0 + c1) + co
    return out


def param_count() -> int:
    return sum(27 * co * (c0 + c1) + co for c0, c1, co in LAYERS)


def unpack(params: np.ndarray) -> List[Tuple[np.ndarray, np.ndarray]]:
    res = []
    for (c0, c1, co), (wo, bo) in zip(LAYERS, layer_offsets()):
        res.append((params[wo:bo].reshape(27, co, c0 + c1), params[bo:bo + co]))
    return res


def init_params(seed: int) -> np.ndarray:
    """He-normal weights (fan-in 27 * cin), zero biases; the head starts at zero so the
    untrained network is the identity (output = input)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    p = np.zeros(param_count(), np.float32)
    for i, ((c0, c1, co), (wo, bo)) in enumerate(zip(LAYERS, layer_offsets())):
        if i == len(LAYERS) - 1:
            continue
        std = np.sqrt(2.0 / (27 * (c0 + c1)))
        p[wo:bo] = rng.normal(0.0, std, bo - wo).astype(np.float32)
    return p


def round_bf16(a: np.ndarray) -> np.ndarray:
    """float -> bfloat16 (round to nearest even) -> float64."""
    f = np.ascontiguousarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    r = np.where(np.isnan(f), u, r).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def _shift(x: np.ndarray, dz: int, dy: int, dx: int) -> np.ndarray:
    """x[..., z + dz, y + dy, x + dx] with zeros outside (dz, dy, dx in {-1, 0, 1})."""
    Z, Y, X = x.shape[-3:]
    out = np.zeros_like(x)
    zs, ys, xs = slice(max(0, -dz), Z - max(0, dz)), slice(max(0, -dy), Y - max(0, dy)), slice(max(0, -dx), X - max(0, dx))
    zd, yd, xd = slice(max(0, dz), Z + min(0, dz)), slice(max(0, dy), Y + min(0, dy)), slice(max(0, dx), X + min(0, dx))
    out[..., zs, ys, xs] = x[..., zd, yd, xd]
    return out


def _taps():
    for t in range(27):
        yield t, t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1


def conv(x: np.ndarray, W: np.ndarray, b) -> np.ndarray:
    """Same-size 3x3x3 convolution: out[b, o, v] = sum_t sum_c x[b, c, v + off(t)] W[t, o, c] + b[o]."""
    B, C, Z, Y, X = x.shape
    out = np.zeros((B, W.shape[1], Z, Y, X))
    for t, dz, dy, dx in _taps():
        out += np.einsum("bczyx,oc->bozyx", _shift(x, dz, dy, dx), W[t], optimize=True)
    if b is not None:
        out += np.asarray(b, np.float64)[None, :, None, None, None]
    return out


def conv_input_grad(g: np.ndarray, W: np.ndarray) -> np.ndarray:
    """Gradient of conv's output g (B, O, ...) with respect to its input (B, C, ...)."""
    out = np.zeros((g.shape[0], W.shape[2]) + g.shape[2:])
    for t, dz, dy, dx in _taps():
        out += np.einsum("bozyx,oc->bczyx", _shift(g, -dz, -dy, -dx), W[t], optimize=True)
    return out


def conv_weight_grad(x: np.ndarray, g: np.ndarray) -> np.ndarray:
    """dW[t, o, c] = sum_{b, v} g[b, o, v] x[b, c, v + off(t)]."""
    dW = np.zeros((27, g.shape[1], x.shape[1]))
    for t, dz, dy, dx in _taps():
        dW[t] = np.einsum("bozyx,bczyx->oc", g, _shift(x, dz, dy, dx), optimize=True)
    return dW


def pool(x: np.ndarray) -> np.ndarray:
    B, C, Z, Y, X = x.shape
    return x.reshape(B, C, Z // 2, 2, Y // 2, 2, X // 2, 2).mean(axis=(3, 5, 7))


def pool_grad(g: np.ndarray) -> np.ndarray:
    return upsample(g) * 0.125


def upsample(x: np.ndarray) -> np.ndarray:
    return x.repeat(2, axis=2).repeat(2, axis=3).repeat(2, axis=4)


def upsample_grad(g: np.ndarray) -> np.ndarray:
    B, C, Z, Y, X = g.shape
    return g.reshape(B, C, Z // 2, 2, Y // 2, 2, X // 2, 2).sum(axis=(3, 5, 7))


def _layer_params(params: np.ndarray, bf16: bool):
    """(W, b) per layer: FP64 as given, or as the CUDA path holds them (BF16 weights,
    FP32 biases)."""
    if bf16:
        return [(round_bf16(W), np.asarray(b, np.float32).astype(np.float64))
                for W, b in unpack(np.asarray(params, np.float32))]
    return unpack(np.asarray(params, np.float64))


def forward(params: np.ndarray, v: np.ndarray, scale: float, bf16: bool = False) -> Tuple[np.ndarray, Dict]:
    """Network output (B, Z, Y, X) = v + scale * net(v / scale), and the activations."""
    R = round_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    P = _layer_params(params, bf16)
    relu = lambda a: np.maximum(a, 0.0)  # noqa: E731
    A: Dict[str, np.ndarray] = {}
    A["x"] = R(np.asarray(v, np.float32)[:, None] * np.float32(1.0 / scale))
    A["e1a"] = R(relu(conv(A["x"], *P[0])))
    A["e1b"] = R(relu(conv(A["e1a"], *P[1])))
    A["p1"] = R(pool(A["e1b"]))
    A["e2a"] = R(relu(conv(A["p1"], *P[2])))
    A["e2b"] = R(relu(conv(A["e2a"], *P[3])))
    A["p2"] = R(pool(A["e2b"]))
    A["e3a"] = R(relu(conv(A["p2"], *P[4])))
    A["e3b"] = R(relu(conv(A["e3a"], *P[5])))
    A["up2"] = upsample(A["e3b"])
    A["d2a"] = R(relu(conv(np.concatenate([A["up2"], A["e2b"]], 1), *P[6])))
    A["d2b"] = R(relu(conv(A["d2a"], *P[7])))
    A["up1"] = upsample(A["d2b"])
    A["d1a"] = R(relu(conv(np.concatenate([A["up1"], A["e1b"]], 1), *P[8])))
    A["d1b"] = R(relu(conv(A["d1a"], *P[9])))
    head = conv(A["d1b"], *P[10])[:, 0]
    out = np.asarray(v, np.float64) + scale * head
    return out, A


def loss_and_grad(params: np.ndarray, v: np.ndarray, target: np.ndarray, scale: float,
                  bf16: bool = False) -> Tuple[float, np.ndarray]:
    """L = mean(((out - target) / scale)^2) and dL/dparams (FP64)."""
    R = round_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    P = _layer_params(params, bf16)
    out, A = forward(params, v, scale, bf16)
    n = out.size
    d = (out - np.asarray(target, np.float64)) / scale
    loss = float(np.mean(d * d))
    grads = [None] * len(LAYERS)

    def step(i, x_in, g):
        grads[i] = (conv_weight_grad(x_in, g), g.sum(axis=(0, 2, 3, 4)))

    mask = lambda a: (a > 0).astype(np.float64)  # noqa: E731
    dy = R((2.0 / n) * d)[:, None]
    step(10, A["d1b"], dy)
    gA1 = R(conv_input_grad(dy, P[10][0]) * mask(A["d1b"]))
    step(9, A["d1a"], gA1)
    gB1 = R(conv_input_grad(gA1, P[9][0]) * mask(A["d1a"]))
    step(8, np.concatenate([A["up1"], A["e1b"]], 1), gB1)
    g8 = R(conv_input_grad(gB1, P[8][0]))
    gUp1, gSkip1 = g8[:, :32], g8[:, 32:]
    gA2 = R(upsample_grad(gUp1) * mask(A["d2b"]))
    step(7, A["d2a"], gA2)
    gB2 = R(conv_input_grad(gA2, P[7][0]) * mask(A["d2a"]))
    step(6, np.concatenate([A["up2"], A["e2b"]], 1), gB2)
    g6 = R(conv_input_grad(gB2, P[6][0]))
    gUp2, gSkip2 = g6[:, :64], g6[:, 64:]
    gA3 = R(upsample_grad(gUp2) * mask(A["e3b"]))
    step(5, A["e3a"], gA3)
    gB3 = R(conv_input_grad(gA3, P[5][0]) * mask(A["e3a"]))
    step(4, A["p2"], gB3)
    dP2 = R(conv_input_grad(gB3, P[4][0]))
    gA2 = R((pool_grad(dP2) + gSkip2) * mask(A["e2b"]))
    step(3, A["e2a"], gA2)
    gB2 = R(conv_input_grad(gA2, P[3][0]) * mask(A["e2a"]))
    step(2, A["p1"], gB2)
    dP1 = R(conv_input_grad(gB2, P[2][0]))
    gA1 = R((pool_grad(dP1) + gSkip1) * mask(A["e1b"]))
    step(1, A["e1a"], gA1)
    gB1 = R(conv_input_grad(gA1, P[1][0]) * mask(A["e1a"]))
    step(0, A["x"], gB1)
    flat = np.zeros(param_count())
    for (dW, db), (wo, bo) in zip(grads, layer_offsets()):
        flat[wo:bo] = dW.ravel()
        flat[bo:bo + db.size] = db
    return loss, flat
