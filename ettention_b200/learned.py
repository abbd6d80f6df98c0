"""Learned warm start for plain SART (host side of the etcu_warmstart_* C ABI).

A 3-level 3-D convolutional encoder-decoder (3x3x3 convolutions, 16 / 32 / 64 channels,
BF16 weights and activations, FP32 accumulation) maps the volume of a few plain SART
iterations to an estimate of the volume many iterations later; plain SART then continues
from that estimate.  Forward, input-gradient and weight-gradient convolutions run on the
GPU's tensor cores inside libettention_b200.so; this module owns the parameter vector,
the training loop over pairs the method itself generates, and the judge that keeps the
warm start only when it lowers the data residual ||Ax - b|| of the plain projector
(otherwise plain zero-initialised SART goes on unchanged).

The reference has no learned component; its warm start enters the reference's loop where
`volume.initFile` does (BlockIterativeConfiguration.cpp:36-41).
"""
from __future__ import annotations

import ctypes
import os
import time
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _abi
from ._abi import EttentionError, lib

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "data", "warmstart_256x256x128.npz")

# (real input channels of source 0, channels of the skip source, output channels) per layer
LAYERS: List[Tuple[int, int, int]] = [
    (1, 0, 16), (16, 0, 16), (16, 0, 32), (32, 0, 32), (32, 0, 64), (64, 0, 64),
    (64, 32, 32), (32, 0, 32), (32, 16, 16), (16, 0, 16), (16, 0, 1),
]


def param_count() -> int:
    return int(lib().etcu_warmstart_param_count())


def layer_offsets() -> List[Tuple[int, int]]:
    out = []
    for l in range(len(LAYERS)):
        info = (ctypes.c_uint32 * 6)()
        _abi.check(lib().etcu_warmstart_layer_info(l, info))
        out.append((int(info[4]), int(info[5])))
    return out


def init_params(seed: int) -> np.ndarray:
    """He-normal weights (fan-in 27 * cin) and zero biases; the head (last layer) starts at
    zero, so the untrained network returns its input unchanged."""
    rng = np.random.Generator(np.random.PCG64(seed))
    p = np.zeros(param_count(), np.float32)
    for i, ((c0, c1, co), (wo, bo)) in enumerate(zip(LAYERS, layer_offsets())):
        if i == len(LAYERS) - 1:
            continue
        p[wo:bo] = rng.normal(0.0, np.sqrt(2.0 / (27 * (c0 + c1))), bo - wo).astype(np.float32)
    return p


def _ptr(t) -> int:
    """Device pointer of a contiguous CUDA float32 tensor, whose pending writes on torch's
    stream are completed first (an int is taken as an address the caller has ordered)."""
    if isinstance(t, int):
        return t
    from .operators import _dptr
    return _dptr(t)


class WarmStartNet:
    """The network on one context, for volumes of `resolution` (x, y, z; multiples of 4)
    and up to `max_batch` volumes per call."""

    def __init__(self, ctx, resolution: Sequence[int], max_batch: int = 1, params: Optional[np.ndarray] = None,
                 scale: float = 1.0):
        self.ctx = ctx
        self.resolution = tuple(int(r) for r in resolution)
        self.max_batch = int(max_batch)
        h = ctypes.c_void_p()
        res = (ctypes.c_uint32 * 3)(*self.resolution)
        ctx.check(lib().etcu_warmstart_create(ctx.handle, res, self.max_batch, ctypes.byref(h)))
        self.handle = h
        self.scale = float(scale)
        self.set_params(init_params(0) if params is None else params, scale)

    def set_params(self, params: np.ndarray, scale: float) -> None:
        p = np.ascontiguousarray(params, np.float32)
        if p.size != param_count():
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, f"expected {param_count()} parameters, got {p.size}")
        self.ctx.check(lib().etcu_warmstart_set_params(self.handle, p.ctypes.data, float(scale)))
        self.scale = float(scale)

    def get_params(self) -> np.ndarray:
        p = np.zeros(param_count(), np.float32)
        s = ctypes.c_float()
        self.ctx.check(lib().etcu_warmstart_get_params(self.handle, p.ctypes.data, ctypes.byref(s)))
        return p

    def infer(self, d_in, d_out, batch: int = 1) -> None:
        """d_out = warm start of d_in (CUDA float32 tensors (batch, z, y, x)), stream-ordered."""
        self.ctx.check(lib().etcu_warmstart_infer(self.handle, _ptr(d_in), _ptr(d_out), int(batch)))

    def train_step(self, d_in, d_target, batch: int = 1, lr: float = 1e-3, want_loss: bool = True):
        loss = ctypes.c_double()
        self.ctx.check(lib().etcu_warmstart_train_step(self.handle, _ptr(d_in), _ptr(d_target), int(batch),
                                                        float(lr), ctypes.byref(loss) if want_loss else None))
        return float(loss.value) if want_loss else None

    def gradients(self, d_in, d_target, batch: int = 1):
        g = np.zeros(param_count(), np.float32)
        loss = ctypes.c_double()
        self.ctx.check(lib().etcu_warmstart_gradients(self.handle, _ptr(d_in), _ptr(d_target), int(batch),
                                                       g.ctypes.data, ctypes.byref(loss)))
        return float(loss.value), g

    def check(self) -> None:
        self.ctx.check(lib().etcu_warmstart_check(self.handle))

    def close(self) -> None:
        if self.handle:
            lib().etcu_warmstart_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def save_weights(path: str, params: np.ndarray, scale: float, **meta) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez_compressed(path, params=np.asarray(params, np.float32), scale=np.float32(scale),
                        **{k: np.asarray(v) for k, v in meta.items()})


def load_weights(path: str = DEFAULT_WEIGHTS):
    with np.load(path) as z:
        meta = {k: z[k] for k in z.files if k not in ("params", "scale")}
        return z["params"].astype(np.float32), float(z["scale"]), meta
