"""CPU checks of the warm-start network's FP64 oracle (oracle/warmstart_oracle.py), the
checker of the CUDA training kernels: its analytic gradient against central finite
differences of its own loss, its BF16 emulation against the exact network, the
parameter layout against the library's table, and the untrained network's identity."""
import numpy as np
import pytest

from oracle import warmstart_oracle as W


def _problem(seed=3, shape=(1, 8, 8, 8)):
    rng = np.random.Generator(np.random.PCG64(seed))
    p = W.init_params(seed).astype(np.float64)
    # a non-zero head and biases so that every layer carries gradient
    for i, (wo, bo) in enumerate(W.layer_offsets()):
        co = W.LAYERS[i][2]
        p[bo:bo + co] = rng.normal(0.0, 0.05, co)
        if i == len(W.LAYERS) - 1:
            p[wo:bo] = rng.normal(0.0, 0.05, bo - wo)
    v = rng.uniform(0.0, 2.0, shape)
    t = v + rng.normal(0.0, 0.3, shape)
    return p, v, t


def test_layout_matches_library_table():
    from ettention_b200 import _abi
    import ctypes
    assert _abi.lib().etcu_warmstart_param_count() == W.param_count()
    offs = W.layer_offsets()
    for l, (c0, c1, co) in enumerate(W.LAYERS):
        info = (ctypes.c_uint32 * 6)()
        assert _abi.lib().etcu_warmstart_layer_info(l, info) == _abi.OK
        assert list(info)[:3] == [c0, c1, co]
        assert (info[4], info[5]) == offs[l]
    assert _abi.lib().etcu_warmstart_layer_info(11, (ctypes.c_uint32 * 6)()) == _abi.ERR_INVALID_ARGUMENT


def test_untrained_head_is_identity():
    p = W.init_params(1)
    v = np.random.default_rng(0).uniform(0, 1, (2, 8, 8, 4))
    out, _ = W.forward(p, v, 0.5)
    assert np.array_equal(out, v)


def test_gradient_matches_finite_differences():
    p, v, t = _problem()
    loss, g = W.loss_and_grad(p, v, t, 0.7)
    rng = np.random.Generator(np.random.PCG64(11))
    checked = 0
    for (wo, bo), (c0, c1, co) in zip(W.layer_offsets(), W.LAYERS):
        for idx in list(rng.integers(wo, bo, 3)) + [bo + int(rng.integers(0, co))]:
            eps = 1e-6
            q = p.copy()
            q[idx] += eps
            lp, _ = W.loss_and_grad(q, v, t, 0.7)
            q[idx] -= 2 * eps
            lm, _ = W.loss_and_grad(q, v, t, 0.7)
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - g[idx]) <= 1e-5 * max(abs(fd), abs(g[idx])) + 1e-9, (idx, fd, g[idx])
            checked += 1
    assert checked == 4 * len(W.LAYERS)
    assert loss > 0


def test_bf16_emulation_close_to_exact():
    p, v, t = _problem(5, (2, 8, 8, 8))
    l64, g64 = W.loss_and_grad(p, v, t, 0.7, bf16=False)
    l16, g16 = W.loss_and_grad(p, v, t, 0.7, bf16=True)
    assert abs(l16 - l64) <= 2e-2 * l64
    assert np.linalg.norm(g16 - g64) <= 5e-2 * np.linalg.norm(g64)


def test_round_bf16_is_round_to_nearest_even():
    # bfloat16 keeps 7 fraction bits: the spacing at 1.0 is 2^-7
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, 1.0 + 2.0 ** -9, -2.5, 0.0],
                 np.float32)
    r = W.round_bf16(x)
    # halfway cases go to the even neighbour: 1 + 2^-8 -> 1, 1 + 3 * 2^-8 -> 1 + 2^-6
    assert list(r) == [1.0, 1.0, 1.0 + 2.0 ** -6, 1.0 + 2.0 ** -7, 1.0, -2.5, 0.0]
