"""GPU tests of the learned warm start's tensor-core kernels (through the C ABI) against
the FP64 CPU oracle of the network (oracle/warmstart_oracle.py):

* the forward pass, with the oracle rounding weights and stored tensors to BF16 where the
  CUDA path does (rel-L2 of the network's correction <= 1e-2) and exactly in FP64;
* the loss and the gradient of every layer's weights and biases (rel-L2 <= 2e-2 against
  the BF16-emulating oracle, <= 1e-1 against the exact FP64 network);
* rows wider than one 128-voxel tile, y extents that leave a tile's last rows outside the
  volume, batches of two and three volumes, and a few Adam steps that lower the loss.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-2
GRAD_TOL = 2e-2
FP64_TOL = 1e-1


@pytest.fixture(scope="module", params=["tensor_copy", "cp_async"])
def loader(request):
    """The convolutions' two operand loaders (ETCU_CONV_LOADER 0: one tensor copy per
    halo, 1: cp.async warps); every result must hold for both."""
    return request.param


@pytest.fixture()
def net_env(loader, monkeypatch):
    monkeypatch.setenv("ETCU_CONV_LOADER", "0" if loader == "tensor_copy" else "1")
    return loader


@pytest.fixture(scope="module")
def ctx():
    import torch
    assert torch.cuda.is_available()
    from ettention_b200.operators import Context
    c = Context(0)
    yield c
    c.close()


def _params(seed):
    from oracle import warmstart_oracle as W
    rng = np.random.Generator(np.random.PCG64(seed))
    p = W.init_params(seed)
    for i, (wo, bo) in enumerate(W.layer_offsets()):
        co = W.LAYERS[i][2]
        p[bo:bo + co] = rng.normal(0.0, 0.05, co)
        if i == len(W.LAYERS) - 1:
            p[wo:bo] = rng.normal(0.0, 0.1, bo - wo)
    return p.astype(np.float32)


def _volumes(res, batch, seed):
    X, Y, Z = res
    rng = np.random.Generator(np.random.PCG64(seed))
    v = rng.uniform(0.0, 1.0, (batch, Z, Y, X)).astype(np.float32)
    t = (v + rng.normal(0.0, 0.2, v.shape)).astype(np.float32)
    return v, t


def _rel(a, b):
    return float(np.linalg.norm((np.asarray(a, np.float64) - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.mark.parametrize("res,batch", [((16, 16, 8), 2), ((160, 8, 4), 1), ((32, 12, 8), 3)])
def test_forward_matches_oracle(ctx, net_env, res, batch):
    import torch
    from oracle import warmstart_oracle as W
    from ettention_b200.learned import WarmStartNet
    p = _params(1)
    v, _ = _volumes(res, batch, 2)
    with WarmStartNet(ctx, res, max_batch=batch, params=p, scale=0.5) as net:
        d_in = torch.as_tensor(v).cuda()
        d_out = torch.zeros_like(d_in)
        net.infer(d_in, d_out, batch)
        ctx.synchronize()
        net.check()
        got = d_out.cpu().numpy()
    ref16, _ = W.forward(p, v, 0.5, bf16=True)
    ref64, _ = W.forward(p, v, 0.5, bf16=False)
    assert _rel(got - v, ref16 - v) <= FWD_TOL
    assert _rel(got - v, ref64 - v) <= FP64_TOL


def test_gradients_match_oracle(ctx, net_env):
    import torch
    from oracle import warmstart_oracle as W
    from ettention_b200.learned import WarmStartNet
    res, batch = (16, 16, 8), 2
    p = _params(3)
    v, t = _volumes(res, batch, 4)
    with WarmStartNet(ctx, res, max_batch=batch, params=p, scale=0.7) as net:
        loss, g = net.gradients(torch.as_tensor(v).cuda(), torch.as_tensor(t).cuda(), batch)
    l16, g16 = W.loss_and_grad(p, v, t, 0.7, bf16=True)
    l64, g64 = W.loss_and_grad(p, v, t, 0.7, bf16=False)
    assert abs(loss - l16) <= 1e-3 * l16
    for i, (wo, bo) in enumerate(W.layer_offsets()):
        co = W.LAYERS[i][2]
        for name, sl in (("W", slice(wo, bo)), ("b", slice(bo, bo + co))):
            e16 = _rel(g[sl], g16[sl])
            e64 = _rel(g[sl], g64[sl])
            assert e16 <= GRAD_TOL, f"layer {i} {name}: rel-L2 {e16} against the BF16-emulating oracle"
            assert e64 <= FP64_TOL, f"layer {i} {name}: rel-L2 {e64} against the FP64 oracle"


def test_adam_steps_lower_the_loss(ctx):
    import torch
    from ettention_b200.learned import WarmStartNet, init_params
    res = (32, 32, 16)
    rng = np.random.Generator(np.random.PCG64(9))
    v = rng.uniform(0.0, 1.0, (1, 16, 32, 32)).astype(np.float32)
    t = (v * np.float32(0.8) + np.float32(0.1)).astype(np.float32)  # a mapping the network can learn
    with WarmStartNet(ctx, res, params=init_params(4), scale=1.0) as net:
        d_in, d_t = torch.as_tensor(v).cuda(), torch.as_tensor(t).cuda()
        losses = [net.train_step(d_in, d_t, 1, lr=2e-3) for _ in range(60)]
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.5 * losses[0], losses[::10]


@pytest.mark.parametrize("res,batch", [((64, 40, 36), 2), ((160, 12, 68), 1)])
def test_zstreamed_convolution_equals_per_tap_kernel(ctx, monkeypatch, res, batch):
    """The 16-output layers as the z-streamed kernel (dz folded into N = 48, the three
    partial sums added in the epilogue; ETCU_CONV_ZFOLD=1, the default) against the
    per-tap kernel (ETCU_CONV_ZFOLD=0), on volumes whose last z segment is partial (36 and
    68 slices over segments of 32), with rows of one partial and of one full plus one
    partial x tile, and a batch of two.  Both stay within FWD_TOL of the BF16-emulating
    oracle, and they agree with each other to 5e-3 of the correction: the two kernels sum
    the same products in different orders, and every layer re-rounds its output to BF16, so
    order-level differences flip a few BF16 roundings that the later layers carry on (the
    difference is spread evenly over z, with no step at the segment boundary)."""
    from oracle import warmstart_oracle as W
    import torch
    from ettention_b200.learned import WarmStartNet
    p = _params(7)
    v, _ = _volumes(res, batch, 8)
    outs = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("ETCU_CONV_ZFOLD", mode)
        with WarmStartNet(ctx, res, max_batch=batch, params=p, scale=0.5) as net:
            d_in = torch.as_tensor(v).cuda()
            d_out = torch.zeros_like(d_in)
            net.infer(d_in, d_out, batch)
            ctx.synchronize()
            net.check()
            outs[mode] = d_out.cpu().numpy()
    corr_ref = outs["0"] - v
    assert np.abs(corr_ref).max() > 0
    assert _rel(outs["1"] - v, corr_ref) <= 5e-3
    if batch == 2:
        ob, _ = W.forward(p, v, 0.5, bf16=True)
        for mode in ("0", "1"):
            assert _rel(outs[mode] - v, ob - v) <= FWD_TOL
