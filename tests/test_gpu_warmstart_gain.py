"""What the trained warm start gains over plain SART, and the residual judge's fallback, on
the learned warm start's workload (ettention_b200/warmstart.py: 256 x 256 x 128 ellipsoid
phantoms, 61 parallel views, Poisson 100 counts, SART lambda 0.03, identity order):

* with the shipped weights, on held-out series: the network's volume has a data residual
  ||Ax - b||^2 at most 0.8 of the three-iteration volume it came from (the judge keeps it),
  and SART continued from it reaches plain SART's 30-iteration residual after at most 8
  further iterations, where plain SART from zero first reaches it at iteration 30;
* with the head of the trained network negated (the network's correction c becomes -c,
  exactly), the judge rejects the warm start -- the residual is a convex quadratic, so
  f(v + c) < f(v) implies f(v - c) > f(v) -- and the reconstruction continues from the
  plain three-iteration volume: after five more iterations the volume equals plain SART's
  eight-iteration volume bit for bit, i.e. the fallback is plain zero-initialised SART.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HELDOUT = (900000, 900003)


@pytest.fixture(scope="module")
def ctx():
    import torch
    assert torch.cuda.is_available()
    from ettention_b200.operators import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def weights():
    from ettention_b200.learned import DEFAULT_WEIGHTS, load_weights
    params, scale, _ = load_weights(DEFAULT_WEIGHTS)
    return params, scale


@pytest.mark.parametrize("seed", HELDOUT)
def test_trained_warm_start_reaches_plain_target_sooner(ctx, weights, seed):
    from ettention_b200 import warmstart as W
    from ettention_b200.learned import WarmStartNet
    params, scale = weights
    s = W.make_series(ctx, seed)
    plain = W.PlainSart(ctx, s)
    plain.set_volume(None)
    r = []
    for _ in range(W.TARGET_ITERS):
        plain.iterate(1)
        r.append(plain.residual())
    plain.close()
    target = r[-1]
    k_plain = next(i + 1 for i, x in enumerate(r) if x <= target)
    assert k_plain == W.TARGET_ITERS  # plain SART's residual falls at every iteration at lambda 0.03
    with WarmStartNet(ctx, W.RES, params=params, scale=scale) as net:
        solver = W.WarmStartSolver(ctx, net, s)
        try:
            assert solver.start()
            r_plain3, r_ws = solver.judge
            assert r_plain3 == pytest.approx(r[W.INPUT_ITERS - 1], rel=1e-6)
            assert r_ws <= 0.8 * r_plain3, solver.judge
            k_ws = 0
            while r_ws > target and k_ws < 8:
                solver.iterate(1)
                k_ws += 1
                r_ws = solver.residual()
            assert r_ws <= target, (k_ws, r_ws, target)
        finally:
            solver.close()
    assert W.INPUT_ITERS + k_ws < k_plain


def test_judge_falls_back_to_plain_sart(ctx, weights):
    import torch
    from oracle import warmstart_oracle as O
    from ettention_b200 import warmstart as W
    from ettention_b200.learned import WarmStartNet
    params, scale = weights
    wo, bo = O.layer_offsets()[-1]
    bad = params.copy()
    bad[wo:bo + O.LAYERS[-1][2]] *= -1.0  # head weights and bias: the correction negated
    s = W.make_series(ctx, HELDOUT[0])
    X, Y, Z = W.RES
    plain = W.PlainSart(ctx, s)
    plain.set_volume(None)
    plain.iterate(W.INPUT_ITERS + 5)
    ref = torch.empty((Z, Y, X), dtype=torch.float32, device="cuda")
    plain.get_volume(ref)
    ctx.synchronize()
    plain.close()
    with WarmStartNet(ctx, W.RES, params=bad, scale=scale) as net:
        solver = W.WarmStartSolver(ctx, net, s)
        try:
            assert not solver.start()
            r_plain3, r_ws = solver.judge
            assert r_ws > r_plain3
            solver.iterate(5)
            got = torch.empty_like(ref)
            solver.sart.get_volume(got)
            ctx.synchronize()
        finally:
            solver.close()
    assert torch.equal(got, ref)
    assert np.isfinite(got.cpu().numpy()).all()
