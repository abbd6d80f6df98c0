"""The launch-shape autotuner (etcu_context_set_autotune): the persistent batched SART
iteration (threads per block, resident blocks per SM), the single-series persistent fused
steps (resident blocks per SM) and the warm-start convolutions (ring stages) time their
candidates once, store the choice in the cache file, and reuse it from there; the
volumes do not depend on the choice (bit for bit against the built-in shapes)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture()
def cache(tmp_path, monkeypatch):
    path = tmp_path / "shapes.txt"
    monkeypatch.setenv("ETCU_TUNE_CACHE", str(path))
    return path


def _batch(ctx, series, p):
    from ettention_b200.operators import BatchReconstructionOperator, GPUMappedVolume
    vols = [GPUMappedVolume(ctx, shape) for shape, _, _ in series]
    batch = BatchReconstructionOperator([(v, g, pr) for v, (_, g, pr) in zip(vols, series)], p)
    batch.runNiterations(2)
    out = batch.getReconstructedVolumes()
    batch.close()
    for v in vols:
        v.close()
    return out


def _single(ctx, shape, geoms, projs, p):
    from ettention_b200.operators import BlockIterativeReconstructionOperator, GPUMappedVolume
    vol = GPUMappedVolume(ctx, shape)
    rec = BlockIterativeReconstructionOperator(vol, geoms, projs, p)
    rec.runNiterations(2)
    out = rec.getReconstructedVolume()
    rec.close()
    vol.close()
    return out


def test_tuned_shapes_are_cached_and_change_nothing(cache):
    import torch
    from ettention_b200 import _abi
    from ettention_b200.learned import WarmStartNet, init_params
    from ettention_b200.operators import AlgebraicParameterSet, Context
    from tests.test_gpu_batch import make_series
    series = make_series(900)
    p = AlgebraicParameterSet(algorithm="sart", block_size=1, iterations=2, lam=0.3, order=_abi.ORDER_IDENTITY)
    shape, geoms, projs = series[0]
    x = torch.rand((1, 16, 32, 64), device="cuda")

    def run(tune):
        ctx = Context(0)
        try:
            if tune:
                ctx.set_autotune(1)
            vb = _batch(ctx, series, p)
            vs = _single(ctx, shape, geoms, projs, p)
            with WarmStartNet(ctx, (64, 32, 16), params=init_params(2), scale=0.5) as net:
                y = torch.empty_like(x)
                net.infer(x, y)
                ctx.synchronize()
                vy = y.cpu().numpy()
            return vb, vs, vy, ctx.tune_report()
        finally:
            ctx.close()

    vb0, vs0, vy0, rep0 = run(False)
    assert rep0 == ""
    vb1, vs1, vy1, rep1 = run(True)
    assert all(np.array_equal(a, b) for a, b in zip(vb0, vb1))
    assert np.array_equal(vs0, vs1) and np.array_equal(vy0, vy1)
    for kind in ("sart_fused_batch|", "sart_fused_persistent|", "warmstart_conv|"):
        lines = [l for l in rep1.splitlines() if l.startswith(kind)]
        assert lines and all("ms" in l for l in lines), (kind, rep1)
    text = cache.read_text()
    assert "sart_fused_batch|" in text and "sart_fused_persistent|" in text and "warmstart_conv|" in text
    vb2, vs2, vy2, rep2 = run(True)
    assert all(np.array_equal(a, b) for a, b in zip(vb0, vb2)) and np.array_equal(vs0, vs2)
    assert "cached" in rep2 and "ms" not in rep2.replace("cached", "")
