"""Weighted back projection on the GPU (etcu_wbp, the WBP plugin's algorithm) against the
oracle: the RamLak filtering of the FFT path restated as a direct circular convolution
(within 1e-5 of the image's range), and the whole reconstruction within the parity
tolerance of the back projector (rel-L2 <= 1e-4), through the operator and through a
WBP parameter file."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "the gpu tests need a CUDA device"
    return t


@pytest.fixture(scope="module")
def ctx(torch):
    from ettention_b200.operators import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("shape", [(128, 128), (30, 100), (1, 256), (130, 300), (8, 1024), (257, 129)])
def test_filter_matches_oracle(torch, ctx, shape):
    from oracle import oracle as O
    from ettention_b200.operators import wbp_filter
    img = np.random.default_rng(shape[0] + 7 * shape[1]).standard_normal(shape).astype(np.float32)
    d_in = torch.tensor(img, device="cuda")
    d_out = torch.zeros_like(d_in)
    wbp_filter(ctx, d_in, d_out)
    ctx.synchronize()
    got = d_out.cpu().numpy()
    want = O.wbp_filter(img)
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()


def test_filter_rejects_too_narrow_images(torch, ctx):
    from ettention_b200.operators import EttentionError, wbp_filter
    d = torch.zeros((8, 5), device="cuda")
    with pytest.raises(EttentionError, match="too small for the mirrored padding"):
        wbp_filter(ctx, d, d.clone())


def _problem(res, det, angles, seed):
    from oracle import oracle as O
    from ettention_b200.operators import mrc_base_geometry
    from tests.helpers import ellipsoid_phantom, oracle_geometry
    truth = ellipsoid_phantom(res, 6, seed=seed)
    vg = O.VolumeGeometry.centered(res)
    geoms = [mrc_base_geometry(*det).rotated(float(a)) for a in angles]
    projs = np.stack([O.forward_project(truth, vg, oracle_geometry(g), 1, 32)[0] for g in geoms]).astype(np.float32)
    return geoms, projs


@pytest.mark.parametrize("res,det,n", [((96, 80, 24), (128, 80), 21), ((128, 64, 32), (100, 64), 13)])
def test_wbp_matches_oracle(ctx, res, det, n):
    from oracle import oracle as O
    from ettention_b200.operators import AlgebraicParameterSet, GPUMappedVolume, WBPOperator
    from tests.helpers import oracle_geometry
    geoms, projs = _problem(res, det, np.linspace(-60, 60, n), seed=res[0] + n)
    p = AlgebraicParameterSet(algorithm="wbp", iterations=1, lam=1.0)
    vol = GPUMappedVolume(ctx, res)
    WBPOperator(vol, geoms, projs, p).run()
    got = vol.download()
    vol.close()
    vo = O.wbp(projs, [oracle_geometry(g) for g in geoms], O.VolumeGeometry.centered(res))
    assert np.abs(vo).max() > 0
    assert O.rel_l2(got, vo) <= 1e-4


def test_wbp_through_a_parameter_file(tmp_path):
    from oracle import oracle as O
    from ettention_b200.operators import MRCStack, XMLParameterSource, mrc_base_geometry, reconstruct_from_config
    from tests.helpers import oracle_geometry
    from tests.test_io_files import write_stack
    res, det = (64, 64, 16), (128, 64)
    angles = np.round(np.linspace(-58.5, 61.25, 17), 2)
    geoms, projs = _problem(res, det, angles, seed=5)
    write_stack(tmp_path / "series.mrc", projs, 2)
    (tmp_path / "series.tlt").write_text("\n".join(f"{a:.2f}" for a in angles) + "\n")
    (tmp_path / "wbp.xml").write_text(
        '<algorithm value="wbp"><numberOfIterations value="1"/><lambda value="1.0"/></algorithm>'
        '<input><projections value="series.mrc"/><tiltAngles value="series.tlt"/></input>'
        '<output><filename value="out.mrc"/><options><orientation value="xyz_order"/></options></output>'
        f'<volume><dimension value="{res[0]} {res[1]} {res[2]}"/></volume>')
    v = reconstruct_from_config(XMLParameterSource(str(tmp_path / "wbp.xml")))
    assert np.array_equal(MRCStack(str(tmp_path / "out.mrc")).load_projections(), v)
    g = [oracle_geometry(mrc_base_geometry(*det).rotated(float(a))) for a in np.float32(angles)]
    vo = O.wbp(projs, g, O.VolumeGeometry.centered(res))
    assert O.rel_l2(v, vo) <= 1e-4
