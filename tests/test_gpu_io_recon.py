"""End to end through the reference's front door: a tilt series in an MRC file with a
tilt-angle file (MRCStack), the reconstruction configured by the reference's keys (a
jason_64_SART-like setup: volume wider than the detector, long-object compensation,
one SART iteration), the volume written as an XZY MRC and read back; compared with
the oracle's block-iterative reconstruction within 1e-3."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_mrc_stack_to_mrc_volume_matches_oracle(tmp_path):
    from oracle import oracle as O
    from ettention_b200.operators import (AlgebraicParameterSet, BlockIterativeReconstructionOperator, Context,
                                          GPUMappedVolume, MRCStack, mrc_base_geometry, write_mrc_volume)
    from tests.helpers import ellipsoid_phantom, oracle_geometry
    from tests.test_io_files import write_stack
    W, H = 32, 32
    X, Y, Z = 64, 64, 16
    angles = np.round(np.linspace(-62.78, 61.5, 21), 2)
    truth = ellipsoid_phantom((X, Y, Z), 8, seed=64)
    vg = O.VolumeGeometry.centered((X, Y, Z))
    geoms = [mrc_base_geometry(W, H).rotated(float(a)) for a in angles]
    projs = np.stack([O.forward_project(truth, vg, oracle_geometry(g), 1, 32)[0] for g in geoms]).astype(np.float32)
    write_stack(tmp_path / "series.ali", projs, 2, extra=b"\0" * 4096)
    (tmp_path / "series.tlt").write_text("\n".join(f"{a:.2f}" for a in angles) + "\n")

    cfg = {"algorithm": "sart", "algorithm.numberOfIterations": "1", "algorithm.useLongObjectCompensation": "true",
           "algorithm.lambda": "0.3", "volume.dimension": f"{X} {Y} {Z}", "volume.initValue": "0.0",
           "hardware.subVolumeCount": "1", "optimization.projectionIteration": "identity"}
    p = AlgebraicParameterSet.from_config(cfg)
    stack = MRCStack(str(tmp_path / "series.ali"), str(tmp_path / "series.tlt"))
    views = stack.geometries()
    data = stack.load_projections()
    assert np.array_equal(data, projs)
    ctx = Context(0)
    try:
        lo, hi = p.bbox()
        vol = GPUMappedVolume(ctx, p.resolution, lo, hi, subvolume_count=p.subvolume_count)
        rec = BlockIterativeReconstructionOperator(vol, views, data, p)
        rec.run()
        v = rec.getReconstructedVolume()
        rec.close()
        vol.close()
    finally:
        ctx.close()
    write_mrc_volume(str(tmp_path / "generated.mrc"), v)  # XZY, the reference's default
    back = MRCStack(str(tmp_path / "generated.mrc")).load_projections()
    assert back.shape == (Y, Z, X) and np.array_equal(back, np.transpose(v, (1, 0, 2)))
    setup = O.ReconstructionSetup(vg, [oracle_geometry(g) for g in views], projs, 0.3, 1, 1, 1, use_loc=True)
    vo = np.zeros((Z, Y, X), np.float32)
    O.block_iterative(setup, vo, 1, 32)
    assert O.rel_l2(v, vo) <= 1e-3
    assert np.abs(v).max() > 0
