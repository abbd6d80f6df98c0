"""Pins the CPU oracle to the reference's own golden fixtures (CPU only).

Each test restates one of the reference's GoogleTest cases
(ettention/test/src/...) with the fixture it compares against, converted to
tests/golden/*.npz by tests/golden/make_golden.py.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import blob_phantom, golden, xzy_to_zyx


@pytest.fixture(scope="module")
def fp45():
    return golden("fp45")


@pytest.mark.parametrize("angle", [45.0, 225.0])
def test_forward_projection_matches_projection_45(fp45, angle):
    """ForwardProjectionTest.cpp:70-95 (Unit_ForwardProjection, _Raysign)."""
    vg = O.VolumeGeometry.centered((64, 64, 64))
    g = O.rotate_geometry(O.projection_test_geometry(), angle)
    for prec in (32, 64):
        p, _ = O.forward_project(blob_phantom(1.0), vg, g, 1, prec)
        assert O.images_equal(p, fp45["projection_45"])
        assert O.rel_l2(p, fp45["projection_45"]) < 2e-6


def test_traversal_length_and_ray_length(fp45):
    """ForwardProjectionTest.cpp:139-161 (Unit_ComputeRayLength, RMS < 0.1) and the
    traversal output of the forward projector against the same image."""
    vg = O.VolumeGeometry.centered((64, 64, 64))
    g = O.rotate_geometry(O.projection_test_geometry(), 45.0)
    rl = O.ray_length(vg, g)
    assert O.rms(rl, fp45["raylength"]) < 0.1
    _, length = O.forward_project(blob_phantom(1.0), vg, g, 1, 32)
    assert O.rel_l2(length, fp45["raylength"]) < 2e-6


@pytest.mark.parametrize("name,angle", [("z", 0.0), ("y", 90.0), ("45", 45.0)])
def test_back_projection_matches_voxel_by_voxel_reference(name, angle):
    """BackprojectionTest.cpp:33-132: lambda 1, 1 sample, ray length from ComputeRayLength;
    StackComparator max slice RMS <= 0.011.  Texture-filter weights (1/256) reproduce
    the fixtures to ~1e-7; exact FP32 weights stay within the reference comparator."""
    bp = golden("bp")
    ref = xzy_to_zyx(bp[f"volume_{name}_xzy"])
    vg = O.VolumeGeometry.centered((64, 64, 64))
    g = O.rotate_geometry(O.projection_test_geometry(), angle)
    L = O.ray_length(vg, g)
    for weights, tol in ((O.WEIGHTS_Q8, 1e-6), (O.WEIGHTS_EXACT, 1e-3)):
        v = np.zeros((64, 64, 64), np.float32)
        O.back_project(v, vg, g, bp[f"projection_{name}"], L, 1.0, 1, 32, weights)
        assert O.max_slice_rms(np.transpose(v, (1, 0, 2)), bp[f"volume_{name}_xzy"]) <= 0.011
        assert O.rel_l2(v, ref) < tol


def test_back_projection_fp64_close_to_fp32_reference():
    bp = golden("bp")
    vg = O.VolumeGeometry.centered((64, 64, 64))
    g = O.rotate_geometry(O.projection_test_geometry(), 45.0)
    L = O.ray_length(vg, g, 64)
    v = np.zeros((64, 64, 64), np.float32)
    O.back_project(v, vg, g, bp["projection_45"], L, 1.0, 1, 64, O.WEIGHTS_Q8)
    assert O.rel_l2(v, xzy_to_zyx(bp["volume_45_xzy"])) < 1e-5


def test_sample_pattern_known_answers():
    """BackprojectionTest.cpp:48-102 (Sampling_Pattern_Generation_*)."""
    base = O.projection_test_geometry()
    vs = (1.0, 1.0, 1.0)
    s1 = O.bp_sample_pattern(O.rotate_geometry(base, 0.0), vs, 1)
    np.testing.assert_allclose(s1, [[0, 0, 0, 1]], atol=1e-7)
    s4 = O.bp_sample_pattern(O.rotate_geometry(base, 0.0), vs, 4)
    np.testing.assert_allclose(s4[:, :3], [[-.25, -.25, 0], [.25, -.25, 0], [-.25, .25, 0], [.25, .25, 0]], atol=1e-7)
    np.testing.assert_allclose(s4[:, 3], 1.0, atol=1e-6)
    s45 = O.bp_sample_pattern(O.rotate_geometry(base, 45.0), vs, 1)
    np.testing.assert_allclose(s45[0, :3], 0.0, atol=1e-7)
    assert abs(s45[0, 3] - np.sqrt(2.0)) < 1e-5
    for bad in (0, 3, 5):
        with pytest.raises(ValueError):
            O.bp_sample_pattern(base, vs, bad)


def test_long_object_compensation_fixture():
    """LongObjectCompensationTest.cpp:129-164: the input images are the forward projection
    of a 32^3 volume of ones with 16x16 sub-rays at 80 degrees; compensation gives the
    constant 32 / cos(80 deg)."""
    loc = golden("loc")
    vg = O.VolumeGeometry.centered((32, 32, 32))
    base = O.ScannerGeometry(np.array([-16., -16., -256.]), np.array([-16., -16., 256.]), np.array([.125, 0, 0]),
                             np.array([0, .125, 0]), 256, 256)
    g = O.rotate_geometry(base, 80.0)
    p, l = O.forward_project(np.ones((32, 32, 32), np.float32), vg, g, 16, 32)
    assert O.images_equal(p, loc["input_virtual"]) and O.rel_l2(p, loc["input_virtual"]) < 1e-6
    assert O.images_equal(l, loc["input_traversal"])
    c = O.traversal_length_through_bbox(g, vg.bmin, vg.bmax)
    assert abs(c - 32.0 / np.cos(np.float32(80.0) / np.float32(180.0) * np.float32(np.pi))) < 0.01
    pc, lc = O.long_object_compensation(loc["input_virtual"], loc["input_traversal"], c)
    assert O.rms(pc, loc["reference"]) < 0.1
    assert np.all(lc == np.float32(c))


def test_perspective_accumulation_identity_and_lengths():
    """ForwardProjectionTest.cpp:163-183 (projection of ones == intersection length) and the
    perspective intersection-length fixture with 8x8 sub-rays."""
    pg = O.perspective_test_geometry()
    vg = O.VolumeGeometry.centered((128, 128, 128))
    ones = np.ones((128, 128, 128), np.float32)
    p, l = O.forward_project(ones, vg, pg, 1, 32)
    assert O.images_equal(p, l)
    p8, l8 = O.forward_project(ones, vg, pg, 8, 32)
    pr = golden("persp")
    assert O.images_equal(l8, pr["intersection_lengths"])
    assert O.rel_l2(l8, pr["intersection_lengths"]) < 1e-6


@pytest.mark.slow
def test_perspective_forward_matches_back():
    """ForwardProjectionTest.cpp:267-304: BP (8^3 samples) of the reference projection, then
    FP (8x8): lengths equal, projection RMS < 2e-2."""
    pr = golden("persp")
    pg = O.perspective_test_geometry()
    vg = O.VolumeGeometry.centered((128, 128, 128))
    v = np.zeros((128, 128, 128), np.float32)
    O.back_project(v, vg, pg, pr["projection"], pr["intersection_lengths"], 1.0, 8, 32, O.WEIGHTS_Q8)
    p2, l2 = O.forward_project(v, vg, pg, 8, 32)
    assert O.images_equal(l2, pr["intersection_lengths"])
    assert O.rms(p2, pr["projection"]) < 2e-2


def test_synthetic_projections_are_forward_projections_of_ground_truth():
    """SyntheticReconstruction.cpp:66-107: the 180 projections of synthetic_3_parallel are
    FP(ground_truth) with the ProjectionTestBase geometry; five are kept as fixtures."""
    syn = golden("synth")
    vg = O.VolumeGeometry.centered((64, 64, 64))
    base = O.projection_test_geometry()
    for a in syn["angles"]:
        p, _ = O.forward_project(syn["ground_truth"], vg, O.rotate_geometry(base, float(a)), 1, 32)
        ref = syn[f"projection_{int(a)}"]
        assert O.images_equal(p, ref)
        assert O.rel_l2(p, ref) < 1e-6


def synthetic_setup(lam, block, fp_samples, bp_samples, angles=None):
    syn = golden("synth")
    base = O.projection_test_geometry()
    angles = list(range(-90, 90)) if angles is None else angles
    views = [O.rotate_geometry(base, float(a)) for a in angles]
    vg = O.VolumeGeometry.centered((64, 64, 64), subvolumes=4)
    vg1 = O.VolumeGeometry.centered((64, 64, 64))
    projs = np.stack([O.forward_project(syn["ground_truth"], vg1, g, 1, 32)[0] for g in views])
    return syn["ground_truth"], O.ReconstructionSetup(vg, views, projs, lam, block, fp_samples, bp_samples)


@pytest.mark.slow
@pytest.mark.parametrize("name,lam,block,fs,bs,iters,limit", [
    ("sart", 0.1, 1, 4, 9, 2, 0.7),
    ("sirt", 1.0, 180, 1, 1, 25, 0.7),
    ("blockIterative", 1.0, 10, 1, 1, 10, 0.2),
])
def test_synthetic_reconstruction_rms(name, lam, block, fs, bs, iters, limit):
    """SyntheticReconstruction.cpp:132-172 with the sart/sirt/blockIterative.xml settings
    (4 sub-volumes), identity order: max slice RMS vs ground truth <= 0.7 / 0.7 / 0.2."""
    gt, setup = synthetic_setup(lam, block, fs, bs)
    v = np.zeros((64, 64, 64), np.float32)
    O.block_iterative(setup, v, iters, 32)
    assert O.max_slice_rms(v, gt) <= limit
