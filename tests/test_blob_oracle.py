"""Blob basis functions on the CPU: the oracle pinned to the reference's BlobTest known
answers and golden fixtures, and the library's host-side tables (the ray-integration
table and the voxelisation kernel, formed on the host before any launch) against the
oracle, bit for bit."""
import ctypes
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import golden


@pytest.fixture(scope="module")
def samples256():
    return O.blob_ray_integration_samples(O.BlobParameters(), 256)


def test_kaiser_bessel_specific_values(samples256):
    """BlobTest.cpp CheckSpecificValues: evaluate(0) = 1, evaluate(a) = 0, the table's first
    entry equals the closed form of the blob's line integral through its centre
    (2^(2m+1) a I_{m+1/2}-series ratio, 200 terms), its last entry 0 (all within 1e-5)."""
    p = O.BlobParameters()
    a, m, alpha = float(np.float32(p.support_radius)), p.degree, float(np.float32(p.density_falloff))
    s1 = s2 = 0.0
    t1 = 1.0 / math.factorial(m)
    t2 = math.factorial(m) / math.factorial(2 * m + 1)
    for n in range(200):
        s1 += t1
        s2 += t2
        t1 *= 0.25 * alpha * alpha / ((n + 1) * (n + m + 1))
        t2 *= alpha * alpha / (2 * (n + 1) * (2 * n + 2 * m + 3))
    ref = 2.0 * 2.0 ** (2 * m) * a * s2 / s1
    assert abs(p.evaluate(0.0) - 1.0) < 1e-5
    assert abs(p.evaluate(a)) < 1e-5
    assert abs(samples256[0] - ref) < 1e-5
    assert abs(samples256[-1]) < 1e-5


def test_voxelizer_golden():
    """BlobTest.cpp Voxelizer: one unit coefficient at (3, 4, 5) of a 16^3 volume, voxelised
    with the default blob, equals voxelized_reference.mrc exactly."""
    b = np.zeros((16, 16, 16), np.float32)
    b[5, 4, 3] = 1.0
    out = O.blob_voxelize(b, O.blob_voxelization_kernel(O.BlobParameters()))
    assert np.array_equal(out, golden("blobs")["voxelized"])


def test_forward_lengths_golden():
    """ForwardProjectionTest.cpp PerspectiveBlobs: the blob traversal lengths of the 128^3
    perspective test case (128-entry table) against intersection_lengths_blobs_reference.tif
    within ImageComparator's RMS bound (0.1); the largest pixel error stays below 3e-4 of the
    image's maximum (the reference's float projection matrix inverse is restated, the
    remaining difference is the OpenCL device's rounding)."""
    vg = O.VolumeGeometry.centered((128, 128, 128))
    _, length = O.forward_project_blobs(np.ones((128, 128, 128), np.float32), vg, O.perspective_test_geometry(),
                                        O.BlobParameters(), 128)
    ref = golden("blobs")["intersection_lengths"]
    assert O.rms(length, ref) < 0.1
    assert np.abs(length - ref).max() < 3e-4 * ref.max()


@pytest.mark.parametrize("params", [(2.0, 2, 3.6), (1.5, 0, 6.0)])
def test_host_tables_match_oracle(params, samples256):
    from ettention_b200 import _abi
    lib = _abi.lib()
    c = _abi.BlobParams(*params)
    p = O.BlobParameters(*params)
    for count in (128, 256):
        want = samples256 if (params == (2.0, 2, 3.6) and count == 256) else O.blob_ray_integration_samples(p, count)
        got = np.zeros(count, np.float32)
        assert lib.etcu_blob_ray_integration_samples(ctypes.byref(c), count, got.ctypes.data) == _abi.OK
        assert np.array_equal(got, want)
    n = ctypes.c_uint32()
    assert lib.etcu_blob_voxelization_kernel(ctypes.byref(c), None, 0, ctypes.byref(n)) == _abi.OK
    k = int(n.value)
    assert k == 2 * math.ceil(params[0]) + 1
    got = np.zeros(k ** 3, np.float32)
    assert lib.etcu_blob_voxelization_kernel(ctypes.byref(c), got.ctypes.data, k ** 3 - 1, ctypes.byref(n)) != _abi.OK
    assert lib.etcu_blob_voxelization_kernel(ctypes.byref(c), got.ctypes.data, k ** 3, ctypes.byref(n)) == _abi.OK
    assert np.array_equal(got.reshape(k, k, k), O.blob_voxelization_kernel(p))


def test_blob_parameters_rejected():
    from ettention_b200 import _abi
    lib = _abi.lib()
    out = np.zeros(8, np.float32)
    for bad in [(0.0, 2, 3.6), (-1.0, 2, 3.6), (2.0, 40, 3.6)]:
        c = _abi.BlobParams(*bad)
        assert lib.etcu_blob_ray_integration_samples(ctypes.byref(c), 8, out.ctypes.data) == _abi.ERR_INVALID_ARGUMENT
    c = _abi.BlobParams(2.0, 2, 3.6)
    assert lib.etcu_blob_ray_integration_samples(ctypes.byref(c), 1, out.ctypes.data) == _abi.ERR_INVALID_ARGUMENT


def test_blob_config_keys():
    """AlgorithmParameterSet.cpp:34-45 and BlobParameterSet.cpp:7-29."""
    from ettention_b200.operators import AlgebraicParameterSet, BlobParameters
    base = {"algorithm": "sart", "algorithm.numberOfIterations": "2", "algorithm.lambda": "0.3"}
    p = AlgebraicParameterSet.from_config(base)
    assert p.basis_functions == "voxels" and p.blob == BlobParameters.createDefault() and not p.enable_voxelization
    p = AlgebraicParameterSet.from_config({**base, "algorithm.basisFunctions": "blobs", "blobs.supportRadius": "2.5",
                                           "blobs.degree": "3", "blobs.densityFalloff": "10.4",
                                           "output.options.enableVoxelization": "true"})
    assert p.basis_functions == "blobs" and p.enable_voxelization
    assert p.blob == BlobParameters.createWithParameters(2.5, 3, 10.4)


def test_oracle_blob_iteration_reduces_residual():
    """The oracle's blob block iteration (SART) on a small perspective case: the squared
    residual of a second iteration is below the first's."""
    g0 = O.ScannerGeometry(np.array([0.0, 0.0, -160.0]), np.array([-0.05, -0.05, -159.0]),
                           np.array([0.003125, 0.0, 0.0]), np.array([0.0, 0.003125, 0.0]), 32, 32, True)
    geoms = [O.rotate_geometry(g0, a) for a in (-40.0, 0.0, 40.0)]
    vg = O.VolumeGeometry.centered((16, 16, 16))
    truth = np.zeros((16, 16, 16), np.float32)
    truth[5:11, 4:12, 6:10] = 1.0
    proj = np.stack([O.forward_project_blobs(truth, vg, g, O.BlobParameters(), 256)[0] for g in geoms])
    vol = np.zeros_like(truth)
    r1 = O.blob_block_iterations(vol, vg, geoms, proj, [0, 1, 2], 1, 0.5, O.BlobParameters())
    r2 = O.blob_block_iterations(vol, vg, geoms, proj, [0, 1, 2], 1, 0.5, O.BlobParameters())
    assert r2 < r1
