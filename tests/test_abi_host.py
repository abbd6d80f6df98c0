"""CPU tests of the C ABI boundary and the product's host-side logic (no GPU needed).

* libettention_b200.so loads and exports every entry point include/ettention_b200.h declares;
* without a GPU the device entry points fail loudly (no CPU fallback);
* the product's C++ geometry (tilt rotation, projection matrices, back-projection
  sample pattern, traversal length, projection orderings) agrees with the oracle;
* config keys parse with the reference's semantics (AlgorithmParameterSet.cpp:8-53).
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from ettention_b200 import _abi
from ettention_b200.operators import (AlgebraicParameterSet, EttentionError, ScannerGeometry, mrc_base_geometry,
                                      projection_order)
from oracle import oracle as O
from tests.helpers import oracle_geometry, product_geometry

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "ettention_b200.h")).read()
    return sorted(set(re.findall(r"ETCU_API\s+[\w\s\*]+?\b(etcu_\w+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 30
    out = subprocess.check_output(["nm", "-D", "--defined-only", _abi.LIB_PATH]).decode()
    exported = set(re.findall(r"\bT\s+(etcu_\w+)", out))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    L = _abi.lib()
    for s in syms:
        assert getattr(L, s) is not None
    assert set(_abi._SIG) == set(syms)
    assert L.etcu_abi_version() == 2


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = _abi.lib().etcu_context_create(0, ctypes.byref(h))
    assert st == _abi.ERR_NO_DEVICE
    assert b"no CUDA device" in _abi.lib().etcu_last_error(None)
    from ettention_b200.operators import Context
    with pytest.raises(EttentionError):
        Context(0)


@pytest.mark.parametrize("w,h,fits", [(1024, 1024, True), (2048, 508, True), (4096, 256, False),
                                       (2048, 1024, False), (1025, 1024, False)])
def test_noalloc_scratch_bound(w, h, fits):
    """The allocation-free update's static image holds (width + 4) x (height + 4) texels of
    at most NOALLOC_SCRATCH_TEXELS and at most NOALLOC_MAX_PIXELS pixels; larger detectors
    are rejected before the device is touched (the buffers below are never dereferenced)."""
    assert ((w + 4) * (h + 4) <= _abi.NOALLOC_SCRATCH_TEXELS and w * h <= _abi.NOALLOC_MAX_PIXELS) == fits
    if fits:
        return
    desc = _abi.VolumeDesc()
    for i, r in enumerate((64, 64, 32)):
        desc.resolution[i] = r
        desc.bbox_min[i] = -0.5 * r
        desc.bbox_max[i] = 0.5 * r
    desc.subvolume_count = 1
    view = mrc_base_geometry(w, h).to_view()
    st = _abi.lib().etcu_sart_view_update_noalloc(ctypes.byref(desc), ctypes.c_void_p(256), ctypes.c_void_p(256),
                                                  ctypes.byref(view), 1, 1, 0.3, None, None)
    assert st == _abi.ERR_INVALID_ARGUMENT
    msg = _abi.lib().etcu_last_error(None)
    assert b"exceeds" in msg and str(_abi.NOALLOC_SCRATCH_TEXELS).encode() in msg


@pytest.mark.parametrize("angle,xt", [(0.0, 0.0), (45.0, 0.0), (-60.0, 0.0), (225.0, 0.0), (37.5, 5.0)])
def test_rotation_and_matrices_match_oracle(angle, xt):
    base = O.projection_test_geometry()
    og = O.rotate_geometry(base, angle, xt)
    pg = product_geometry(base).rotated(angle, xt)
    for name in ("source", "detector", "hpitch", "vpitch"):
        np.testing.assert_allclose(getattr(pg, name), getattr(og, name), rtol=2e-6, atol=2e-5)
    np.testing.assert_allclose(pg.projection_matrix(), O.projection_matrix(og), rtol=1e-5, atol=1e-4)


def test_perspective_matrix_matches_oracle():
    og = O.perspective_test_geometry()
    pg = product_geometry(og)
    np.testing.assert_allclose(pg.projection_matrix(), O.projection_matrix(og), rtol=1e-4, atol=1e-3)


def test_sample_pattern_known_answers_and_errors():
    """BackprojectionTest.cpp:48-102."""
    g = product_geometry(O.projection_test_geometry())
    s1 = g.sample_pattern([1, 1, 1], 1)
    np.testing.assert_allclose(s1, [[0, 0, 0, 1]], atol=1e-7)
    s4 = g.sample_pattern([1, 1, 1], 4)
    np.testing.assert_allclose(s4[:, :3], [[-.25, -.25, 0], [.25, -.25, 0], [-.25, .25, 0], [.25, .25, 0]], atol=1e-7)
    np.testing.assert_allclose(s4[:, 3], 1.0, atol=1e-6)
    s45 = g.rotated(45.0).sample_pattern([1, 1, 1], 1)
    assert abs(s45[0, 3] - np.sqrt(2)) < 1e-5
    for bad, msg in ((0, "zero samples"), (3, "non-square"), (5, "non-square")):
        with pytest.raises(EttentionError, match=msg):
            g.sample_pattern([1, 1, 1], bad)
    for n in (1, 4, 9, 16):
        gg = g.rotated(33.0)
        np.testing.assert_allclose(gg.sample_pattern([1, 1, 1], n),
                                   O.bp_sample_pattern(oracle_geometry(gg), (1, 1, 1), n), rtol=1e-5, atol=1e-6)


def test_traversal_length():
    """LongObjectCompensationTest.cpp:33-45: 32 / cos(80 deg) within 0.01; perspective throws."""
    base = ScannerGeometry([-16, -16, -256], [-16, -16, 256], [.125, 0, 0], [0, .125, 0], 256, 256)
    g = base.rotated(80.0)
    c = g.traversal_length([-16, -16, -16], [16, 16, 16])
    assert abs(c - 32.0 / np.cos(np.float32(80.0) / np.float32(180.0) * np.float32(np.pi))) < 0.01
    with pytest.raises(EttentionError, match="only supported for parallel"):
        product_geometry(O.perspective_test_geometry()).traversal_length([-1, -1, -1], [1, 1, 1])


def test_projection_orders():
    """ProjectionSetTest.cpp:24-82 (permutation property) plus the exact orders of the
    deterministic schemes against the oracle restatement."""
    for n in (1, 5, 61, 180):
        ident = projection_order(_abi.ORDER_IDENTITY, n)
        assert ident == list(range(n))
        assert projection_order(_abi.ORDER_MAXANGLE, n) == O.order_maxangle(list(range(n)))
        assert projection_order(_abi.ORDER_BUCKETS, n) == O.order_buckets(list(range(n)))
        rnd = projection_order(_abi.ORDER_RANDOM, n)
        assert sorted(rnd) == list(range(n))
        assert rnd == projection_order(_abi.ORDER_RANDOM, n)  # fixed default seed
    assert projection_order(_abi.ORDER_IDENTITY, 6, skip=[1, 4]) == [0, 2, 3, 5]
    assert projection_order(_abi.ORDER_MAXANGLE, 5) == [2, 0, 3, 1, 4]
    # the random scheme renumbers 0..n-1 after skipping (ProjectionSetRandom.cpp:32-35)
    assert sorted(projection_order(_abi.ORDER_RANDOM, 6, skip=[1, 4])) == [0, 1, 2, 3]


def test_config_keys():
    sart = AlgebraicParameterSet.from_config({"algorithm": "sart", "algorithm.numberOfIterations": "2",
                                              "algorithm.lambda": "0.1", "backProjection.samples": "9",
                                              "forwardProjection.samples": "4", "hardware.subVolumeCount": "4",
                                              "volume.dimension": "64 64 64"})
    assert (sart.block_size, sart.iterations, sart.bp_samples, sart.fp_samples, sart.subvolume_count) == (1, 2, 9, 4, 4)
    assert sart.order == _abi.ORDER_RANDOM  # OptimizationParameterSet.cpp:19-21 default
    assert sart.bbox() == ([-32.0] * 3, [32.0] * 3)
    sirt = AlgebraicParameterSet.from_config({"algorithm": "sirt", "algorithm.numberOfIterations": "25",
                                              "algorithm.lambda": "1.0", "algorithm.blockSize": "7"})
    assert sirt.block_size == _abi.BLOCK_ALL
    bi = AlgebraicParameterSet.from_config({"algorithm": "blockIterative", "algorithm.blockSize": "10",
                                            "algorithm.numberOfIterations": "10", "algorithm.lambda": "1",
                                            "optimization.projectionIteration": "identity",
                                            "optimization.internalVoxelRepresentationType": "half"})
    assert (bi.block_size, bi.order, bi.voxel_type) == (10, _abi.ORDER_IDENTITY, _abi.VOXEL_HALF16)
    nb = AlgebraicParameterSet.from_config({"algorithm": "blockIterative", "algorithm.numberOfIterations": "1",
                                            "algorithm.lambda": "1"})
    assert nb.block_size == _abi.BLOCK_ALL  # no blockSize key: SIRT block (AlgorithmParameterSet.cpp:11)
    with pytest.raises(EttentionError, match="Illegal ProjectionBlockSize"):
        AlgebraicParameterSet.from_config({"algorithm": "blockIterative", "algorithm.blockSize": "0",
                                           "algorithm.numberOfIterations": "1", "algorithm.lambda": "1"})
    with pytest.raises(EttentionError, match="Illegal ProjectionSetType"):
        AlgebraicParameterSet.from_config({"algorithm": "sart", "algorithm.numberOfIterations": "1",
                                           "algorithm.lambda": "1", "optimization.projectionIteration": "zigzag"})
    with pytest.raises(EttentionError, match="basisFunctions"):
        AlgebraicParameterSet.from_config({"algorithm": "sart", "algorithm.numberOfIterations": "1",
                                           "algorithm.lambda": "1", "algorithm.basisFunctions": "cubes"})


def test_mrc_base_geometry():
    """MRCStack.cpp:250-261."""
    g = mrc_base_geometry(128, 96)
    assert list(g.source) == [-64.0, -48.0, 128.0] and list(g.detector) == [-64.0, -48.0, -128.0]
    og = O.mrc_base_geometry(128, 96)
    np.testing.assert_allclose(g.projection_matrix(), O.projection_matrix(og), atol=1e-5)
