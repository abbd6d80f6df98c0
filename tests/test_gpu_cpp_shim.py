"""Forward projection, back projection and a SART reconstruction driven through the
C++ operator surface (include/ettention_b200.hpp, tests/cpp/shim_gpu.cpp), compared
with the oracle: projections and back projection within 1e-4 relative L2, the
2-iteration SART volume within 1e-3."""
import os

import numpy as np
import pytest

from tests.test_cpp_shim import build_and_run

pytestmark = pytest.mark.gpu

X, Y, Z, NV = 96, 80, 40, 15


def phantom():
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    return (np.float32(0.01) * ((x * 7 + y * 13 + z * 29) % 17).astype(np.float32) / np.float32(16.0)).astype(np.float32)


def test_cpp_shim_projectors_and_sart_match_oracle(tmp_path):
    import subprocess
    from oracle import oracle as O
    from ettention_b200.operators import mrc_base_geometry
    from tests.helpers import oracle_geometry
    exe = build_and_run(tmp_path, "shim_gpu.cpp", ("-I", "/usr/local/cuda/include", "-lcudart"))
    out = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    load = lambda n, shape: np.fromfile(tmp_path / n, np.float32).reshape(shape)
    vol = phantom()
    vg = O.VolumeGeometry.centered((X, Y, Z))
    g = mrc_base_geometry(X, Y).rotated(25.0)
    po, lo = O.forward_project(vol, vg, oracle_geometry(g), 1, 32)
    pv, pl = load("fp_virtual.bin", (Y, X)), load("fp_length.bin", (Y, X))
    assert O.rel_l2(pv, po) <= 1e-4 and O.rel_l2(pl, lo) <= 1e-4
    i = np.arange(X * Y, dtype=np.int64)
    res = (((i * 37) % 101 - 50).astype(np.float32) / np.float32(50.0)).reshape(Y, X)
    vb = np.zeros((Z, Y, X), np.float32)
    O.back_project(vb, vg, oracle_geometry(g), res, pl, 0.5, 1, 32, O.WEIGHTS_Q8)
    assert O.rel_l2(load("bp_volume.bin", (Z, Y, X)), vb) <= 1e-4
    geoms = [mrc_base_geometry(X, Y).rotated(float(-60.0 + 120.0 * k / (NV - 1))) for k in range(NV)]
    projs = load("projections.bin", (NV, Y, X))
    setup = O.ReconstructionSetup(vg, [oracle_geometry(q) for q in geoms], projs, 0.3, 1, 1, 1)
    vo = np.zeros((Z, Y, X), np.float32)
    O.block_iterative(setup, vo, 2, 32)
    assert O.rel_l2(load("sart_volume.bin", (Z, Y, X)), vo) <= 1e-3
    vw = O.wbp(projs, [oracle_geometry(q) for q in geoms], vg)
    assert O.rel_l2(load("wbp_volume.bin", (Z, Y, X)), vw) <= 1e-4
    # blob basis functions: forward projections, one blob SART iteration, voxelisation
    from ettention_b200.operators import ScannerGeometry
    B, D = 24, 32
    i = np.arange(B ** 3, dtype=np.int64)
    ph = (((i * 7 + (i // B) * 13) % 11).astype(np.float32) / np.float32(10.0)).reshape(B, B, B)
    base = ScannerGeometry([0.0, 0.0, -160.0], [-0.05, -0.05, -159.0], [0.1 / D, 0, 0], [0, 0.1 / D, 0], D, D, True)
    bgeoms = [oracle_geometry(base.rotated(-45.0 + 30.0 * k)) for k in range(4)]
    bvg = O.VolumeGeometry.centered((B, B, B))
    bprojs = load("blob_projections.bin", (4, D, D))
    want = np.stack([O.forward_project_blobs(ph, bvg, q, O.BlobParameters(), 256)[0] for q in bgeoms])
    assert O.rel_l2(bprojs, want) <= 1e-5
    coeff = np.zeros((B, B, B), np.float32)
    O.blob_block_iterations(coeff, bvg, bgeoms, bprojs, [0, 1, 2, 3], 1, 0.5, O.BlobParameters())
    got = load("blob_coefficients.bin", (B, B, B))
    assert O.rel_l2(got, coeff) <= 1e-4
    vox = O.blob_voxelize(got, O.blob_voxelization_kernel(O.BlobParameters()))
    assert np.array_equal(load("blob_voxels.bin", (B, B, B)), vox)
