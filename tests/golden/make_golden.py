"""Converts the reference's own test fixtures into compact NumPy archives.

Run in a container where the reference checkout is mounted (read-only):

    python tests/golden/make_golden.py /path/to/ettention-checkout

It reads the TIFF and MRC fixtures under ``ettention/test/data`` (the files the
reference's GoogleTest suites compare against) and writes ``tests/golden/*.npz``.
The archives hold the fixture arrays unchanged (float32), so tests on machines
without the reference checkout compare against exactly the same numbers.

Fixtures (reference test that uses each one):
  fp45.npz    forward_projection/projection_45.tif, raylength_reference.tif
              (test/src/unit/sart_components/forwardprojection/ForwardProjectionTest.cpp:51-161)
  bp.npz      back_projection/projection_{z,y,45}.tif and
              voxel_by_voxel_reference_{z,y,45}.mrc
              (test/src/unit/sart_components/backprojection/BackprojectionTest.cpp:33-132)
  loc.npz     long_object_compensation/{input_virtual_projection,input_traversal_length,
              virtual_projection_reference}.tif (test/src/unit/LongObjectCompensationTest.cpp:129-164)
  persp.npz   perspective/{projection,intersection_lengths}_reference.tif
              (ForwardProjectionTest.cpp:163-183, :267-304)
  blobs.npz   blobs/voxelized_reference.mrc (test/src/unit/BlobTest.cpp:113-131) and
              perspective/intersection_lengths_blobs_reference.tif
              (ForwardProjectionTest.cpp:238-265, :306-338)
  synth.npz   synthetic_3_parallel/ground_truth.mrc plus five of its 180 projections
              (test/src/integration/SyntheticReconstruction.cpp:66-172); the other
              projections are forward projections of ground_truth and are regenerated.
"""
from __future__ import annotations

import os
import struct
import sys

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))
SYNTH_ANGLES = (-90, -37, 0, 45, 89)


def read_tif(path: str) -> np.ndarray:
    from PIL import Image
    return np.array(Image.open(path), np.float32)


def read_mrc(path: str) -> np.ndarray:
    """MRC mode-2 volume as stored: array[nz][ny][nx] (nx fastest)."""
    with open(path, "rb") as f:
        b = f.read()
    nx, ny, nz, mode = struct.unpack("<4i", b[:16])
    if mode != 2:
        raise ValueError(f"{path}: MRC mode {mode} is not float32")
    next_ = struct.unpack("<i", b[92:96])[0]
    return np.frombuffer(b[1024 + next_:], np.float32, nx * ny * nz).reshape(nz, ny, nx).copy()


def main(root: str) -> None:
    d = os.path.join(root, "ettention", "test", "data")
    np.savez_compressed(os.path.join(OUT, "fp45.npz"),
                        projection_45=read_tif(os.path.join(d, "forward_projection", "projection_45.tif")),
                        raylength=read_tif(os.path.join(d, "forward_projection", "raylength_reference.tif")))
    bp = {}
    for n in ("z", "y", "45"):
        bp[f"projection_{n}"] = read_tif(os.path.join(d, "back_projection", f"projection_{n}.tif"))
        bp[f"volume_{n}_xzy"] = read_mrc(os.path.join(d, "back_projection", f"voxel_by_voxel_reference_{n}.mrc"))
    np.savez_compressed(os.path.join(OUT, "bp.npz"), **bp)
    lo = os.path.join(d, "long_object_compensation")
    np.savez_compressed(os.path.join(OUT, "loc.npz"),
                        input_virtual=read_tif(os.path.join(lo, "input_virtual_projection.tif")),
                        input_traversal=read_tif(os.path.join(lo, "input_traversal_length.tif")),
                        reference=read_tif(os.path.join(lo, "virtual_projection_reference.tif")))
    pe = os.path.join(d, "perspective")
    np.savez_compressed(os.path.join(OUT, "persp.npz"),
                        projection=read_tif(os.path.join(pe, "projection_reference.tif")),
                        intersection_lengths=read_tif(os.path.join(pe, "intersection_lengths_reference.tif")))
    np.savez_compressed(os.path.join(OUT, "blobs.npz"),
                        voxelized=read_mrc(os.path.join(d, "blobs", "voxelized_reference.mrc")),
                        intersection_lengths=read_tif(os.path.join(pe, "intersection_lengths_blobs_reference.tif")))
    sy = os.path.join(d, "synthetic_3_parallel")
    syn = {"ground_truth": read_mrc(os.path.join(sy, "ground_truth.mrc")),
           "angles": np.array(SYNTH_ANGLES, np.float32)}
    for a in SYNTH_ANGLES:
        syn[f"projection_{a}"] = read_tif(os.path.join(sy, f"projection{a}.tif"))
    np.savez_compressed(os.path.join(OUT, "synth.npz"), **syn)
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ETTENTION_REFERENCE", "")
    if not ref:
        sys.exit("usage: make_golden.py <reference checkout> (or set ETTENTION_REFERENCE)")
    main(ref)
