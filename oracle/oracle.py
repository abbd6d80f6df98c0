"""TEST INFRASTRUCTURE ONLY -- the checker, never the product.

Python face of the CPU oracle for Ettention's block-iterative hot path.  Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module; the product package ``ettention_b200`` never does.

The numeric kernels live in ``oracle/ettention_oracle.c`` (built into
``oracle/liboracle.so``); this module restates the reference's HOST geometry
(scanner geometry, tilt rotation, projection matrices, back-projection sample
pattern, sub-volume split, projection orderings) in NumPy float64 and rounds
to float32 where the reference stores float.  Every function cites the
reference file:line it follows (paths relative to
``ettention/libReconstruction/src`` unless stated).
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

WEIGHTS_EXACT, WEIGHTS_Q8, WEIGHTS_Q8_TRUNC = 0, 1, 2
FLT_MAX = float(np.finfo(np.float32).max)


# ----------------------------------------------------------------------------
# ctypes plumbing
# ----------------------------------------------------------------------------
class _View(ctypes.Structure):
    _fields_ = [("source", ctypes.c_double * 3), ("detector", ctypes.c_double * 3),
                ("hpitch", ctypes.c_double * 3), ("vpitch", ctypes.c_double * 3),
                ("ray", ctypes.c_double * 3), ("width", ctypes.c_int), ("height", ctypes.c_int),
                ("perspective", ctypes.c_int)]


class _VolGeom(ctypes.Structure):
    _fields_ = [("res", ctypes.c_int * 3), ("bmin", ctypes.c_double * 3), ("bmax", ctypes.c_double * 3),
                ("cmin", ctypes.c_double * 3), ("cmax", ctypes.c_double * 3), ("voxel", ctypes.c_double * 3)]


_lib = None


def build() -> None:
    """Compile liboracle.so with the committed recipe."""
    import subprocess
    subprocess.check_call([os.path.join(_HERE, "build_oracle.sh")])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        L.orc_forward.argtypes = [ctypes.c_int, ctypes.POINTER(_View), ctypes.POINTER(_VolGeom), P, ctypes.c_int,
                                  P, ctypes.c_int, P, P]
        L.orc_back_parallel.argtypes = [ctypes.c_int, ctypes.POINTER(_VolGeom), P, P, ctypes.c_int, P, P,
                                        ctypes.c_int, ctypes.c_int, P, ctypes.c_int, P, ctypes.c_float, ctypes.c_int]
        L.orc_back_perspective.argtypes = [ctypes.c_int, ctypes.POINTER(_VolGeom), P, P, ctypes.c_int, P, P,
                                           ctypes.c_int, ctypes.c_int, P, ctypes.c_int, P, ctypes.c_float,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_float]
        L.orc_ray_length.argtypes = [ctypes.c_int, ctypes.POINTER(_View), ctypes.POINTER(_VolGeom), P]
        L.orc_compare.argtypes = [P, P, P, ctypes.c_long]
        L.orc_long_object_compensation.argtypes = [P, P, ctypes.c_float, ctypes.c_long]
        L.orc_half_from_float.argtypes = [P, P, ctypes.c_long]
        L.orc_float_from_half.argtypes = [P, P, ctypes.c_long]
        L.orc_block_iterative.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_View), P, ctypes.c_int,
                                          ctypes.POINTER(_VolGeom), ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, P, P, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int, P,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_float]
        L.orc_block_iterative.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


# ----------------------------------------------------------------------------
# Geometry (host side of the reference)
# ----------------------------------------------------------------------------
def _f32(v) -> np.ndarray:
    return np.asarray(v, dtype=np.float32).astype(np.float64)


def _normalize32(v) -> np.ndarray:
    """Vec3f doNormalize in float: v / |v| (framework/math/Vec3.h)."""
    v = np.asarray(v, dtype=np.float32)
    n = np.float32(np.sqrt(np.float32(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])))
    return (v / n).astype(np.float32).astype(np.float64)


@dataclass
class ScannerGeometry:
    """model/geometry/ScannerGeometry.cpp:39-46: source/detector base, pitches, resolution."""
    source: np.ndarray
    detector: np.ndarray
    hpitch: np.ndarray
    vpitch: np.ndarray
    width: int
    height: int
    perspective: bool = False

    def ray_direction(self) -> np.ndarray:
        """ParallelScannerGeometry.cpp:44-47 / PerspectiveScannerGeometry.cpp:37-40."""
        if self.perspective:
            return _normalize32(self.detector_center() - self.source)
        return _normalize32(np.asarray(self.detector, np.float32) - np.asarray(self.source, np.float32))

    def detector_center(self) -> np.ndarray:
        """ScannerGeometry.cpp:80-83."""
        return _f32(np.asarray(self.detector, np.float32) + np.float32(0.5) * (
            np.float32(self.width) * np.asarray(self.hpitch, np.float32)
            + np.float32(self.height) * np.asarray(self.vpitch, np.float32)))

    def to_c(self) -> _View:
        v = _View()
        for name in ("source", "detector", "hpitch", "vpitch"):
            arr = getattr(v, name)
            for i in range(3):
                arr[i] = float(np.float32(getattr(self, name)[i]))
        r = self.ray_direction()
        for i in range(3):
            v.ray[i] = float(r[i])
        v.width, v.height, v.perspective = int(self.width), int(self.height), int(self.perspective)
        return v


def rotate_geometry(base: ScannerGeometry, tilt_deg: float, xaxis_tilt_deg: float = 0.0) -> ScannerGeometry:
    """SingleAxisTiltRotator.cpp:42-78: rotate source, detector and both
    pitches by -tilt about +y (optionally about a y axis pre-tilted about x)."""
    t = np.float32(-np.float32(tilt_deg) / np.float32(180.0) * np.float32(math.pi))
    xt = np.float32(np.float32(xaxis_tilt_deg) / np.float32(180.0) * np.float32(math.pi))
    c, s = np.float32(np.cos(t)), np.float32(np.sin(t))

    def rot(p):
        p = np.asarray(p, np.float32)
        if xt == 0.0:
            return np.array([p[0] * c - p[2] * s, p[1], p[0] * s + p[2] * c], np.float32)
        cx, sx = np.float32(np.cos(xt)), np.float32(np.sin(xt))
        q = np.array([p[0], p[1] * cx + p[2] * sx, -p[1] * sx + p[2] * cx], np.float32)
        ax = _normalize32([0.0, cx, -sx]).astype(np.float32)
        one = np.float32(1.0)
        return np.array([
            (c + (one - c) * ax[0] * ax[0]) * q[0] + ((one - c) * ax[0] * ax[1] - s * ax[2]) * q[1]
            + ((one - c) * ax[0] * ax[2] + s * ax[1]) * q[2],
            ((one - c) * ax[0] * ax[1] + s * ax[2]) * q[0] + (c + (one - c) * ax[1] * ax[1]) * q[1]
            + ((one - c) * ax[1] * ax[2] - s * ax[0]) * q[2],
            ((one - c) * ax[0] * ax[2] - s * ax[1]) * q[0] + ((one - c) * ax[1] * ax[2] + s * ax[0]) * q[1]
            + (c + (one - c) * ax[2] * ax[2]) * q[2]], np.float32)

    return ScannerGeometry(_f32(rot(base.source)), _f32(rot(base.detector)), _f32(rot(base.hpitch)),
                           _f32(rot(base.vpitch)), base.width, base.height, base.perspective)


def mrc_base_geometry(nx: int, ny: int) -> ScannerGeometry:
    """io/datasource/MRCStack.cpp:250-261: parallel base geometry of an MRC stack."""
    return ScannerGeometry(np.array([-0.5 * nx, -0.5 * ny, float(nx)]), np.array([-0.5 * nx, -0.5 * ny, -float(nx)]),
                           np.array([1.0, 0.0, 0.0]), np.array([0.0, 1.0, 0.0]), nx, ny, False)


def projection_test_geometry() -> ScannerGeometry:
    """framework/test/ProjectionTestBase.cpp:105-119 (256^2 detector, pitch 0.5)."""
    return ScannerGeometry(np.array([-64.0, -64.0, -128.0]), np.array([-64.0, -64.0, 128.0]),
                           np.array([0.5, 0.0, 0.0]), np.array([0.0, 0.5, 0.0]), 256, 256, False)


def perspective_test_geometry() -> ScannerGeometry:
    """framework/test/ProjectionTestBase.cpp:137-145."""
    return ScannerGeometry(_f32([0.0, 0.0, -700.0]), _f32([-0.10510424, -0.10510424, -699.0]),
                           _f32([0.0016422537, 0.0, 0.0]), _f32([0.0, 0.0016422537, 0.0]), 128, 128, True)


def _mat_from_columns(c0, c1, c2, c3) -> np.ndarray:
    """framework/math/Matrix4x4.cpp:44-63 (column vectors) -> 4x4 row/col array."""
    return np.array([c0, c1, c2, c3], dtype=np.float64).T


def parallel_projection_matrix(g: ScannerGeometry) -> np.ndarray:
    """ParallelScannerGeometry.cpp:49-62: T(res/2 + 0.5) * inverse[h, v, ray, e4].
    Returned as 16 column-major values (Matrix4x4::values layout)."""
    ray = g.ray_direction()
    m = np.linalg.inv(_mat_from_columns(list(_f32(g.hpitch)) + [0.0], list(_f32(g.vpitch)) + [0.0],
                                        list(ray) + [0.0], [0.0, 0.0, 0.0, 1.0]))
    v = 0.5 * np.array([g.width, g.height], np.float64) + 0.5
    coord = _mat_from_columns([1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [v[0], v[1], 0.0, 1.0])
    full = coord @ m
    return _f32(full.T.reshape(-1))


def perspective_projection_matrix(g: ScannerGeometry) -> np.ndarray:
    """framework/math/Matrix4x4.cpp:376-399 getPerspectiveProjection."""
    src = _f32(g.source)
    dc = g.detector_center()
    view = np.linalg.inv(_mat_from_columns(list(_f32(g.hpitch)) + [0.0], list(_f32(g.vpitch)) + [0.0],
                                           list(dc - src) + [0.0], list(src) + [1.0]))
    zn = 1e-2
    proj = _mat_from_columns([1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1.0 / (1.0 - zn), 1.0], [0, 0, -zn / (1.0 - zn), 0])
    tr = _mat_from_columns([1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0.5 * g.width, 0.5 * g.height, 0.0, 1.0])
    full = tr @ proj @ view
    return _f32(full.T.reshape(-1))


def projection_matrix(g: ScannerGeometry) -> np.ndarray:
    return perspective_projection_matrix(g) if g.perspective else parallel_projection_matrix(g)


def bp_sample_pattern(g: ScannerGeometry, voxel_size: Sequence[float], samples: int) -> np.ndarray:
    """ParallelBeamsBackProjectionKernel.cpp:55-98: per-voxel detector-plane
    offsets scaled by the largest voxel edge, each with the chord of the ray
    through the voxel's AABB at that offset.  Raises on non-square counts."""
    if samples == 0:
        raise ValueError("zero samples not supported for BackProjection")
    n = int(math.sqrt(float(samples)))
    if n * n != samples:
        raise ValueError("non-square root number of samples not supported for BackProjection")
    vs = np.asarray(voxel_size, np.float32)
    mvs = np.float32(max(vs))
    h = (_normalize32(g.hpitch) * mvs).astype(np.float32)
    v = (_normalize32(g.vpitch) * mvs).astype(np.float32)
    ray = g.ray_direction().astype(np.float32)
    inv = np.array([np.float32(1.0) / r if r != 0 else np.float32(FLT_MAX) for r in ray], np.float32)
    out = np.zeros((samples, 4), np.float32)
    k = 0
    for y in range(n):
        yp = np.float32((np.float32(y) + np.float32(0.5)) / np.float32(n)) - np.float32(0.5)
        for x in range(n):
            xp = np.float32((np.float32(x) + np.float32(0.5)) / np.float32(n)) - np.float32(0.5)
            p = (xp * h + yp * v).astype(np.float32)
            with np.errstate(invalid="ignore", over="ignore"):
                t0 = (-0.5 * vs - p) * inv
                t1 = (0.5 * vs - p) * inv
            tmin = np.minimum(t0, t1)
            tmax = np.maximum(t0, t1)
            d = np.float32(min(tmax)) - np.float32(max(tmin))
            out[k] = [p[0], p[1], p[2], d]
            k += 1
    return out


def traversal_length_through_bbox(g: ScannerGeometry, bmin, bmax) -> float:
    """ParallelScannerGeometry.cpp:64-69 (long-object constant length)."""
    if g.perspective:
        raise ValueError("Calculation of traversal length is only supported for parallel scanner geometry!")
    ray = g.ray_direction()
    zin = np.float32((np.float32(bmin[2]) - np.float32(g.source[2])) / np.float32(ray[2]))
    zout = np.float32((np.float32(bmax[2]) - np.float32(g.source[2])) / np.float32(ray[2]))
    return float(np.float32(max(zin, zout) - min(zin, zout)))


@dataclass
class VolumeGeometry:
    """model/volume/VolumeProperties.cpp:21-27 and :74-98."""
    resolution: tuple
    bmin: np.ndarray
    bmax: np.ndarray
    subvolumes: int = 1

    @classmethod
    def centered(cls, resolution, dimension=None, origin=(0.0, 0.0, 0.0), subvolumes=1):
        """setup/parameterset/VolumeParameterSet.cpp:68-71 bbox = origin +- dim/2."""
        dim = np.asarray(resolution if dimension is None else dimension, np.float64)
        o = np.asarray(origin, np.float64)
        return cls(tuple(int(r) for r in resolution), _f32(o - 0.5 * dim), _f32(o + 0.5 * dim), subvolumes)

    @property
    def voxel_size(self) -> np.ndarray:
        return _f32((np.asarray(self.bmax, np.float32) - np.asarray(self.bmin, np.float32))
                    / np.asarray(self.resolution, np.float32))

    def slabs(self) -> List[dict]:
        """VolumeProperties.cpp:74-98: z split, remainder to the first slabs."""
        X, Y, Z = self.resolution
        cnt = self.subvolumes
        if Z < cnt:
            raise ValueError(f"Volume of size {Z} in z direction cannot be split into {cnt} subvolumes!")
        base = Z // cnt
        rem = Z - cnt * base
        vs = np.asarray(self.voxel_size, np.float32)
        nxt = np.asarray(self.bmin, np.float32).copy()
        z0 = 0
        out = []
        for i in range(cnt):
            rz = base + 1 if i < rem else base
            res = (X, Y, rz)
            bmin = nxt.copy()
            bmax = (nxt + np.asarray(res, np.float32) * vs).astype(np.float32)
            nxt = nxt.copy()
            nxt[2] = bmax[2]
            out.append(dict(res=res, z0=z0, bmin=_f32(bmin), bmax=_f32(bmax)))
            z0 += rz
        return out

    def to_c(self, slab: Optional[dict] = None) -> _VolGeom:
        if slab is None:
            slab = dict(res=self.resolution, bmin=self.bmin, bmax=self.bmax)
        g = _VolGeom()
        vs = self.voxel_size
        for i in range(3):
            g.res[i] = int(slab["res"][i])
            g.bmin[i] = float(slab["bmin"][i])
            g.bmax[i] = float(slab["bmax"][i])
            g.cmin[i] = float(self.bmin[i])
            g.cmax[i] = float(self.bmax[i])
            g.voxel[i] = float(vs[i])
        return g


# ----------------------------------------------------------------------------
# Kernels
# ----------------------------------------------------------------------------
def forward_project(volume: np.ndarray, vg: VolumeGeometry, g: ScannerGeometry, samples: int = 1, prec: int = 32,
                    mask: Optional[np.ndarray] = None, slab: Optional[dict] = None,
                    proj: Optional[np.ndarray] = None, length: Optional[np.ndarray] = None):
    """Forward projection of one (sub-)volume into (proj, length), accumulated (+=)."""
    half = volume.dtype == np.float16
    vol = np.ascontiguousarray(volume.view(np.uint16) if half else volume.astype(np.float32, copy=False))
    if proj is None:
        proj = np.zeros((g.height, g.width), np.float32)
    if length is None:
        length = np.zeros((g.height, g.width), np.float32)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    gv, gg = g.to_c(), vg.to_c(slab)
    lib().orc_forward(prec, ctypes.byref(gv), ctypes.byref(gg), _ptr(vol), int(half), _ptr(m), samples,
                      _ptr(proj), _ptr(length))
    return proj, length


def back_project(volume: np.ndarray, vg: VolumeGeometry, g: ScannerGeometry, residual: np.ndarray,
                 raylength: np.ndarray, lam: float, samples: int = 1, prec: int = 32, weights: int = WEIGHTS_Q8,
                 mask: Optional[np.ndarray] = None, slab: Optional[dict] = None, vmin=None, vmax=None):
    """In-place voxel-driven back projection of one view into ``volume``."""
    half = volume.dtype == np.float16
    assert volume.flags["C_CONTIGUOUS"]
    buf = volume.view(np.uint16) if half else volume
    assert buf.dtype in (np.float32, np.uint16)
    res = np.ascontiguousarray(residual, np.float32)
    rl = np.ascontiguousarray(raylength, np.float32)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    mat = np.ascontiguousarray(projection_matrix(g), np.float64)
    gg = vg.to_c(slab)
    if not g.perspective:
        pattern = np.ascontiguousarray(bp_sample_pattern(g, vg.voxel_size, samples))
        lib().orc_back_parallel(prec, ctypes.byref(gg), _ptr(mat), _ptr(pattern), samples, _ptr(res), _ptr(rl),
                                g.width, g.height, _ptr(buf), int(half), _ptr(m), float(lam), weights)
    else:
        src = np.ascontiguousarray(_f32(g.source), np.float64)
        lib().orc_back_perspective(prec, ctypes.byref(gg), _ptr(mat), _ptr(src), samples, _ptr(res), _ptr(rl),
                                   g.width, g.height, _ptr(buf), int(half), _ptr(m), float(lam), weights,
                                   int(vmin is not None), float(vmin or 0.0), int(vmax is not None),
                                   float(vmax or 0.0))
    return volume


def perspective_sampling_factor(proj_res, vol_res, samples_per_voxel: int) -> int:
    """PerspectiveBeamsBackProjectionKernel.cpp:72-81 computeSamplingFactor."""
    if samples_per_voxel != 0:
        return samples_per_voxel
    return max(1, max(proj_res) // max(vol_res))


def ray_length(vg: VolumeGeometry, g: ScannerGeometry, prec: int = 32) -> np.ndarray:
    out = np.zeros((g.height, g.width), np.float32)
    gv, gg = g.to_c(), vg.to_c()
    lib().orc_ray_length(prec, ctypes.byref(gv), ctypes.byref(gg), _ptr(out))
    return out


# ----------------------------------------------------------------------------
# Weighted back projection (plugins/WBPPlugin/src/reconstruction/WBP.cpp)
# ----------------------------------------------------------------------------
def ramlak_kernel(resolution: int = 128) -> np.ndarray:
    """ocl_src/GenerateRamLakKernel.cl: value at position gid - resolution/2, float32."""
    out = np.zeros(resolution, np.float32)
    pi2 = np.float32(np.float32(np.pi) * np.float32(np.pi))
    for gid in range(resolution):
        pos = gid - resolution // 2
        if pos == 0:
            out[gid] = np.float32(0.25)
        elif pos % 2 != 0:
            out[gid] = np.float32(-1.0) / np.float32(np.float32(pos * pos) * pi2)
    return out


def _next_pow2(n: int) -> int:
    """framework/NumericalAlgorithms.cpp:20-31."""
    v = n - 1
    for k in (1, 2, 4, 8, 16):
        v |= v >> k
    return v + 1


def _pad_index(i: np.ndarray, n: int, nu: int) -> np.ndarray:
    """ocl_src/PaddingForFFT.cl computePaddedCopyForFourierSpace, one axis."""
    b, e = (nu - n) // 2, (nu + n) // 2
    out = np.where((i >= b) & (i < e), i - b, np.where(i < e, b - i, (n + e - 1) - i))
    if out.min() < 0 or out.max() >= n:  # the reference would read outside the image
        raise ValueError(f"mirrored padding of {n} to {nu} leaves the image")
    return out


def wbp_filter(image: np.ndarray, filter_resolution: int = 128) -> np.ndarray:
    """algorithm/imagemanipulation/convolution/ConvolutionFourierSpaceImplementation.cpp
    with kernelRequiresOriginShifting (WBP.cpp:40-42): source padded (mirrored, centred)
    to the power-of-two grid, kernel zero-padded centred (PaddingForFFT.cl) and its origin
    moved (MoveOriginToCenter.cl), product of the FFTs, inverse FFT with 1/N, centred crop
    (CroppingForFFT.cl).  FP64 FFT here; float32 out."""
    img = np.asarray(image, np.float64)
    H, W = img.shape
    Wu, Hu = _next_pow2(max(W, filter_resolution)), _next_pow2(max(H, 1))
    ys = _pad_index(np.arange(Hu), H, Hu)
    xs = _pad_index(np.arange(Wu), W, Wu)
    src = img[ys][:, xs]
    padded = np.zeros((Hu, Wu))
    bx, by = (Wu - filter_resolution) // 2, (Hu - 1) // 2
    padded[by, bx:bx + filter_resolution] = ramlak_kernel(filter_resolution)
    shifted = np.roll(np.roll(padded, -(Hu // 2), axis=0), -(Wu // 2), axis=1)
    full = np.real(np.fft.ifft2(np.fft.fft2(src) * np.fft.fft2(shifted)))
    cx, cy = Wu // 2 - W // 2, Hu // 2 - H // 2
    return full[cy:cy + H, cx:cx + W].astype(np.float32)


def wbp(projections: np.ndarray, geometries, vg: "VolumeGeometry", lam: float = 1.0, samples: int = 1,
        prec: int = 32, weights: int = WEIGHTS_Q8, volume: Optional[np.ndarray] = None) -> np.ndarray:
    """WBP::runNiterations (WBP.cpp:72-83): per view the filtered projection and its ray
    lengths through the complete volume are back projected with lambda / N."""
    X, Y, Z = vg.resolution
    vol = np.zeros((Z, Y, X), np.float32) if volume is None else volume
    lamb = np.float32(lam) / np.float32(len(geometries))
    for i, g in enumerate(geometries):
        back_project(vol, vg, g, wbp_filter(projections[i]), ray_length(vg, g, prec), lamb, samples, prec, weights)
    return vol


# ----------------------------------------------------------------------------
# Blob basis functions (model/blobs, algorithm/blobs, ocl_src/BlobRaytracer.hl)
# ----------------------------------------------------------------------------
@dataclass
class BlobParameters:
    """model/blobs/BlobParameters.cpp: Kaiser-Bessel blob (support radius a, degree m,
    density fall-off alpha); createDefault() = (2.0, 2, 3.6)."""
    support_radius: float = 2.0
    degree: int = 2
    density_falloff: float = 3.6

    def _bessel(self, x: float, n: int = 40) -> float:
        """evaluateModifiedBessel: I_m(x) by 40 series terms (m = the degree)."""
        m = self.degree
        total, summand = 0.0, _uint_pow(0.5 * x, m) / float(math.factorial(m))
        for k in range(n):
            total += summand
            summand *= 0.25 * x * x / float((k + 1) * (k + m + 1))
        return total

    def evaluate(self, x: float) -> float:
        """BlobParameters::evaluate (Lewitt 1992)."""
        a, m, alpha = float(np.float32(self.support_radius)), self.degree, float(np.float32(self.density_falloff))
        if 0 <= x <= a:
            root = math.sqrt(1.0 - (x * x) / (a * a))
            return 1.0 / self._bessel(alpha) * _uint_pow(root, m) * self._bessel(alpha * root)
        return 0.0


def _uint_pow(base: float, e: int) -> float:
    """framework/NumericalAlgorithms.cpp uintPow (square and multiply)."""
    if e == 0:
        return 1.0
    if e == 1:
        return base
    f = _uint_pow(base, e // 2)
    return f * f * (1.0 if e % 2 == 0 else base)


_BLOB_TABLES: Dict[tuple, np.ndarray] = {}


def blob_ray_integration_samples(p: BlobParameters, count: int) -> np.ndarray:
    """algorithm/blobs/BlobRayIntegrationSampler.cpp: line integral through the blob at
    distance w = i * a / (count - 1), trapezoid-like sum of 1000 steps (kept per
    parameters and count: the sums take seconds in Python)."""
    key = (float(p.support_radius), int(p.degree), float(p.density_falloff), int(count))
    if key not in _BLOB_TABLES:
        _BLOB_TABLES[key] = _blob_ray_integration_samples(p, count)
    return _BLOB_TABLES[key].copy()


def _blob_ray_integration_samples(p: BlobParameters, count: int) -> np.ndarray:
    a = float(np.float32(p.support_radius))
    out = np.zeros(count, np.float32)
    n = 1000
    for i in range(count):
        w = float(i) * a / float(count - 1)
        d = math.sqrt(a * a - w * w)
        delta = d / n
        total = sum(p.evaluate(math.sqrt(w * w + float(k * k) * delta * delta)) for k in range(1, n + 1))
        out[i] = np.float32(delta * (2.0 * total + p.evaluate(w)))
    return out


def blob_voxelization_kernel(p: BlobParameters) -> np.ndarray:
    """algorithm/blobs/BlobVoxelizationKernelValues.cpp:49-67: the blob integrated over each
    voxel of the (2 ceil(a) + 1)^3 neighbourhood with 20^3 samples summed one after another
    in double (z, y, x order; a cumulative sum keeps that order), float32, [dz][dy][dx]."""
    r = int(math.ceil(float(np.float32(p.support_radius))))
    s = (np.arange(20) + 0.5) / 20.0
    out = np.zeros((2 * r + 1,) * 3, np.float32)
    ev = np.vectorize(p.evaluate)
    for dz in range(-r, r + 1):
        for dy in range(-r, r + 1):
            for dx in range(-r, r + 1):
                zz, yy, xx = np.meshgrid(dz - 0.5 + s, dy - 0.5 + s, dx - 0.5 + s, indexing="ij")
                vals = ev(np.sqrt(xx * xx + yy * yy + zz * zz)).ravel()
                out[dz + r, dy + r, dx + r] = np.float32(np.cumsum(vals)[-1] / 8000.0)
    return out


def blob_voxelize(blobs: np.ndarray, kernel: np.ndarray) -> np.ndarray:
    """BlobVoxelizerOperator: VolumeConvolution.cl over the blob coefficients with a zero
    border of the kernel radius (VolumeConvolutionOperator.cpp:30-37); float32 sums in
    kernel order z, y, x."""
    Z, Y, X = blobs.shape
    r = kernel.shape[0] // 2
    pad = np.zeros((Z + 2 * r, Y + 2 * r, X + 2 * r), np.float32)
    pad[r:r + Z, r:r + Y, r:r + X] = blobs
    out = np.zeros_like(blobs, dtype=np.float32)
    for kz in range(kernel.shape[0]):
        for ky in range(kernel.shape[1]):
            for kx in range(kernel.shape[2]):
                out = (out + kernel[kz, ky, kx] * pad[kz:kz + Z, ky:ky + Y, kx:kx + X]).astype(np.float32)
    return out


def _sample_blob(samples: np.ndarray, t: np.ndarray) -> np.ndarray:
    """BlobRaytracer.hl SampleBlob: linear interpolation of the ray-integration table."""
    n = samples.shape[0]
    # OpenCL clamp(t, 0, 1) = min(max(t, 0), 1); a NaN distance (sqrt of a rounded-negative
    # square) becomes 0 as fmax / fmin return the non-NaN operand
    coord = (np.fmin(np.fmax(t, np.float32(0.0)), np.float32(1.0)) * np.float32(n - 1)).astype(np.float32)
    left = np.floor(coord).astype(np.int64)
    lv = samples[left]
    rv = samples[np.minimum(n - 1, left + 1)]
    f = (coord - left.astype(np.float32)).astype(np.float32)
    return (lv + (rv - lv) * f).astype(np.float32)


class _FloatMat4:
    """framework/math/Matrix4x4.cpp in float32, step by step: at(column, row), multiply
    (:312-328), determinantOfMinor / determinant / inverse by cofactors (:90-119, :208-220)."""

    def __init__(self, cols=None):
        self.v = [np.float32(0)] * 16
        if cols is not None:
            for c in range(4):
                for r in range(4):
                    self.v[4 * c + r] = np.float32(cols[c][r])

    def at(self, c, r):
        return self.v[4 * c + r]

    def minor(self, dc, dr):
        f = np.float32
        c = [i if i < dc else i + 1 for i in range(3)]
        r = [i if i < dr else i + 1 for i in range(3)]
        a = self.at
        t1 = f(f(a(c[1], r[1]) * a(c[2], r[2])) - f(a(c[1], r[2]) * a(c[2], r[1])))
        t2 = f(f(a(c[1], r[0]) * a(c[2], r[2])) - f(a(c[1], r[2]) * a(c[2], r[0])))
        t3 = f(f(a(c[1], r[0]) * a(c[2], r[1])) - f(a(c[1], r[1]) * a(c[2], r[0])))
        return f(f(f(a(c[0], r[0]) * t1) - f(a(c[0], r[1]) * t2)) + f(a(c[0], r[2]) * t3))

    def inverse(self):
        f = np.float32
        a = self.at
        det = f(f(f(f(a(0, 0) * self.minor(0, 0)) - f(a(0, 1) * self.minor(0, 1))) + f(a(0, 2) * self.minor(0, 2)))
                - f(a(0, 3) * self.minor(0, 3)))
        o = f(f(1.0) / det)
        out = _FloatMat4()
        for c in range(4):
            for r in range(4):
                x = f(self.minor(c, r) * o)
                if (r + c) % 2 == 1:
                    x = f(x * f(-1.0))
                out.v[4 * r + c] = x
        return out

    def __matmul__(self, b):
        out = _FloatMat4()
        for i in range(4):
            for j in range(4):
                v = np.float32(0)
                for k in range(4):
                    v = np.float32(v + np.float32(self.at(k, j) * b.at(i, k)))
                out.v[4 * i + j] = v
        return out


def float_perspective_projection(g: ScannerGeometry) -> "_FloatMat4":
    """Matrix4x4::getPerspectiveProjection (Matrix4x4.cpp:376-399) in float32."""
    f = np.float32
    src, det = _f32(g.source).astype(f), _f32(g.detector).astype(f)
    hp, vp = _f32(g.hpitch).astype(f), _f32(g.vpitch).astype(f)
    dc = (det + f(0.5) * (f(g.width) * hp + f(g.height) * vp)).astype(f)
    view = _FloatMat4([list(hp) + [0], list(vp) + [0], list((dc - src).astype(f)) + [0], list(src) + [1]]).inverse()
    zn = f(1e-2)
    proj = _FloatMat4([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, f(f(1) / f(f(1) - zn)), 1], [0, 0, f(-zn / f(f(1) - zn)), 0]])
    tr = _FloatMat4([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [f(0.5) * f(g.width), f(0.5) * f(g.height), 0, 1]])
    return tr @ proj @ view


def projection_to_world(g: ScannerGeometry) -> np.ndarray:
    """The blob kernels' projection2world: world2projection.inverse() of the float
    perspective projection (PerspectiveBeamsForwardProjectionWithBlobsKernel.cpp:39-41),
    as a row-major 4x4 float32 array."""
    return np.array(float_perspective_projection(g).inverse().v, np.float32).reshape(4, 4).T


def forward_project_blobs(volume: np.ndarray, vg: "VolumeGeometry", g: ScannerGeometry, p: BlobParameters,
                          sample_count: int = 128) -> tuple:
    """PerspectiveBeamsForwardProjectionWithBlobs.cl + BlobRaytracer.hl BlobTraverseRay:
    the ray through pixel (x, y) (TransformCoordG of (x, y, 1) by projection_to_world)
    steps slice by slice along its dominant axis; every voxel within
    ceil(1.415 R / vs) of the pierced voxel whose centre is closer than R = a * vs.x to the
    ray adds table(dist / R) * value (and table(dist / R) to the traversal length).
    Vectorised over the rays, float32."""
    f32 = np.float32
    samples = blob_ray_integration_samples(p, sample_count)
    inv = projection_to_world(g)
    H, W = g.height, g.width
    yy, xx = np.meshgrid(np.arange(H, dtype=np.float32), np.arange(W, dtype=np.float32), indexing="ij")
    v = np.stack([xx.ravel(), yy.ravel(), np.ones(H * W, np.float32), np.ones(H * W, np.float32)])
    wp = (inv @ v).astype(np.float32)
    world = (wp[:3] / wp[3]).astype(np.float32)
    src = _f32(g.source).astype(np.float32)[:, None]
    d = (world - src).astype(np.float32)
    ray = (d / np.sqrt((d * d).sum(0))).astype(np.float32)
    X, Y, Z = vg.resolution
    res = np.array([X, Y, Z])
    vs = np.asarray(vg.voxel_size, np.float32)[:, None]
    bmin = np.asarray(vg.bmin, np.float32)[:, None]
    R = f32(f32(p.support_radius) * vs[0, 0])
    grid = int(math.ceil(f32(1.415) * R / vs[0, 0]))
    with np.errstate(divide="ignore", invalid="ignore"):
        tmin = ((bmin + f32(0.5) * vs - src) / ray).astype(np.float32)
    absr = np.abs(ray)
    axis = np.where((absr[0] >= np.maximum(absr[1], absr[2])), 0, np.where(absr[1] >= np.maximum(absr[0], absr[2]), 1, 2))
    val = np.zeros(H * W, np.float32)
    length = np.zeros(H * W, np.float32)
    vol = np.asarray(volume, np.float32)
    for ax in (0, 1, 2):
        sel = np.nonzero(axis == ax)[0]
        if sel.size == 0:
            continue
        r_ = ray[:, sel]
        point = (src + tmin[ax, sel] * r_).astype(np.float32)
        step = (r_ / r_[ax] * vs).astype(np.float32)
        ex, ey = [(1, 2), (2, 0), (0, 1)][ax]
        for _ in range(res[ax]):
            base = np.floor((point - bmin) / vs).astype(np.int64)
            for dy in range(-grid, grid + 1):
                for dx in range(-grid, grid + 1):
                    gc = base.copy()
                    gc[ex] += dx
                    gc[ey] += dy
                    inside = np.all((gc >= 0) & (gc < res[:, None]), axis=0)
                    if not inside.any():
                        continue
                    gci = gc[:, inside]
                    ids = sel[inside]
                    centre = (bmin + f32(0.5) * vs + gci.astype(np.float32) * vs).astype(np.float32)
                    rr = r_[:, inside]
                    sc = (src - centre).astype(np.float32)
                    t = (-(sc * rr).sum(0)).astype(np.float32)
                    c2r = (src + t * rr - centre).astype(np.float32)
                    d2 = (c2r * c2r).sum(0).astype(np.float32)
                    hit = d2 < R * R
                    if not hit.any():
                        continue
                    wgt = _sample_blob(samples, (np.sqrt(d2[hit]) / R).astype(np.float32))
                    gh = gci[:, hit]
                    np.add.at(val, ids[hit], wgt * vol[gh[2], gh[1], gh[0]])
                    np.add.at(length, ids[hit], wgt)
            point = (point + step).astype(np.float32)
    return val.reshape(H, W), length.reshape(H, W)


def back_project_blobs(volume: np.ndarray, vg: "VolumeGeometry", g: ScannerGeometry, residual: np.ndarray,
                       raylength: np.ndarray, lam: float, p: BlobParameters, sample_count: int = 256,
                       mask: Optional[np.ndarray] = None) -> np.ndarray:
    """PerspectiveBeamsBackProjectionWithBlobs.cl correct(), in place: every blob centre is
    projected, the detector window its footprint can reach is bounded (asin / acos / sin of
    the view angles), and every pixel of the window with a nonzero residual and a ray
    length above 1 whose ray passes closer than R = a * vs.x to the centre adds
    residual * table(dist / R) / length; the blob takes lambda * sum / sum(table) when the
    weights exceed 1e-2, times mask / 255 with a prior-knowledge mask (uint8).  Vectorised
    over the voxels, float32."""
    f = np.float32
    table = blob_ray_integration_samples(p, sample_count)
    X, Y, Z = vg.resolution
    vs = np.asarray(vg.voxel_size, f)
    R = f(f(p.support_radius) * vs[0])
    fp = float_perspective_projection(g)
    w2p = np.array(fp.v, f).reshape(4, 4).T  # the float projection matrix, row-major
    p2w = np.array(fp.inverse().v, f).reshape(4, 4).T
    src = _f32(g.source).astype(f)
    det = _f32(g.detector).astype(f)
    hp, vp = _f32(g.hpitch).astype(f), _f32(g.vpitch).astype(f)
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    centre = np.stack([np.asarray(vg.bmin, f)[i] + (g_.astype(f) + f(0.5)) * vs[i]
                       for i, g_ in enumerate((xx.ravel(), yy.ravel(), zz.ravel()))]).astype(f)
    c4 = np.vstack([centre, np.ones((1, centre.shape[1]), f)])
    proj = (w2p @ c4).astype(f)
    params = (proj[:2] / proj[3]).astype(f)
    ok = proj[3] > 0
    pv = (det[:, None] + params[0] * hp[:, None] + params[1] * vp[:, None] - src[:, None]).astype(f)
    q = (centre - src[:, None]).astype(f)
    lp = np.sqrt((pv * pv).sum(0)).astype(f)
    lq = np.sqrt((q * q).sum(0)).astype(f)
    ldx, ldy = f(np.sqrt((hp * hp).sum())), f(np.sqrt((vp * vp).sum()))
    r = (R * lp / lq).astype(f)
    alpha = np.arcsin(R / lq).astype(f)
    bx = np.arccos(((hp[:, None] * pv).sum(0) / (ldx * lp)).astype(f)).astype(f)
    by = np.arccos(((vp[:, None] * pv).sum(0) / (ldy * lp)).astype(f)).astype(f)
    with np.errstate(divide="ignore", invalid="ignore"):
        wx = (np.maximum(r / np.sin(bx - alpha), r / np.sin(bx + alpha)) / ldx).astype(f)
        wy = (np.maximum(r / np.sin(by - alpha), r / np.sin(by + alpha)) / ldy).astype(f)
    ok &= (wx < 4096) & (wy < 4096)  # windows that are not finite or wider than any detector: skipped
    sx = np.where(ok, np.ceil(np.where(ok, wx, 0)), 0).astype(np.int64)
    sy = np.where(ok, np.ceil(np.where(ok, wy, 0)), 0).astype(np.int64)
    base = np.trunc(params + f(0.5) * np.sign(params)).astype(np.int64)
    H, W = residual.shape
    val = np.zeros(centre.shape[1], f)
    acc = np.zeros(centre.shape[1], f)
    R2 = f(R * R)
    for dy in range(-int(sy.max()), int(sy.max()) + 1):
        for dx in range(-int(sx.max()), int(sx.max()) + 1):
            use = ok & (np.abs(dx) <= sx) & (np.abs(dy) <= sy)
            px, py = base[0] + dx, base[1] + dy
            use &= (px >= 0) & (py >= 0) & (px < W) & (py < H)
            ids = np.nonzero(use)[0]
            if ids.size == 0:
                continue
            pxs, pys = px[ids], py[ids]
            ln = raylength[pys, pxs]
            res = residual[pys, pxs]
            take = (res != 0) & (ln > 1.0)
            ids, pxs, pys, ln, res = ids[take], pxs[take], pys[take], ln[take], res[take]
            if ids.size == 0:
                continue
            pc = (p2w @ np.vstack([pxs.astype(f), pys.astype(f), np.ones_like(ln), np.ones_like(ln)])).astype(f)
            d = (pc[:3] / pc[3] - src[:, None]).astype(f)
            d = (d / np.sqrt((d * d).sum(0))).astype(f)
            s2b = q[:, ids]
            t0 = (d * s2b).sum(0).astype(f)
            dist2 = ((s2b * s2b).sum(0) - t0 * t0).astype(f)
            hit = R2 > dist2
            with np.errstate(invalid="ignore"):
                wgt = _sample_blob(table, np.sqrt(dist2[hit] / R2).astype(f))
            np.add.at(acc, ids[hit], wgt)
            np.add.at(val, ids[hit], (res[hit] * wgt / ln[hit]).astype(f))
    upd = acc > f(1e-2)
    flat = volume.reshape(-1)
    step = (f(lam) * val[upd]).astype(f)
    if mask is not None:
        step = (step * (mask.reshape(-1)[upd].astype(f) / f(255.0)).astype(f)).astype(f)
    flat[upd] = (flat[upd] + step / acc[upd]).astype(f)
    return volume


def blob_block_iterations(volume: np.ndarray, vg: "VolumeGeometry", geometries, projections: np.ndarray,
                          order, block_size: int, lam: float, p: BlobParameters, iterations: int = 1) -> float:
    """BlockIterativeReconstructionOperator.cpp:84-160 with blob basis functions, in place:
    per block of ``order``, the blob forward projection (256-entry table,
    DefaultForwardProjectionCreator.cpp:56) of every view into cleared images, residual =
    measured - virtual, then the blob back projection of every view with lambda / block
    size.  Returns the sum of squared residuals of the last iteration."""
    order = list(order)
    rsq = 0.0
    for _ in range(iterations):
        rsq = 0.0
        for b0 in range(0, len(order), block_size):
            blk = order[b0:b0 + block_size]
            fps = [forward_project_blobs(volume, vg, geometries[i], p, 256) for i in blk]
            res = [(projections[i] - fps[j][0]).astype(np.float32) for j, i in enumerate(blk)]
            rsq += float(sum((r.astype(np.float64) ** 2).sum() for r in res))
            for j, i in enumerate(blk):
                back_project_blobs(volume, vg, geometries[i], res[j], fps[j][1],
                                   float(np.float32(lam) / np.float32(len(blk))), p)
    return rsq


def long_object_compensation(proj: np.ndarray, length: np.ndarray, constant_length: float):
    p = np.ascontiguousarray(proj, np.float32).copy()
    l = np.ascontiguousarray(length, np.float32).copy()
    lib().orc_long_object_compensation(_ptr(p), _ptr(l), float(constant_length), p.size)
    return p, l


def to_half(a: np.ndarray) -> np.ndarray:
    src = np.ascontiguousarray(a, np.float32)
    out = np.empty(src.shape, np.uint16)
    lib().orc_half_from_float(_ptr(src), _ptr(out), src.size)
    return out.view(np.float16)


# ----------------------------------------------------------------------------
# Projection orderings (model/projectionset/*.cpp)
# ----------------------------------------------------------------------------
def order_identity(n: int, skip=()) -> List[int]:
    """ProjectionSet.cpp:14-25 + ProjectionSetIdentity.cpp."""
    return [i for i in range(n) if i not in set(skip)]


def order_maxangle(indices: List[int]) -> List[int]:
    """ProjectionSetMaxAngle.cpp:16-38: alternate middle-out and front."""
    n = len(indices)
    out = [0] * n
    j, k = n // 2, 0
    for i in range(n):
        if i % 2 == 0:
            out[i] = indices[j]; j += 1
        else:
            out[i] = indices[k]; k += 1
    return out


def order_buckets(indices: List[int]) -> List[int]:
    """ProjectionSetBuckets.cpp:16-42: four interleaved angle groups."""
    n = len(indices)
    cur = [i * n // 4 for i in range(4)]
    out = [0] * n
    for i in range(n):
        s = i % 4
        out[i] = indices[cur[s]]
        cur[s] += 1
    return out


# ----------------------------------------------------------------------------
# Block-iterative driver
# ----------------------------------------------------------------------------
@dataclass
class ReconstructionSetup:
    vg: VolumeGeometry
    views: List[ScannerGeometry]
    projections: np.ndarray          # (N, H, W) float32, in iteration order
    lam: float
    block_size: int
    fp_samples: int = 1
    bp_samples: int = 1
    use_loc: bool = False
    weights: int = WEIGHTS_Q8
    vmin: Optional[float] = None
    vmax: Optional[float] = None
    mask: Optional[np.ndarray] = None


def block_iterative(setup: ReconstructionSetup, volume: np.ndarray, iterations: int, prec: int = 32) -> np.ndarray:
    """BlockIterativeReconstructionOperator.cpp:92-142 on the CPU, in place.
    ``volume`` is (Z, Y, X) float32 (or float16 for the half path)."""
    vg = setup.vg
    slabs = vg.slabs()
    N = len(setup.views)
    half = volume.dtype == np.float16
    buf = volume.view(np.uint16) if half else volume
    esz = buf.itemsize
    X, Y, Z = vg.resolution
    vol_ptrs = (ctypes.c_void_p * len(slabs))()
    mask_ptrs = None
    if setup.mask is not None:
        mk = np.ascontiguousarray(setup.mask, np.uint8)
        mask_ptrs = (ctypes.c_void_p * len(slabs))()
    for i, s in enumerate(slabs):
        vol_ptrs[i] = buf.ctypes.data + s["z0"] * X * Y * esz
        if mask_ptrs is not None:
            mask_ptrs[i] = mk.ctypes.data + s["z0"] * X * Y
    c_slabs = (_VolGeom * len(slabs))(*[vg.to_c(s) for s in slabs])
    c_views = (_View * N)(*[g.to_c() for g in setup.views])
    mats = np.ascontiguousarray(np.stack([projection_matrix(g) for g in setup.views]), np.float64)
    persp = setup.views[0].perspective
    if persp:
        pattern = np.zeros((N, 1, 4), np.float32)
        nbp = 1
        pn = perspective_sampling_factor((setup.views[0].width, setup.views[0].height), slabs[0]["res"],
                                         setup.bp_samples)
    else:
        pattern = np.ascontiguousarray(np.stack([bp_sample_pattern(g, vg.voxel_size, setup.bp_samples)
                                                 for g in setup.views]), np.float32)
        nbp = setup.bp_samples
        pn = 1
    loc = np.zeros(N, np.float32)
    if setup.use_loc:
        loc = np.array([traversal_length_through_bbox(g, vg.bmin, vg.bmax) for g in setup.views], np.float32)
    proj = np.ascontiguousarray(setup.projections, np.float32)
    rc = lib().orc_block_iterative(prec, N, c_views, _ptr(proj), len(slabs), c_slabs, vol_ptrs, int(half),
                                   mask_ptrs, setup.fp_samples, _ptr(mats), _ptr(pattern), nbp, pn,
                                   float(setup.lam), int(setup.block_size), int(iterations), int(setup.use_loc),
                                   _ptr(loc), setup.weights, int(setup.vmin is not None), float(setup.vmin or 0.0),
                                   int(setup.vmax is not None), float(setup.vmax or 0.0))
    if rc != 0:
        raise RuntimeError(f"oracle block_iterative failed ({rc})")
    return volume


# ----------------------------------------------------------------------------
# Comparators (model/image/ImageComparator.cpp:109-122, model/volume/StackComparator.cpp:12)
# ----------------------------------------------------------------------------
def rms(a: np.ndarray, b: np.ndarray) -> float:
    d = np.asarray(a, np.float64) - np.asarray(b, np.float64)
    return float(np.sqrt(np.mean(d * d)))


def images_equal(a: np.ndarray, b: np.ndarray) -> bool:
    """ImageComparator::assertImagesAreEqual: RMS <= 0.1 and max |d| <= 1e-5 * max."""
    if rms(a, b) > 0.1:
        return False
    thr = max(float(np.max(a)), float(np.max(b))) * 1e-5
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)))) <= thr


def max_slice_rms(a: np.ndarray, b: np.ndarray) -> float:
    """StackComparator::getMaxRMS over the file's slices (first axis)."""
    return max(rms(a[i], b[i]) for i in range(a.shape[0]))


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))
