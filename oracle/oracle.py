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
from typing import List, Optional, Sequence

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
