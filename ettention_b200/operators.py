"""Python face of the CUDA path, mirroring libReconstruction's operator surface.

Names, argument meaning and error behaviour follow the reference
(LR = ettention/libReconstruction/src):

  ScannerGeometry / rotate          LR/model/geometry/{Parallel,Perspective}ScannerGeometry.cpp,
                                    LR/model/geometry/SingleAxisTiltRotator.cpp
  GPUMappedVolume                   LR/model/volume/GPUMappedVolume.cpp (device-resident here)
  ForwardProjectionOperator         LR/algorithm/projections/forward/ForwardProjectionOperator.cpp
  BackProjectionOperator            LR/algorithm/projections/back/BackProjectionOperator.cpp
  BlockIterativeReconstructionOperator
                                    LR/algorithm/reconstruction/blockiterative/
                                    BlockIterativeReconstructionOperator.cpp
  AlgebraicParameterSet.from_config LR/setup/parameterset/*ParameterSet.cpp (same config keys)
  BlobParameters, BlobRayIntegrationSampler, BlobVoxelizationKernelValues,
  BlobVoxelizerOperator             LR/model/blobs, LR/algorithm/blobs (blob basis functions)

Every compute call goes through ``libettention_b200.so``; device images are
CUDA ``torch.Tensor`` objects (float32, contiguous) used as plain device
memory.
"""
from __future__ import annotations

import ctypes
import os
import weakref
from dataclasses import dataclass, field
from typing import Dict, Iterable, List, Optional, Sequence

import numpy as np

from . import _abi
from ._abi import EttentionError, View, VolumeDesc, ReconParams, check, lib


# ----------------------------------------------------------------------------- geometry
@dataclass
class ScannerGeometry:
    """LR/model/geometry/ScannerGeometry.cpp:39-46 (+ Parallel/Perspective subclass)."""
    source: Sequence[float]
    detector: Sequence[float]
    hpitch: Sequence[float]
    vpitch: Sequence[float]
    width: int
    height: int
    perspective: bool = False

    def to_view(self) -> View:
        v = View()
        for name in ("source", "detector", "hpitch", "vpitch"):
            arr = getattr(v, name)
            val = getattr(self, name)
            for i in range(3):
                arr[i] = float(val[i])
        v.width, v.height, v.perspective = int(self.width), int(self.height), int(bool(self.perspective))
        return v

    @classmethod
    def from_view(cls, v: View) -> "ScannerGeometry":
        return cls(list(v.source), list(v.detector), list(v.hpitch), list(v.vpitch), v.width, v.height,
                   bool(v.perspective))

    def rotated(self, tilt_deg: float, xaxis_tilt_deg: float = 0.0) -> "ScannerGeometry":
        """SingleAxisTiltRotator::createRotatedScannerGeometry."""
        out = View()
        check(lib().etcu_view_rotate(ctypes.byref(self.to_view()), float(tilt_deg), float(xaxis_tilt_deg),
                                     ctypes.byref(out)))
        return ScannerGeometry.from_view(out)

    def projection_matrix(self) -> np.ndarray:
        m = np.zeros(16, np.float32)
        check(lib().etcu_view_projection_matrix(ctypes.byref(self.to_view()), m.ctypes.data))
        return m

    def sample_pattern(self, voxel_size: Sequence[float], samples: int) -> np.ndarray:
        """ParallelBeamsBackProjectionKernel::setSamples + generateSamplingPatternForPerVoxelSampling."""
        vs = np.asarray(voxel_size, np.float32)
        out = np.zeros((max(int(samples), 1), 4), np.float32)
        check(lib().etcu_view_sample_pattern(ctypes.byref(self.to_view()), vs.ctypes.data, int(samples),
                                             out.ctypes.data))
        return out

    def traversal_length(self, bbox_min: Sequence[float], bbox_max: Sequence[float]) -> float:
        lo = np.asarray(bbox_min, np.float32)
        hi = np.asarray(bbox_max, np.float32)
        r = ctypes.c_float()
        check(lib().etcu_view_traversal_length(ctypes.byref(self.to_view()), lo.ctypes.data, hi.ctypes.data,
                                               ctypes.byref(r)))
        return float(r.value)


def mrc_base_geometry(nx: int, ny: int) -> ScannerGeometry:
    """LR/io/datasource/MRCStack.cpp:250-261: base parallel geometry of an MRC tilt series."""
    return ScannerGeometry([-0.5 * nx, -0.5 * ny, float(nx)], [-0.5 * nx, -0.5 * ny, -float(nx)],
                           [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], nx, ny, False)


def tilt_series(base: ScannerGeometry, angles: Iterable[float], xaxis_tilt_deg: float = 0.0) -> List[ScannerGeometry]:
    return [base.rotated(a, xaxis_tilt_deg) for a in angles]


def projection_order(order: int, n: int, skip: Sequence[int] = ()) -> List[int]:
    """LR/model/projectionset/factory/ProjectionIteratorFactory.cpp:11-22 orderings."""
    sk = np.asarray(list(skip), np.uint32)
    out = np.zeros(max(n, 1), np.uint32)
    cnt = ctypes.c_uint32()
    check(lib().etcu_projection_order(int(order), int(n), sk.ctypes.data if len(sk) else None, len(sk),
                                      out.ctypes.data, ctypes.byref(cnt)))
    return [int(i) for i in out[: cnt.value]]


class MRCStack:
    """LR/io/datasource/MRCStack.cpp: a tilt series in an MRC file (modes 0/1/2/6) with an
    optional tilt-angle file; projections as float32 (log-transformed when
    ``logarithmize``, the reference's input.logarithmize), the MRC base geometry and
    SingleAxisTiltRotator views."""

    def __init__(self, path: str, tilt_path: Optional[str] = None, logarithmize: bool = False):
        self.path = str(path)
        info = _abi.MrcInfo()
        _check_free(lib().etcu_mrc_read_info(self.path.encode(), ctypes.byref(info)))
        self.info = info
        self.logarithmize = bool(logarithmize)
        if tilt_path is None:
            self.tilt_angles = [0.0] * info.nz  # MRCStack::setEmptyTiltAngles
        else:
            self.tilt_angles = read_tilt_angles(tilt_path)
            if len(self.tilt_angles) != info.nz:  # ImageStackDatasource.cpp:75-78
                raise EttentionError(_abi.ERR_INVALID_ARGUMENT,
                                     f"Number of projections DIFFERS from number of Tilt Angles given in {tilt_path}")

    def getNumberOfProjections(self) -> int:
        return int(self.info.nz)

    def getResolution(self):
        return int(self.info.nx), int(self.info.ny)

    def load_projections(self) -> np.ndarray:
        """All projections, (nz, ny, nx) float32."""
        out = np.empty((self.info.nz, self.info.ny, self.info.nx), np.float32)
        _check_free(lib().etcu_mrc_read_stack(self.path.encode(), int(self.logarithmize), out.ctypes.data, out.size))
        return out

    def createScannerGeometry(self, index: int, xaxis_tilt_deg: float = 0.0) -> "ScannerGeometry":
        return mrc_base_geometry(*self.getResolution()).rotated(float(self.tilt_angles[index]), xaxis_tilt_deg)

    def geometries(self, xaxis_tilt_deg: float = 0.0) -> List["ScannerGeometry"]:
        return [self.createScannerGeometry(i, xaxis_tilt_deg) for i in range(self.getNumberOfProjections())]


def _check_free(status: int) -> None:
    if status != _abi.OK:
        msg = lib().etcu_last_error(None)
        raise EttentionError(status, (msg or b"").decode() or f"etcu status {status}")


def read_tilt_angles(path: str) -> List[float]:
    """ImageStackDatasource::readTiltAngles: every whitespace-separated float of the file."""
    n = ctypes.c_uint32()
    _check_free(lib().etcu_read_tilt_angles(str(path).encode(), None, 0, ctypes.byref(n)))
    out = np.zeros(max(1, n.value), np.float32)
    _check_free(lib().etcu_read_tilt_angles(str(path).encode(), out.ctypes.data, n.value, ctypes.byref(n)))
    return [float(a) for a in out[: n.value]]


OUTPUT_VOXEL_TYPES = {"unsigned8": 0, "signed16": 1, "float32": 2, "unsigned16": 6}


def write_mrc_volume(path: str, volume: np.ndarray, orientation: str = "xzy", voxel_type: str = "float32",
                     invert: bool = False) -> None:
    """VolumeFileFormatWriter + MRCWriter: ``volume`` is (z, y, x); orientation 'xzy' (the
    reference's default output.options.orientation) or 'xyz'; voxel_type one of
    output.options.voxelType's values (IOEnumerations.cpp:39-61: unsigned8, unsigned16,
    signed16, float32); invert = output.options.invert."""
    if voxel_type not in OUTPUT_VOXEL_TYPES:
        raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "ParseVoxelValueType: Unknown file mode ")
    v = np.ascontiguousarray(volume, np.float32)
    res = np.array([v.shape[2], v.shape[1], v.shape[0]], np.uint32)
    axes = {"xyz": _abi.AXES_XYZ, "xzy": _abi.AXES_XZY}[orientation.lower()]
    _check_free(lib().etcu_mrc_write_volume_typed(str(path).encode(), v.ctypes.data, res.ctypes.data, axes,
                                                  OUTPUT_VOXEL_TYPES[voxel_type], int(bool(invert))))


def read_tiff(path: str, page: int = 0) -> np.ndarray:
    """ImageDeserializer::readImage / readImageFromStack (LR/io/deserializer/
    ImageDeserializer.cpp:10-62): one page as (height, width) float32, row 0 the file's
    first row; 8-bit grey / 255, 16-bit grey / 65535, 32-bit float as is."""
    info = _abi.ImageInfo()
    _check_free(lib().etcu_tiff_read_info(str(path).encode(), int(page), ctypes.byref(info)))
    out = np.empty((info.height, info.width), np.float32)
    _check_free(lib().etcu_tiff_read(str(path).encode(), int(page), out.ctypes.data, out.size))
    return out


def tiff_page_count(path: str) -> int:
    """ImageDeserializer::getNumberOfImagesInStack."""
    info = _abi.ImageInfo()
    _check_free(lib().etcu_tiff_read_info(str(path).encode(), 0, ctypes.byref(info)))
    return int(info.pages)


def write_tiff(path: str, image: np.ndarray) -> None:
    """ImageSerializer::writeImage(..., TIFF_GRAY_32): (height, width) as 32-bit float grey."""
    a = np.ascontiguousarray(image, np.float32)
    if a.ndim != 2:
        raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "an image is a 2-D array")
    _check_free(lib().etcu_tiff_write(str(path).encode(), a.ctypes.data, a.shape[1], a.shape[0]))


class ImageStackDirectoryDatasource:
    """LR/io/datasource/ImageStackDirectoryDatasource.cpp: a directory of projection
    images described by metadata.xml (base parallel geometry, one tilt angle per
    image, optional <logscale/>, multi-page <projectionstack> entries); the detector
    size is the first image's; views are SingleAxisTiltRotator rotations of the base
    geometry."""

    METADATA = "metadata.xml"

    def __init__(self, directory: str):
        self.directory = str(directory)
        h = ctypes.c_void_p()
        _check_free(lib().etcu_image_stack_open(self.directory.encode(), ctypes.byref(h)))
        self.handle = h
        info = _abi.ImageStackInfo()
        _check_free(lib().etcu_image_stack_info_get(h, ctypes.byref(info)))
        self.count, self.width, self.height = int(info.count), int(info.width), int(info.height)
        self.base_geometry = ScannerGeometry.from_view(info.base)
        a = np.zeros(max(1, self.count), np.float32)
        _check_free(lib().etcu_image_stack_tilt_angles(h, a.ctypes.data, self.count))
        self.tilt_angles = [float(x) for x in a[: self.count]]

    @staticmethod
    def canHandleResource(path: str) -> bool:
        """:74-87: a directory that holds metadata.xml."""
        return os.path.isdir(path) and os.path.exists(os.path.join(path, ImageStackDirectoryDatasource.METADATA))

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().etcu_image_stack_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def getNumberOfProjections(self) -> int:
        return self.count

    def getResolution(self):
        return self.width, self.height

    def getTiltAngle(self, index: int) -> float:
        return self.tilt_angles[index]

    def load_projections(self, first: int = 0, count: Optional[int] = None) -> np.ndarray:
        """Projections first .. first + count - 1 as (count, height, width) float32."""
        n = self.count - int(first) if count is None else int(count)
        out = np.empty((n, self.height, self.width), np.float32)
        _check_free(lib().etcu_image_stack_load(self.handle, int(first), n, out.ctypes.data, out.size))
        return out

    def getProjectionImage(self, index: int) -> np.ndarray:
        return self.load_projections(index, 1)[0]

    def createScannerGeometry(self, index: int, xaxis_tilt_deg: float = 0.0) -> ScannerGeometry:
        return self.base_geometry.rotated(self.tilt_angles[index], xaxis_tilt_deg)

    def geometries(self, xaxis_tilt_deg: float = 0.0) -> List[ScannerGeometry]:
        return [self.createScannerGeometry(i, xaxis_tilt_deg) for i in range(self.count)]

    @staticmethod
    def writeMetaDataFile(path: str, tilt_angles: Sequence[float], filenames: Sequence[str],
                          base: ScannerGeometry, volume_resolution: Sequence[int]) -> None:
        """:121-175: base geometry, volume dimensions, one <projection> per image."""
        if len(tilt_angles) != len(filenames):
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "Filename count does not match tilt angle count!")
        a = np.asarray(tilt_angles, np.float32)
        names = (ctypes.c_char_p * max(1, len(filenames)))(*[str(f).encode() for f in filenames])
        res = np.asarray(volume_resolution, np.uint32)
        _check_free(lib().etcu_image_stack_write_metadata(str(path).encode(), a.ctypes.data, names, len(filenames),
                                                          ctypes.byref(base.to_view()), res.ctypes.data))


def mrc_can_handle(path: str) -> bool:
    """MRCStack::canHandleResource (MRCStack.cpp:70-83): a file ending in .mrc or .ali."""
    return os.path.isfile(path) and os.path.splitext(path)[1] in (".mrc", ".ali")


def open_image_stack(projections: str, tilt_angles: Optional[str] = None, logarithmize: bool = False):
    """ImageStackDatasourceFactory::instantiate (LR/io/ImageStackDataSourceFactory.cpp:19-44):
    the directory datasource is asked first, then the MRC stack."""
    if ImageStackDirectoryDatasource.canHandleResource(projections):
        return ImageStackDirectoryDatasource(projections)
    if mrc_can_handle(projections):
        return MRCStack(projections, tilt_angles, logarithmize)
    raise EttentionError(_abi.ERR_INVALID_ARGUMENT,
                         f"Unable to open image stack {projections}! Incorrect filename or plugin missing?")


PATH_PARAMETERS = ("input.projections", "input.tiltAngles", "output.filename", "volume.initFile",
                   "priorknowledge.maskVolumeFilename", "debug.performanceReportFile", "debug.infoPath",
                   "debug.meshExportPath")


class XMLParameterSource:
    """LR/setup/parametersource/XMLParameterSource.cpp: the value attribute of every
    element by its dotted path; path parameters use '/' for '\\' and are relative to
    the file's directory (:24-35)."""

    def __init__(self, filename: str):
        self.filename = str(filename)
        n = ctypes.c_size_t()
        _check_free(lib().etcu_xml_config_read(self.filename.encode(), None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        _check_free(lib().etcu_xml_config_read(self.filename.encode(), buf, n.value, ctypes.byref(n)))
        self.values: Dict[str, str] = {}
        for line in buf.value.decode().splitlines():
            key, _, value = line.partition("\t")
            self.values[key] = value

    def parameterExists(self, name: str) -> bool:
        return name in self.values

    def getStringParameter(self, name: str) -> str:
        if name not in self.values:
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, f"xml config file entry does not exist: {name}")
        return self.values[name]

    def getPathParameter(self, name: str) -> str:
        p = self.getStringParameter(name).replace("\\", "/")
        if not os.path.isabs(p):
            p = os.path.join(os.path.dirname(os.path.abspath(self.filename)), p)
        return os.path.normpath(p)

    def config(self) -> Dict[str, str]:
        """Every value, path parameters resolved: the input of AlgebraicParameterSet.from_config."""
        cfg = dict(self.values)
        for k in PATH_PARAMETERS:
            if k in cfg:
                cfg[k] = self.getPathParameter(k)
        return cfg


def _true(v) -> bool:
    return str(v).strip().lower() in ("true", "1", "yes")


# CoordinateOrder (LR/setup/parameterset/IOEnumerations.cpp:7-35, "xzy_order" ...):
# working coordinate k = file coordinate perm[k] (BlockIterativeConfiguration.cpp:176-197).
_ORIENTATIONS = {"xyz": (0, 1, 2), "xzy": (0, 2, 1), "yxz": (1, 0, 2), "yzx": (2, 0, 1), "zxy": (1, 2, 0),
                 "zyx": (2, 1, 0)}


def _coordinate_order(value: str) -> str:
    v = str(value).strip().lower()
    v = v[:-len("_order")] if v.endswith("_order") else v
    if v not in _ORIENTATIONS:
        raise EttentionError(_abi.ERR_INVALID_ARGUMENT, f"Unknown CoordinateOrder given: {value}")
    return v


def load_init_volume(path: str, orientation: str, resolution: Sequence[int]) -> np.ndarray:
    """volume.initFile (BlockIterativeConfiguration.cpp:36-40, :155-198): an MRC volume
    whose file coordinates map to the working volume's by ``orientation``; returns
    the (z, y, x) float32 working volume."""
    X, Y, Z = (int(r) for r in resolution)
    perm = _ORIENTATIONS[_coordinate_order(orientation)]
    raw = MRCStack(path).load_projections()  # (nz, ny, nx): file coordinates (x, y, z)
    work_xyz = np.transpose(np.transpose(raw, (2, 1, 0)), perm)
    if work_xyz.shape != (X, Y, Z):
        raise EttentionError(_abi.ERR_INVALID_ARGUMENT,
                             f"Resolution of volume from file {path} does not match resolution given in config file!")
    return np.ascontiguousarray(np.transpose(work_xyz, (2, 1, 0)), np.float32)


def load_mask_volume(path: str, resolution: Sequence[int]) -> np.ndarray:
    """priorknowledge.maskVolumeFilename (BlockIterativeConfiguration.cpp:46-50,
    VolumeDeserializer.cpp:15-47): an MRC volume in file order, each value cast to an
    8-bit voxel (ByteVolume::convertValueFromFloat; clamped to 0..255 here)."""
    X, Y, Z = (int(r) for r in resolution)
    m = MRCStack(path).load_projections()
    if m.shape != (Z, Y, X):
        raise EttentionError(_abi.ERR_INVALID_ARGUMENT, f"mask volume {path} does not match the volume's resolution")
    return np.clip(m, 0, 255).astype(np.uint8)


def reconstruct_from_config(config, device: int = 0, write_output: bool = True) -> np.ndarray:
    """A block-iterative run as the reference's frontend performs it from a parameter
    file: parameters (XMLParameterSource or a dict of keys with resolved paths),
    the projections through open_image_stack (input.projections, input.tiltAngles,
    input.logarithmize, input.xAxisTilt), the volume from volume.* and
    hardware.subVolumeCount, optionally volume.initFile (MRC in
    volume.initFileOrientation, XZY by default; BlockIterativeConfiguration.cpp:36-40,
    :155-198) and priorknowledge.maskVolumeFilename (MRC read in file order, values
    cast to 8 bits; :46-50), the iterations of BlockIterativeReconstructionOperator
    on the GPU (or, for algorithm "wbp", the WBP plugin's weighted back projection), and Framework::writeFinalVolume to output.filename (MRC of output.options.voxelType with
    output.options.invert, output.options.orientation xyz_order or xzy_order, XZY by
    default).  Returns the
    (z, y, x) volume."""
    cfg = config.config() if isinstance(config, XMLParameterSource) else dict(config)
    p = AlgebraicParameterSet.from_config(cfg)
    if p.resolution is None:
        raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "xml config file entry does not exist: volume.dimension")
    if "input.projections" not in cfg:
        raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "xml config file entry does not exist: input.projections")
    vt = cfg.get("output.options.voxelType", "float32")
    if vt not in OUTPUT_VOXEL_TYPES:  # OutputParameterSet.cpp:29-33
        raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "ParseVoxelValueType: Unknown file mode ")
    invert = _true(cfg.get("output.options.invert", "false"))
    out_order = _coordinate_order(cfg.get("output.options.orientation", "xzy_order"))
    if write_output and "output.filename" in cfg and out_order not in ("xyz", "xzy"):
        raise EttentionError(_abi.ERR_UNSUPPORTED, f"output orientation {out_order}: XYZ and XZY are written")
    stack = open_image_stack(cfg["input.projections"], cfg.get("input.tiltAngles"),
                             _true(cfg.get("input.logarithmize", "false")))
    views = stack.geometries(p.xaxis_tilt)
    data = stack.load_projections()
    X, Y, Z = (int(r) for r in p.resolution)
    init = None
    if "volume.initFile" in cfg:
        init = load_init_volume(cfg["volume.initFile"], cfg.get("volume.initFileOrientation", "xzy_order"), (X, Y, Z))
    mask = None
    if "priorknowledge.maskVolumeFilename" in cfg:
        mask = load_mask_volume(cfg["priorknowledge.maskVolumeFilename"], (X, Y, Z))
    ctx = Context(device)
    try:
        lo, hi = p.bbox()
        vol = GPUMappedVolume(ctx, (X, Y, Z), lo, hi, voxel_type=p.voxel_type, init_value=p.init_value,
                              subvolume_count=p.subvolume_count)
        if init is not None:
            vol.upload(init)
        if mask is not None:
            vol.set_mask(mask)
        if p.algorithm == "wbp":  # the WBP plugin's algorithm (WBPPlugin.cpp)
            WBPOperator(vol, views, data, p).run()
            v = vol.download()
        else:
            rec = BlockIterativeReconstructionOperator(vol, views, data, p)
            rec.run()
            v = rec.getReconstructedVolume()
    finally:
        ctx.close()
        if isinstance(stack, ImageStackDirectoryDatasource):
            stack.close()
    if write_output and "output.filename" in cfg:
        write_mrc_volume(cfg["output.filename"], v, out_order, vt, invert)
    return v


ORDERS = {"identity": _abi.ORDER_IDENTITY, "random": _abi.ORDER_RANDOM, "maxangle": _abi.ORDER_MAXANGLE,
          "buckets": _abi.ORDER_BUCKETS}
VOXEL_TYPES = {"float": _abi.VOXEL_FLOAT32, "float32": _abi.VOXEL_FLOAT32, "half": _abi.VOXEL_HALF16,
               "half_master": _abi.VOXEL_F16_MASTER, "bf16_master": _abi.VOXEL_BF16_MASTER}


# ----------------------------------------------------------------------------- context / volume
class Context:
    """One device, one stream (replaces CLAbstractionLayer's context and queue)."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        check(lib().etcu_context_create(int(device), ctypes.byref(h)))
        self.handle = h
        self.device = device
        self._children = weakref.WeakSet()

    def _adopt(self, obj) -> None:
        self._children.add(obj)

    def close(self) -> None:
        """Destroys the context after every volume / reconstruction created on it."""
        if self.handle:
            for child in [c for c in self._children if not isinstance(c, GPUMappedVolume)]:
                child.close()
            for child in list(self._children):
                child.close()
            lib().etcu_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self) -> None:
        check(lib().etcu_synchronize(self.handle), self.handle)

    def set_stream(self, stream_ptr: Optional[int]) -> None:
        check(lib().etcu_set_stream(self.handle, stream_ptr), self.handle)

    @property
    def stream_handle(self) -> int:
        """cudaStream_t of the library's work on this context (for CUDA events)."""
        return int(lib().etcu_context_stream(self.handle) or 0)

    @property
    def device_bytes(self) -> int:
        return int(lib().etcu_device_bytes(self.handle))

    def set_autotune(self, mode: int = 1) -> None:
        """Launch shapes from the autotuner's cache, timed on the real problem on a miss
        (etcu_context_set_autotune); results do not depend on the choice."""
        check(lib().etcu_context_set_autotune(self.handle, int(mode)), self.handle)

    def tune_report(self) -> str:
        """The autotuner's choices on this context, one line each."""
        n = ctypes.c_size_t()
        check(lib().etcu_context_tune_report(self.handle, None, 0, ctypes.byref(n)), self.handle)
        buf = ctypes.create_string_buffer(n.value)
        check(lib().etcu_context_tune_report(self.handle, buf, n.value, None), self.handle)
        return buf.value.decode()

    def check(self, status: int) -> None:
        check(status, self.handle)


def _dptr(t) -> int:
    """Device address of a CUDA tensor (float32, contiguous).  The tensor's pending
    writes on torch's stream are completed first, so the library's stream sees them."""
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "device images must be CUDA tensors")
    if t.dtype != torch.float32 or not t.is_contiguous():
        raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "device images must be contiguous float32")
    torch.cuda.current_stream(t.device).synchronize()
    return t.data_ptr()


class GPUMappedVolume:
    """Device-resident volume (LR/model/volume/GPUMappedVolume.cpp:9-41)."""

    def __init__(self, ctx: Context, resolution: Sequence[int], bbox_min: Optional[Sequence[float]] = None,
                 bbox_max: Optional[Sequence[float]] = None, voxel_type: int = _abi.VOXEL_FLOAT32,
                 init_value: float = 0.0, subvolume_count: int = 1):
        self.ctx = ctx
        res = [int(r) for r in resolution]
        if bbox_min is None:  # VolumeParameterSet.cpp:40-46: dimension = resolution, origin 0
            bbox_min = [-0.5 * r for r in res]
            bbox_max = [0.5 * r for r in res]
        d = VolumeDesc()
        for i in range(3):
            d.resolution[i] = res[i]
            d.bbox_min[i] = float(bbox_min[i])
            d.bbox_max[i] = float(bbox_max[i])
        d.subvolume_count = int(subvolume_count)
        self.desc = d
        self.resolution = tuple(res)
        self.bbox_min = tuple(float(np.float32(b)) for b in bbox_min)
        self.bbox_max = tuple(float(np.float32(b)) for b in bbox_max)
        self.voxel_type = voxel_type
        h = ctypes.c_void_p()
        ctx.check(lib().etcu_volume_create(ctx.handle, ctypes.byref(d), int(voxel_type), float(init_value),
                                           ctypes.byref(h)))
        self.handle = h
        ctx._adopt(self)

    @property
    def voxel_size(self) -> np.ndarray:
        return ((np.asarray(self.bbox_max, np.float32) - np.asarray(self.bbox_min, np.float32))
                / np.asarray(self.resolution, np.float32)).astype(np.float32)

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().etcu_volume_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, data: np.ndarray) -> None:
        """data: (z, y, x) float32 array, x fastest."""
        X, Y, Z = self.resolution
        a = np.ascontiguousarray(data, np.float32)
        if a.size != X * Y * Z:
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "volume data has the wrong size")
        self.ctx.check(lib().etcu_volume_upload(self.handle, a.ctypes.data))

    def download(self) -> np.ndarray:
        X, Y, Z = self.resolution
        out = np.empty((Z, Y, X), np.float32)
        self.ctx.check(lib().etcu_volume_download(self.handle, out.ctypes.data))
        return out

    def set_mask(self, mask: Optional[np.ndarray]) -> None:
        if mask is None:
            self.ctx.check(lib().etcu_volume_set_mask(self.handle, None))
            return
        m = np.ascontiguousarray(mask, np.uint8)
        self.ctx.check(lib().etcu_volume_set_mask(self.handle, m.ctypes.data))

    def set_intensity_clamp(self, vmin: Optional[float] = None, vmax: Optional[float] = None) -> None:
        self.ctx.check(lib().etcu_volume_set_intensity_clamp(self.handle, int(vmin is not None), float(vmin or 0.0),
                                                              int(vmax is not None), float(vmax or 0.0)))

    def device_ptr(self) -> int:
        return int(lib().etcu_volume_device_ptr(self.handle) or 0)

    def upload_device(self, t) -> None:
        """Copies a CUDA float32 tensor (z, y, x) into the volume on the library's stream."""
        self.ctx.check(lib().etcu_volume_upload_device(self.handle, _dptr(t)))

    def download_device(self, t) -> None:
        """Copies the volume into a CUDA float32 tensor (z, y, x) on the library's stream
        (synchronise the context before reading it on another stream)."""
        self.ctx.check(lib().etcu_volume_download_device(self.handle, _dptr(t)))


# ----------------------------------------------------------------------------- operators
class ForwardProjectionOperator:
    """ForwardProjectionOperator (ForwardProjectionOperator.cpp:11-55): SetOutput + Execute(subVolume).
    The outputs are ACCUMULATED (+=), as in the reference."""

    def __init__(self, volume: GPUMappedVolume, samples: int = 1, blob_parameters: Optional["BlobParameters"] = None,
                 blob_samples: int = 256):
        self.volume = volume
        self.samples = samples
        self.blob_parameters = blob_parameters  # algorithm.basisFunctions = blobs
        self.blob_samples = blob_samples
        self.geometry: Optional[ScannerGeometry] = None
        self.virtual = None
        self.traversal = None

    def setScannerGeometry(self, g: ScannerGeometry) -> None:
        self.geometry = g

    def SetOutput(self, virtual_projection, traversal_length) -> None:
        if (virtual_projection is None) != (traversal_length is None):
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT,
                                 "Virtual projection and traversal length must either be set both or none of them!")
        if virtual_projection is not None and tuple(virtual_projection.shape) != tuple(traversal_length.shape):
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT,
                                 "Virtual projection and traversal length images differ in size!")
        self.virtual, self.traversal = virtual_projection, traversal_length

    def Execute(self, subvolume: int = 0) -> None:
        if self.virtual is None:
            raise EttentionError(_abi.ERR_STATE, "ForwardProjectionKernel cannot be run without setting output "
                                 "images! Be sure to call setOutput() before with non-null parameters.")
        g = self.geometry
        if tuple(self.virtual.shape) != (g.height, g.width):
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "output image does not match the detector resolution")
        if self.blob_parameters is not None:
            forward_project_blobs(self.volume, g, self.blob_parameters, self.virtual, self.traversal, subvolume,
                                  self.blob_samples)
            return
        v = g.to_view()
        self.volume.ctx.check(lib().etcu_forward_project(self.volume.handle, ctypes.byref(v), int(subvolume),
                                                         int(self.samples), _dptr(self.virtual),
                                                         _dptr(self.traversal)))
        self.volume.ctx.synchronize()  # the reference waits after every launch (CLKernel.cpp:177-179)


class BackProjectionOperator:
    """BackProjectionOperator (BackProjectionOperator.cpp:13-98): setInput(residual, traversal,
    blockSize) + execute(subVolume | ALL_SUB_VOLUMES); lambda / blockSize per update."""

    ALL_SUB_VOLUMES = _abi.ALL_SUBVOLUMES

    def __init__(self, volume: GPUMappedVolume, lam: float, samples: int = 1,
                 sampling: int = _abi.SAMPLING_Q8, blob_parameters: Optional["BlobParameters"] = None):
        self.volume = volume
        self.blob_parameters = blob_parameters  # algorithm.basisFunctions = blobs
        self.lam = float(lam)
        self.samples = int(samples)
        self.sampling = sampling
        self.geometry: Optional[ScannerGeometry] = None
        self.residual = None
        self.traversal = None
        self.block_size = 1

    def setScannerGeometry(self, g: ScannerGeometry) -> None:
        self.geometry = g

    def setInput(self, residual, traversal_length, block_size: int = 1) -> None:
        if (residual is None) != (traversal_length is None):
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT,
                                 "Either residual and traversalLength images must be provided both or none of them!")
        if residual is not None and tuple(residual.shape) != tuple(traversal_length.shape):
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "Residual and traversalLength differ in size!")
        self.residual, self.traversal, self.block_size = residual, traversal_length, int(block_size)

    def execute(self, subvolume: int = _abi.ALL_SUBVOLUMES) -> None:
        if self.residual is None:
            raise EttentionError(_abi.ERR_STATE, "Residual and traversalLength images must both be provided via "
                                 "SetInput() before kernel launch!")
        if self.blob_parameters is not None:
            back_project_blobs(self.volume, self.geometry, self.blob_parameters, self.residual, self.traversal,
                               self.lam, self.block_size, subvolume)
            return
        v = self.geometry.to_view()
        self.volume.ctx.check(lib().etcu_back_project(self.volume.handle, ctypes.byref(v), int(subvolume),
                                                      self.samples, self.lam, self.block_size,
                                                      _dptr(self.residual), _dptr(self.traversal),
                                                      int(self.sampling)))
        self.volume.ctx.synchronize()


def compare(ctx: Context, real, virtual, residual) -> None:
    """CompareKernel (ocl_src/Compare.cl): residual = real - virtual."""
    ctx.check(lib().etcu_compare(ctx.handle, _dptr(real), _dptr(virtual), _dptr(residual), real.numel()))
    ctx.synchronize()


def long_object_compensation(ctx: Context, virtual, traversal, constant_length: float) -> None:
    """VirtualProjectionKernel (ocl_src/VirtualProjection.cl), in place."""
    ctx.check(lib().etcu_long_object_compensation(ctx.handle, _dptr(virtual), _dptr(traversal),
                                                  float(constant_length), virtual.numel()))
    ctx.synchronize()


def compute_ray_length(volume: GPUMappedVolume, g: ScannerGeometry, out) -> None:
    """ComputeRayLengthKernel (ocl_src/ComputeRayLength.cl)."""
    v = g.to_view()
    volume.ctx.check(lib().etcu_compute_ray_length(volume.handle, ctypes.byref(v), _dptr(out)))
    volume.ctx.synchronize()


# ----------------------------------------------------------------------------- blob basis functions
@dataclass
class BlobParameters:
    """model/blobs/BlobParameters.cpp: Kaiser-Bessel blob of support radius a (voxels),
    degree m and density fall-off alpha; createDefault() = (2.0, 2, 3.6)."""
    support_radius: float = 2.0
    degree: int = 2
    density_falloff: float = 3.6

    @classmethod
    def createDefault(cls) -> "BlobParameters":
        return cls()

    @classmethod
    def createWithParameters(cls, support_radius: float, degree: int, density_falloff: float) -> "BlobParameters":
        return cls(float(support_radius), int(degree), float(density_falloff))

    @classmethod
    def from_config(cls, cfg: Dict[str, str]) -> "BlobParameters":
        """BlobParameterSet.cpp:7-29: blobs.supportRadius, blobs.degree, blobs.densityFalloff."""
        return cls(float(cfg.get("blobs.supportRadius", 2.0)), int(cfg.get("blobs.degree", 2)),
                   float(cfg.get("blobs.densityFalloff", 3.6)))

    def getSupportRadius(self) -> float:
        return self.support_radius

    def getDegree(self) -> int:
        return self.degree

    def getDensityFallOff(self) -> float:
        return self.density_falloff

    def to_c(self) -> "_abi.BlobParams":
        return _abi.BlobParams(float(self.support_radius), int(self.degree), float(self.density_falloff))


class BlobRayIntegrationSampler:
    """algorithm/blobs/BlobRayIntegrationSampler.cpp: the blob's line integral at
    ``count`` distances from 0 to a (etcu_blob_ray_integration_samples)."""

    def __init__(self, params: BlobParameters, count: int):
        self.params = params
        self.samples = np.zeros(int(count), np.float32)
        c = params.to_c()
        check(lib().etcu_blob_ray_integration_samples(ctypes.byref(c), int(count), self.samples.ctypes.data))

    def getSamples(self) -> np.ndarray:
        return self.samples

    def getSampleCount(self) -> int:
        return int(self.samples.shape[0])

    def getParameters(self) -> BlobParameters:
        return self.params


class BlobVoxelizationKernelValues:
    """algorithm/blobs/BlobVoxelizationKernelValues.cpp: the blob integrated over every
    voxel of its (2 ceil(a) + 1)^3 neighbourhood, [dz][dy][dx]."""

    def __init__(self, params: BlobParameters):
        c = params.to_c()
        n = ctypes.c_uint32()
        check(lib().etcu_blob_voxelization_kernel(ctypes.byref(c), None, 0, ctypes.byref(n)))
        k = int(n.value)
        self.values = np.zeros((k, k, k), np.float32)
        check(lib().etcu_blob_voxelization_kernel(ctypes.byref(c), self.values.ctypes.data, k ** 3, ctypes.byref(n)))

    def getValuesPerDimension(self) -> int:
        return int(self.values.shape[0])

    def getKernelValues(self) -> np.ndarray:
        return self.values


def forward_project_blobs(volume: "GPUMappedVolume", g: ScannerGeometry, params: BlobParameters, projection,
                          traversal, subvolume: int = _abi.ALL_SUBVOLUMES, sample_count: int = 256) -> None:
    """PerspectiveBeamsForwardProjectionWithBlobsKernel: ADDS the blob line integrals of the
    coefficients and their weights into two device images."""
    v, c = g.to_view(), params.to_c()
    volume.ctx.check(lib().etcu_forward_project_blobs(volume.handle, ctypes.byref(v), int(subvolume), ctypes.byref(c),
                                                      int(sample_count), _dptr(projection), _dptr(traversal)))


def back_project_blobs(volume: "GPUMappedVolume", g: ScannerGeometry, params: BlobParameters, residual, traversal,
                       lam: float, block_size: int = 1, subvolume: int = _abi.ALL_SUBVOLUMES) -> None:
    """PerspectiveBeamsBackProjectionWithBlobsKernel: every blob takes lambda / block size times
    the weighted mean of residual / ray length over the pixels whose rays pass within its radius."""
    v, c = g.to_view(), params.to_c()
    volume.ctx.check(lib().etcu_back_project_blobs(volume.handle, ctypes.byref(v), int(subvolume), ctypes.byref(c),
                                                   float(lam), int(block_size), _dptr(residual), _dptr(traversal)))


class BlobVoxelizerOperator:
    """algorithm/blobs/BlobVoxelizerOperator.cpp: the blob coefficients convolved with the
    voxelisation kernel into a second volume of the same resolution and box."""

    def __init__(self, volume: "GPUMappedVolume", params: BlobParameters):
        self.volume = volume
        self.params = params
        self.voxels = GPUMappedVolume(volume.ctx, volume.resolution, volume.bbox_min, volume.bbox_max)

    def voxelize(self) -> None:
        c = self.params.to_c()
        self.volume.ctx.check(lib().etcu_blob_voxelize(self.volume.handle, self.voxels.handle, ctypes.byref(c)))

    def getVoxelVolume(self) -> "GPUMappedVolume":
        return self.voxels


class _BlobBlockIterations:
    """BlockIterativeReconstructionOperator.cpp:84-160 with blob basis functions
    (algorithm.basisFunctions = blobs, etcu_blob_recon_*): per block, the blob forward
    projection of every view into cleared images, residual = measured - virtual, then the
    blob back projection of every view with lambda / block size.  With
    output.options.enableVoxelization the coefficients are voxelised after every
    runNiterations (:66-79) and the voxel volume is the result."""

    def __init__(self, volume: "GPUMappedVolume", geometries: Sequence[ScannerGeometry], projections,
                 params: "AlgebraicParameterSet"):
        self.volume = volume
        self.params = params
        self._views = (View * len(geometries))(*[g.to_view() for g in geometries])
        rp = params.recon_params(False)
        self._skip = (ctypes.c_uint32 * max(1, len(params.skip)))(*[int(s) for s in params.skip])
        if len(params.skip):
            rp.skip = ctypes.cast(self._skip, ctypes.POINTER(ctypes.c_uint32))
            rp.skip_count = len(params.skip)
        blob = params.blob.to_c()
        h = ctypes.c_void_p()
        if isinstance(projections, np.ndarray):
            host = np.ascontiguousarray(projections, np.float32)
            if host.shape[0] != len(geometries):
                raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "one projection per geometry")
            volume.ctx.check(lib().etcu_blob_recon_create(volume.handle, self._views, len(geometries), host.ctypes.data,
                                                          ctypes.byref(rp), ctypes.byref(blob), ctypes.byref(h)))
        else:
            self._dev = projections
            volume.ctx.check(lib().etcu_blob_recon_create_device(volume.handle, self._views, len(geometries),
                                                                 _dptr(projections), ctypes.byref(rp),
                                                                 ctypes.byref(blob), ctypes.byref(h)))
        self.handle = h
        self.voxelizer = BlobVoxelizerOperator(volume, params.blob) if params.enable_voxelization else None

    @property
    def order(self) -> List[int]:
        n = len(self._views)
        out = np.zeros(n, np.uint32)
        cnt = ctypes.c_uint32()
        self.volume.ctx.check(lib().etcu_blob_recon_view_order(self.handle, out.ctypes.data, n, ctypes.byref(cnt)))
        return [int(i) for i in out[: cnt.value]]

    @property
    def residual_sq(self) -> float:
        r = ctypes.c_double()
        self.volume.ctx.check(lib().etcu_blob_recon_last_residual_sq(self.handle, ctypes.byref(r)))
        return float(r.value)

    @property
    def launches(self) -> int:
        return int(lib().etcu_blob_recon_launches_per_iteration(self.handle))

    def profile_iteration(self):
        """One iteration with CUDA events around every launch:
        {kind: (total ms, launches)} for 'forward', 'residual', 'back'."""
        ms = np.zeros(3, np.float32)
        cnt = np.zeros(3, np.uint32)
        self.volume.ctx.check(lib().etcu_blob_recon_profile_iteration(self.handle, ms.ctypes.data, cnt.ctypes.data))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(("forward", "residual", "back"))}

    def run(self, n: int) -> None:
        self.volume.ctx.check(lib().etcu_blob_recon_run(self.handle, int(n)))
        if self.voxelizer is not None:
            self.voxelizer.voxelize()

    def result(self) -> np.ndarray:
        return (self.voxelizer.getVoxelVolume() if self.voxelizer is not None else self.volume).download()

    def close(self) -> None:
        if self.voxelizer is not None:
            self.voxelizer.voxels.close()
            self.voxelizer = None
        if getattr(self, "handle", None):
            lib().etcu_blob_recon_destroy(self.handle)
            self.handle = None


# ----------------------------------------------------------------------------- parameters
@dataclass
class AlgebraicParameterSet:
    """The hot-path keys of AlgorithmParameterSet, OptimizationParameterSet,
    Forward/BackProjectionParameterSet, HardwareParameterSet, VolumeParameterSet,
    InputParameterSet and PriorKnowledgeParameterSet (LR/setup/parameterset)."""
    algorithm: str = "sart"
    block_size: int = 1
    iterations: int = 1
    lam: float = 1.0
    use_long_object_compensation: bool = False
    fp_samples: int = 1
    bp_samples: int = 1
    voxel_type: int = _abi.VOXEL_FLOAT32
    order: int = _abi.ORDER_RANDOM
    subvolume_count: int = 1
    dimension: Optional[Sequence[float]] = None
    resolution: Optional[Sequence[int]] = None
    origin: Sequence[float] = (0.0, 0.0, 0.0)
    init_value: float = 0.0
    skip: Sequence[int] = ()
    xaxis_tilt: float = 0.0
    vmin: Optional[float] = None
    vmax: Optional[float] = None
    sampling: int = _abi.SAMPLING_Q8
    basis_functions: str = "voxels"
    blob: BlobParameters = field(default_factory=BlobParameters)
    enable_voxelization: bool = False
    projection_storage: int = _abi.PROJ_F32  # device storage of the tilt series (FP32, FP16 or BF16)

    @classmethod
    def from_config(cls, cfg: Dict[str, str]) -> "AlgebraicParameterSet":
        def vec(s):
            return [float(x) for x in str(s).replace(",", " ").split()]

        p = cls()
        if "algorithm" not in cfg:
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "missing parameter algorithm")
        p.algorithm = cfg["algorithm"]
        # AlgorithmParameterSet.cpp:10-23
        p.block_size = _abi.BLOCK_ALL
        if p.algorithm == "sart":
            p.block_size = 1
        elif p.algorithm == "sirt":
            p.block_size = _abi.BLOCK_ALL
        elif "algorithm.blockSize" in cfg:
            p.block_size = int(cfg["algorithm.blockSize"])
        p.iterations = int(cfg["algorithm.numberOfIterations"])
        p.lam = float(cfg["algorithm.lambda"])
        p.use_long_object_compensation = str(cfg.get("algorithm.useLongObjectCompensation", "false")).lower() in (
            "true", "1", "yes")
        basis = cfg.get("algorithm.basisFunctions", "voxels")  # AlgorithmParameterSet.cpp:34-45
        if basis not in ("voxels", "blobs"):
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT,
                                 f'Illegal value for parameter "algorithm.basisFunctions": {basis}!')
        p.basis_functions = basis
        p.blob = BlobParameters.from_config(cfg)
        p.enable_voxelization = str(cfg.get("output.options.enableVoxelization", "false")).lower() in (
            "true", "1", "yes")
        p.fp_samples = int(cfg.get("forwardProjection.samples", 1))
        p.bp_samples = int(cfg.get("backProjection.samples", 1))
        vt = cfg.get("optimization.internalVoxelRepresentationType", "float")
        if vt not in VOXEL_TYPES:
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT,
                                 "UChar is not supported as a valid internal voxel storage data type.")
        p.voxel_type = VOXEL_TYPES[vt]
        order = cfg.get("optimization.projectionIteration", "random")
        if order not in ORDERS:
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "Illegal ProjectionSetType!")
        p.order = ORDERS[order]
        p.subvolume_count = int(cfg.get("hardware.subVolumeCount", 1))
        if "volume.dimension" in cfg:
            p.dimension = vec(cfg["volume.dimension"])
            p.resolution = [int(x) for x in p.dimension]
        if "volume.resolution" in cfg:
            p.resolution = [int(x) for x in vec(cfg["volume.resolution"])]
        if "volume.origin" in cfg:
            p.origin = vec(cfg["volume.origin"])
        p.init_value = float(cfg.get("volume.initValue", 0.0))
        if "input.skipProjections" in cfg:
            p.skip = [int(x) for x in vec(cfg["input.skipProjections"])]
        p.xaxis_tilt = float(cfg.get("input.xAxisTilt", 0.0))
        if "priorknowledge.volumeMinimumIntensity" in cfg:
            p.vmin = float(cfg["priorknowledge.volumeMinimumIntensity"])
        if "priorknowledge.volumeMaximumIntensity" in cfg:
            p.vmax = float(cfg["priorknowledge.volumeMaximumIntensity"])
        if p.block_size == 0:
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "Illegal ProjectionBlockSize!")
        return p

    def bbox(self):
        dim = np.asarray(self.dimension if self.dimension is not None else self.resolution, np.float64)
        o = np.asarray(self.origin, np.float64)
        return list(o - 0.5 * dim), list(o + 0.5 * dim)

    def recon_params(self, use_graph: bool = True) -> ReconParams:
        rp = ReconParams()
        rp.lam = float(self.lam)
        rp.block_size = int(self.block_size)
        rp.fp_samples = int(self.fp_samples)
        rp.bp_samples = int(self.bp_samples)
        rp.use_long_object_compensation = int(bool(self.use_long_object_compensation))
        rp.order = int(self.order)
        rp.sampling = int(self.sampling)
        rp.use_graph = int(bool(use_graph))
        rp.projection_storage = int(self.projection_storage)
        return rp


class BlockIterativeReconstructionOperator:
    """BlockIterativeReconstructionOperator (BlockIterativeReconstructionOperator.cpp:26-185):
    SART (blockSize 1), SIRT (one block of every view) and general block sizes.

    ``projections`` is an (N, H, W) float32 NumPy array (uploaded once) or a CUDA
    tensor already in device memory."""

    def __init__(self, volume: GPUMappedVolume, geometries: Sequence[ScannerGeometry], projections,
                 params: AlgebraicParameterSet, use_graph: bool = True):
        self.volume = volume
        self.params = params
        self.handle = None
        self._blobs = None
        if params.basis_functions == "blobs":
            self._blobs = _BlobBlockIterations(volume, geometries, projections, params)
            volume.ctx._adopt(self)
            return
        self._views = (View * len(geometries))(*[g.to_view() for g in geometries])
        rp = params.recon_params(use_graph)
        self._skip = (ctypes.c_uint32 * max(1, len(params.skip)))(*[int(s) for s in params.skip])
        if len(params.skip):
            rp.skip = ctypes.cast(self._skip, ctypes.POINTER(ctypes.c_uint32))
            rp.skip_count = len(params.skip)
        self._rp = rp
        if params.vmin is not None or params.vmax is not None:
            volume.set_intensity_clamp(params.vmin, params.vmax)
        h = ctypes.c_void_p()
        if isinstance(projections, np.ndarray):
            self._host = np.ascontiguousarray(projections, np.float32)
            volume.ctx.check(lib().etcu_recon_create(volume.handle, self._views, len(geometries),
                                                     self._host.ctypes.data, ctypes.byref(rp), ctypes.byref(h)))
        else:
            self._dev = projections
            volume.ctx.check(lib().etcu_recon_create_device(volume.handle, self._views, len(geometries),
                                                            _dptr(projections), ctypes.byref(rp), ctypes.byref(h)))
        self.handle = h
        volume.ctx._adopt(self)

    def close(self) -> None:
        if getattr(self, "_blobs", None) is not None:
            self._blobs.close()
            self._blobs = None
        if getattr(self, "handle", None):
            lib().etcu_recon_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _voxels_only(self, what: str) -> None:
        if self._blobs is not None:
            raise EttentionError(_abi.ERR_UNSUPPORTED, f"{what} is reported for voxel basis functions only")

    def runNiterations(self, n: int = 1) -> None:
        if self._blobs is not None:
            self._blobs.run(n)
            return
        self.volume.ctx.check(lib().etcu_recon_run(self.handle, int(n)))

    def run(self) -> None:
        self.runNiterations(self.params.iterations)

    def runSingleIteration(self) -> None:
        self.runNiterations(1)

    def getReconstructedVolume(self) -> np.ndarray:
        if self._blobs is not None:
            return self._blobs.result()
        return self.volume.download()

    def last_residual_sq(self) -> float:
        if self._blobs is not None:
            return self._blobs.residual_sq
        r = ctypes.c_double()
        self.volume.ctx.check(lib().etcu_recon_last_residual_sq(self.handle, ctypes.byref(r)))
        return float(r.value)

    def data_residual_sq(self) -> float:
        self._voxels_only("the data residual")
        r = ctypes.c_double()
        self.volume.ctx.check(lib().etcu_recon_data_residual_sq(self.handle, ctypes.byref(r)))
        return float(r.value)

    def view_order(self) -> List[int]:
        if self._blobs is not None:
            return list(self._blobs.order)
        n = len(self._views)
        out = np.zeros(n, np.uint32)
        cnt = ctypes.c_uint32()
        self.volume.ctx.check(lib().etcu_recon_view_order(self.handle, out.ctypes.data, n, ctypes.byref(cnt)))
        return [int(i) for i in out[: cnt.value]]

    @property
    def launches_per_iteration(self) -> int:
        if self._blobs is not None:
            return self._blobs.launches
        return int(lib().etcu_recon_launches_per_iteration(self.handle))

    def profile_steps(self):
        """Runs one iteration as run() does, each step timed: [(kind, ms, launches)],
        kind 'forward', 'back' or 'fused' (etcu_recon_profile_steps)."""
        self._voxels_only("the step profile")
        n = ctypes.c_uint32()
        self.volume.ctx.check(lib().etcu_recon_profile_steps(self.handle, None, None, None, 0, ctypes.byref(n)))
        ms = np.zeros(n.value, np.float32)
        kinds = np.zeros(n.value, np.uint32)
        launches = np.zeros(n.value, np.uint32)
        self.volume.ctx.check(lib().etcu_recon_profile_steps(self.handle, ms.ctypes.data, kinds.ctypes.data,
                                                             launches.ctypes.data, n.value, ctypes.byref(n)))
        names = ("forward", "back", "fused")
        return [(names[int(k)], float(t), int(l)) for k, t, l in zip(kinds, ms, launches)]

    def profile_iteration(self):
        """Runs one iteration with per-launch CUDA events: (fp_ms, bp_ms, fp_launches, bp_launches)."""
        if self._blobs is not None:
            k = self._blobs.profile_iteration()
            return k["forward"][0], k["back"][0], k["forward"][1], k["back"][1]
        f, b = ctypes.c_float(), ctypes.c_float()
        nf, nb = ctypes.c_uint32(), ctypes.c_uint32()
        self.volume.ctx.check(lib().etcu_recon_profile_iteration(self.handle, ctypes.byref(f), ctypes.byref(b),
                                                                 ctypes.byref(nf), ctypes.byref(nb)))
        return float(f.value), float(b.value), int(nf.value), int(nb.value)


def wbp_filter(ctx: "Context", image, out, filter_width: int = 128) -> None:
    """The WBP plugin's RamLak filtering of one device image (etcu_wbp_filter)."""
    H, W = int(image.shape[-2]), int(image.shape[-1])
    ctx.check(lib().etcu_wbp_filter(ctx.handle, _dptr(image), _dptr(out), W, H, int(filter_width)))


class WBPOperator:
    """WBP plugin (plugins/WBPPlugin/src/reconstruction/WBP.cpp): every projection
    RamLak-filtered, back projected with its ray lengths and lambda / N; ``run`` adds
    the weighted back projection of all views to the volume."""

    def __init__(self, volume: GPUMappedVolume, geometries: Sequence[ScannerGeometry], projections: np.ndarray,
                 params: AlgebraicParameterSet):
        self.volume = volume
        self.params = params
        self._views = (View * len(geometries))(*[g.to_view() for g in geometries])
        self._host = np.ascontiguousarray(projections, np.float32)
        if self._host.shape[0] != len(geometries):
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "one projection per geometry")

    def run(self) -> None:
        p = self.params
        self.volume.ctx.check(lib().etcu_wbp(self.volume.handle, self._views, len(self._views), self._host.ctypes.data,
                                             float(p.lam), int(p.bp_samples), int(p.sampling)))

    def getReconstructedVolume(self) -> np.ndarray:
        return self.volume.download()


class BatchReconstructionOperator:
    """Many independent tilt series of uneven sizes reconstructed together with SART:
    each iteration of all series is one persistent launch when every series can run the
    fused step, else every step runs one forward-projection and one back-projection
    launch over all series, each iteration one CUDA graph (etcu_batch_*).  No counterpart in the
    reference, which reconstructs one series per run.

    ``series`` is a list of (GPUMappedVolume, [ScannerGeometry], projections (N, H, W)
    float32 array); the volumes share one Context."""

    def __init__(self, series, params: AlgebraicParameterSet, use_graph: bool = True):
        if not series:
            raise EttentionError(_abi.ERR_INVALID_ARGUMENT, "no series")
        self.volumes = [v for v, _, _ in series]
        self.params = params
        ctx = self.volumes[0].ctx
        self._views = [(View * len(g))(*[x.to_view() for x in g]) for _, g, _ in series]
        self._projs = [np.ascontiguousarray(p, np.float32) for _, _, p in series]
        arr = (_abi.BatchSeries * len(series))()
        for i, (vol, geoms, _) in enumerate(series):
            arr[i].volume = vol.handle
            arr[i].views = ctypes.cast(self._views[i], ctypes.POINTER(View))
            arr[i].n_views = len(geoms)
            arr[i].host_projections = self._projs[i].ctypes.data
        rp = params.recon_params(use_graph)
        self._skip = (ctypes.c_uint32 * max(1, len(params.skip)))(*[int(s) for s in params.skip])
        if len(params.skip):
            rp.skip = ctypes.cast(self._skip, ctypes.POINTER(ctypes.c_uint32))
            rp.skip_count = len(params.skip)
        h = ctypes.c_void_p()
        ctx.check(lib().etcu_batch_create(ctx.handle, arr, len(series), ctypes.byref(rp), ctypes.byref(h)))
        self.handle = h
        self.ctx = ctx
        ctx._adopt(self)

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().etcu_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def runNiterations(self, n: int = 1) -> None:
        self.ctx.check(lib().etcu_batch_run(self.handle, int(n)))

    def run(self) -> None:
        self.runNiterations(self.params.iterations)

    def getReconstructedVolumes(self) -> List[np.ndarray]:
        return [v.download() for v in self.volumes]

    def last_residual_sq(self) -> List[float]:
        out = np.zeros(len(self.volumes), np.float64)
        self.ctx.check(lib().etcu_batch_last_residual_sq(self.handle, out.ctypes.data))
        return [float(x) for x in out]

    @property
    def launches_per_iteration(self) -> int:
        return int(lib().etcu_batch_launches_per_iteration(self.handle))
