"""ctypes binding of include/ettention_b200.h (libettention_b200.so).

The library is the only compute path: there is no CPU fallback.  Importing
this module does not need a GPU; calls that touch the device return
ETCU_ERR_NO_DEVICE / raise ``EttentionError`` when none is present.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libettention_b200.so")

OK = 0
ERR_INVALID_ARGUMENT, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_STATE, ERR_UNSUPPORTED, ERR_NO_DEVICE = 1, 2, 3, 4, 5, 6
VOXEL_FLOAT32, VOXEL_HALF16, VOXEL_F16_MASTER, VOXEL_BF16_MASTER = 0, 1, 2, 3
SAMPLING_Q8, SAMPLING_EXACT, SAMPLING_HW_TEXTURE = 0, 1, 2
ORDER_IDENTITY, ORDER_RANDOM, ORDER_MAXANGLE, ORDER_BUCKETS = 0, 1, 2, 3
ALL_SUBVOLUMES = 0xFFFFFFFF
NOALLOC_MAX_PIXELS = 1024 * 1024
NOALLOC_SCRATCH_TEXELS = NOALLOC_MAX_PIXELS + 8208
BLOCK_ALL = 0xFFFFFFFF


class EttentionError(RuntimeError):
    """Raised for every non-OK status (the reference raises ettention::Exception / GPUException)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class View(ctypes.Structure):
    _fields_ = [("source", ctypes.c_float * 3), ("detector", ctypes.c_float * 3),
                ("hpitch", ctypes.c_float * 3), ("vpitch", ctypes.c_float * 3),
                ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("perspective", ctypes.c_int32)]


class VolumeDesc(ctypes.Structure):
    _fields_ = [("resolution", ctypes.c_uint32 * 3), ("bbox_min", ctypes.c_float * 3),
                ("bbox_max", ctypes.c_float * 3), ("subvolume_count", ctypes.c_uint32)]


class ReconParams(ctypes.Structure):
    _fields_ = [("lam", ctypes.c_float), ("block_size", ctypes.c_uint32), ("fp_samples", ctypes.c_uint32),
                ("bp_samples", ctypes.c_uint32), ("use_long_object_compensation", ctypes.c_int32),
                ("order", ctypes.c_int), ("sampling", ctypes.c_int), ("skip", ctypes.POINTER(ctypes.c_uint32)),
                ("skip_count", ctypes.c_uint32), ("use_graph", ctypes.c_int32), ("projection_storage", ctypes.c_int)]


PROJ_F32, PROJ_F16, PROJ_BF16 = 0, 1, 2


class MrcInfo(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_uint32), ("ny", ctypes.c_uint32), ("nz", ctypes.c_uint32), ("mode", ctypes.c_int32),
                ("dmin", ctypes.c_float), ("dmax", ctypes.c_float), ("dmean", ctypes.c_float),
                ("extended_bytes", ctypes.c_uint32)]


AXES_XYZ, AXES_XZY = 0, 1


class ImageInfo(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("pages", ctypes.c_uint32),
                ("bits_per_sample", ctypes.c_uint32), ("sample_format", ctypes.c_uint32),
                ("compression", ctypes.c_uint32)]


class ImageStackInfo(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint32), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("base", View)]


class BlobParams(ctypes.Structure):
    _fields_ = [("support_radius", ctypes.c_float), ("degree", ctypes.c_uint32), ("density_falloff", ctypes.c_float)]


class BatchSeries(ctypes.Structure):
    _fields_ = [("volume", ctypes.c_void_p), ("views", ctypes.POINTER(View)), ("n_views", ctypes.c_uint32),
                ("host_projections", ctypes.c_void_p)]


_lib = None

# name -> (restype, argtypes)
_P = ctypes.c_void_p
_U = ctypes.c_uint32
_F = ctypes.c_float
_I = ctypes.c_int
_S = ctypes.c_int  # etcu_status
_SIG = {
    "etcu_abi_version": (_I, []),
    "etcu_context_create": (_S, [_I, ctypes.POINTER(_P)]),
    "etcu_context_destroy": (_S, [_P]),
    "etcu_last_error": (ctypes.c_char_p, [_P]),
    "etcu_synchronize": (_S, [_P]),
    "etcu_set_stream": (_S, [_P, _P]),
    "etcu_device_bytes": (ctypes.c_size_t, [_P]),
    "etcu_context_set_autotune": (_S, [_P, _I]),
    "etcu_context_tune_report": (_S, [_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "etcu_context_stream": (_P, [_P]),
    "etcu_view_rotate": (_S, [ctypes.POINTER(View), _F, _F, ctypes.POINTER(View)]),
    "etcu_view_projection_matrix": (_S, [ctypes.POINTER(View), _P]),
    "etcu_view_sample_pattern": (_S, [ctypes.POINTER(View), _P, _U, _P]),
    "etcu_view_traversal_length": (_S, [ctypes.POINTER(View), _P, _P, ctypes.POINTER(_F)]),
    "etcu_volume_create": (_S, [_P, ctypes.POINTER(VolumeDesc), _I, _F, ctypes.POINTER(_P)]),
    "etcu_volume_destroy": (_S, [_P]),
    "etcu_volume_upload": (_S, [_P, _P]),
    "etcu_volume_download": (_S, [_P, _P]),
    "etcu_volume_upload_device": (_S, [_P, _P]),
    "etcu_volume_download_device": (_S, [_P, _P]),
    "etcu_volume_set_mask": (_S, [_P, _P]),
    "etcu_volume_device_ptr": (_P, [_P]),
    "etcu_volume_set_intensity_clamp": (_S, [_P, _I, _F, _I, _F]),
    "etcu_forward_project": (_S, [_P, ctypes.POINTER(View), _U, _U, _P, _P]),
    "etcu_back_project": (_S, [_P, ctypes.POINTER(View), _U, _U, _F, _U, _P, _P, _I]),
    "etcu_compare": (_S, [_P, _P, _P, _P, ctypes.c_size_t]),
    "etcu_long_object_compensation": (_S, [_P, _P, _P, _F, ctypes.c_size_t]),
    "etcu_compute_ray_length": (_S, [_P, ctypes.POINTER(View), _P]),
    "etcu_recon_create": (_S, [_P, ctypes.POINTER(View), _U, _P, ctypes.POINTER(ReconParams), ctypes.POINTER(_P)]),
    "etcu_recon_create_device": (_S, [_P, ctypes.POINTER(View), _U, _P, ctypes.POINTER(ReconParams),
                                      ctypes.POINTER(_P)]),
    "etcu_recon_destroy": (_S, [_P]),
    "etcu_recon_run": (_S, [_P, _U]),
    "etcu_recon_last_residual_sq": (_S, [_P, ctypes.POINTER(ctypes.c_double)]),
    "etcu_recon_data_residual_sq": (_S, [_P, ctypes.POINTER(ctypes.c_double)]),
    "etcu_recon_view_order": (_S, [_P, _P, _U, ctypes.POINTER(_U)]),
    "etcu_recon_launches_per_iteration": (_U, [_P]),
    "etcu_recon_block_count": (_S, [_P, ctypes.POINTER(_U), ctypes.POINTER(_U)]),
    "etcu_recon_set_complete_bbox": (_S, [_P, _P, _P]),
    "etcu_recon_slab_forward": (_S, [_P, _U, _P]),
    "etcu_recon_slab_backward": (_S, [_P, _U, _P]),
    "etcu_recon_slab_step": (_S, [_P, _U, _P, _P]),
    "etcu_recon_profile_iteration": (_S, [_P, ctypes.POINTER(_F), ctypes.POINTER(_F), ctypes.POINTER(_U),
                                         ctypes.POINTER(_U)]),
    "etcu_recon_profile_steps": (_S, [_P, _P, _P, _P, _U, ctypes.POINTER(_U)]),
    "etcu_reconstruct": (_S, [_P, ctypes.POINTER(VolumeDesc), _I, ctypes.POINTER(View), _U, _P,
                              ctypes.POINTER(ReconParams), _U, _P]),
    "etcu_projection_order": (_S, [_I, _U, _P, _U, _P, ctypes.POINTER(_U)]),
    "etcu_mrc_read_info": (_S, [ctypes.c_char_p, ctypes.POINTER(MrcInfo)]),
    "etcu_mrc_read_stack": (_S, [ctypes.c_char_p, _I, _P, ctypes.c_size_t]),
    "etcu_read_tilt_angles": (_S, [ctypes.c_char_p, _P, _U, ctypes.POINTER(_U)]),
    "etcu_mrc_write_volume": (_S, [ctypes.c_char_p, _P, _P, _I]),
    "etcu_mrc_write_volume_typed": (_S, [ctypes.c_char_p, _P, _P, _I, _I, _I]),
    "etcu_tiff_read_info": (_S, [ctypes.c_char_p, _U, ctypes.POINTER(ImageInfo)]),
    "etcu_tiff_read": (_S, [ctypes.c_char_p, _U, _P, ctypes.c_size_t]),
    "etcu_tiff_write": (_S, [ctypes.c_char_p, _P, _U, _U]),
    "etcu_image_stack_open": (_S, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "etcu_image_stack_destroy": (None, [_P]),
    "etcu_image_stack_info_get": (_S, [_P, ctypes.POINTER(ImageStackInfo)]),
    "etcu_image_stack_tilt_angles": (_S, [_P, _P, _U]),
    "etcu_image_stack_load": (_S, [_P, _U, _U, _P, ctypes.c_size_t]),
    "etcu_image_stack_write_metadata": (_S, [ctypes.c_char_p, _P, ctypes.POINTER(ctypes.c_char_p), _U,
                                             ctypes.POINTER(View), _P]),
    "etcu_xml_config_read": (_S, [ctypes.c_char_p, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "etcu_wbp": (_S, [_P, ctypes.POINTER(View), _U, _P, _F, _U, _I]),
    "etcu_wbp_filter": (_S, [_P, _P, _P, _U, _U, _U]),
    "etcu_blob_ray_integration_samples": (_S, [ctypes.POINTER(BlobParams), _U, _P]),
    "etcu_blob_voxelization_kernel": (_S, [ctypes.POINTER(BlobParams), _P, _U, ctypes.POINTER(_U)]),
    "etcu_forward_project_blobs": (_S, [_P, ctypes.POINTER(View), _U, ctypes.POINTER(BlobParams), _U, _P, _P]),
    "etcu_back_project_blobs": (_S, [_P, ctypes.POINTER(View), _U, ctypes.POINTER(BlobParams), _F, _U, _P, _P]),
    "etcu_blob_voxelize": (_S, [_P, _P, ctypes.POINTER(BlobParams)]),
    "etcu_blob_recon_create": (_S, [_P, ctypes.POINTER(View), _U, _P, ctypes.POINTER(ReconParams),
                                    ctypes.POINTER(BlobParams), ctypes.POINTER(_P)]),
    "etcu_blob_recon_create_device": (_S, [_P, ctypes.POINTER(View), _U, _P, ctypes.POINTER(ReconParams),
                                           ctypes.POINTER(BlobParams), ctypes.POINTER(_P)]),
    "etcu_blob_recon_run": (_S, [_P, _U]),
    "etcu_blob_recon_last_residual_sq": (_S, [_P, ctypes.POINTER(ctypes.c_double)]),
    "etcu_blob_recon_view_order": (_S, [_P, _P, _U, ctypes.POINTER(_U)]),
    "etcu_blob_recon_launches_per_iteration": (_U, [_P]),
    "etcu_blob_recon_profile_iteration": (_S, [_P, _P, _P]),
    "etcu_blob_recon_destroy": (_S, [_P]),
    "etcu_batch_create": (_S, [_P, ctypes.POINTER(BatchSeries), _U, ctypes.POINTER(ReconParams), ctypes.POINTER(_P)]),
    "etcu_batch_destroy": (_S, [_P]),
    "etcu_batch_run": (_S, [_P, _U]),
    "etcu_batch_last_residual_sq": (_S, [_P, _P]),
    "etcu_batch_launches_per_iteration": (_U, [_P]),
    "etcu_sart_view_update_noalloc": (_S, [ctypes.POINTER(VolumeDesc), _P, _P, ctypes.POINTER(View), _U, _U, _F, _P,
                                           ctypes.POINTER(ctypes.c_double)]),
    "etcu_warmstart_param_count": (_U, []),
    "etcu_warmstart_layer_info": (_S, [_U, _P]),
    "etcu_warmstart_create": (_S, [_P, _P, _U, ctypes.POINTER(_P)]),
    "etcu_warmstart_destroy": (_S, [_P]),
    "etcu_warmstart_set_params": (_S, [_P, _P, _F]),
    "etcu_warmstart_get_params": (_S, [_P, _P, ctypes.POINTER(_F)]),
    "etcu_warmstart_infer": (_S, [_P, _P, _P, _U]),
    "etcu_warmstart_train_step": (_S, [_P, _P, _P, _U, _F, ctypes.POINTER(ctypes.c_double)]),
    "etcu_warmstart_gradients": (_S, [_P, _P, _P, _U, _P, ctypes.POINTER(ctypes.c_double)]),
    "etcu_warmstart_check": (_S, [_P]),
}


def lib() -> ctypes.CDLL:
    """Load the in-tree CUDA library; raise loudly when it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m ettention_b200.build` "
                              "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIG.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, ctx=None) -> None:
    if status != OK:
        msg = lib().etcu_last_error(ctx)
        raise EttentionError(status, (msg or b"").decode() or f"etcu status {status}")
