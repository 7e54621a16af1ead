"""ctypes binding of the C ABI in include/cr/cr.h (libsatincr.so).

The library is built in-tree by ``build.py`` into ``_lib/libsatincr.so``.
Loading fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsatincr.so")

CR_OK = 0
STATUS_NAMES = {0: "CR_OK", 1: "CR_ERR_INVALID_ARGUMENT", 2: "CR_ERR_OUT_OF_MEMORY",
                3: "CR_ERR_CUDA", 4: "CR_ERR_UNSUPPORTED", 5: "CR_ERR_CAPACITY",
                6: "CR_ERR_TIMEOUT", 7: "CR_ERR_NO_DEVICE", 8: "CR_ERR_INTERNAL"}

# numpy views of the shared structs (ComputeRasteriserTypes.h:11-57).
BATCH_DTYPE = np.dtype([("state", "<i4"), ("minX", "<f4"), ("minY", "<f4"), ("minZ", "<f4"),
                        ("maxX", "<f4"), ("maxY", "<f4"), ("maxZ", "<f4"),
                        ("numPoints", "<u4"), ("firstPoint", "<u4"), ("fileIndex", "<u4"),
                        ("lodCum01", "<u4"), ("lodCum23", "<u4"), ("lodCum45", "<u4"),
                        ("lodCum67", "<u4"), ("padding7", "<u4"), ("padding8", "<u4")])
FILE_DTYPE = np.dtype([("transform", "<f4", 16), ("transformFrustum", "<f4", 16),
                       ("world", "<f4", 16), ("prevTransform", "<f4", 16)])
PIXEL_DTYPE = np.dtype([("depth", "<u4"), ("red", "<u4"), ("green", "<u4"), ("blue", "<u4"),
                        ("count", "<u4"), ("weight", "<u4"), ("padding", "<u4", 2)])
VISIBLE_DTYPE = np.dtype([("batchIndex", "<u4"), ("level", "<i4"), ("lodThreshold", "<f4"),
                          ("activePoints", "<u4")])


class cr_config(C.Structure):
    _fields_ = [("mode", C.c_int32), ("depthTolerance", C.c_float),
                ("backgroundColor", C.c_float * 4), ("enableFrustumCulling", C.c_int32),
                ("lodBias", C.c_int32), ("enableCLOD", C.c_int32), ("enableLODDither", C.c_int32),
                ("holeFillIterations", C.c_int32), ("colorizeChunks", C.c_int32),
                ("colorizeOverdraw", C.c_int32), ("pointSizeMode", C.c_int32),
                ("minimumPointSize", C.c_float), ("maximumPointSize", C.c_float),
                ("pointSizeScale", C.c_float), ("applyDisplacement", C.c_int32),
                ("applyTint", C.c_int32), ("tintAlphaIsCoverage", C.c_int32),
                ("writesSceneDepth", C.c_int32), ("motionBlur", C.c_float),
                ("motionBlurSamples", C.c_int32), ("motionBlurMaxSpread", C.c_float)]


class cr_camera(C.Structure):
    _fields_ = [("view", C.c_float * 16), ("projection", C.c_float * 16)]


class cr_capacity(C.Structure):
    _fields_ = [("maxResidentBatches", C.c_uint32), ("pointsPerBatch", C.c_uint32)]


class cr_pack_input(C.Structure):
    _fields_ = [("positions", C.c_void_p), ("positionStrideBytes", C.c_uint32),
                ("colors", C.c_void_p), ("colorStrideBytes", C.c_uint32),
                ("colorFormat", C.c_int32)]


class cr_pack_params(C.Structure):
    _fields_ = [("lodLevels", C.c_int32), ("coarseVoxelDivisions", C.c_int32),
                ("mortonBits", C.c_int32)]


class cr_synth_terrain(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("extent", C.c_float), ("amplitude", C.c_float),
                ("baseWavelength", C.c_float), ("octaves", C.c_int32),
                ("lacunarity", C.c_float), ("gain", C.c_float), ("outlierFraction", C.c_float),
                ("outlierMargin", C.c_float), ("colorNoiseSigma", C.c_float)]


class cr_frame_planes(C.Structure):
    _fields_ = [("depth", C.c_void_p), ("accum", C.c_void_p), ("pixels", C.c_uint64),
                ("stream", C.c_void_p)]


class cr_ply_header(C.Structure):
    _fields_ = [("vertexCount", C.c_uint64), ("bodyOffset", C.c_uint64), ("format", C.c_uint32),
                ("propertyCount", C.c_uint32), ("stride", C.c_uint32),
                ("colorProperties", C.c_uint32)]


class cr_cloud_arrays(C.Structure):
    _fields_ = [("batches", C.c_void_p), ("xyzLow", C.c_void_p), ("xyzMed", C.c_void_p),
                ("xyzHigh", C.c_void_p), ("colors", C.c_void_p), ("levels", C.c_void_p),
                ("points", C.c_uint64), ("slots", C.c_uint32), ("pointsPerBatch", C.c_uint32)]


class cr_tuning(C.Structure):
    _fields_ = [("chunkPoints", C.c_int32), ("useTiles", C.c_int32),
                ("viewGroupPixels", C.c_int32), ("cullSpinLimit", C.c_int32)]


class cr_cloud_info(C.Structure):
    _fields_ = [("capacity", cr_capacity), ("residentBatchCount", C.c_uint32),
                ("pointCount", C.c_uint64), ("freeSlotCount", C.c_uint32),
                ("fileCount", C.c_uint32)]


P = C.c_void_p
VP = C.POINTER(C.c_void_p)
i32 = C.c_int32
u32 = C.c_uint32
u64 = C.c_uint64

# name -> (restype, argtypes); every symbol the header declares.
PROTOTYPES = {
    "cr_status_string": (C.c_char_p, [C.c_int]),
    "cr_last_error_detail": (C.c_char_p, []),
    "cr_layout_sizes": (C.c_int, [P]),
    "cr_config_default": (C.c_int, [C.POINTER(cr_config)]),
    "cr_context_create": (C.c_int, [C.c_int, VP]),
    "cr_context_destroy": (C.c_int, [P]),
    "cr_context_synchronize": (C.c_int, [P]),
    "cr_context_stream": (C.c_int, [P, VP]),
    "cr_context_trim": (C.c_int, [P]),
    "cr_cloud_create": (C.c_int, [P, cr_capacity, P, u32, VP]),
    "cr_cloud_destroy": (C.c_int, [P]),
    "cr_cloud_reallocate": (C.c_int, [P, cr_capacity, P, u32]),
    "cr_cloud_set_files": (C.c_int, [P, P, u32]),
    "cr_cloud_add_batches": (C.c_int, [P, P, P, P, P, P, u64, P, u32, C.c_int, P]),
    "cr_cloud_remove_batches": (C.c_int, [P, P, u32, C.c_int]),
    "cr_cloud_commit": (C.c_int, [P]),
    "cr_cloud_clear": (C.c_int, [P]),
    "cr_cloud_update_files": (C.c_int, [P, P, P, P, P]),
    "cr_cloud_info_get": (C.c_int, [P, C.POINTER(cr_cloud_info)]),
    "cr_cloud_read_files": (C.c_int, [P, P, u32]),
    "cr_cloud_read_batches": (C.c_int, [P, P, u32, u32]),
    "cr_cloud_read_points": (C.c_int, [P, u64, u64, P, P, P, P, P]),
    "cr_cloud_read_visible": (C.c_int, [P, P, u32, C.POINTER(u32)]),
    "cr_frame_create": (C.c_int, [P, C.c_int, C.c_int, VP]),
    "cr_frame_destroy": (C.c_int, [P]),
    "cr_render": (C.c_int, [P, P, P, u32, C.POINTER(cr_config), C.POINTER(cr_camera)]),
    "cr_cloud_add_batches_async": (C.c_int, [P, P, P, P, P, P, u64, P, u32, u32, P]),
    "cr_cloud_poll_uploads": (C.c_int, [P, C.c_int, P, P]),
    "cr_cloud_wait_uploads": (C.c_int, [P, C.c_int]),
    "cr_cloud_set_upload_staging": (C.c_int, [P, u64]),
    "cr_ply_read_header": (C.c_int, [P, u64, C.POINTER(cr_ply_header)]),
    "cr_ply_parse": (C.c_int, [P, u64, C.c_int, P, P]),
    "cr_file_map": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]),
    "cr_file_unmap": (C.c_int, [P, u64]),
    "cr_cloud_attribute": (C.c_int, [P, i32, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]),
    "cr_cloud_release_attribute": (C.c_int, [P, i32]),
    "cr_cloud_device_arrays": (C.c_int, [P, C.POINTER(cr_cloud_arrays)]),
    "cr_render_stages": (C.c_int, [P, P, P, u32, C.POINTER(cr_config), C.POINTER(cr_camera),
                                   u32]),
    "cr_frame_device_planes": (C.c_int, [P, C.POINTER(cr_frame_planes)]),
    "cr_frame_flip_depth_order": (C.c_int, [P]),
    "cr_frame_read_rgba8": (C.c_int, [P, P]),
    "cr_frame_read_rgba8_async": (C.c_int, [P, P]),
    "cr_frame_read_wait": (C.c_int, [P]),
    "cr_frame_read_wait_keep": (C.c_int, [P, C.c_int]),
    "cr_frame_read_depth_f32": (C.c_int, [P, P]),
    "cr_frame_read_pixels": (C.c_int, [P, P]),
    "cr_frame_read_nearest_depth": (C.c_int, [P, P]),
    "cr_frame_read_nearest_index": (C.c_int, [P, P]),
    "cr_frame_read_nearest_index_rows": (C.c_int, [P, C.c_int, C.c_int, P]),
    "cr_pick": (C.c_int, [P, P, P, P, C.POINTER(cr_config), C.POINTER(cr_camera), C.c_int,
                          C.POINTER(u32), C.POINTER(C.c_int)]),
    "cr_pack_params_default": (C.c_int, [C.POINTER(cr_pack_params)]),
    "cr_buffer_create": (C.c_int, [P, u64, VP]),
    "cr_buffer_destroy": (C.c_int, [P, P]),
    "cr_buffer_upload": (C.c_int, [P, P, P, u64]),
    "cr_buffer_download": (C.c_int, [P, P, P, u64]),
    "cr_host_alloc": (C.c_int, [u64, VP]),
    "cr_host_free": (C.c_int, [P]),
    "cr_context_set_profiling": (C.c_int, [P, C.c_int]),
    "cr_context_get_tuning": (C.c_int, [P, C.POINTER(cr_tuning)]),
    "cr_context_set_tuning": (C.c_int, [P, C.POINTER(cr_tuning)]),
    "cr_context_pass_times": (C.c_int, [P, i32, P, C.POINTER(i32)]),
    "cr_synth_terrain_default": (C.c_int, [C.POINTER(cr_synth_terrain)]),
    "cr_synth_terrain_height": (C.c_float, [C.POINTER(cr_synth_terrain), C.c_float, C.c_float]),
    "cr_synth_terrain_points": (C.c_int, [P, C.POINTER(cr_synth_terrain), u64, u64, P]),
    "cr_synth_lattice_points": (C.c_int, [P, u64, u32, C.c_float, C.c_float, C.c_float, P]),
    "cr_cull_noalloc": (C.c_int, [P, u32, P, u32, C.POINTER(cr_config), C.POINTER(cr_camera),
                                  C.c_int, C.c_int, P, P, P]),
    "cr_render_multiview": (C.c_int, [P, P, P, u32, P, P, u32, C.POINTER(cr_config)]),
    "cr_hqs_forward_f32": (C.c_int, [P, P, P, C.POINTER(cr_config), C.POINTER(cr_camera), P,
                                     P]),
    "cr_hqs_backward_colors": (C.c_int, [P, P, P, C.POINTER(cr_config), C.POINTER(cr_camera),
                                         P, P]),
    "cr_l2_loss": (C.c_int, [P, P, P, u64, C.c_float, P, C.POINTER(C.c_double)]),
    "cr_autotune_multiview": (C.c_int, [P, P, P, u32, P, P, u32, C.POINTER(cr_config),
                                        C.c_char_p, C.c_int, C.POINTER(cr_tuning),
                                        C.POINTER(C.c_float)]),
    "cr_pack": (C.c_int, [P, P, C.POINTER(cr_pack_input), u64, C.POINTER(cr_pack_params),
                          C.c_int, P]),
    "cr_pack_chunks": (C.c_int, [P, P, P, P, u32, C.POINTER(cr_pack_params), C.c_int, P,
                                 C.POINTER(u32)]),
}

_lib = None


class CRError(RuntimeError):
    """A cr_status other than CR_OK, with the library's detail string."""

    def __init__(self, status: int, detail: str):
        self.status = status
        self.detail = detail
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {detail}")


def lib():
    """Load libsatincr.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with build.py "
                           "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error_detail() -> str:
    return lib().cr_last_error_detail().decode(errors="replace")


def check(status: int) -> None:
    if status != CR_OK:
        detail = lib().cr_last_error_detail().decode(errors="replace")
        raise CRError(status, detail)


def ptr(a):
    if a is None:
        return None
    return C.c_void_p(a.ctypes.data)
