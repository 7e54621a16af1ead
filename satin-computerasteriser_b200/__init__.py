"""B200 point-cloud compute rasteriser — host mirror of Satin-ComputeRasteriser's API.

The classes here mirror the reference's Swift surface for the render path
(same names, argument meaning and error behaviour) on top of the C ABI in
``include/cr/cr.h``:

  ComputeRasteriserConfiguration  ComputeRasteriserTypes.swift:26-142
  ComputeRasteriserCapacity       ComputeRasteriserPointCloud.swift:23-40
  ComputeRasteriserPointCloud     ComputeRasteriserPointCloud.swift:59-678
  ComputeRasteriser               ComputeRasteriser.swift:5-888
  PackedPointCloud                ComputeRasteriserTypes.swift:269-320

Swift preconditions become ``CRError`` exceptions.  All GPU work runs in
``_lib/libsatincr.so`` (CUDA, sm_100a); nothing here computes pixels.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field, fields

import numpy as np

from . import _native as N
from ._native import (BATCH_DTYPE, FILE_DTYPE, PIXEL_DTYPE, VISIBLE_DTYPE, CRError)

__all__ = ["Context", "ComputeRasteriserConfiguration", "ComputeRasteriserCapacity",
           "ComputeRasteriserPointCloud", "ComputeRasteriser", "PackedPointCloud",
           "PerspectiveCamera", "CRError", "BATCH_DTYPE", "FILE_DTYPE", "PIXEL_DTYPE",
           "VISIBLE_DTYPE", "computeRasteriserThreadsPerGroup", "MODE_HQS", "MODE_NEAREST",
           "identity_files", "matrix_multiply", "GPUPacker", "PackInput", "DeviceBuffer",
           "HostBuffer", "TerrainParams", "synth_terrain", "synth_lattice", "terrain_height",
           "PASS_NAMES", "MultiViewRasteriser", "l2_loss", "STAGE_DEPTH", "STAGE_COLOR",
           "STAGE_RESOLVE", "STAGE_ALL", "PLYPointCloudLoader", "PLYPointCloudLoaderError",
           "DeviceView", "DisplacementPass", "TintPass", "ATTR_DISPLACEMENT",
           "ATTR_PREV_DISPLACEMENT", "ATTR_TINT"]

PASS_NAMES = ("clear", "cull", "depth", "color", "resolve", "hole_fill")
STAGE_DEPTH, STAGE_COLOR, STAGE_RESOLVE, STAGE_ALL = 1, 2, 4, 7  # cr_stage

computeRasteriserThreadsPerGroup = 128
MODE_HQS = 0      # ComputeRasteriserMode.highQualityAverage
MODE_NEAREST = 1  # ComputeRasteriserMode.nearestPoint
SCREEN_SPACE = 0  # PointSizeMode.screenSpace
WORLD_SPACE = 1   # PointSizeMode.worldSpace


def _mat16(m) -> np.ndarray:
    """A 4x4 matrix as the column-major float[16] the ABI takes.

    Accepts a flat 16-vector (already column-major) or a 4x4 array in
    row-major math notation (m[row][col]), which is transposed."""
    a = np.asarray(m, dtype=np.float32)
    if a.shape == (4, 4):
        a = a.T
    return np.ascontiguousarray(a.reshape(16))


def matrix_multiply(a, b) -> np.ndarray:
    """a * b for column-major float[16] matrices with the library's fixed
    operation order (rows summed k = 0..3 left to right, no FMA)."""
    A, B = _mat16(a).reshape(4, 4), _mat16(b).reshape(4, 4)  # A[k][r] = a[4k + r]
    # Element (c, r): ((a[r] b[4c] + a[4+r] b[4c+1]) + a[8+r] b[4c+2]) + a[12+r] b[4c+3],
    # every product and sum rounded to float32, for all 16 elements at once.
    s = np.multiply.outer(B[:, 0], A[0]) + np.multiply.outer(B[:, 1], A[1])
    s = s + np.multiply.outer(B[:, 2], A[2])
    s = s + np.multiply.outer(B[:, 3], A[3])
    return np.ascontiguousarray(s, dtype=np.float32).reshape(16)


def identity_files(n: int = 1) -> np.ndarray:
    """RasterFile() defaults (ComputeRasteriserTypes.swift:235-244): identity matrices."""
    f = np.zeros(n, FILE_DTYPE)
    eye = np.eye(4, dtype=np.float32).reshape(16)
    for k in FILE_DTYPE.names:
        f[k][:] = eye
    return f


class Context:
    """Device + stream (the role of Satin's Context / MTLCommandQueue)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        N.check(N.lib().cr_context_create(device, C.byref(self._h)))
        self.device = device

    @property
    def handle(self):
        return self._h

    def synchronize(self):
        N.check(N.lib().cr_context_synchronize(self._h))

    def stream(self) -> int:
        s = C.c_void_p()
        N.check(N.lib().cr_context_stream(self._h, C.byref(s)))
        return s.value or 0

    def trim(self):
        """Release the packer's scratch memory."""
        N.check(N.lib().cr_context_trim(self._h))

    def tuning(self) -> dict:
        t = N.cr_tuning()
        N.check(N.lib().cr_context_get_tuning(self._h, C.byref(t)))
        return {"chunkPoints": t.chunkPoints, "useTiles": bool(t.useTiles),
                "viewGroupPixels": t.viewGroupPixels, "cullSpinLimit": t.cullSpinLimit}

    def set_tuning(self, chunkPoints: int | None = None, useTiles: bool | None = None,
                   viewGroupPixels: int | None = None, cullSpinLimit: int | None = None):
        """Launch tuning of the point passes (results do not depend on it).

        cullSpinLimit bounds the cull's wait for its predecessors' counts; a
        wait that runs out makes the next synchronising call raise CRError
        with CR_ERR_TIMEOUT (0 gives up at once, to exercise that path)."""
        cur = self.tuning()
        t = N.cr_tuning(int(cur["chunkPoints"] if chunkPoints is None else chunkPoints),
                        int(cur["useTiles"] if useTiles is None else useTiles),
                        int(cur["viewGroupPixels"] if viewGroupPixels is None
                            else viewGroupPixels),
                        int(cur["cullSpinLimit"] if cullSpinLimit is None else cullSpinLimit))
        N.check(N.lib().cr_context_set_tuning(self._h, C.byref(t)))

    def set_profiling(self, enable: bool):
        """Bracket every pass of every cr_render with CUDA events (ring of 256 frames)."""
        N.check(N.lib().cr_context_set_profiling(self._h, int(enable)))

    def pass_times(self, nframes: int = 256) -> np.ndarray:
        """(frames, 6) device milliseconds per pass (PASS_NAMES order), oldest first."""
        out = np.zeros((max(nframes, 1), len(PASS_NAMES)), np.float32)
        got = C.c_int32()
        N.check(N.lib().cr_context_pass_times(self._h, nframes, N.ptr(out), C.byref(got)))
        return out[:got.value].copy()

    def close(self):
        if self._h:
            N.lib().cr_context_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceBuffer:
    """Device memory owned through the C ABI (cr_buffer_*); exposes
    __cuda_array_interface__ so it can be handed to the packer or to torch."""

    def __init__(self, context: Context, nbytes: int, shape=None, dtype=np.uint8):
        self.context = context
        self.nbytes = int(nbytes)
        self.dtype = np.dtype(dtype)
        self.shape = tuple(shape) if shape is not None else (self.nbytes // self.dtype.itemsize,)
        p = C.c_void_p()
        N.check(N.lib().cr_buffer_create(context.handle, self.nbytes, C.byref(p)))
        self.ptr = p.value

    @property
    def __cuda_array_interface__(self):
        return {"shape": self.shape, "typestr": self.dtype.str, "data": (self.ptr, False),
                "version": 3, "strides": None}

    def upload(self, host: np.ndarray):
        """Copy host data in: raw bytes into a byte (uint8) buffer, otherwise
        converted to the buffer's dtype."""
        if self.dtype == np.uint8:
            h = np.ascontiguousarray(host)
        else:
            h = np.ascontiguousarray(host, dtype=self.dtype)
        N.check(N.lib().cr_buffer_upload(self.context.handle, C.c_void_p(self.ptr), N.ptr(h),
                                         min(h.nbytes, self.nbytes)))

    def download(self) -> np.ndarray:
        out = np.empty(self.shape, self.dtype)
        N.check(N.lib().cr_buffer_download(self.context.handle, N.ptr(out), C.c_void_p(self.ptr),
                                           out.nbytes))
        return out

    def close(self):
        # A buffer outliving its context (interpreter shutdown frees objects in
        # no fixed order) was released with it.
        if self.ptr and self.context.handle:
            N.lib().cr_buffer_destroy(self.context.handle, C.c_void_p(self.ptr))
        self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HostBuffer:
    """Pinned (page-locked) host memory as a numpy array (cr_host_alloc)."""

    def __init__(self, shape, dtype=np.uint8):
        dt = np.dtype(dtype)
        n = int(np.prod(shape)) * dt.itemsize
        p = C.c_void_p()
        N.check(N.lib().cr_host_alloc(n, C.byref(p)))
        self._p = p
        buf = (C.c_uint8 * max(n, 1)).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dt, count=int(np.prod(shape))).reshape(shape)

    def close(self):
        if self._p:
            self.array = None
            N.lib().cr_host_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class TerrainParams:
    """cr_synth_terrain: the 4 km x 4 km fractal heightfield workload."""
    seed: int = 0xC0FFEE02
    extent: float = 4000.0
    amplitude: float = 200.0
    baseWavelength: float = 1500.0
    octaves: int = 6
    lacunarity: float = 2.0
    gain: float = 0.5
    outlierFraction: float = 0.05
    outlierMargin: float = 50.0
    colorNoiseSigma: float = 10.0

    def to_c(self) -> N.cr_synth_terrain:
        return N.cr_synth_terrain(self.seed, self.extent, self.amplitude, self.baseWavelength,
                                  self.octaves, self.lacunarity, self.gain, self.outlierFraction,
                                  self.outlierMargin, self.colorNoiseSigma)


def terrain_height(params: TerrainParams, x: float, y: float) -> float:
    t = params.to_c()
    return float(N.lib().cr_synth_terrain_height(C.byref(t), float(x), float(y)))


def synth_terrain(context: Context, params: TerrainParams, count: int,
                  out: DeviceBuffer | None = None, first: int = 0) -> DeviceBuffer:
    """count 16-byte records {x, y, z, rgba8} of the heightfield in device memory."""
    buf = out or DeviceBuffer(context, count * 16, (count, 4), np.float32)
    t = params.to_c()
    N.check(N.lib().cr_synth_terrain_points(context.handle, C.byref(t), first, count,
                                            C.c_void_p(buf.ptr)))
    return buf


def synth_lattice(context: Context, n_axis: int, seed: int = 0xC0FFEE01, lo: float = -1.0,
                  hi: float = 1.0, jitter: float = 0.002) -> DeviceBuffer:
    """n_axis^3 jittered lattice records {x, y, z, rgba8} in device memory."""
    count = n_axis ** 3
    buf = DeviceBuffer(context, count * 16, (count, 4), np.float32)
    N.check(N.lib().cr_synth_lattice_points(context.handle, seed, n_axis, lo, hi, jitter,
                                            C.c_void_p(buf.ptr)))
    return buf


@dataclass
class ComputeRasteriserConfiguration:
    """ComputeRasteriserConfiguration (ComputeRasteriserTypes.swift:26-142), same defaults."""
    mode: int = MODE_HQS
    depthTolerance: float = 0.01
    backgroundColor: tuple = (0.0, 0.0, 0.0, 0.0)
    enableFrustumCulling: bool = True
    lodBias: int = 0
    enableCLOD: bool = True
    enableLODDither: bool = True
    holeFillIterations: int = 0
    colorizeChunks: bool = False
    colorizeOverdraw: bool = False
    pointSizeMode: int = SCREEN_SPACE
    minimumPointSize: float = 1.0
    maximumPointSize: float = 1.0
    pointSizeScale: float = 1.0
    applyDisplacement: bool = False
    applyTint: bool = False
    tintAlphaIsCoverage: bool = False
    writesSceneDepth: bool = True
    motionBlur: float = 0.0
    motionBlurSamples: int = 8
    motionBlurMaxSpread: float = 64.0

    def to_c(self) -> N.cr_config:
        c = N.cr_config()
        for f in fields(self):
            v = getattr(self, f.name)
            if f.name == "backgroundColor":
                c.backgroundColor[:] = [float(x) for x in v]
            elif isinstance(getattr(c, f.name), float):
                setattr(c, f.name, float(v))
            else:
                setattr(c, f.name, int(v))
        return c


@dataclass(frozen=True)
class ComputeRasteriserCapacity:
    """ComputeRasteriserCapacity (ComputeRasteriserPointCloud.swift:23-40)."""
    maxResidentBatches: int
    pointsPerBatch: int = computeRasteriserThreadsPerGroup * 80

    def __post_init__(self):
        if self.maxResidentBatches <= 0:
            raise CRError(1, "maxResidentBatches must be positive")
        if self.pointsPerBatch <= 0:
            raise CRError(1, "pointsPerBatch must be positive")

    @property
    def maxResidentPoints(self) -> int:
        return self.maxResidentBatches * self.pointsPerBatch

    def to_c(self) -> N.cr_capacity:
        return N.cr_capacity(self.maxResidentBatches, self.pointsPerBatch)


@dataclass
class PackedPointCloud:
    """PackedPointCloud (ComputeRasteriserTypes.swift:269-320) as numpy arrays."""
    batches: np.ndarray
    files: np.ndarray
    xyzLow: np.ndarray
    xyzMed: np.ndarray
    xyzHigh: np.ndarray
    colors: np.ndarray
    levels: np.ndarray
    boundsMin: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))
    boundsMax: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))
    orderedPositions: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float32))
    sourceIndices: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))

    @property
    def pointCount(self) -> int:
        return len(self.colors)

    @property
    def batchCount(self) -> int:
        return len(self.batches)


class DeviceView:
    """A device array owned by the library (a cloud's attribute or pool
    array), with __cuda_array_interface__ for torch / CuPy / numba kernels and
    host upload / download through the C ABI."""

    def __init__(self, context: Context, ptr: int, shape, dtype, owner=None):
        self.context = context
        self.ptr = int(ptr)
        self.shape = tuple(int(d) for d in shape)
        self.dtype = np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        self._owner = owner  # keeps the cloud alive

    @property
    def __cuda_array_interface__(self):
        return {"shape": self.shape, "typestr": self.dtype.str, "data": (self.ptr, False),
                "version": 3, "strides": None}

    def upload(self, host: np.ndarray):
        h = np.ascontiguousarray(host, dtype=self.dtype)
        N.check(N.lib().cr_buffer_upload(self.context.handle, C.c_void_p(self.ptr), N.ptr(h),
                                         min(h.nbytes, self.nbytes)))

    def download(self) -> np.ndarray:
        out = np.empty(self.shape, self.dtype)
        N.check(N.lib().cr_buffer_download(self.context.handle, N.ptr(out),
                                           C.c_void_p(self.ptr), out.nbytes))
        return out


ATTR_DISPLACEMENT, ATTR_PREV_DISPLACEMENT, ATTR_TINT = 0, 1, 2  # cr_attribute


class ComputeRasteriserPointCloud:
    """ComputeRasteriserPointCloud (ComputeRasteriserPointCloud.swift:59-678).

    A fixed-size slot pool on the device: per-point xyzLow/Med/High, colours
    and levels, one RasterBatch per slot, and the per-file transform table.
    """

    def __init__(self, context: Context, capacity: ComputeRasteriserCapacity | None = None,
                 files=None, packed: PackedPointCloud | None = None,
                 label: str = "ComputeRasteriserPointCloud"):
        self.context = context
        self.label = label
        self.visible = True
        self.worldMatrix = np.eye(4, dtype=np.float32).reshape(16)
        if packed is not None and capacity is None:
            # Convenience init (ComputeRasteriserPointCloud.swift:222-236).
            ppb = int(packed.batches["numPoints"].max()) if packed.batchCount else \
                computeRasteriserThreadsPerGroup * 80
            capacity = ComputeRasteriserCapacity(max(1, packed.batchCount), max(1, ppb))
            files = packed.files
        if capacity is None:
            raise CRError(1, "capacity or packed is required")
        files = identity_files() if files is None else np.ascontiguousarray(files, FILE_DTYPE)
        self._h = C.c_void_p()
        N.check(N.lib().cr_cloud_create(context.handle, capacity.to_c(), N.ptr(files), len(files),
                                        C.byref(self._h)))
        self._capacity = capacity
        if packed is not None and packed.batchCount > 0:
            self._upload_packed(packed)

    # --- Satin Object transform (position only, enough for the render path) ---
    @property
    def position(self):
        return tuple(self.worldMatrix[12:15])

    @position.setter
    def position(self, p):
        m = np.eye(4, dtype=np.float32).reshape(16)
        m[12:15] = np.asarray(p, np.float32)
        self.worldMatrix = m

    @property
    def handle(self):
        return self._h

    def _info(self) -> N.cr_cloud_info:
        info = N.cr_cloud_info()
        N.check(N.lib().cr_cloud_info_get(self._h, C.byref(info)))
        return info

    @property
    def capacity(self) -> ComputeRasteriserCapacity:
        return self._capacity

    @property
    def batchCount(self) -> int:
        return self._capacity.maxResidentBatches

    @property
    def residentBatchCount(self) -> int:
        return self._info().residentBatchCount

    @property
    def pointCount(self) -> int:
        return self._info().pointCount

    @property
    def freeSlotCount(self) -> int:
        return self._info().freeSlotCount

    def addBatches(self, positionsXYZLow, positionsXYZMed, positionsXYZHigh, colors, levels,
                   batches, commit: bool = True) -> list[int]:
        """addBatches (ComputeRasteriserPointCloud.swift:410-452)."""
        low = np.ascontiguousarray(positionsXYZLow, np.uint32)
        med = np.ascontiguousarray(positionsXYZMed, np.uint32)
        high = np.ascontiguousarray(positionsXYZHigh, np.uint32)
        col = np.ascontiguousarray(colors, np.uint32)
        lv = np.ascontiguousarray(levels, np.uint8)
        b = np.ascontiguousarray(batches, BATCH_DTYPE)
        n = min(len(low), len(med), len(high), len(col), len(lv))
        slots = np.zeros(max(len(b), 1), np.int32)
        N.check(N.lib().cr_cloud_add_batches(self._h, N.ptr(low), N.ptr(med), N.ptr(high),
                                             N.ptr(col), N.ptr(lv), n, N.ptr(b), len(b),
                                             int(commit), N.ptr(slots)))
        return slots[:len(b)].tolist()

    def addBatchesAsync(self, positionsXYZLow, positionsXYZMed, positionsXYZHigh, colors,
                        levels, batches, borrow: bool = False) -> list[int]:
        """addBatches with an asynchronous copy (cr_cloud_add_batches_async): the
        slots are taken now and become resident when pollUploads / waitUploads
        sees their copy landed.  The arrays may be reused when this returns;
        with borrow=True they must be page-locked (HostBuffer arrays) and stay
        unchanged until the upload is published (no staging copy)."""
        if borrow:
            for a, dt in ((positionsXYZLow, np.uint32), (positionsXYZMed, np.uint32),
                          (positionsXYZHigh, np.uint32), (colors, np.uint32),
                          (levels, np.uint8)):
                if a.dtype != dt or not a.flags.c_contiguous:
                    raise CRError(1, "borrowed arrays must be C-contiguous of the pool's types")
        low = np.ascontiguousarray(positionsXYZLow, np.uint32)
        med = np.ascontiguousarray(positionsXYZMed, np.uint32)
        high = np.ascontiguousarray(positionsXYZHigh, np.uint32)
        col = np.ascontiguousarray(colors, np.uint32)
        lv = np.ascontiguousarray(levels, np.uint8)
        b = np.ascontiguousarray(batches, BATCH_DTYPE)
        n = min(len(low), len(med), len(high), len(col), len(lv))
        slots = np.zeros(max(len(b), 1), np.int32)
        N.check(N.lib().cr_cloud_add_batches_async(self._h, N.ptr(low), N.ptr(med), N.ptr(high),
                                                   N.ptr(col), N.ptr(lv), n, N.ptr(b), len(b),
                                                   1 if borrow else 0, N.ptr(slots)))
        return slots[:len(b)].tolist()

    def pollUploads(self, commit: bool = True) -> tuple[int, int]:
        """Publishes the asynchronous uploads that have landed (non-blocking);
        returns (batches published now, batches still in flight)."""
        landed, flying = C.c_uint32(0), C.c_uint32(0)
        N.check(N.lib().cr_cloud_poll_uploads(self._h, int(commit), C.byref(landed),
                                              C.byref(flying)))
        return landed.value, flying.value

    def waitUploads(self, commit: bool = True):
        """Waits for every asynchronous upload in flight and publishes it."""
        N.check(N.lib().cr_cloud_wait_uploads(self._h, int(commit)))

    def setUploadStaging(self, nbytes: int):
        """Size of the page-locked staging ring of the asynchronous uploads."""
        N.check(N.lib().cr_cloud_set_upload_staging(self._h, int(nbytes)))

    # --- colour-variant attributes (displacementBuffer / tintBuffer) ---
    def _attribute(self, which: int) -> DeviceView:
        p, n = C.c_void_p(), C.c_uint64()
        N.check(N.lib().cr_cloud_attribute(self._h, which, C.byref(p), C.byref(n)))
        return DeviceView(self.context, p.value, (n.value, 4), np.float32, owner=self)

    def displacementBuffer(self) -> DeviceView:
        """The per-point float4 displacement (xyz) buffer, allocated zeroed on
        first use (makeDisplacementBuffer, ComputeRasteriserPointCloud.swift)."""
        return self._attribute(ATTR_DISPLACEMENT)

    def prevDisplacementBuffer(self) -> DeviceView:
        """The previous frame's displacement (motion blur)."""
        return self._attribute(ATTR_PREV_DISPLACEMENT)

    def tintBuffer(self) -> DeviceView:
        """The per-point float4 tint (rgba) buffer (makeTintBuffer)."""
        return self._attribute(ATTR_TINT)

    def releaseAttribute(self, which: int):
        N.check(N.lib().cr_cloud_release_attribute(self._h, which))

    def deviceArrays(self) -> dict:
        """The pool's device arrays for user kernels (read-only): batches
        (BATCH_DTYPE per slot), xyzLow / xyzMed / xyzHigh / colors (uint32 per
        point), levels (uint8 per point)."""
        a = N.cr_cloud_arrays()
        N.check(N.lib().cr_cloud_device_arrays(self._h, C.byref(a)))
        ctx, n = self.context, int(a.points)
        return {"batches": DeviceView(ctx, a.batches, (a.slots, BATCH_DTYPE.itemsize), np.uint8,
                                      self),
                "xyzLow": DeviceView(ctx, a.xyzLow, (n,), np.uint32, self),
                "xyzMed": DeviceView(ctx, a.xyzMed, (n,), np.uint32, self),
                "xyzHigh": DeviceView(ctx, a.xyzHigh, (n,), np.uint32, self),
                "colors": DeviceView(ctx, a.colors, (n,), np.uint32, self),
                "levels": DeviceView(ctx, a.levels, (n,), np.uint8, self),
                "pointsPerBatch": int(a.pointsPerBatch)}

    def removeBatches(self, slots, commit: bool = True):
        """removeBatches (ComputeRasteriserPointCloud.swift:460-473)."""
        s = np.ascontiguousarray(slots, np.int32)
        N.check(N.lib().cr_cloud_remove_batches(self._h, N.ptr(s), len(s), int(commit)))

    def commitBatchUpdates(self):
        N.check(N.lib().cr_cloud_commit(self._h))

    def clearAllBatches(self):
        N.check(N.lib().cr_cloud_clear(self._h))

    def replacePackedPointCloud(self, packed: PackedPointCloud):
        """replacePackedPointCloud (ComputeRasteriserPointCloud.swift:246-264)."""
        needed = max(1, packed.batchCount)
        ppb = int(packed.batches["numPoints"].max()) if packed.batchCount else \
            self._capacity.pointsPerBatch
        files = np.ascontiguousarray(packed.files, FILE_DTYPE)
        if needed > self._capacity.maxResidentBatches or ppb > self._capacity.pointsPerBatch:
            cap = ComputeRasteriserCapacity(needed, max(ppb, self._capacity.pointsPerBatch))
            N.check(N.lib().cr_cloud_reallocate(self._h, cap.to_c(), N.ptr(files), len(files)))
            self._capacity = cap
        else:
            N.check(N.lib().cr_cloud_set_files(self._h, N.ptr(files), len(files)))
            self.clearAllBatches()
        if packed.batchCount > 0:
            self._upload_packed(packed)

    def replacePackedPointCloudGPU(self, packer: "GPUPacker", positions=None, colors=None,
                                   count=None, records=None):
        """replacePackedPointCloud(packer:queue:positions:colors:count:) (GPUPacker.swift:507-519)."""
        return packer.pack(positions, colors, count, into=self, records=records)

    def addRawChunksGPU(self, packer: "GPUPacker", chunks, maxConcurrent: int = 1) -> list[int]:
        """addRawChunksGPU(packer:queue:chunks:maxConcurrent:) (GPUPacker.swift:545-577):
        chunks are (positions, colors) pairs or PackInput objects."""
        return packer.addRawChunks(self, chunks)

    def _sync_capacity(self):
        info = self._info()
        self._capacity = ComputeRasteriserCapacity(info.capacity.maxResidentBatches,
                                                   info.capacity.pointsPerBatch)

    def _upload_packed(self, packed: PackedPointCloud):
        self.addBatches(packed.xyzLow, packed.xyzMed, packed.xyzHigh, packed.colors,
                        packed.levels, packed.batches)

    def updateFiles(self, viewProjection, modelMatrix, frustumTransform=None,
                    prevViewProjection=None):
        """updateFiles (ComputeRasteriserPointCloud.swift:487-515)."""
        vp, mm = _mat16(viewProjection), _mat16(modelMatrix)
        fr = None if frustumTransform is None else _mat16(frustumTransform)
        pv = None if prevViewProjection is None else _mat16(prevViewProjection)
        N.check(N.lib().cr_cloud_update_files(self._h, N.ptr(vp), N.ptr(mm), N.ptr(fr),
                                              N.ptr(pv)))

    # --- read-backs (for tests and tools) ---
    def files(self) -> np.ndarray:
        out = np.zeros(self._info().fileCount, FILE_DTYPE)
        N.check(N.lib().cr_cloud_read_files(self._h, N.ptr(out), len(out)))
        return out

    def batches(self, first: int = 0, n: int | None = None) -> np.ndarray:
        n = self.batchCount - first if n is None else n
        out = np.zeros(max(n, 0), BATCH_DTYPE)
        N.check(N.lib().cr_cloud_read_batches(self._h, N.ptr(out), first, n))
        return out

    def points(self, first: int = 0, n: int | None = None) -> dict:
        n = self._capacity.maxResidentPoints - first if n is None else n
        out = {k: np.zeros(n, np.uint32) for k in ("xyzLow", "xyzMed", "xyzHigh", "colors")}
        out["levels"] = np.zeros(n, np.uint8)
        N.check(N.lib().cr_cloud_read_points(self._h, first, n, N.ptr(out["xyzLow"]),
                                             N.ptr(out["xyzMed"]), N.ptr(out["xyzHigh"]),
                                             N.ptr(out["colors"]), N.ptr(out["levels"])))
        return out

    def visibleBatches(self) -> np.ndarray:
        out = np.zeros(self.batchCount, VISIBLE_DTYPE)
        count = C.c_uint32()
        N.check(N.lib().cr_cloud_read_visible(self._h, N.ptr(out), len(out), C.byref(count)))
        return out[:count.value].copy()

    def close(self):
        if self._h and self.context.handle:
            N.lib().cr_cloud_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PackInput:
    """Raw points for the GPU packer: one of
      * positions (n, 3) float32 (12-byte stride) or (n, 4) float32 (the
        reference's 16-byte float3 slots), with colours (n, 4) float32 RGBA
        in [0, 1] or (n,) uint32 packed RGBA8;
      * records: (n, 4) of 16-byte records {float x, y, z; uint32 rgba8}
        given as a float32 or uint32 view.
    Arrays may live on the host (numpy) or on the device (any object with
    __cuda_array_interface__, e.g. a CUDA torch tensor)."""

    def __init__(self, positions=None, colors=None, records=None):
        self._keep = []
        if records is not None:
            base, dev, n, row = self._view(records)
            if row != 16:
                raise CRError(1, "records must be 16 bytes each")
            self.on_device, self.count = dev, n
            self.c = N.cr_pack_input(base, 16, base + 12, 16, 1)
            return
        pb, pdev, n, prow = self._view(positions)
        cb, cdev, nc, crow = self._view(colors)
        if pdev != cdev:
            raise CRError(1, "positions and colors must both be host or both device arrays")
        if n != nc:
            raise CRError(1, "positions and colors must have the same count")
        if prow not in (12, 16):
            raise CRError(1, "positions must be (n, 3) or (n, 4) float32")
        fmt = 1 if crow == 4 else 0
        if crow not in (4, 16):
            raise CRError(1, "colors must be (n, 4) float32 or (n,) uint32 RGBA8")
        self.on_device, self.count = pdev, n
        self.c = N.cr_pack_input(pb, prow, cb, crow, fmt)

    def _view(self, a):
        if hasattr(a, "__cuda_array_interface__"):
            ai = a.__cuda_array_interface__
            shape = ai["shape"]
            itemsize = np.dtype(ai["typestr"]).itemsize
            if ai.get("strides") not in (None,) and ai["strides"] is not None:
                exp = [itemsize]
                for d in reversed(shape[1:]):
                    exp.insert(0, exp[0] * d)
                if tuple(ai["strides"]) != tuple(exp):
                    raise CRError(1, "device arrays must be C-contiguous")
            row = itemsize * (int(np.prod(shape[1:])) if len(shape) > 1 else 1)
            self._keep.append(a)
            return int(ai["data"][0]), True, int(shape[0]) if shape else 0, row
        arr = np.ascontiguousarray(a)
        if arr.dtype == np.float64:
            arr = arr.astype(np.float32)
        self._keep.append(arr)
        row = arr.dtype.itemsize * (int(np.prod(arr.shape[1:])) if arr.ndim > 1 else 1)
        return int(arr.ctypes.data), False, int(arr.shape[0]) if arr.ndim else 0, row


class GPUPacker:
    """GPUPacker (GPUPacker.swift:27-392): packs raw points on the GPU straight
    into a cloud's slot pool, decode-identical to the CPU pack.

    mortonBits = 10 reproduces the reference's 30-bit Morton order;
    mortonBits = 21 sorts 63-bit keys (21 bits per axis)."""

    def __init__(self, context: Context, lodLevels: int = 4, coarseVoxelDivisions: int = 64,
                 mortonBits: int = 10):
        self.context = context
        self.lodLevels = max(1, min(int(lodLevels), 8))
        self.coarseVoxelDivisions = max(1, int(coarseVoxelDivisions))
        self.mortonBits = int(mortonBits)

    def _params(self) -> N.cr_pack_params:
        return N.cr_pack_params(self.lodLevels, self.coarseVoxelDivisions, self.mortonBits)

    def pack(self, positions=None, colors=None, count=None, into=None, records=None,
             sourceIndices: bool = False):
        """pack(positions:colors:count:into:commandBuffer:) (GPUPacker.swift:140-160),
        synchronous.  Returns the source-index permutation when asked."""
        if into is None:
            raise CRError(1, "into (a ComputeRasteriserPointCloud) is required")
        inp = PackInput(positions, colors, records)
        n = inp.count if count is None else int(count)
        if n > inp.count:
            raise CRError(1, "count exceeds the input length")
        src = np.zeros(max(n, 1), np.uint32) if sourceIndices else None
        N.check(N.lib().cr_pack(self.context.handle, into.handle, C.byref(inp.c), n,
                                C.byref(self._params()), int(inp.on_device), N.ptr(src)))
        into._sync_capacity()
        return src[:n] if sourceIndices else None

    def addRawChunks(self, cloud, chunks) -> list[int]:
        """The packing half of addRawChunksGPU (GPUPacker.swift:545-577)."""
        inputs = [c if isinstance(c, PackInput) else PackInput(*c) for c in chunks]
        if len({i.on_device for i in inputs}) > 1:
            raise CRError(1, "chunks must all be host or all be device arrays")
        arr = (N.cr_pack_input * max(len(inputs), 1))(*[i.c for i in inputs])
        counts = np.array([i.count for i in inputs] or [0], np.uint64)
        firsts = np.zeros(max(len(inputs), 1), np.int32)
        placed = C.c_uint32()
        on_dev = int(inputs[0].on_device) if inputs else 0
        N.check(N.lib().cr_pack_chunks(self.context.handle, cloud.handle, arr, N.ptr(counts),
                                       len(inputs), C.byref(self._params()), on_dev,
                                       N.ptr(firsts), C.byref(placed)))
        return firsts[:placed.value].tolist()


class _Frame:
    def __init__(self, context: Context, width: int, height: int):
        self.context = context
        self.width, self.height = width, height
        self._h = C.c_void_p()
        self._pending = []  # host arrays of enqueued asynchronous read-backs
        N.check(N.lib().cr_frame_create(context.handle, width, height, C.byref(self._h)))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h and self.context.handle:
            N.lib().cr_frame_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # Read-backs (synchronise the context's stream; row 0 = top).
    def rgba8(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.zeros((self.height, self.width, 4), np.uint8)
        elif out.nbytes < self.width * self.height * 4 or not out.flags.c_contiguous:
            raise CRError(1, "out is too small or not contiguous")
        N.check(N.lib().cr_frame_read_rgba8(self._h, N.ptr(out)))
        return out

    def rgba8_async(self, out: np.ndarray) -> np.ndarray:
        """Enqueues the RGBA8 read-back into `out` and returns at once; the
        array is held until wait()."""
        if out.nbytes < self.width * self.height * 4 or not out.flags.c_contiguous:
            raise CRError(1, "out is too small or not contiguous")
        N.check(N.lib().cr_frame_read_rgba8_async(self._h, N.ptr(out)))
        self._pending.append(out)
        return out

    def wait(self, keep: int = 0):
        """Waits until at most the `keep` most recent read-backs may still be
        in flight (0: all done); the arrays of the finished ones are released."""
        N.check(N.lib().cr_frame_read_wait_keep(self._h, int(keep)))
        del self._pending[:len(self._pending) - int(keep) if keep else None]

    def depth_f32(self) -> np.ndarray:
        out = np.zeros((self.height, self.width), np.float32)
        N.check(N.lib().cr_frame_read_depth_f32(self._h, N.ptr(out)))
        return out

    def pixels(self) -> np.ndarray:
        out = np.zeros((self.height, self.width), PIXEL_DTYPE)
        N.check(N.lib().cr_frame_read_pixels(self._h, N.ptr(out)))
        return out


class PerspectiveCamera:
    """A Satin-style perspective camera: right-handed view (looks down -Z) and
    a reverse-Z projection for Metal's [0, 1] clip depth (near -> 1, far -> 0)."""

    def __init__(self, position=(0.0, 0.0, 5.0), near: float = 0.1, far: float = 100.0,
                 fov: float = 45.0, aspect: float = 1.0):
        self.position = np.asarray(position, np.float64)
        self.near, self.far, self.fov, self.aspect = near, far, fov, aspect
        self.target = np.zeros(3)
        self.up = np.array([0.0, 1.0, 0.0])

    def lookAt(self, target, up=(0.0, 1.0, 0.0)):
        self.target = np.asarray(target, np.float64)
        self.up = np.asarray(up, np.float64)

    # The matrices are recomputed only when the pose or the lens changes (a
    # render loop reads them several times per frame).
    @property
    def viewMatrix(self) -> np.ndarray:
        key = (np.asarray(self.position, np.float64).tobytes(),
               np.asarray(self.target, np.float64).tobytes(),
               np.asarray(self.up, np.float64).tobytes())
        if getattr(self, "_view_key", None) != key:
            self._view = self._compute_view()
            self._view_key = key
        return self._view.copy()

    @property
    def projectionMatrix(self) -> np.ndarray:
        key = (self.near, self.far, self.fov, self.aspect)
        if getattr(self, "_proj_key", None) != key:
            self._proj = self._compute_projection()
            self._proj_key = key
        return self._proj.copy()

    def _compute_view(self) -> np.ndarray:
        f = self.target - self.position
        f = f / np.linalg.norm(f)
        s = np.cross(f, self.up)
        s = s / np.linalg.norm(s)
        u = np.cross(s, f)
        m = np.eye(4)
        m[0, :3], m[1, :3], m[2, :3] = s, u, -f
        m[0, 3], m[1, 3], m[2, 3] = -s @ self.position, -u @ self.position, f @ self.position
        return _mat16(m)

    def _compute_projection(self) -> np.ndarray:
        t = 1.0 / math.tan(math.radians(self.fov) * 0.5)
        n, fa = self.near, self.far
        m = np.zeros((4, 4))
        m[0, 0] = t / self.aspect
        m[1, 1] = t
        m[2, 2] = n / (fa - n)
        m[2, 3] = fa * n / (fa - n)
        m[3, 2] = -1.0
        return _mat16(m)


def _camera_c(camera) -> N.cr_camera:
    c = N.cr_camera()
    C.memmove(c.view, _mat16(camera.viewMatrix).ctypes.data, 64)
    C.memmove(c.projection, _mat16(camera.projectionMatrix).ctypes.data, 64)
    return c


class ComputeRasteriser:
    """ComputeRasteriser (ComputeRasteriser.swift:5-888): the per-frame render API.

    ``update`` sets the camera and refreshes every visible cloud's file
    table; ``encode`` enqueues the frame (HQS or nearest, then hole fill).
    Outputs are device buffers read back with ``outputRGBA8`` and friends.
    Per-viewport buffers are cached for the four most recent sizes
    (ComputeRasteriser.swift:43-53, 766-838).
    """
    resourceCacheCap = 4

    def __init__(self, context: Context, label: str = "ComputeRasteriser"):
        self.context = context
        self.label = label
        self.configuration = ComputeRasteriserConfiguration()
        self.visible = True
        self._clouds: list[ComputeRasteriserPointCloud] = []
        self._cache: dict[tuple, _Frame] = {}
        self._lru: list[tuple] = []
        self._frame: _Frame | None = None
        self._camera = None
        self._prev_vp: dict[int, np.ndarray] = {}

    def addPointCloud(self, cloud: ComputeRasteriserPointCloud) -> ComputeRasteriserPointCloud:
        self._clouds.append(cloud)
        return cloud

    def removePointCloud(self, cloud: ComputeRasteriserPointCloud):
        self._clouds = [c for c in self._clouds if c is not cloud]

    @property
    def pointClouds(self):
        return list(self._clouds)

    @property
    def visiblePointClouds(self):
        return [c for c in self._clouds if c.visible]

    def resize(self, size):
        w, h = int(size[0]), int(size[1])
        if w <= 0 or h <= 0:
            return
        key = (w, h)
        frame = self._cache.get(key)
        if frame is None:
            while len(self._lru) >= self.resourceCacheCap:
                old = self._lru.pop(0)
                self._cache.pop(old).close()
            frame = _Frame(self.context, w, h)
            self._cache[key] = frame
        if key in self._lru:
            self._lru.remove(key)
        self._lru.append(key)
        self._frame = frame

    @property
    def viewportSize(self):
        return None if self._frame is None else (self._frame.width, self._frame.height)

    def update(self, camera, viewport=None):
        """update(renderContext:camera:viewport:index:) (ComputeRasteriser.swift:201-268)."""
        if not self.visible:
            return
        if viewport is not None:
            w, h = int(viewport[-2]), int(viewport[-1])
            if self.viewportSize != (w, h):
                self.resize((w, h))
        self._camera = camera
        vp = matrix_multiply(camera.projectionMatrix, camera.viewMatrix)
        prev = self._prev_vp.get(id(camera), vp)
        for cloud in self.visiblePointClouds:
            cloud.updateFiles(vp, cloud.worldMatrix, prevViewProjection=prev)
        self._prev_vp[id(camera)] = vp

    def encode(self):
        """encode(_:) (ComputeRasteriser.swift:277-296)."""
        if not self.visible or self._frame is None or self._camera is None:
            return
        clouds = self.visiblePointClouds
        arr = (C.c_void_p * max(len(clouds), 1))(*[c.handle.value for c in clouds])
        cfg = self.configuration.to_c()
        cam = _camera_c(self._camera)
        N.check(N.lib().cr_render(self.context.handle, self._frame.handle, arr, len(clouds),
                                  C.byref(cfg), C.byref(cam)))

    def encodeStages(self, stages: int):
        """Some HQS stages of encode() (cr_render_stages): STAGE_DEPTH (clear,
        cull, depth pass), STAGE_COLOR (colour pass against the frame's depth
        plane), STAGE_RESOLVE (resolve, hole fill), or a union of them.  Used
        to combine several frames' planes between the stages (a frame split
        by points over GPUs, see sharded.PointShardedRasteriser)."""
        if not self.visible or self._frame is None or self._camera is None:
            return
        clouds = self.visiblePointClouds
        arr = (C.c_void_p * max(len(clouds), 1))(*[c.handle.value for c in clouds])
        cfg = self.configuration.to_c()
        cam = _camera_c(self._camera)
        N.check(N.lib().cr_render_stages(self.context.handle, self._frame.handle, arr,
                                         len(clouds), C.byref(cfg), C.byref(cam), int(stages)))

    def devicePlanes(self) -> dict:
        """Device pointers of the frame's depth plane (uint32 per pixel) and
        accumulators (uint32 R, G, B, count per pixel), the pixel count and
        the context's CUDA stream (cr_frame_device_planes)."""
        f = self._require_frame()
        pl = N.cr_frame_planes()
        N.check(N.lib().cr_frame_device_planes(f.handle, C.byref(pl)))
        return {"depth": pl.depth, "accum": pl.accum, "pixels": int(pl.pixels),
                "stream": pl.stream or 0, "device": self.context.device}

    def flipDepthOrder(self):
        """XOR the top bit of every depth word (cr_frame_flip_depth_order):
        unsigned depth order <-> signed int32 order, around an int32 max."""
        N.check(N.lib().cr_frame_flip_depth_order(self._require_frame().handle))

    # --- outputs (row 0 = top of the viewport) ---
    def outputRGBA8(self, out: np.ndarray | None = None) -> np.ndarray:
        """The final RGBA8 image (row 0 at the top); `out` may be a pinned HostBuffer array."""
        f = self._require_frame()
        if out is None:
            out = np.zeros((f.height, f.width, 4), np.uint8)
        elif out.nbytes < f.width * f.height * 4 or not out.flags.c_contiguous:
            raise CRError(1, "out is too small or not contiguous")
        N.check(N.lib().cr_frame_read_rgba8(f.handle, N.ptr(out)))
        return out

    def outputRGBA8Async(self, out: np.ndarray) -> np.ndarray:
        """Enqueues the read-back of the final RGBA8 image into `out` (page-locked
        host memory, e.g. HostBuffer((h, w, 4), np.uint8).array, for the copy
        to be asynchronous) and returns at once; `out` holds the image after
        waitOutput().  The next encode() into this frame waits on the device
        for the copy before its resolve rewrites the image, so a render loop
        that reads every frame keeps the GPU busy while the images travel."""
        return self._require_frame().rgba8_async(out)

    def waitOutput(self, keep: int = 0):
        """Waits for the read-backs enqueued by outputRGBA8Async: all of them,
        or all but the `keep` (at most 3) most recent."""
        self._require_frame().wait(keep)

    def depthTexture(self) -> np.ndarray:
        f = self._require_frame()
        out = np.zeros((f.height, f.width), np.float32)
        N.check(N.lib().cr_frame_read_depth_f32(f.handle, N.ptr(out)))
        return out

    def pixels(self) -> np.ndarray:
        f = self._require_frame()
        out = np.zeros((f.height, f.width), PIXEL_DTYPE)
        N.check(N.lib().cr_frame_read_pixels(f.handle, N.ptr(out)))
        return out

    def nearestDepths(self) -> np.ndarray:
        f = self._require_frame()
        out = np.zeros((f.height, f.width), np.uint32)
        N.check(N.lib().cr_frame_read_nearest_depth(f.handle, N.ptr(out)))
        return out

    def nearestIndices(self) -> np.ndarray:
        f = self._require_frame()
        out = np.zeros((f.height, f.width), np.uint32)
        N.check(N.lib().cr_frame_read_nearest_index(f.handle, N.ptr(out)))
        return out

    # --- differentiable colours (FP32 variant of the colour pass) ---
    def forwardF32(self, cloud: ComputeRasteriserPointCloud, colors: DeviceBuffer,
                   image: DeviceBuffer):
        """Image (height x width x 3 float32, device) of `cloud` with learnable
        colours (pool points x 3 float32, device) at the camera of the last
        update (cr_hqs_forward_f32)."""
        f = self._require_frame()
        cfg = self.configuration.to_c()
        cam = _camera_c(self._camera)
        N.check(N.lib().cr_hqs_forward_f32(self.context.handle, f.handle, cloud.handle,
                                           C.byref(cfg), C.byref(cam), C.c_void_p(colors.ptr),
                                           C.c_void_p(image.ptr)))

    def backwardColors(self, cloud: ComputeRasteriserPointCloud, dL_dimage: DeviceBuffer,
                       dL_dcolors: DeviceBuffer):
        """Adds dL/dcolors of the last forwardF32 to dL_dcolors (cr_hqs_backward_colors)."""
        f = self._require_frame()
        cfg = self.configuration.to_c()
        cam = _camera_c(self._camera)
        N.check(N.lib().cr_hqs_backward_colors(self.context.handle, f.handle, cloud.handle,
                                               C.byref(cfg), C.byref(cam),
                                               C.c_void_p(dL_dimage.ptr),
                                               C.c_void_p(dL_dcolors.ptr)))

    def pickPointIndex(self, atNDC, cloud: ComputeRasteriserPointCloud, camera,
                       searchRadius: int = 10):
        """pickPointIndex(atNDC:in:camera:searchRadius:) (ComputeRasteriser.swift:609-670)."""
        if self._frame is None or cloud.residentBatchCount == 0:
            return None
        vp = matrix_multiply(camera.projectionMatrix, camera.viewMatrix)
        cloud.updateFiles(vp, cloud.worldMatrix)
        ndc = np.asarray(atNDC, np.float32)
        cfg = self.configuration.to_c()
        cam = _camera_c(camera)
        idx = C.c_uint32()
        found = C.c_int()
        N.check(N.lib().cr_pick(self.context.handle, self._frame.handle, cloud.handle,
                                N.ptr(ndc), C.byref(cfg), C.byref(cam), int(searchRadius),
                                C.byref(idx), C.byref(found)))
        return int(idx.value) if found.value else None

    def _require_frame(self) -> _Frame:
        if self._frame is None:
            raise CRError(1, "no viewport: call resize or update first")
        return self._frame


class _UserAttributePass:
    """Shared machinery of DisplacementPass and TintPass (DisplacementPass.swift,
    TintPass.swift): per frame, make sure the target cloud has the attribute
    buffer, run the user kernel on the library's stream with the cloud's
    device arrays and the output buffer, and switch the variant on in the
    rasteriser's configuration.  The kernel is any Python callable that
    launches CUDA work (a torch / CuPy / numba kernel, a custom extension):
        kernel(arrays: dict, out: DeviceView, stream: int, **user)
    with arrays from ComputeRasteriserPointCloud.deviceArrays() and stream the
    context's cudaStream_t (the kernel must run on it, or synchronise)."""

    _which = ATTR_DISPLACEMENT

    def __init__(self, rasteriser: ComputeRasteriser, kernel, **user):
        self.rasteriser = rasteriser
        self.kernel = kernel
        self.user = user

    def _flip(self, cfg):
        raise NotImplementedError

    def encode(self, cloud: ComputeRasteriserPointCloud | None = None):
        """Runs the kernel for `cloud` (default: the rasteriser's first cloud);
        call before encode() so the frame sees this frame's values."""
        target = cloud or (self.rasteriser.pointClouds[0] if self.rasteriser.pointClouds
                           else None)
        if target is None:
            return
        out = target._attribute(self._which)
        self.kernel(target.deviceArrays(), out, self.rasteriser.context.stream(), **self.user)
        self._flip(self.rasteriser.configuration)


class DisplacementPass(_UserAttributePass):
    """Per-point displacement written by a user kernel (xyz added to each
    decoded position; a NaN component drops the point); sets
    configuration.applyDisplacement."""

    _which = ATTR_DISPLACEMENT

    def _flip(self, cfg):
        cfg.applyDisplacement = True


class TintPass(_UserAttributePass):
    """Per-point tint written by a user kernel (rgba: mix weight a, a < 0
    drops the point's colour); sets configuration.applyTint, and with
    alphaIsCoverage tintAlphaIsCoverage (translucent defocus: a is the
    circle of confusion, coverage = 1 - a, weighted-blended accumulation)."""

    _which = ATTR_TINT

    def __init__(self, rasteriser, kernel, alphaIsCoverage: bool = False, **user):
        super().__init__(rasteriser, kernel, **user)
        self.alphaIsCoverage = alphaIsCoverage

    def _flip(self, cfg):
        cfg.applyTint = True
        cfg.tintAlphaIsCoverage = bool(self.alphaIsCoverage)


class MultiViewRasteriser:
    """Batched HQS rendering of many views of the same clouds in one CUDA-graph
    launch (cr_render_multiview); no counterpart in the reference, whose
    ComputeRasteriser draws one viewport per encode.

    ``sizes`` fixes the views' (width, height); ``render(cameras)`` draws view
    i with cameras[i] into its own frame, bit-identical to a ComputeRasteriser
    update + encode of that camera at that size.  ``autotune`` picks the
    launch shape (cr_autotune_multiview), optionally cached in a JSON-lines
    file.
    """

    def __init__(self, context: Context, sizes):
        sizes = list(sizes)
        if not 1 <= len(sizes) <= 256:
            raise CRError(1, "between 1 and 256 views")
        self.context = context
        self.configuration = ComputeRasteriserConfiguration()
        self._clouds: list[ComputeRasteriserPointCloud] = []
        self.frames = [_Frame(context, int(w), int(h)) for w, h in sizes]

    def addPointCloud(self, cloud: ComputeRasteriserPointCloud) -> ComputeRasteriserPointCloud:
        self._clouds.append(cloud)
        return cloud

    def removePointCloud(self, cloud: ComputeRasteriserPointCloud):
        self._clouds = [c for c in self._clouds if c is not cloud]

    @property
    def viewCount(self) -> int:
        return len(self.frames)

    def _args(self, cameras):
        if len(cameras) != len(self.frames):
            raise CRError(1, "one camera per view")
        frames = (C.c_void_p * len(self.frames))(*[f.handle.value for f in self.frames])
        cams = (N.cr_camera * len(cameras))(*[_camera_c(c) for c in cameras])
        clouds = [c for c in self._clouds if c.visible]
        arr = (C.c_void_p * max(len(clouds), 1))(*[c.handle.value for c in clouds])
        models = np.zeros((max(len(clouds), 1), 16), np.float32)
        for i, c in enumerate(clouds):
            models[i] = _mat16(c.worldMatrix)
        return frames, cams, arr, len(clouds), models

    def render(self, cameras):
        frames, cams, arr, n, models = self._args(cameras)
        cfg = self.configuration.to_c()
        N.check(N.lib().cr_render_multiview(self.context.handle, frames, cams, len(self.frames),
                                            arr, N.ptr(models), n, C.byref(cfg)))

    def autotune(self, cameras, cachePath: str | None = None, reps: int = 5) -> dict:
        frames, cams, arr, n, models = self._args(cameras)
        cfg = self.configuration.to_c()
        best = N.cr_tuning()
        ms = C.c_float()
        path = None if cachePath is None else os.fsencode(cachePath)
        N.check(N.lib().cr_autotune_multiview(self.context.handle, frames, cams,
                                              len(self.frames), arr, N.ptr(models), n,
                                              C.byref(cfg), path, int(reps), C.byref(best),
                                              C.byref(ms)))
        return {"chunkPoints": best.chunkPoints, "useTiles": bool(best.useTiles),
                "viewGroupPixels": best.viewGroupPixels, "ms": float(ms.value)}

    def outputRGBA8(self, view: int, out: np.ndarray | None = None) -> np.ndarray:
        return self.frames[view].rgba8(out)

    def depthTexture(self, view: int) -> np.ndarray:
        return self.frames[view].depth_f32()

    def pixels(self, view: int) -> np.ndarray:
        return self.frames[view].pixels()

    def close(self):
        for f in self.frames:
            f.close()


def l2_loss(context: Context, image: DeviceBuffer, target: DeviceBuffer, scale: float,
            dL_dimage: DeviceBuffer, want_loss: bool = True):
    """dL_dimage = 2 * scale * (image - target); returns scale * sum (image -
    target)^2 (FP64, synchronises) when want_loss (cr_l2_loss)."""
    n = image.nbytes // 4
    loss = C.c_double()
    N.check(N.lib().cr_l2_loss(context.handle, C.c_void_p(image.ptr), C.c_void_p(target.ptr), n,
                               float(scale), C.c_void_p(dL_dimage.ptr),
                               C.byref(loss) if want_loss else None))
    return loss.value if want_loss else None


from .ply import PLYPointCloudLoader, PLYPointCloudLoaderError  # noqa: E402
