"""CPU oracle of the point-cloud compute rasteriser (test infrastructure).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this package, and only as the checker.  It wraps
``oracle/_build/liboracle.so`` (built by ``oracle/Makefile`` from the C++
restatement in ``cr_oracle.cpp`` / ``cr_oracle_pack.cpp``) with numpy.

Parity is pinned against the reference's own known-answer tests
(Tests/SatinComputeRasteriserTests/NearestPointReferenceTests.swift:5-62,
LayoutTests.swift:5-134, LODBucketingTests.swift:50-153) restated in
``tests/test_oracle_known_answers.py``; the reference itself (Swift + Metal)
cannot be built or run on Linux, so no output of it is available.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class orc_batch(C.Structure):
    _fields_ = [("state", C.c_int32)] + [(n, C.c_float) for n in
                                         ("minX", "minY", "minZ", "maxX", "maxY", "maxZ")] + \
               [(n, C.c_uint32) for n in ("numPoints", "firstPoint", "fileIndex", "lodCum01",
                                          "lodCum23", "lodCum45", "lodCum67", "padding7",
                                          "padding8")]


class orc_file(C.Structure):
    _fields_ = [("transform", C.c_float * 16), ("transformFrustum", C.c_float * 16),
                ("world", C.c_float * 16), ("prevTransform", C.c_float * 16)]


class orc_visible(C.Structure):
    _fields_ = [("batchIndex", C.c_uint32), ("level", C.c_int32), ("lodThreshold", C.c_float),
                ("activePoints", C.c_uint32)]


class orc_config(C.Structure):
    _fields_ = [("mode", C.c_int32), ("depthTolerance", C.c_float),
                ("backgroundColor", C.c_float * 4), ("enableFrustumCulling", C.c_int32),
                ("lodBias", C.c_int32), ("enableCLOD", C.c_int32), ("enableLODDither", C.c_int32),
                ("holeFillIterations", C.c_int32), ("colorizeChunks", C.c_int32),
                ("colorizeOverdraw", C.c_int32), ("pointSizeMode", C.c_int32),
                ("minimumPointSize", C.c_float), ("maximumPointSize", C.c_float),
                ("pointSizeScale", C.c_float), ("applyDisplacement", C.c_int32),
                ("applyTint", C.c_int32), ("tintAlphaIsCoverage", C.c_int32),
                ("motionBlur", C.c_float), ("motionBlurSamples", C.c_int32),
                ("motionBlurMaxSpread", C.c_float)]


class orc_cloud(C.Structure):
    _fields_ = [("batches", C.POINTER(orc_batch)), ("batchCount", C.c_uint32),
                ("files", C.POINTER(orc_file)), ("fileCount", C.c_uint32),
                ("xyzLow", C.POINTER(C.c_uint32)), ("xyzMed", C.POINTER(C.c_uint32)),
                ("xyzHigh", C.POINTER(C.c_uint32)), ("colors", C.POINTER(C.c_uint32)),
                ("levels", C.POINTER(C.c_uint8)), ("displacements", C.c_void_p),
                ("prevDisplacements", C.c_void_p), ("tints", C.c_void_p)]


# numpy dtypes with the same layouts (RasterBatch 64 B, RasterFile 256 B, VisibleBatch 16 B).
BATCH_DTYPE = np.dtype([("state", "<i4"), ("minX", "<f4"), ("minY", "<f4"), ("minZ", "<f4"),
                        ("maxX", "<f4"), ("maxY", "<f4"), ("maxZ", "<f4"),
                        ("numPoints", "<u4"), ("firstPoint", "<u4"), ("fileIndex", "<u4"),
                        ("lodCum01", "<u4"), ("lodCum23", "<u4"), ("lodCum45", "<u4"),
                        ("lodCum67", "<u4"), ("padding7", "<u4"), ("padding8", "<u4")])
FILE_DTYPE = np.dtype([("transform", "<f4", 16), ("transformFrustum", "<f4", 16),
                       ("world", "<f4", 16), ("prevTransform", "<f4", 16)])
VISIBLE_DTYPE = np.dtype([("batchIndex", "<u4"), ("level", "<i4"), ("lodThreshold", "<f4"),
                          ("activePoints", "<u4")])


class orc_terrain(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("extent", C.c_float), ("amplitude", C.c_float),
                ("baseWavelength", C.c_float), ("octaves", C.c_int32), ("lacunarity", C.c_float),
                ("gain", C.c_float), ("outlierFraction", C.c_float),
                ("outlierMargin", C.c_float), ("colorNoiseSigma", C.c_float)]


@dataclass
class Terrain:
    """Parameters of the seeded fractal heightfield (the library's defaults)."""
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

    def to_c(self) -> orc_terrain:
        return orc_terrain(self.seed, self.extent, self.amplitude, self.baseWavelength,
                           self.octaves, self.lacunarity, self.gain, self.outlierFraction,
                           self.outlierMargin, self.colorNoiseSigma)


def terrain_height(t: Terrain, x: float, y: float) -> float:
    """Height of the heightfield's noise surface at (x, y)."""
    return float(_load().orc_terrain_height(C.byref(t.to_c()), x, y))


def synth_terrain(t: Terrain, count: int, first: int = 0, threads: int = 1) -> np.ndarray:
    """(count, 4) float32 records {x, y, z, rgba8 bits} of points [first, first+count),
    bit-identical to the library's device generator."""
    out = np.empty((count, 4), np.float32)
    if _load().orc_synth_terrain(C.byref(t.to_c()), first, count, _ptr(out), threads) != 0:
        raise ValueError("bad terrain parameters")
    return out


def synth_lattice(n_axis: int, seed: int = 0xC0FFEE01, lo: float = -1.0, hi: float = 1.0,
                  jitter: float = 0.002, threads: int = 1) -> np.ndarray:
    """(n^3, 4) float32 records of the jittered lattice, bit-identical to the
    library's device generator."""
    out = np.empty((n_axis ** 3, 4), np.float32)
    _load().orc_synth_lattice(seed, n_axis, lo, hi, jitter, _ptr(out), threads)
    return out


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = C.CDLL(_LIB_PATH)
    P = C.c_void_p
    lib.orc_log2f.restype = C.c_float
    lib.orc_log2f.argtypes = [C.c_float]
    lib.orc_exp_neg.restype = C.c_float
    lib.orc_exp_neg.argtypes = [C.c_float]
    lib.orc_hash_unit.restype = C.c_float
    lib.orc_hash_unit.argtypes = [C.c_uint32]
    lib.orc_depth_to_uint.restype = C.c_uint32
    lib.orc_depth_to_uint.argtypes = [C.c_float]
    lib.orc_mat4_mul.argtypes = [P, P, P]
    lib.orc_update_files.argtypes = [P, C.c_uint32, P, P, P, P, P]
    lib.orc_cull.restype = C.c_uint32
    lib.orc_cull.argtypes = [C.POINTER(orc_cloud), C.POINTER(orc_config), P, P, C.c_int,
                             C.c_int, P, C.c_uint32]
    lib.orc_render.restype = C.c_int
    lib.orc_render.argtypes = [C.POINTER(orc_cloud), C.c_uint32, C.POINTER(orc_config), P, P,
                               C.c_int, C.c_int, P, P, P, P, P, P, P, C.c_uint32, P, C.c_int]
    lib.orc_hole_fill.argtypes = [P, C.c_int, C.c_int, C.c_int]
    lib.orc_hqs_stage.restype = C.c_int
    lib.orc_hqs_stage.argtypes = [C.POINTER(orc_cloud), C.c_uint32, C.POINTER(orc_config), P, P,
                                  C.c_int, C.c_int, C.c_uint32, P, P, P, P, C.c_int]
    lib.orc_hqs_grad_f64.restype = C.c_int
    lib.orc_hqs_grad_f64.argtypes = [C.POINTER(orc_cloud), C.POINTER(orc_config), P, P,
                                     C.c_int, C.c_int, P, P, C.c_double, P, P, P, P,
                                     C.c_uint32, C.c_double, P, C.c_int]
    lib.orc_nearest_cpu_reference.argtypes = [C.POINTER(orc_cloud), C.c_int, C.c_int, P, P,
                                              C.c_int, P, P]
    lib.orc_pick_scan.restype = C.c_int
    lib.orc_pick_scan.argtypes = [P, C.c_int, C.c_int, P, C.c_int, P]
    lib.orc_pack.restype = C.c_int
    lib.orc_pack.argtypes = [P, P, P, C.c_uint64, C.c_uint32, C.c_int, C.c_int, C.c_int,
                             P, P, P, P, P, P, P, P, P]
    lib.orc_pack_threads.restype = C.c_int
    lib.orc_pack_threads.argtypes = [P, P, P, C.c_uint64, C.c_uint32, C.c_int, C.c_int, C.c_int,
                                     P, P, P, P, P, P, P, P, P, C.c_int]
    lib.orc_terrain_height.restype = C.c_float
    lib.orc_terrain_height.argtypes = [C.POINTER(orc_terrain), C.c_float, C.c_float]
    lib.orc_synth_terrain.restype = C.c_int
    lib.orc_synth_terrain.argtypes = [C.POINTER(orc_terrain), C.c_uint64, C.c_uint64, P, C.c_int]
    lib.orc_synth_lattice.restype = C.c_int
    lib.orc_synth_lattice.argtypes = [C.c_uint64, C.c_uint32, C.c_float, C.c_float, C.c_float, P,
                                      C.c_int]
    lib.orc_ln_unit.restype = C.c_float
    lib.orc_ln_unit.argtypes = [C.c_float]
    lib.orc_cos_2pi.restype = C.c_float
    lib.orc_cos_2pi.argtypes = [C.c_float]
    _lib = lib
    return lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _mat(m):
    m = np.ascontiguousarray(np.asarray(m, dtype=np.float32).reshape(16))
    return m


def log2f(x: float) -> float:
    return _load().orc_log2f(x)


def exp_neg(x: float) -> float:
    """The project's e^-x (x >= 0) shared by the coverage resolve and the oracle."""
    return _load().orc_exp_neg(x)


def hash_unit(x: int) -> float:
    return _load().orc_hash_unit(x)


def depth_to_uint(z: float) -> int:
    return _load().orc_depth_to_uint(z)


def mat4_mul(a, b):
    out = np.zeros(16, np.float32)
    a, b = _mat(a), _mat(b)
    _load().orc_mat4_mul(_ptr(a), _ptr(b), _ptr(out))
    return out


def identity_file():
    f = np.zeros(1, FILE_DTYPE)
    eye = np.eye(4, dtype=np.float32).reshape(16)
    for k in FILE_DTYPE.names:
        f[k][0] = eye
    return f


def update_files(base_files, vp, model, frustum=None, prev_vp=None):
    """updateFiles (ComputeRasteriserPointCloud.swift:487-515) on a FILE_DTYPE array."""
    base = np.ascontiguousarray(base_files, dtype=FILE_DTYPE)
    out = np.zeros_like(base)
    vp, model = _mat(vp), _mat(model)
    fr = None if frustum is None else _mat(frustum)
    pv = None if prev_vp is None else _mat(prev_vp)
    _load().orc_update_files(_ptr(base), len(base), _ptr(vp), _ptr(model), _ptr(fr), _ptr(pv),
                             _ptr(out))
    return out


@dataclass
class Config:
    """Mirror of the pass-relevant ComputeRasteriserConfiguration fields and defaults
    (ComputeRasteriserTypes.swift:97-119)."""
    mode: int = 0
    depthTolerance: float = 0.01
    backgroundColor: tuple = (0.0, 0.0, 0.0, 0.0)
    enableFrustumCulling: bool = True
    lodBias: int = 0
    enableCLOD: bool = True
    enableLODDither: bool = True
    holeFillIterations: int = 0
    colorizeChunks: bool = False
    colorizeOverdraw: bool = False
    pointSizeMode: int = 0
    minimumPointSize: float = 1.0
    maximumPointSize: float = 1.0
    pointSizeScale: float = 1.0
    applyDisplacement: bool = False
    applyTint: bool = False
    tintAlphaIsCoverage: bool = False
    motionBlur: float = 0.0
    motionBlurSamples: int = 8
    motionBlurMaxSpread: float = 64.0

    def to_c(self) -> orc_config:
        c = orc_config()
        for name, _ in orc_config._fields_:
            v = getattr(self, name)
            if name == "backgroundColor":
                c.backgroundColor[:] = [float(x) for x in v]
            else:
                setattr(c, name, type(getattr(c, name))(v) if not isinstance(v, bool) else int(v))
        return c


@dataclass
class Cloud:
    """A slot pool as the device holds it (the arrays cull/draw passes read)."""
    batches: np.ndarray
    files: np.ndarray
    xyzLow: np.ndarray
    xyzMed: np.ndarray
    xyzHigh: np.ndarray
    colors: np.ndarray
    levels: np.ndarray
    displacements: np.ndarray | None = None      # float32 [points, 4]
    prevDisplacements: np.ndarray | None = None  # float32 [points, 4]
    tints: np.ndarray | None = None              # float32 [points, 4]
    _keep: list = field(default_factory=list, repr=False)

    def to_c(self) -> orc_cloud:
        arrs = [np.ascontiguousarray(self.batches, dtype=BATCH_DTYPE),
                np.ascontiguousarray(self.files, dtype=FILE_DTYPE),
                np.ascontiguousarray(self.xyzLow, dtype=np.uint32),
                np.ascontiguousarray(self.xyzMed, dtype=np.uint32),
                np.ascontiguousarray(self.xyzHigh, dtype=np.uint32),
                np.ascontiguousarray(self.colors, dtype=np.uint32),
                np.ascontiguousarray(self.levels, dtype=np.uint8)]
        self._keep = arrs
        c = orc_cloud()
        c.batches = arrs[0].ctypes.data_as(C.POINTER(orc_batch))
        c.batchCount = len(arrs[0])
        c.files = arrs[1].ctypes.data_as(C.POINTER(orc_file))
        c.fileCount = len(arrs[1])
        c.xyzLow = arrs[2].ctypes.data_as(C.POINTER(C.c_uint32))
        c.xyzMed = arrs[3].ctypes.data_as(C.POINTER(C.c_uint32))
        c.xyzHigh = arrs[4].ctypes.data_as(C.POINTER(C.c_uint32))
        c.colors = arrs[5].ctypes.data_as(C.POINTER(C.c_uint32))
        c.levels = arrs[6].ctypes.data_as(C.POINTER(C.c_uint8))
        for name in ("displacements", "prevDisplacements", "tints"):
            a = getattr(self, name)
            if a is not None:
                a = np.ascontiguousarray(a, dtype=np.float32).reshape(-1, 4)
                self._keep.append(a)
                setattr(c, name, a.ctypes.data)
        return c


@dataclass
class Packed:
    """PackedPointCloud (ComputeRasteriserTypes.swift:269-320)."""
    batches: np.ndarray
    files: np.ndarray
    xyzLow: np.ndarray
    xyzMed: np.ndarray
    xyzHigh: np.ndarray
    colors: np.ndarray
    levels: np.ndarray
    boundsMin: np.ndarray
    boundsMax: np.ndarray
    orderedPositions: np.ndarray
    sourceIndices: np.ndarray

    @property
    def pointCount(self) -> int:
        return len(self.colors)

    @property
    def batchCount(self) -> int:
        return len(self.batches)

    def cloud(self, files=None) -> Cloud:
        return Cloud(self.batches, self.files if files is None else files, self.xyzLow,
                     self.xyzMed, self.xyzHigh, self.colors, self.levels)


def pack(positions, colors=None, colors_rgba8=None, pointsPerBatch: int = 10240,
         lodLevels: int = 4, coarseVoxelDivisions: int = 64, morton_bits: int = 10,
         threads: int = 1) -> Packed:
    """PackedPointCloudFixtures.pack (PackedPointCloudFixtures.swift:30-167).

    threads > 1 runs the bit-identical multi-threaded pack (orc_pack_threads)."""
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float32).reshape(-1, 3))
    n = len(pos)
    if n == 0:
        return Packed(np.zeros(0, BATCH_DTYPE), identity_file(), *(np.zeros(0, np.uint32),) * 4,
                      np.zeros(0, np.uint8), np.zeros(3, np.float32), np.zeros(3, np.float32),
                      np.zeros((0, 3), np.float32), np.zeros(0, np.uint32))
    cf = None if colors is None else np.ascontiguousarray(
        np.asarray(colors, dtype=np.float32).reshape(-1, 4))
    c8 = None if colors_rgba8 is None else np.ascontiguousarray(colors_rgba8, dtype=np.uint32)
    if cf is None and c8 is None:
        raise ValueError("colors or colors_rgba8 required")
    if (cf is not None and len(cf) != n) or (c8 is not None and len(c8) != n):
        raise ValueError("positions and colors must have the same count")
    nb = (n + pointsPerBatch - 1) // pointsPerBatch
    batches = np.zeros(nb, BATCH_DTYPE)
    low, med, high, cols = (np.zeros(n, np.uint32) for _ in range(4))
    levels = np.zeros(n, np.uint8)
    src = np.zeros(n, np.uint32)
    opos = np.zeros((n, 3), np.float32)
    bounds = np.zeros(6, np.float32)
    args = (_ptr(pos), _ptr(cf), _ptr(c8), n, pointsPerBatch, lodLevels, coarseVoxelDivisions,
            morton_bits, _ptr(batches), _ptr(low), _ptr(med), _ptr(high), _ptr(cols),
            _ptr(levels), _ptr(src), _ptr(opos), _ptr(bounds))
    rc = _load().orc_pack(*args) if threads <= 1 else _load().orc_pack_threads(*args, threads)
    if rc != 0:
        raise ValueError(f"orc_pack failed ({rc})")
    return Packed(batches, identity_file(), low, med, high, cols, levels, bounds[:3].copy(),
                  bounds[3:].copy(), opos, src)


def cube_grid(pointsPerAxis: int = 24) -> Packed:
    """PackedPointCloudFixtures.cubeGrid (PackedPointCloudFixtures.swift:5-25)."""
    n = max(pointsPerAxis, 2)
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    fx = x.reshape(-1).astype(np.float32) / np.float32(n - 1)
    fy = y.reshape(-1).astype(np.float32) / np.float32(n - 1)
    fz = z.reshape(-1).astype(np.float32) / np.float32(n - 1)
    pos = np.stack([fx - np.float32(0.5), fy - np.float32(0.5), fz - np.float32(0.5)], 1)
    col = np.stack([fx, fy, fz, np.ones_like(fx)], 1)
    return pack(pos, col)


def cull(cloud: Cloud, cfg: Config, view, proj, width: int, height: int) -> np.ndarray:
    cc = cloud.to_c()
    out = np.zeros(max(len(cloud.batches), 1), VISIBLE_DTYPE)
    c = cfg.to_c()
    v, p = _mat(view), _mat(proj)
    n = _load().orc_cull(C.byref(cc), C.byref(c), _ptr(v), _ptr(p), width, height, _ptr(out),
                         len(out))
    return out[:n].copy()


@dataclass
class Frame:
    rgba: np.ndarray
    depthf: np.ndarray
    depth: np.ndarray | None = None
    accum: np.ndarray | None = None
    nearest_depth: np.ndarray | None = None
    nearest_index: np.ndarray | None = None
    visible: list | None = None
    rc: int = 0


def render(clouds, cfg: Config, view, proj, width: int, height: int, threads: int = 1) -> Frame:
    """Full frame (ComputeRasteriser.encode, ComputeRasteriser.swift:277-553)."""
    if isinstance(clouds, Cloud):
        clouds = [clouds]
    ccs = (orc_cloud * max(len(clouds), 1))()
    for i, cl in enumerate(clouds):
        ccs[i] = cl.to_c()
    c = cfg.to_c()
    v, p = _mat(view), _mat(proj)
    npix = width * height
    depth = np.zeros(npix, np.uint32)
    accum = np.zeros(npix * 4, np.uint32)
    nd = np.zeros(npix, np.uint32)
    ni = np.full(npix, 0xFFFFFFFF, np.uint32)
    rgba = np.zeros(npix * 4, np.uint8)
    depthf = np.zeros(npix, np.float32)
    stride = max([len(cl.batches) for cl in clouds] + [1])
    vis = np.zeros(max(len(clouds), 1) * stride, VISIBLE_DTYPE)
    vcount = np.zeros(max(len(clouds), 1), np.uint32)
    rc = _load().orc_render(ccs, len(clouds), C.byref(c), _ptr(v), _ptr(p), width, height,
                            _ptr(depth), _ptr(accum), _ptr(nd), _ptr(ni), _ptr(rgba),
                            _ptr(depthf), _ptr(vis), stride, _ptr(vcount), threads)
    visible = [vis[i * stride:i * stride + vcount[i]].copy() for i in range(len(clouds))]
    return Frame(rgba.reshape(height, width, 4), depthf.reshape(height, width),
                 depth.reshape(height, width), accum.reshape(height, width, 4),
                 nd.reshape(height, width), ni.reshape(height, width), visible, rc)


def hqs_stage(clouds, cfg: Config, view, proj, width: int, height: int, stage: int,
              depth: np.ndarray, accum: np.ndarray, rgba: np.ndarray | None = None,
              depthf: np.ndarray | None = None, threads: int = 1) -> None:
    """One HQS stage of a frame split by points (cr_render_stages): 1 = clear,
    cull and depth pass into depth (uint32[h*w]); 2 = cull and colour pass
    against depth, added into accum (uint32[h*w*4]); 4 = resolve and hole fill
    into rgba (uint8[h*w*4]) and depthf (float32[h*w]).  The arrays must be
    C-contiguous and are written in place."""
    if isinstance(clouds, Cloud):
        clouds = [clouds]
    for a, dt, n in ((depth, np.uint32, width * height), (accum, np.uint32, width * height * 4)):
        if a.dtype != dt or a.size != n or not a.flags.c_contiguous:
            raise ValueError("depth / accum: wrong dtype, size or layout")
    ccs = (orc_cloud * max(len(clouds), 1))()
    for i, cl in enumerate(clouds):
        ccs[i] = cl.to_c()
    c = cfg.to_c()
    v, p = _mat(view), _mat(proj)
    rc = _load().orc_hqs_stage(ccs, len(clouds), C.byref(c), _ptr(v), _ptr(p), width, height,
                               stage, _ptr(depth), _ptr(accum),
                               None if rgba is None else _ptr(rgba),
                               None if depthf is None else _ptr(depthf), threads)
    if rc != 0:
        raise ValueError(f"orc_hqs_stage failed ({rc})")


def hqs_grad_f64(cloud: Cloud, cfg: Config, view, proj, width: int, height: int, colors,
                 target, scale: float, grad=None, fd_points=None, fd_h: float = 1e-3,
                 fd=None, threads: int = 1) -> dict:
    """Differentiable HQS colours in FP64 for one view (orc_hqs_grad_f64):
    colours (pool points x 3) and target (height x width x 3) in float64.
    Returns the image, the loss, and grad / fd, which accumulate into the
    arrays given (several views)."""
    cc = cloud.to_c()
    c = cfg.to_c()
    v, p = _mat(view), _mat(proj)
    colors = np.ascontiguousarray(colors, np.float64)
    target = np.ascontiguousarray(target, np.float64)
    image = np.zeros((height, width, 3), np.float64)
    loss = np.zeros(1, np.float64)
    if grad is None:
        grad = np.zeros_like(colors)
    pts = None if fd_points is None else np.ascontiguousarray(fd_points, np.uint32)
    n_fd = 0 if pts is None else len(pts)
    if n_fd and fd is None:
        fd = np.zeros((n_fd, 3), np.float64)
    rc = _load().orc_hqs_grad_f64(C.byref(cc), C.byref(c), _ptr(v), _ptr(p), width, height,
                                  _ptr(colors), _ptr(target), float(scale), _ptr(image),
                                  _ptr(loss), _ptr(grad), _ptr(pts), n_fd, float(fd_h),
                                  _ptr(fd) if n_fd else None, threads)
    if rc:
        raise RuntimeError(f"orc_hqs_grad_f64 failed ({rc})")
    return {"image": image, "loss": float(loss[0]), "grad": grad, "fd": fd}


def hole_fill(rgba: np.ndarray, iterations: int) -> np.ndarray:
    img = np.ascontiguousarray(rgba, dtype=np.uint8).copy()
    h, w = img.shape[:2]
    _load().orc_hole_fill(_ptr(img), w, h, iterations)
    return img


def nearest_cpu_reference(cloud: Cloud, width: int, height: int, view=None, proj=None,
                          enable_frustum: bool = False):
    """NearestPointCPUReference.render (NearestPointCPUReference.swift:16-81)."""
    view = np.eye(4, dtype=np.float32) if view is None else view
    proj = np.eye(4, dtype=np.float32) if proj is None else proj
    cc = cloud.to_c()
    npix = max(width, 0) * max(height, 0)
    d = np.zeros(max(npix, 1), np.uint32)
    ix = np.zeros(max(npix, 1), np.uint32)
    v, p = _mat(view), _mat(proj)
    _load().orc_nearest_cpu_reference(C.byref(cc), width, height, _ptr(v), _ptr(p),
                                      int(enable_frustum), _ptr(d), _ptr(ix))
    return d[:npix], ix[:npix]


def pick_scan(nindex: np.ndarray, ndc, radius: int = 10):
    idx = np.ascontiguousarray(nindex, dtype=np.uint32)
    h, w = idx.shape
    nd = np.asarray(ndc, dtype=np.float32)
    out = np.zeros(1, np.uint32)
    found = _load().orc_pick_scan(_ptr(idx), w, h, _ptr(nd), radius, _ptr(out))
    return int(out[0]) if found else None
