"""The allocation-free cull (cr_cull_noalloc) against the cull cr_render runs.

Callers that cannot allocate device memory (plug-ins whose host application
owns every device allocation, real-time loops that cannot take cudaMalloc's
device-wide synchronisation mid-frame) pass their own device arrays to
cr_cull_noalloc, whose scratch is a fixed array inside the library.  This
test calls it through the C ABI twice in a row on the same inputs and
requires both results to equal, bit for bit, the ordered survivor list that
the regular render path's cull produced for the same cloud and camera.  It
lives in its own file, collected last, so a failure here leaves every other
test already run.
"""
import ctypes as C
import importlib

import numpy as np
import pytest

from scenes import blob_cloud, to_product_packed

pytestmark = pytest.mark.gpu


def test_cull_noalloc_matches_render_cull(cr, orc):
    native = importlib.import_module("satin-computerasteriser_b200._native")
    ctx = cr.Context(0)
    pos, rgba = blob_cloud(200000, 44, scale=3.0)
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=300)
    cloud = cr.ComputeRasteriserPointCloud(ctx, packed=to_product_packed(cr, packed))
    cloud.removeBatches(list(range(0, cloud.batchCount, 7)))  # some empty slots
    w, h = 640, 360
    cam = cr.PerspectiveCamera(position=(0.4, 0.3, 2.0), near=0.01, far=100.0, fov=60.0,
                               aspect=w / h)
    cam.lookAt((0.0, 0.0, 0.0))
    cfg = cr.ComputeRasteriserConfiguration(lodBias=1)
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cfg
    ras.addPointCloud(cloud)
    ras.resize((w, h))
    ras.update(cam)
    ras.encode()
    expect = cloud.visibleBatches()
    assert 20 < len(expect) < cloud.residentBatchCount

    batches = cloud.batches()
    files = cloud.files()
    d_batches = cr.DeviceBuffer(ctx, batches.nbytes)
    d_batches.upload(batches)
    d_files = cr.DeviceBuffer(ctx, files.nbytes)
    d_files.upload(files)
    d_visible = cr.DeviceBuffer(ctx, len(batches) * cr.VISIBLE_DTYPE.itemsize,
                                (len(batches),), cr.VISIBLE_DTYPE)
    d_count = cr.DeviceBuffer(ctx, 4, (1,), np.uint32)
    ccfg = cfg.to_c()
    ccam = native.cr_camera()
    ccam.view[:] = cr._mat16(cam.viewMatrix).tolist()
    ccam.projection[:] = cr._mat16(cam.projectionMatrix).tolist()
    lib = native.lib()
    for _ in range(2):
        d_visible.upload(np.full(d_visible.nbytes, 0xFF, np.uint8))  # stale contents
        st = lib.cr_cull_noalloc(C.c_void_p(d_batches.ptr), len(batches), C.c_void_p(d_files.ptr),
                                 len(files), C.byref(ccfg), C.byref(ccam), w, h,
                                 C.c_void_p(d_visible.ptr), C.c_void_p(d_count.ptr),
                                 C.c_void_p(ctx.stream()))
        native.check(st)
        count = int(d_count.download()[0])
        got = d_visible.download()[:count]
        assert count == len(expect)
        assert got.tobytes() == expect.tobytes()


def test_cull_noalloc_rejects_oversized_input(cr):
    native = importlib.import_module("satin-computerasteriser_b200._native")
    lib = native.lib()
    ctx = cr.Context(0)
    ccfg = cr.ComputeRasteriserConfiguration().to_c()
    ccam = native.cr_camera()
    small = cr.DeviceBuffer(ctx, 4096)  # the size check rejects the call before any launch
    p = C.c_void_p(small.ptr)
    st = lib.cr_cull_noalloc(p, (1 << 20) + 1, p, 1, C.byref(ccfg), C.byref(ccam), 8, 8, p, p,
                             C.c_void_p(ctx.stream()))
    assert st == 5  # CR_ERR_CAPACITY
    assert b"1048576" in lib.cr_last_error_detail()
