"""Asynchronous slot-pool uploads (cr_cloud_add_batches_async) and the
streaming adapter on the GPU.

* chunks uploaded asynchronously then published give the same slots, pool
  contents and image as the same chunks added synchronously;
* slots whose copy is in flight are not drawn before they are published,
  and removing them cancels the upload (the slots come back free);
* a staging ring smaller than the uploads wraps and waits, with the same
  result;
* the streaming adapter over a camera path: the invariants each tick, and
  the final image equals the oracle's render of the device's own pool.
"""
import importlib

import numpy as np
import pytest

from scenes import blob_cloud, oracle_cloud_from_device, oracle_config

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(cr):
    return cr.Context(0)


@pytest.fixture(scope="module")
def streaming():
    return importlib.import_module("satin-computerasteriser_b200.streaming")


def chunks_of(orc, streaming, n, seed, ppb=512, per=3):
    pos, rgba = blob_cloud(n, seed)
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=ppb)
    return packed, streaming.chunks_from_packed(packed, per)


def render(cr, ctx, cloud, size=(200, 150), eye=(1.1, 0.6, 1.9)):
    ras = cr.ComputeRasteriser(ctx)
    ras.addPointCloud(cloud)
    ras.resize(size)
    cam = cr.PerspectiveCamera(position=eye, near=0.01, far=100.0, fov=55.0,
                               aspect=size[0] / size[1])
    cam.lookAt((0.0, 0.0, 0.0))
    ras.update(cam)
    ras.encode()
    return ras.outputRGBA8(), ras.pixels()


def new_cloud(cr, ctx, packed, slots):
    return cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(slots, 512),
                                          files=packed.files)


def test_async_upload_matches_sync_add(cr, orc, ctx, streaming):
    packed, chunks = chunks_of(orc, streaming, 120000, 3)
    a = new_cloud(cr, ctx, packed, 400)
    b = new_cloud(cr, ctx, packed, 400)
    sa, sb = [], []
    for c in chunks:
        sa += a.addBatchesAsync(c.xyzLow, c.xyzMed, c.xyzHigh, c.colors, c.levels, c.batches)
        sb += b.addBatches(c.xyzLow, c.xyzMed, c.xyzHigh, c.colors, c.levels, c.batches)
    assert sa == sb
    a.waitUploads()
    assert a.residentBatchCount == b.residentBatchCount == len(packed.batches)
    assert a.pointCount == b.pointCount
    assert np.array_equal(a.batches(), b.batches())
    pa, pb = a.points(), b.points()
    for f in ("xyzLow", "xyzMed", "xyzHigh", "colors", "levels"):
        assert np.array_equal(pa[f], pb[f]), f
    ia, ib = render(cr, ctx, a), render(cr, ctx, b)
    assert np.array_equal(ia[0], ib[0]) and np.array_equal(ia[1], ib[1])
    assert ia[1]["count"].any()
    # Borrowed page-locked arrays (no staging copy): the same pool.
    arena = streaming.pin_chunks(chunks)
    c2 = new_cloud(cr, ctx, packed, 400)
    sc = []
    for c in chunks:
        sc += c2.addBatchesAsync(c.xyzLow, c.xyzMed, c.xyzHigh, c.colors, c.levels, c.batches,
                                 borrow=True)
    c2.waitUploads()
    assert sc == sa
    pc = c2.points()
    for f in ("xyzLow", "xyzMed", "xyzHigh", "colors", "levels"):
        assert np.array_equal(pc[f], pb[f]), f
    assert np.array_equal(c2.batches(), b.batches())
    c2.close()
    arena.close()


def test_unpublished_slots_are_not_drawn_and_removal_cancels(cr, orc, ctx, streaming):
    packed, chunks = chunks_of(orc, streaming, 60000, 8)
    cl = new_cloud(cr, ctx, packed, 200)
    slots = []
    for c in chunks:
        slots += cl.addBatchesAsync(c.xyzLow, c.xyzMed, c.xyzHigh, c.colors, c.levels,
                                    c.batches)
    # Not published yet: nothing resident, nothing drawn, slots taken.
    assert cl.residentBatchCount == 0 and cl.pointCount == 0
    assert cl.freeSlotCount == 200 - len(slots)
    _, px = render(cr, ctx, cl)
    assert not px["count"].any()
    # Cancel half of them while (possibly) in flight, then publish.
    cl.removeBatches(slots[::2])
    cl.waitUploads()
    assert cl.residentBatchCount == len(slots[1::2])
    assert cl.freeSlotCount == 200 - len(slots[1::2])
    b = cl.batches()
    assert all(b["state"][s] == 1 for s in slots[1::2])
    assert all(b["state"][s] == 0 for s in slots[::2])
    # Removing published slots frees them as usual.
    cl.removeBatches(slots[1::2])
    assert cl.residentBatchCount == 0 and cl.freeSlotCount == 200


def test_small_staging_ring_wraps(cr, orc, ctx, streaming):
    packed, chunks = chunks_of(orc, streaming, 90000, 12, per=2)
    a = new_cloud(cr, ctx, packed, 300)
    b = new_cloud(cr, ctx, packed, 300)
    a.setUploadStaging(3 * 2 * 512 * 17)  # about three chunks
    for k, c in enumerate(chunks):
        a.addBatchesAsync(c.xyzLow, c.xyzMed, c.xyzHigh, c.colors, c.levels, c.batches)
        b.addBatches(c.xyzLow, c.xyzMed, c.xyzHigh, c.colors, c.levels, c.batches)
        if k % 5 == 4:
            a.pollUploads()
    a.waitUploads()
    pa, pb = a.points(), b.points()
    for f in ("xyzLow", "xyzMed", "xyzHigh", "colors", "levels"):
        assert np.array_equal(pa[f], pb[f]), f
    assert np.array_equal(a.batches(), b.batches())


def test_streaming_adapter_on_device(cr, orc, ctx, streaming):
    packed, chunks = chunks_of(orc, streaming, 200000, 21, per=4)
    cloud = new_cloud(cr, ctx, packed, 120)
    src = streaming.InMemoryStreamingSource(chunks, budget_bytes=150 * 512 * 17)
    ad = streaming.StreamingAdapter(src, cloud)
    ad.maxChunkUploadsPerTick = 6
    ras = cr.ComputeRasteriser(ctx)
    ras.addPointCloud(cloud)
    ras.resize((192, 108))
    path = [(0, 0, 3.0)] * 6 + [(0.5, 0.5, 0.8)] * 6 + \
        [(1.1 * np.cos(a), 0.3, 1.1 * np.sin(a)) for a in np.linspace(0, 2 * np.pi, 12)]
    full = False
    for eye in path:
        cam = cr.PerspectiveCamera(position=eye, near=0.01, far=100.0, fov=45.0,
                                   aspect=192 / 108)
        cam.lookAt((0.0, 0.0, 0.0))
        ad.update(cam, (192, 108))
        ras.update(cam)
        ras.encode()  # draws whatever is published
        assert len(src.believed) - ad.residentChunks - ad.pendingUploadCount == 0
        assert ad.residentPoints == cloud.pointCount
        full |= ad.lastError is not None
    assert full  # the pool was under pressure
    cloud.waitUploads()
    ad.update(cam, (192, 108))
    cloud.waitUploads()
    # Published slots hold exactly the adapter's chunks.
    want = sum(len(chunks[i[1]].batches) for i in ad.slotsByChunk)
    assert cloud.residentBatchCount == want
    ras.update(cam)
    ras.encode()
    got = ras.pixels()
    ocl = oracle_cloud_from_device(orc, cloud)
    ref = orc.render(ocl, oracle_config(orc, ras.configuration), cam.viewMatrix,
                     cam.projectionMatrix, 192, 108)
    assert np.array_equal(got["depth"], ref.depth)
    assert np.array_equal(got["count"], ref.accum[..., 3])
    assert np.array_equal(ras.outputRGBA8(), ref.rgba)
    assert ref.accum[..., 3].any()
