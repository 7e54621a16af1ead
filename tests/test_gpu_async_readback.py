"""Asynchronous RGBA8 read-back (cr_frame_read_rgba8_async): a render loop
that reads every frame while the next one renders gets, in each host buffer,
the image of the frame it was enqueued after — bit-identical to a blocking
read of a render of the same camera."""
import numpy as np
import pytest

from scenes import blob_cloud, to_product_packed

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(cr):
    return cr.Context(0)


def make_cloud(cr, orc, ctx, n=80000, seed=3):
    pos, rgba = blob_cloud(n, seed)
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=1024)
    return cr.ComputeRasteriserPointCloud(ctx, packed=to_product_packed(cr, packed))


def camera(cr, k, aspect):
    a = 0.7 * k
    cam = cr.PerspectiveCamera(position=(2.4 * np.sin(a), 0.3 * k - 0.5, 2.4 * np.cos(a)),
                               near=0.01, far=100.0, fov=55.0, aspect=aspect)
    cam.lookAt((0.0, 0.0, 0.0))
    return cam


@pytest.mark.parametrize("hole_fill", [0, 2])
def test_pipelined_readback_matches_blocking(cr, orc, ctx, hole_fill):
    cloud = make_cloud(cr, orc, ctx)
    w, h = 320, 200
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cr.ComputeRasteriserConfiguration(holeFillIterations=hole_fill)
    ras.addPointCloud(cloud)
    ras.resize((w, h))
    frames = 6
    expect = []
    for k in range(frames):
        ras.update(camera(cr, k, w / h))
        ras.encode()
        expect.append(ras.outputRGBA8())
    assert len({e.tobytes() for e in expect}) == frames  # every camera differs

    # Every frame into its own buffer, nothing waited for until the end: each
    # render's resolve waits on the device for the previous frame's copy.
    bufs = [cr.HostBuffer((h, w, 4), np.uint8) for _ in range(frames)]
    for k in range(frames):
        ras.update(camera(cr, k, w / h))
        ras.encode()
        ras.outputRGBA8Async(bufs[k].array)
    ras.waitOutput()
    for k in range(frames):
        assert np.array_equal(bufs[k].array, expect[k]), f"frame {k}"

    # Two buffers, waiting for frame k-1's copy before enqueueing frame k's.
    ring = bufs[:2]
    for k in range(frames):
        ras.update(camera(cr, k, w / h))
        ras.encode()
        ras.waitOutput()
        if k >= 1:
            assert np.array_equal(ring[(k - 1) & 1].array, expect[k - 1]), f"ring frame {k - 1}"
        ras.outputRGBA8Async(ring[k & 1].array)
    ras.waitOutput()
    assert np.array_equal(ring[(frames - 1) & 1].array, expect[-1])

    # Three buffers, waiting only until frame k-2's copy is done (keep=1:
    # frame k-1's may still travel) before enqueueing frame k's.
    ring = bufs[:3]
    for k in range(frames):
        ras.update(camera(cr, k, w / h))
        ras.encode()
        ras.waitOutput(keep=1)
        if k >= 2:
            assert np.array_equal(ring[(k - 2) % 3].array, expect[k - 2]), f"ring3 frame {k - 2}"
        ras.outputRGBA8Async(ring[k % 3].array)
    ras.waitOutput()
    for k in (frames - 2, frames - 1):
        assert np.array_equal(ring[k % 3].array, expect[k]), f"ring3 frame {k}"
    for b in bufs:
        b.close()


def test_wait_keep_is_validated(cr, ctx):
    ras = cr.ComputeRasteriser(ctx)
    ras.resize((64, 48))
    ras.waitOutput(keep=3)  # nothing enqueued: returns at once
    with pytest.raises(cr.CRError):
        ras.waitOutput(keep=4)
    with pytest.raises(cr.CRError):
        ras.waitOutput(keep=-1)


def test_readback_then_batched_views_render(cr, orc, ctx):
    """A batched-view render waits for the frames' pending read-backs."""
    cloud = make_cloud(cr, orc, ctx, 60000, 5)
    sizes = [(128, 96), (200, 120)]
    mv = cr.MultiViewRasteriser(ctx, sizes)
    mv.addPointCloud(cloud)
    cams_a = [camera(cr, 1, 128 / 96), camera(cr, 2, 200 / 120)]
    cams_b = [camera(cr, 4, 128 / 96), camera(cr, 5, 200 / 120)]
    mv.render(cams_a)
    want = [mv.outputRGBA8(i) for i in range(2)]
    bufs = [cr.HostBuffer((hh, ww, 4), np.uint8) for ww, hh in sizes]
    for _ in range(3):
        mv.render(cams_a)
        for i in range(2):
            mv.frames[i].rgba8_async(bufs[i].array)
        mv.render(cams_b)
        for i in range(2):
            mv.frames[i].wait()
            assert np.array_equal(bufs[i].array, want[i]), i
    for b in bufs:
        b.close()


def test_resize_and_close_with_a_pending_readback(cr, orc, ctx):
    cloud = make_cloud(cr, orc, ctx, 20000, 9)
    ras = cr.ComputeRasteriser(ctx)
    ras.addPointCloud(cloud)
    ras.resize((64, 64))
    ras.update(camera(cr, 0, 1.0))
    ras.encode()
    buf = cr.HostBuffer((64, 64, 4), np.uint8)
    ras.outputRGBA8Async(buf.array)
    ras.resize((96, 64))  # destroys the frame: waits for its copy first
    ras.update(camera(cr, 0, 1.5))
    ras.encode()
    assert ras.outputRGBA8().shape == (64, 96, 4)
    ras.waitOutput()  # nothing pending on the new frame
    with pytest.raises(cr.CRError):
        ras.outputRGBA8Async(np.zeros((8, 8, 4), np.uint8))
    buf.close()
