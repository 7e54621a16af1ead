"""Device-side status: a bounded wait of the one-view cull that gives up is
reported to the host as CR_ERR_TIMEOUT.

The cull's CTAs each wait (a bounded number of polls) for the survivor counts
of the CTAs before them.  With cullSpinLimit = 0 every CTA after the first
gives up at once: nothing waits and nothing hangs, the frame's survivor list
is incomplete, and the next synchronising call must say so.  The reference
reports nothing from the GPU (its guards are silent no-ops,
ComputeRasteriser.swift:278-283); here the error is not silent.
"""
import numpy as np
import pytest

from scenes import blob_cloud, oracle_cloud_from_device, oracle_config, to_product_packed

pytestmark = pytest.mark.gpu

CR_ERR_TIMEOUT = 6


@pytest.fixture(scope="module")
def ctx(cr):
    c = cr.Context(0)
    yield c
    c.close()


def many_slot_cloud(cr, orc, ctx):
    # 2,500 batches of 16 points: ten cull CTAs of 256 slots.
    pos, rgba = blob_cloud(40000, 21, scale=2.0)
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=16)
    assert len(packed.batches) > 4 * 256
    return cr.ComputeRasteriserPointCloud(ctx, packed=to_product_packed(cr, packed))


def render(cr, ctx, cloud, mode, w=192, h=128):
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cr.ComputeRasteriserConfiguration(mode=mode)
    ras.addPointCloud(cloud)
    ras.resize((w, h))
    cam = cr.PerspectiveCamera(position=(0.6, 0.4, 2.2), near=0.01, far=100, fov=60,
                               aspect=w / h)
    cam.lookAt((0, 0, 0))
    ras.update(cam)
    ras.encode()
    return ras, cam


@pytest.mark.parametrize("mode", [0, 1])
def test_cull_wait_timeout_is_reported(cr, orc, ctx, mode):
    cloud = many_slot_cloud(cr, orc, ctx)
    saved = ctx.tuning()
    try:
        ctx.set_tuning(cullSpinLimit=0)
        render(cr, ctx, cloud, mode)
        with pytest.raises(cr.CRError) as err:
            ctx.synchronize()
        assert err.value.status == CR_ERR_TIMEOUT
        assert "cull" in str(err.value)
        # The status word was cleared by the report.
        ctx.synchronize()
        # A read-back reports a timed-out frame too.
        ras, _ = render(cr, ctx, cloud, mode)
        with pytest.raises(cr.CRError) as err:
            ras.outputRGBA8()
        assert err.value.status == CR_ERR_TIMEOUT
    finally:
        ctx.set_tuning(cullSpinLimit=saved["cullSpinLimit"])
    # With the default limit the same frame is complete and bit-exact.
    ras, cam = render(cr, ctx, cloud, mode)
    img = ras.outputRGBA8()
    ref = orc.render(oracle_cloud_from_device(orc, cloud), oracle_config(orc, ras.configuration),
                     cam.viewMatrix, cam.projectionMatrix, 192, 128)
    assert np.array_equal(img, ref.rgba)
    assert np.array_equal(cloud.visibleBatches(), ref.visible[0])
    assert len(ref.visible[0]) > 256
    cloud.close()


def test_spin_limit_is_validated(cr, ctx):
    with pytest.raises(cr.CRError):
        ctx.set_tuning(cullSpinLimit=-1)
    assert ctx.tuning()["cullSpinLimit"] == 1 << 20
