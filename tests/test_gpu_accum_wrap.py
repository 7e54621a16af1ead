"""HQS accumulators past 2^32: the colour pass adds R | G << 32 and
B | count << 32 as 64-bit words, which stays exact while a pixel holds at
most 16,843,009 samples (255 * 16843009 = 2^32 - 1).  Past that the resolve
detects the pixel and the frame is re-run with one 32-bit add per field, so
every field still ends as its 32-bit sum modulo 2^32, as the reference's
atomic_uint adds wrap (ColorPass/Shaders.metal, integer path).

The scenes stack whole batches of one white point at the origin, so a
single pixel receives every sample; CLOD and dither are off so that all
points are drawn.
"""
import numpy as np
import pytest

from scenes import oracle_cloud_from_device, oracle_config

pytestmark = pytest.mark.gpu

PPB = 10240
LIMIT = 16843009  # largest count whose 8-bit channel sums fit 32 bits
W = H = 16


@pytest.fixture(scope="module")
def ctx(cr):
    return cr.Context(0)


def stacked_cloud(cr, ctx, samples: int):
    """`samples` copies of one white point at the origin, in batches of PPB."""
    nb = (samples + PPB - 1) // PPB
    zeros = np.zeros(PPB, np.uint32)
    white = np.full(PPB, 0xFFFFFFFF, np.uint32)
    levels = np.zeros(PPB, np.uint8)
    b = np.zeros(nb, cr.BATCH_DTYPE)
    b["state"] = 1
    b["numPoints"] = PPB
    b["numPoints"][-1] = samples - (nb - 1) * PPB
    b["firstPoint"] = 0  # every record copies the same source points
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(nb, PPB))
    cloud.addBatches(zeros, zeros, zeros, white, levels, b)
    return cloud


def render(cr, ctx, cloud):
    cfg = cr.ComputeRasteriserConfiguration(enableCLOD=False, enableLODDither=False)
    cam = cr.PerspectiveCamera(position=(0.0, 0.0, 3.0), near=0.01, far=100.0, fov=60.0,
                               aspect=1.0)
    cam.lookAt((0.0, 0.0, 0.0))
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cfg
    ras.addPointCloud(cloud)
    ras.resize((W, H))
    ras.update(cam)
    ras.encode()
    px = ras.pixels()
    acc = np.stack([px["red"], px["green"], px["blue"], px["count"]], -1)
    return ras, cfg, cam, acc


@pytest.mark.parametrize("samples", [LIMIT, LIMIT + 1, 1700 * PPB])
def test_single_pixel_sums_wrap_like_32_bit_adds(cr, ctx, samples):
    cloud = stacked_cloud(cr, ctx, samples)
    _, _, _, acc = render(cr, ctx, cloud)
    hit = np.argwhere(acc[..., 3] != 0)
    assert len(hit) == 1
    y, x = hit[0]
    s = (255 * samples) % (1 << 32)
    assert acc[y, x].tolist() == [s, s, s, samples % (1 << 32)]
    rest = acc.copy()
    rest[y, x] = 0
    assert not rest.any()


def test_wrapped_frame_matches_oracle(cr, orc, ctx):
    samples = 1700 * PPB
    cloud = stacked_cloud(cr, ctx, samples)
    ras, cfg, cam, acc = render(cr, ctx, cloud)
    ref = orc.render([oracle_cloud_from_device(orc, cloud)], oracle_config(orc, cfg),
                     cam.viewMatrix, cam.projectionMatrix, W, H, threads=8)
    assert np.array_equal(acc, ref.accum)
    assert np.array_equal(ras.outputRGBA8(), ref.rgba)
    assert np.array_equal(ras.depthTexture().view(np.uint32), ref.depthf.view(np.uint32))
