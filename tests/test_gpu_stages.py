"""Staged HQS rendering (cr_render_stages) and the frame split by points.

* depth / colour / resolve as three calls give encode()'s planes and image;
* two parts of the batches rendered into two frames, depth planes combined
  by max (in signed order, through cr_frame_flip_depth_order), colour
  stages against that depth, accumulators summed: both frames resolve to the
  single render of all batches, bit for bit;
* PointShardedRasteriser over a one-rank NCCL group gives encode()'s image.
"""
import importlib
import os
import socket

import numpy as np
import pytest

from scenes import blob_cloud, lattice_cloud, to_product_packed

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(cr):
    return cr.Context(0)


def make_cloud(cr, orc, ctx, pos, rgba, ppb=1024):
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=ppb)
    return cr.ComputeRasteriserPointCloud(ctx, packed=to_product_packed(cr, packed))


def camera(cr, aspect, eye=(1.3, 0.8, 2.1)):
    cam = cr.PerspectiveCamera(position=eye, near=0.01, far=100.0, fov=55.0, aspect=aspect)
    cam.lookAt((0.0, 0.0, 0.0))
    return cam


def outputs(ras):
    px = ras.pixels()
    return ras.outputRGBA8(), ras.depthTexture().view(np.uint32), px


def assert_same(a, b):
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1], b[1])
    for f in ("depth", "red", "green", "blue", "count"):
        assert np.array_equal(a[2][f], b[2][f]), f


CONFIGS = {
    "default": {},
    "holes_tolerance": dict(holeFillIterations=2, depthTolerance=0.05),
    "footprint": dict(minimumPointSize=1.0, maximumPointSize=3.0, pointSizeScale=2.0),
}


@pytest.mark.parametrize("name", list(CONFIGS))
def test_stages_compose_to_encode(cr, orc, ctx, name):
    pos, rgba = blob_cloud(90000, 23)
    cloud = make_cloud(cr, orc, ctx, pos, rgba)
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cr.ComputeRasteriserConfiguration(**CONFIGS[name])
    ras.addPointCloud(cloud)
    ras.resize((240, 160))
    ras.update(camera(cr, 1.5))
    ras.encode()
    want = outputs(ras)
    assert want[2]["count"].any()
    for split in ([cr.STAGE_DEPTH, cr.STAGE_COLOR, cr.STAGE_RESOLVE],
                  [cr.STAGE_DEPTH | cr.STAGE_COLOR, cr.STAGE_RESOLVE],
                  [cr.STAGE_DEPTH, cr.STAGE_COLOR | cr.STAGE_RESOLVE]):
        for st in split:
            ras.encodeStages(st)
        assert_same(outputs(ras), want)


def _parts(cr, orc, ctx, pos, rgba, nparts):
    """Clouds with the same slot layout, each keeping one part of the batches."""
    sharded = importlib.import_module("satin-computerasteriser_b200.sharded")
    clouds = []
    for r in range(nparts):
        c = make_cloud(cr, orc, ctx, pos, rgba)
        lo, hi = sharded.shard_range(c.residentBatchCount, r, nparts)
        drop = [s for s in range(c.residentBatchCount) if not lo <= s < hi]
        if drop:
            c.removeBatches(drop)
        clouds.append(c)
    return clouds


@pytest.mark.parametrize("nparts", [2, 3])
def test_parts_combined_by_max_and_sum_match_single_render(cr, orc, ctx, nparts):
    import torch

    pos, rgba = lattice_cloud(36, 5)
    full = make_cloud(cr, orc, ctx, pos, rgba)
    parts = _parts(cr, orc, ctx, pos, rgba, nparts)
    assert sum(p.residentBatchCount for p in parts) == full.residentBatchCount
    cfg = cr.ComputeRasteriserConfiguration(holeFillIterations=1)
    cam = camera(cr, 1.25, eye=(0.4, 0.5, 2.6))

    ref = cr.ComputeRasteriser(ctx)
    ref.configuration = cfg
    ref.addPointCloud(full)
    ref.resize((200, 160))
    ref.update(cam)
    ref.encode()
    want = outputs(ref)

    rs = []
    for p in parts:
        r = cr.ComputeRasteriser(ctx)
        r.configuration = cfg
        r.addPointCloud(p)
        r.resize((200, 160))
        r.update(cam)
        rs.append(r)
    sharded = importlib.import_module("satin-computerasteriser_b200.sharded")
    planes = []
    for r in rs:
        pl = r.devicePlanes()
        planes.append((torch.as_tensor(sharded._DevicePlane(pl["depth"], pl["pixels"]),
                                       device="cuda:0"),
                       torch.as_tensor(sharded._DevicePlane(pl["accum"], 4 * pl["pixels"]),
                                       device="cuda:0")))
    for r in rs:
        r.encodeStages(cr.STAGE_DEPTH)
        r.flipDepthOrder()
    ctx.synchronize()
    m = planes[0][0].clone()
    for d, _ in planes[1:]:
        m = torch.maximum(m, d)
    torch.cuda.synchronize()
    for d, _ in planes:
        d.copy_(m)
    torch.cuda.synchronize()
    for r in rs:
        r.flipDepthOrder()
        r.encodeStages(cr.STAGE_COLOR)
    ctx.synchronize()
    acc = planes[0][1].clone()
    for _, a in planes[1:]:
        acc += a
    torch.cuda.synchronize()
    for _, a in planes:
        a.copy_(acc)
    torch.cuda.synchronize()
    for r in rs:
        r.encodeStages(cr.STAGE_RESOLVE)
        assert_same(outputs(r), want)
    # Each part alone draws less than the whole.
    assert all(p.pointCount < full.pointCount for p in parts)


def test_flip_depth_order_is_an_involution(cr, orc, ctx):
    pos, rgba = blob_cloud(20000, 2)
    cloud = make_cloud(cr, orc, ctx, pos, rgba)
    ras = cr.ComputeRasteriser(ctx)
    ras.addPointCloud(cloud)
    ras.resize((37, 23))  # pixel count not a multiple of 4
    ras.update(camera(cr, 37 / 23))
    ras.encode()
    d0 = ras.pixels()["depth"].copy()
    ras.flipDepthOrder()
    d1 = ras.pixels()["depth"]
    assert np.array_equal(d1, d0 ^ np.uint32(0x80000000))
    ras.flipDepthOrder()
    assert np.array_equal(ras.pixels()["depth"], d0)


def test_separate_stages_reject_nearest_and_bad_bits(cr, orc, ctx):
    pos, rgba = blob_cloud(3000, 1)
    cloud = make_cloud(cr, orc, ctx, pos, rgba)
    ras = cr.ComputeRasteriser(ctx)
    ras.addPointCloud(cloud)
    ras.resize((32, 32))
    ras.update(camera(cr, 1.0))
    with pytest.raises(cr.CRError):
        ras.encodeStages(0)
    with pytest.raises(cr.CRError):
        ras.encodeStages(8)
    ras.configuration = cr.ComputeRasteriserConfiguration(mode=cr.MODE_NEAREST)
    with pytest.raises(cr.CRError) as e:
        ras.encodeStages(cr.STAGE_DEPTH)
    assert e.value.status == 4
    ras.encodeStages(cr.STAGE_ALL)  # the whole frame is fine


def test_point_sharded_rasteriser_one_rank_nccl(cr, orc, ctx):
    import torch.distributed as dist

    sharded = importlib.import_module("satin-computerasteriser_b200.sharded")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0,
                            world_size=1)
    try:
        pos, rgba = blob_cloud(70000, 8)
        cloud = make_cloud(cr, orc, ctx, pos, rgba)
        ras = cr.ComputeRasteriser(ctx)
        ras.configuration = cr.ComputeRasteriserConfiguration(holeFillIterations=1)
        ras.addPointCloud(cloud)
        ras.resize((160, 120))
        ras.update(camera(cr, 160 / 120))
        ras.encode()
        want = outputs(ras)
        sh = sharded.PointShardedRasteriser(ras)
        for _ in range(2):
            sh.encode()
            assert_same(outputs(ras), want)
    finally:
        dist.destroy_process_group()
