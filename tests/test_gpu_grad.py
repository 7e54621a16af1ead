"""Differentiable HQS colours on the GPU (FP32) against the FP64 oracle.

Scene: learnable colours initialised to 0.5; targets rendered by the oracle
from a hidden colour field c(x) = 0.5 + 0.5 sin(k . x + phi) per channel;
L2 loss over several views of different sizes.  Checked:

* the FP32 forward images against the FP64 images (|diff| <= 1e-5);
* the loss against the FP64 loss (relative 1e-5);
* the gradient on 1,000 seeded points visible in some view against the
  FP64 adjoint and the FP64 central differences (step 1e-3), with the
  relative error of a point
      max_c |g_c - g64_c| / max(max_c |g64_c|, 1e-2 * max over points |g64|)
  at most 1e-5 (the floor keeps points whose gradient nearly cancels
  across views from dividing by ~0);
* one gradient step lowers the loss.
"""
import numpy as np
import pytest

from scenes import blob_cloud, oracle_cloud_from_device, oracle_config, to_product_packed

pytestmark = pytest.mark.gpu

SIZES = [(96, 96), (128, 80), (64, 112), (100, 100)]


@pytest.fixture(scope="module")
def ctx(cr):
    return cr.Context(0)


def pool_positions(cloud, packed, ppb):
    """Float positions of every pool point (the packed order mapped to slots)."""
    dev = cloud.batches(0, packed.batchCount)
    n = cloud.capacity.maxResidentPoints
    pos = np.zeros((n, 3), np.float64)
    for i, b in enumerate(packed.batches):
        k0, cnt, f0 = int(b["firstPoint"]), int(b["numPoints"]), int(dev["firstPoint"][i])
        pos[f0:f0 + cnt] = packed.orderedPositions[k0:k0 + cnt, :3]
    return pos


def cameras(cr, seed):
    rng = np.random.default_rng(seed)
    cams = []
    for w, h in SIZES:
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        cam = cr.PerspectiveCamera(position=tuple(d * 2.2), near=0.01, far=100.0, fov=55.0,
                                   aspect=w / h)
        cam.lookAt((0.0, 0.0, 0.0))
        cams.append(cam)
    return cams


def test_fp32_gradient_matches_fp64_oracle_and_differences(cr, orc, ctx):
    ppb = 1024
    pos, rgba = blob_cloud(120000, 31)
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=ppb)
    cloud = cr.ComputeRasteriserPointCloud(ctx, packed=to_product_packed(cr, packed))
    n = cloud.capacity.maxResidentPoints
    xyz = pool_positions(cloud, packed, ppb)
    k = np.array([[3.1, -2.3, 1.7], [-1.9, 2.7, 2.2], [2.4, 1.3, -3.0]])
    phi = np.array([0.3, 1.1, -0.7])
    hidden = (0.5 + 0.5 * np.sin(xyz @ k.T + phi)).astype(np.float32)
    learn = np.full((n, 3), 0.5, np.float32)
    cfg = cr.ComputeRasteriserConfiguration()
    ocfg = oracle_config(orc, cfg)
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cfg
    ras.addPointCloud(cloud)
    ocl = oracle_cloud_from_device(orc, cloud)
    cams = cameras(cr, 7)
    total_px = sum(w * h for w, h in SIZES)
    scale = 1.0 / (3 * total_px)

    d_colors = cr.DeviceBuffer(ctx, n * 12, (n, 3), np.float32)
    d_grad = cr.DeviceBuffer(ctx, n * 12, (n, 3), np.float32)
    d_colors.upload(learn)
    d_grad.upload(np.zeros((n, 3), np.float32))
    targets, grad64 = [], np.zeros((n, 3))
    loss_gpu = loss64 = 0.0
    img64 = []
    for cam, (w, h) in zip(cams, SIZES):
        ras.resize((w, h))
        ras.update(cam)
        ocl.files = cloud.files()
        # Target: the oracle's FP64 image of the hidden colours.
        t = orc.hqs_grad_f64(ocl, ocfg, cam.viewMatrix, cam.projectionMatrix, w, h,
                             hidden.astype(np.float64), np.zeros((h, w, 3)), 1.0,
                             threads=8)["image"].astype(np.float32)
        targets.append(t)
        d_img = cr.DeviceBuffer(ctx, h * w * 12, (h, w, 3), np.float32)
        d_tgt = cr.DeviceBuffer(ctx, h * w * 12, (h, w, 3), np.float32)
        d_dl = cr.DeviceBuffer(ctx, h * w * 12, (h, w, 3), np.float32)
        d_tgt.upload(t)
        ras.forwardF32(cloud, d_colors, d_img)
        loss_gpu += cr.l2_loss(ctx, d_img, d_tgt, scale, d_dl)
        ras.backwardColors(cloud, d_dl, d_grad)
        ref = orc.hqs_grad_f64(ocl, ocfg, cam.viewMatrix, cam.projectionMatrix, w, h,
                               learn.astype(np.float64), t.astype(np.float64), scale,
                               grad=grad64, threads=8)
        loss64 += ref["loss"]
        img64.append(ref["image"])
        assert np.abs(d_img.download() - ref["image"]).max() <= 1e-5
    g = d_grad.download().astype(np.float64)
    assert abs(loss_gpu - loss64) <= 1e-5 * loss64

    visible = np.flatnonzero(np.abs(grad64).max(axis=1) > 0)
    assert len(visible) > 5000
    pts = np.sort(np.random.default_rng(0x5EED).choice(visible, 1000, replace=False))
    fd = np.zeros((1000, 3))
    for cam, (w, h), t in zip(cams, SIZES, targets):
        ras.resize((w, h))
        ras.update(cam)
        ocl.files = cloud.files()
        orc.hqs_grad_f64(ocl, ocfg, cam.viewMatrix, cam.projectionMatrix, w, h,
                         learn.astype(np.float64), t.astype(np.float64), scale,
                         fd_points=pts.astype(np.uint32), fd_h=1e-3, fd=fd, threads=8)
    floor = 1e-2 * np.abs(grad64[pts]).max()

    def rel(a, b):
        return (np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), floor)).max()

    assert rel(fd, grad64[pts]) <= 1e-8          # FP64 differences vs FP64 adjoint
    assert rel(g[pts], fd) <= 1e-5               # FP32 adjoint vs FP64 differences
    assert rel(g[pts], grad64[pts]) <= 1e-5      # FP32 adjoint vs FP64 adjoint

    # One gradient step lowers the loss.
    d_colors.upload((learn - 0.5 * g / np.abs(g).max()).astype(np.float32))
    loss_after = 0.0
    for cam, (w, h), t in zip(cams, SIZES, targets):
        ras.resize((w, h))
        ras.update(cam)
        d_img = cr.DeviceBuffer(ctx, h * w * 12, (h, w, 3), np.float32)
        d_tgt = cr.DeviceBuffer(ctx, h * w * 12, (h, w, 3), np.float32)
        d_dl = cr.DeviceBuffer(ctx, h * w * 12, (h, w, 3), np.float32)
        d_tgt.upload(t)
        ras.forwardF32(cloud, d_colors, d_img)
        loss_after += cr.l2_loss(ctx, d_img, d_tgt, scale, d_dl)
    assert loss_after < loss_gpu


def test_backward_needs_a_forward_and_rejects_colorize(cr, orc, ctx):
    pos, rgba = blob_cloud(3000, 2)
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=512)
    cloud = cr.ComputeRasteriserPointCloud(ctx, packed=to_product_packed(cr, packed))
    n = cloud.capacity.maxResidentPoints
    ras = cr.ComputeRasteriser(ctx)
    ras.addPointCloud(cloud)
    ras.resize((32, 32))
    cam = cr.PerspectiveCamera(position=(0.0, 0.0, 3.0), near=0.01, far=100.0, aspect=1.0)
    cam.lookAt((0.0, 0.0, 0.0))
    ras.update(cam)
    buf = cr.DeviceBuffer(ctx, n * 12, (n, 3), np.float32)
    img = cr.DeviceBuffer(ctx, 32 * 32 * 12, (32, 32, 3), np.float32)
    with pytest.raises(cr.CRError):
        ras.backwardColors(cloud, img, buf)
    ras.configuration = cr.ComputeRasteriserConfiguration(colorizeChunks=True)
    with pytest.raises(cr.CRError) as e:
        ras.forwardF32(cloud, buf, img)
    assert e.value.status == 4
