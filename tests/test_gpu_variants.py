"""The colour variants of the reference's colour pass
(Pipelines/ColorPass/Shaders.metal:106-199: displacement, tint,
translucent-defocus coverage, motion blur; Resolve/Shaders.metal:27-45) on
the GPU against the oracle, bit for bit on every plane: RGBA8, depth, R, G,
B, count, depth f32.

The per-point attributes are written into the cloud's device buffers (here
with uploads, and through DisplacementPass / TintPass with a torch kernel),
read back, and handed to the oracle with the device's own pool."""
import numpy as np
import pytest

from scenes import blob_cloud, oracle_cloud_from_device, oracle_config, to_product_packed

pytestmark = pytest.mark.gpu

W, H = 200, 150


@pytest.fixture(scope="module")
def ctx(cr):
    return cr.Context(0)


def setup(cr, orc, ctx, seed=4, n=70000, **cfg):
    pos, rgba = blob_cloud(n, seed)
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=1024)
    cloud = cr.ComputeRasteriserPointCloud(ctx, packed=to_product_packed(cr, packed))
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cr.ComputeRasteriserConfiguration(**cfg)
    ras.addPointCloud(cloud)
    ras.resize((W, H))
    return cloud, ras


def camera(cr, eye=(1.2, 0.7, 1.9)):
    cam = cr.PerspectiveCamera(position=eye, near=0.01, far=100.0, fov=55.0, aspect=W / H)
    cam.lookAt((0.0, 0.0, 0.0))
    return cam


def check(cr, orc, ras, cloud, cam, disp=None, prev=None, tint=None):
    ocl = oracle_cloud_from_device(orc, cloud)
    ocl.displacements, ocl.prevDisplacements, ocl.tints = disp, prev, tint
    ref = orc.render(ocl, oracle_cfg(orc, ras.configuration), cam.viewMatrix,
                     cam.projectionMatrix, W, H)
    px = ras.pixels()
    assert np.array_equal(px["depth"], ref.depth)
    for k, f in enumerate(("red", "green", "blue", "count")):
        assert np.array_equal(px[f], ref.accum[..., k]), f
    assert np.array_equal(ras.outputRGBA8(), ref.rgba)
    assert np.array_equal(ras.depthTexture().view(np.uint32), ref.depthf.view(np.uint32))
    assert ref.accum[..., 3].any()
    return ref


def oracle_cfg(orc, cfg):
    o = oracle_config(orc, cfg)
    for name in ("applyDisplacement", "applyTint", "tintAlphaIsCoverage", "motionBlur",
                 "motionBlurSamples", "motionBlurMaxSpread"):
        setattr(o, name, getattr(cfg, name))
    return o


def rand_disp(rng, n, scale=0.02, nan_frac=0.02):
    d = np.zeros((n, 4), np.float32)
    d[:, :3] = rng.normal(0, scale, (n, 3))
    d[rng.random(n) < nan_frac, 1] = np.nan
    return d


def rand_tint(rng, n, neg_frac=0.05, hi=1.3):
    t = rng.uniform(-0.2, hi, (n, 4)).astype(np.float32)
    t[:, 3] = rng.uniform(0.0, hi, n)
    t[rng.random(n) < neg_frac, 3] = -0.5
    return t


@pytest.mark.parametrize("point_size", [1.0, 3.0])
def test_displacement(cr, orc, ctx, point_size):
    cloud, ras = setup(cr, orc, ctx, applyDisplacement=True, maximumPointSize=point_size,
                       pointSizeScale=3.0)
    d = rand_disp(np.random.default_rng(1), cloud.displacementBuffer().shape[0])
    cloud.displacementBuffer().upload(d)
    cam = camera(cr)
    ras.update(cam)
    ras.encode()
    check(cr, orc, ras, cloud, cam, disp=d)


@pytest.mark.parametrize("colorize", [False, True])
def test_tint_mix_and_discard(cr, orc, ctx, colorize):
    cloud, ras = setup(cr, orc, ctx, applyTint=True, colorizeChunks=colorize)
    t = rand_tint(np.random.default_rng(2), cloud.tintBuffer().shape[0])
    cloud.tintBuffer().upload(t)
    cam = camera(cr)
    ras.update(cam)
    ras.encode()
    check(cr, orc, ras, cloud, cam, tint=t)


@pytest.mark.parametrize("holes", [0, 1])
def test_tint_coverage(cr, orc, ctx, holes):
    cloud, ras = setup(cr, orc, ctx, applyTint=True, tintAlphaIsCoverage=True,
                       holeFillIterations=holes, backgroundColor=(0.1, 0.2, 0.3, 1.0))
    t = rand_tint(np.random.default_rng(3), cloud.tintBuffer().shape[0])
    cloud.tintBuffer().upload(t)
    cam = camera(cr)
    ras.update(cam)
    ras.encode()
    ref = check(cr, orc, ras, cloud, cam, tint=t)
    a = ref.rgba[..., 3]
    assert ((a > 0) & (a < 255)).any()  # translucent pixels


def test_motion_blur_camera_and_displacement(cr, orc, ctx):
    cloud, ras = setup(cr, orc, ctx, applyDisplacement=True, motionBlur=1.0,
                       motionBlurSamples=6, motionBlurMaxSpread=9.0)
    rng = np.random.default_rng(5)
    n = cloud.displacementBuffer().shape[0]
    d1, d2 = rand_disp(rng, n, 0.01, 0.0), rand_disp(rng, n, 0.01, 0.01)
    cam = camera(cr)
    cloud.displacementBuffer().upload(d1)
    ras.update(cam)
    ras.encode()  # first frame: previous = current
    check(cr, orc, ras, cloud, cam, disp=d1)
    cam.position = np.array([1.3, 0.75, 1.85])
    cam.lookAt((0.02, 0.0, 0.0))
    cloud.displacementBuffer().upload(d2)
    ras.update(cam)  # previous view-projection = the first frame's
    ras.encode()
    # Snapshot after the colour pass: next frame's previous displacement.
    assert np.array_equal(cloud.prevDisplacementBuffer().download().view(np.uint32),
                          d2.view(np.uint32))
    ref = check(cr, orc, ras, cloud, cam, disp=d2, prev=d1)
    assert (ref.accum[..., 3] > 0).sum() > 100


def test_user_passes_with_a_torch_kernel(cr, orc, ctx):
    import torch

    cloud, ras = setup(cr, orc, ctx)

    def tint_kernel(arrays, out, stream, gain):
        dev = torch.device("cuda", 0)
        with torch.cuda.stream(torch.cuda.ExternalStream(stream, device=dev)):
            col = torch.as_tensor(arrays["colors"], device=dev).to(torch.int64)
            o = torch.as_tensor(out, device=dev)
            r = (col & 255).to(torch.float32) / 255.0
            o[:, 0] = 1.0 - r
            o[:, 1] = r * gain
            o[:, 2] = 0.25
            o[:, 3] = torch.where((col >> 8) & 1 == 1, 0.6, -1.0)

    def disp_kernel(arrays, out, stream):
        dev = torch.device("cuda", 0)
        with torch.cuda.stream(torch.cuda.ExternalStream(stream, device=dev)):
            lv = torch.as_tensor(arrays["levels"], device=dev).to(torch.float32)
            o = torch.as_tensor(out, device=dev)
            o[:, 0] = 0.01 * lv
            o[:, 1] = -0.005 * lv

    tp = cr.TintPass(ras, tint_kernel, gain=0.5)
    dp = cr.DisplacementPass(ras, disp_kernel)
    cam = camera(cr)
    ras.update(cam)
    tp.encode()
    dp.encode()
    assert ras.configuration.applyTint and ras.configuration.applyDisplacement
    ras.encode()
    check(cr, orc, ras, cloud, cam, disp=cloud.displacementBuffer().download(),
          tint=cloud.tintBuffer().download())


def test_variants_rejected_where_not_built(cr, orc, ctx):
    cloud, ras = setup(cr, orc, ctx, n=5000)
    mv = cr.MultiViewRasteriser(ctx, [(32, 32)])
    mv.addPointCloud(cloud)
    mv.configuration = cr.ComputeRasteriserConfiguration(applyTint=True)
    with pytest.raises(cr.CRError) as e:
        mv.render([camera(cr)])
    assert e.value.status == 4
    ras.configuration = cr.ComputeRasteriserConfiguration(motionBlur=1.0, motionBlurSamples=0)
    ras.update(camera(cr))
    with pytest.raises(cr.CRError) as e:
        ras.encode()
    assert e.value.status == 1
