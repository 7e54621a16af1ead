"""GPU parity of the render path against the CPU oracle (bit-exact).

Every test renders with the CUDA library through the C ABI and compares the
device outputs with the oracle run on the very same device slot pool (read
back), at sizes the oracle finishes in seconds.
"""
import numpy as np
import pytest

from scenes import (blob_cloud, lattice_cloud, oracle_cloud_from_device, oracle_config,
                    to_product_packed)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(cr):
    return cr.Context(0)


def make_cloud(cr, orc, ctx, pos, rgba, ppb=10240, **kw):
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=ppb, **kw)
    return cr.ComputeRasteriserPointCloud(ctx, packed=to_product_packed(cr, packed)), packed


def render_both(cr, orc, ctx, clouds, cfg, cam, w, h):
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cfg
    for c in clouds:
        ras.addPointCloud(c)
    ras.resize((w, h))
    ras.update(cam)
    ras.encode()
    gpu = {"rgba": ras.outputRGBA8(), "depthf": ras.depthTexture()}
    if cfg.mode == cr.MODE_HQS:
        px = ras.pixels()
        gpu["depth"] = px["depth"]
        gpu["accum"] = np.stack([px["red"], px["green"], px["blue"], px["count"]], -1)
    else:
        gpu["nd"] = ras.nearestDepths()
        gpu["ni"] = ras.nearestIndices()
    gpu["visible"] = [c.visibleBatches() for c in clouds]
    ocl = [oracle_cloud_from_device(orc, c) for c in clouds]
    ref = orc.render(ocl, oracle_config(orc, cfg), cam.viewMatrix, cam.projectionMatrix, w, h)
    return ras, gpu, ref


def assert_same(cr, cfg, gpu, ref, clouds=1, nearest_only_first=True):
    assert np.array_equal(gpu["rgba"], ref.rgba)
    assert np.array_equal(gpu["depthf"].view(np.uint32), ref.depthf.view(np.uint32))
    if cfg.mode == cr.MODE_HQS:
        assert np.array_equal(gpu["depth"], ref.depth)
        assert np.array_equal(gpu["accum"], ref.accum)
        for g, r in zip(gpu["visible"], ref.visible):
            assert np.array_equal(g, r)
    else:
        assert np.array_equal(gpu["nd"], ref.nearest_depth)
        assert np.array_equal(gpu["ni"], ref.nearest_index)
        assert np.array_equal(gpu["visible"][0], ref.visible[0])


def camera(cr, pos, target=(0, 0, 0), w=320, h=180, fov=60.0, near=0.01, far=100.0):
    cam = cr.PerspectiveCamera(position=pos, near=near, far=far, fov=fov, aspect=w / h)
    cam.lookAt(target)
    return cam


def test_update_files_bit_identical_to_oracle(cr, orc, ctx):
    pos, rgba = lattice_cloud(12, 1)
    cloud, packed = make_cloud(cr, orc, ctx, pos, rgba)
    cloud.position = (0.25, -0.5, 1.0)
    cam = camera(cr, (0.3, 0.4, 3.0))
    vp = cr.matrix_multiply(cam.projectionMatrix, cam.viewMatrix)
    cloud.updateFiles(vp, cloud.worldMatrix)
    ref = orc.update_files(packed.files, vp, cloud.worldMatrix)
    assert cloud.files().tobytes() == ref.tobytes()


@pytest.mark.parametrize("mode", [0, 1])
def test_lattice_frame_bit_exact(cr, orc, ctx, mode):
    """The 1M-point lattice workload's shape at 40^3 points, 320x180."""
    pos, rgba = lattice_cloud(40, 7)
    cloud, _ = make_cloud(cr, orc, ctx, pos, rgba)
    cfg = cr.ComputeRasteriserConfiguration(mode=mode)
    cam = camera(cr, (0, 0, 3))
    ras, gpu, ref = render_both(cr, orc, ctx, [cloud], cfg, cam, 320, 180)
    assert_same(cr, cfg, gpu, ref)
    assert (ref.accum[..., 3] > 0).sum() > 1000 or mode == 1


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("variant", ["footprint", "worldspace", "noclod", "holefill",
                                     "colorize", "lodbias", "nofrustum"])
def test_config_variants_bit_exact(cr, orc, ctx, mode, variant):
    pos, rgba = blob_cloud(60000, 11, scale=2.0)
    cloud, _ = make_cloud(cr, orc, ctx, pos, rgba, ppb=4096)
    cfg = cr.ComputeRasteriserConfiguration(mode=mode, backgroundColor=(0.1, 0.2, 0.3, 1.0))
    if variant == "footprint":
        cfg.minimumPointSize, cfg.maximumPointSize, cfg.pointSizeScale = 1.0, 7.0, 6.0
    elif variant == "worldspace":
        cfg.pointSizeMode, cfg.minimumPointSize, cfg.maximumPointSize = 1, 1.0, 9.0
        cfg.pointSizeScale = 0.01
    elif variant == "noclod":
        cfg.enableCLOD, cfg.enableLODDither = False, False
    elif variant == "holefill":
        cfg.holeFillIterations = 3
    elif variant == "colorize":
        cfg.colorizeChunks = True
    elif variant == "lodbias":
        cfg.lodBias = -2
    elif variant == "nofrustum":
        cfg.enableFrustumCulling = False
    cam = camera(cr, (0.7, 0.5, 1.6), w=256, h=160)
    ras, gpu, ref = render_both(cr, orc, ctx, [cloud], cfg, cam, 256, 160)
    assert_same(cr, cfg, gpu, ref)


def test_multi_cloud_occlusion_independent_of_order(cr, orc, ctx):
    """MultiCloudDepthOrderTests.swift:131-162: near red cube occludes far blue cube
    in both insertion orders; here both orders are also bit-exact to the oracle."""
    n = 16
    g = np.linspace(0, 1, n, dtype=np.float32)
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    cube = np.stack([x.ravel() - 0.5, y.ravel() - 0.5, z.ravel() - 0.5], 1).astype(np.float32)
    red = np.full(len(cube), 0xFF0000FF, np.uint32)
    blue = np.full(len(cube), 0xFFFF0000, np.uint32)
    cfg = cr.ComputeRasteriserConfiguration(depthTolerance=0.002, backgroundColor=(0, 0, 0, 1),
                                            enableFrustumCulling=False, enableCLOD=False,
                                            enableLODDither=False, minimumPointSize=8,
                                            maximumPointSize=64, pointSizeScale=32)
    cam = camera(cr, (0, 0, 5), w=64, h=64, fov=45, near=0.1)
    texels = []
    for order in (("near", "far"), ("far", "near")):
        clouds = []
        for name in order:
            c, _ = make_cloud(cr, orc, ctx, cube, red if name == "near" else blue)
            c.position = (0, 0, 1) if name == "near" else (0, 0, -1)
            clouds.append(c)
        ras, gpu, ref = render_both(cr, orc, ctx, clouds, cfg, cam, 64, 64)
        assert_same(cr, cfg, gpu, ref)
        texels.append(gpu["rgba"][32, 32].astype(int))
    assert np.array_equal(texels[0], texels[1])
    assert texels[0][0] > 0.6 * 255 and texels[0][2] < 0.2 * 255


def test_pick_matches_oracle_and_source_indices(cr, orc, ctx):
    """PickPointIndexTests.swift:49-114."""
    positions = np.array([[-0.8, 0, 0], [0, 0, 0], [0.8, 0, 0]], np.float32)
    colors = np.array([[1, 0, 0, 1], [0, 1, 0, 1], [0, 0, 1, 1]], np.float32)
    packed = orc.pack(positions, colors)
    cloud = cr.ComputeRasteriserPointCloud(ctx, packed=to_product_packed(cr, packed))
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cr.ComputeRasteriserConfiguration(
        backgroundColor=(0, 0, 0, 1), enableFrustumCulling=False, enableCLOD=False,
        enableLODDither=False)
    ras.addPointCloud(cloud)
    ras.resize((64, 64))
    cam = camera(cr, (0, 0, 5), w=64, h=64, fov=45, near=0.1)
    for _ in range(3):
        ras.update(cam)
        ras.encode()
    cloud.updateFiles(cr.matrix_multiply(cam.projectionMatrix, cam.viewMatrix), cloud.worldMatrix)
    oc = oracle_cloud_from_device(orc, cloud)
    d, ix = orc.nearest_cpu_reference(oc, 64, 64, cam.viewMatrix, cam.projectionMatrix)
    vp = cr.matrix_multiply(cam.projectionMatrix, cam.viewMatrix).reshape(4, 4).T.astype(np.float64)
    for orig, p in enumerate(positions):
        clip = vp @ np.array([*p, 1.0])
        ndc = (clip[0] / clip[3], clip[1] / clip[3])
        picked = ras.pickPointIndex(ndc, cloud, cam)
        assert picked is not None
        assert packed.sourceIndices[picked] == orig
        px = min(max(int((np.float32(ndc[0]) * np.float32(0.5) + np.float32(0.5)) * 64), 0), 63)
        pyb = int((np.float32(ndc[1]) * np.float32(0.5) + np.float32(0.5)) * 64)
        py = min(max(63 - pyb, 0), 63)
        assert ix.reshape(64, 64)[py, px] == picked


def test_pick_empty_space_returns_none(cr, orc, ctx):
    packed = orc.pack(np.zeros((1, 3), np.float32), np.ones((1, 4), np.float32))
    cloud = cr.ComputeRasteriserPointCloud(ctx, packed=to_product_packed(cr, packed))
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cr.ComputeRasteriserConfiguration(
        backgroundColor=(0, 0, 0, 1), enableFrustumCulling=False, enableCLOD=False,
        enableLODDither=False)
    ras.addPointCloud(cloud)
    ras.resize((64, 64))
    cam = camera(cr, (0, 0, 5), w=64, h=64, fov=45, near=0.1)
    ras.update(cam)
    ras.encode()
    assert ras.pickPointIndex((0.95, 0.95), cloud, cam) is None


def test_slot_pool_add_remove_and_render(cr, orc, ctx):
    """Streaming-style residency: LIFO slots, rebased firstPoint, removed slots
    skipped by the cull (state == 0), render stays bit-exact."""
    pos, rgba = blob_cloud(20000, 3)
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=1024)
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(40, 1024))
    slots = cloud.addBatches(packed.xyzLow, packed.xyzMed, packed.xyzHigh, packed.colors,
                             packed.levels, packed.batches, commit=False)
    assert slots == list(range(packed.batchCount))
    cloud.commitBatchUpdates()
    assert cloud.residentBatchCount == packed.batchCount
    assert cloud.pointCount == 20000
    gb = cloud.batches(0, packed.batchCount)
    assert np.array_equal(gb["firstPoint"], np.arange(packed.batchCount) * 1024)
    cloud.removeBatches([1, 3, 5])
    assert cloud.freeSlotCount == 40 - packed.batchCount + 3
    # LIFO reuse: the newest freed slot is handed out first.
    again = cloud.addBatches(packed.xyzLow, packed.xyzMed, packed.xyzHigh, packed.colors,
                             packed.levels, packed.batches[:2])
    assert again == [5, 3]
    cfg = cr.ComputeRasteriserConfiguration()
    cam = camera(cr, (0.2, 0.3, 1.5), w=200, h=150)
    ras, gpu, ref = render_both(cr, orc, ctx, [cloud], cfg, cam, 200, 150)
    assert_same(cr, cfg, gpu, ref)


def test_empty_and_nonresident_clouds(cr, orc, ctx):
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(4, 128))
    cfg = cr.ComputeRasteriserConfiguration(backgroundColor=(1.0, 0.5, 0.0, 1.0))
    cam = camera(cr, (0, 0, 3), w=32, h=16)
    ras, gpu, ref = render_both(cr, orc, ctx, [cloud], cfg, cam, 32, 16)
    assert_same(cr, cfg, gpu, ref)
    assert np.all(gpu["rgba"][..., 0] == 255) and np.all(gpu["rgba"][..., 3] == 0)


def test_colour_variant_flags_render_on_an_empty_cloud(cr, orc, ctx):
    """The colour variants (parity in test_gpu_variants.py) render through
    cr_render, clouds without attribute buffers reading zeros; a motion blur
    with no sample allowed is an argument error."""
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(1, 16))
    ras = cr.ComputeRasteriser(ctx)
    ras.addPointCloud(cloud)
    ras.resize((8, 8))
    ras.update(camera(cr, (0, 0, 3), w=8, h=8))
    for kw in ({"applyTint": True}, {"applyDisplacement": True},
               {"applyTint": True, "tintAlphaIsCoverage": True}, {"motionBlur": 0.5}):
        ras.configuration = cr.ComputeRasteriserConfiguration(**kw)
        ras.encode()
        assert not ras.pixels()["count"].any()
    ras.configuration = cr.ComputeRasteriserConfiguration(motionBlur=0.5, motionBlurSamples=0)
    with pytest.raises(cr.CRError) as e:
        ras.encode()
    assert e.value.status == 1


def test_capacity_errors(cr, orc, ctx):
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(2, 8))
    packed = orc.pack(np.random.default_rng(0).normal(size=(40, 3)).astype(np.float32),
                      np.ones((40, 4), np.float32), pointsPerBatch=8)
    with pytest.raises(cr.CRError) as e:
        cloud.addBatches(packed.xyzLow, packed.xyzMed, packed.xyzHigh, packed.colors,
                         packed.levels, packed.batches)
    assert e.value.status == 5
    with pytest.raises(cr.CRError):
        cloud.removeBatches([7])


def test_render_is_deterministic(cr, orc, ctx):
    pos, rgba = blob_cloud(80000, 21)
    cloud, _ = make_cloud(cr, orc, ctx, pos, rgba, ppb=2048)
    ras = cr.ComputeRasteriser(ctx)
    ras.addPointCloud(cloud)
    ras.resize((300, 200))
    ras.update(camera(cr, (0.1, 0.2, 1.2), w=300, h=200))
    outs = []
    for _ in range(3):
        ras.encode()
        outs.append((ras.outputRGBA8(), ras.pixels()))
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0]) and np.array_equal(o[1], outs[0][1])


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("chunk,tiles", [(256, True), (777, False), (2048, True), (65536, True),
                                         (2048, False)])
def test_tuning_does_not_change_results(cr, orc, ctx, mode, chunk, tiles):
    """Chunk size and shared-memory tiles are launch choices only: every setting
    renders the oracle's frame bit for bit (dense far-field cloud: many points
    per pixel, so the tiles are exercised)."""
    pos, rgba = blob_cloud(120000, 31, scale=1.0)
    cloud, _ = make_cloud(cr, orc, ctx, pos, rgba, ppb=4096)
    ctx.set_tuning(chunkPoints=chunk, useTiles=tiles)
    try:
        cfg = cr.ComputeRasteriserConfiguration(mode=mode, enableCLOD=False,
                                                enableLODDither=False)
        cam = camera(cr, (0.0, 0.0, 6.0), w=320, h=200, fov=40.0)
        ras, gpu, ref = render_both(cr, orc, ctx, [cloud], cfg, cam, 320, 200)
        assert_same(cr, cfg, gpu, ref)
        if mode == 0:
            assert ref.accum[..., 3].max() > 10  # many points per pixel
    finally:
        ctx.set_tuning(chunkPoints=2048, useTiles=True)


@pytest.mark.parametrize("mode", [0, 1])
def test_lattice_1m_1280x720_bit_exact(cr, orc, ctx, mode):
    """The small plain configuration at its stated size: 1,000,000 points on the
    100^3 lattice over [-1, 1]^3 with +-0.002 jitter and uniform RGB8 (the
    seeded generator, seed 0xC0FFEE01), packed into 10,240-point Morton
    batches (98 batches), one camera at (0, 0, 3) looking at the origin (fov
    60, near 0.01, far 100), 1280x720, depth tolerance 1 %.  The depth plane,
    the R, G, B, count planes, the survivor list, the RGBA8 image and the
    float depth are compared bit for bit with the oracle (HQS); the nearest
    depth and index planes in the nearest mode."""
    recs = orc.synth_lattice(100, seed=0xC0FFEE01, threads=8)
    packed = orc.pack(np.ascontiguousarray(recs[:, :3]), colors_rgba8=recs[:, 3].view(np.uint32),
                      pointsPerBatch=10240, threads=8)
    assert packed.batchCount == 98
    cloud = cr.ComputeRasteriserPointCloud(ctx, packed=to_product_packed(cr, packed))
    cfg = cr.ComputeRasteriserConfiguration(mode=mode, depthTolerance=0.01)
    cam = camera(cr, (0, 0, 3), w=1280, h=720, fov=60.0, near=0.01, far=100.0)
    ras, gpu, ref = render_both(cr, orc, ctx, [cloud], cfg, cam, 1280, 720)
    assert_same(cr, cfg, gpu, ref)
    if mode == 0:
        assert (ref.accum[..., 3] > 0).sum() > 100_000
        assert ref.visible[0]["activePoints"].sum() > 100_000
    else:
        assert (ref.nearest_index != 0xFFFFFFFF).sum() > 100_000
    cloud.close()
