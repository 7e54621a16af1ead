"""Batched views (cr_render_multiview): every view bit-identical to a
per-view ComputeRasteriser update + encode of the same camera and size.

The per-view path with single-pixel footprints runs the fragment passes
(depth pass emits fragments, colour pass reads them); the batched path
decodes and projects the points again in its colour pass.  The two must
agree bit for bit on every plane: depth, R, G, B, count, RGBA8, depth f32.
"""
import os

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


def cameras(cr, sizes, seed, radius=2.5):
    rng = np.random.default_rng(seed)
    cams = []
    for w, h in sizes:
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        cam = cr.PerspectiveCamera(position=tuple(d * rng.uniform(0.8, 1.2) * radius),
                                   near=0.01, far=100.0, fov=float(rng.uniform(40, 75)),
                                   aspect=w / h)
        cam.lookAt(tuple(rng.uniform(-0.2, 0.2, 3)))
        cams.append(cam)
    return cams


def per_view(cr, ctx, clouds, cfg, cam, size):
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cfg
    for c in clouds:
        ras.addPointCloud(c)
    ras.resize(size)
    ras.update(cam)
    ras.encode()
    return ras.outputRGBA8(), ras.depthTexture(), ras.pixels()


def assert_views_match(cr, ctx, mv, clouds, cfg, cams, sizes):
    for i, (cam, size) in enumerate(zip(cams, sizes)):
        rgba, depthf, px = per_view(cr, ctx, clouds, cfg, cam, size)
        assert np.array_equal(mv.outputRGBA8(i), rgba), f"view {i} rgba"
        assert np.array_equal(mv.depthTexture(i).view(np.uint32), depthf.view(np.uint32)), i
        got = mv.pixels(i)
        for f in ("depth", "red", "green", "blue", "count"):
            assert np.array_equal(got[f], px[f]), f"view {i} {f}"
        assert px["count"].any(), f"view {i} drew nothing"


SIZES = [(64, 64), (128, 96), (320, 180), (96, 160), (200, 150), (32, 32), (256, 256)]


def test_batched_views_match_per_view_renders(cr, orc, ctx):
    pos, rgba = lattice_cloud(40, 11)
    cloud = make_cloud(cr, orc, ctx, pos, rgba)
    mv = cr.MultiViewRasteriser(ctx, SIZES)
    mv.addPointCloud(cloud)
    cams = cameras(cr, SIZES, 5)
    mv.render(cams)
    assert_views_match(cr, ctx, mv, [cloud], mv.configuration, cams, SIZES)


def test_graph_replay_with_new_cameras(cr, orc, ctx):
    """Three calls with different cameras reuse the captured graph (alternating
    staging blocks); each call's images match its own per-view renders."""
    pos, rgba = blob_cloud(60000, 4)
    cloud = make_cloud(cr, orc, ctx, pos, rgba)
    mv = cr.MultiViewRasteriser(ctx, SIZES[:4])
    mv.addPointCloud(cloud)
    for seed in (1, 2, 3):
        cams = cameras(cr, SIZES[:4], seed)
        mv.render(cams)
        assert_views_match(cr, ctx, mv, [cloud], mv.configuration, cams, SIZES[:4])


def test_batched_views_two_clouds_models_and_options(cr, orc, ctx):
    pos, rgba = blob_cloud(30000, 7)
    a = make_cloud(cr, orc, ctx, pos, rgba)
    pos2, rgba2 = lattice_cloud(24, 8, lo=-0.6, hi=0.6)
    b = make_cloud(cr, orc, ctx, pos2, rgba2, ppb=512)
    b.position = (0.3, -0.2, 0.1)
    cfg = cr.ComputeRasteriserConfiguration(depthTolerance=0.05, holeFillIterations=2,
                                            backgroundColor=(0.2, 0.4, 0.6, 1.0))
    mv = cr.MultiViewRasteriser(ctx, SIZES[:5])
    mv.configuration = cfg
    mv.addPointCloud(a)
    mv.addPointCloud(b)
    cams = cameras(cr, SIZES[:5], 9)
    mv.render(cams)
    assert_views_match(cr, ctx, mv, [a, b], cfg, cams, SIZES[:5])


@pytest.mark.parametrize("variant", ["footprint", "no_clod", "colorize"])
def test_batched_views_config_variants(cr, orc, ctx, variant):
    pos, rgba = lattice_cloud(32, 3)
    cloud = make_cloud(cr, orc, ctx, pos, rgba)
    kw = {"footprint": dict(minimumPointSize=1.0, maximumPointSize=4.0, pointSizeScale=3.0),
          "no_clod": dict(enableCLOD=False, enableLODDither=False),
          "colorize": dict(colorizeChunks=True)}[variant]
    cfg = cr.ComputeRasteriserConfiguration(**kw)
    sizes = SIZES[:3]
    mv = cr.MultiViewRasteriser(ctx, sizes)
    mv.configuration = cfg
    mv.addPointCloud(cloud)
    cams = cameras(cr, sizes, 21)
    mv.render(cams)
    assert_views_match(cr, ctx, mv, [cloud], cfg, cams, sizes)


def test_autotune_sets_and_caches_the_launch_shape(cr, orc, ctx, tmp_path):
    pos, rgba = blob_cloud(40000, 12)
    cloud = make_cloud(cr, orc, ctx, pos, rgba)
    mv = cr.MultiViewRasteriser(ctx, SIZES[:3])
    mv.addPointCloud(cloud)
    cams = cameras(cr, SIZES[:3], 2)
    path = os.path.join(tmp_path, "tune.jsonl")
    try:
        best = mv.autotune(cams, cachePath=path, reps=2)
        assert best["chunkPoints"] in (1024, 2048, 4096)
        assert best["viewGroupPixels"] in (0, 1048576, 2097152, 4194304, 8388608)
        assert ctx.tuning()["chunkPoints"] == best["chunkPoints"]
        lines = open(path).read().splitlines()
        assert len(lines) == 1 and '"candidates"' in lines[0]
        again = mv.autotune(cams, cachePath=path, reps=2)
        assert again["chunkPoints"] == best["chunkPoints"]
        assert again["useTiles"] == best["useTiles"]
        assert again["viewGroupPixels"] == best["viewGroupPixels"]
        assert len(open(path).read().splitlines()) == 1  # read, not re-timed
        mv.render(cams)
        assert_views_match(cr, ctx, mv, [cloud], mv.configuration, cams, SIZES[:3])
    finally:
        ctx.set_tuning(chunkPoints=2048, useTiles=True, viewGroupPixels=4194304)


@pytest.mark.parametrize("group_pixels", [1, 40000, 0])
def test_view_groups_do_not_change_results(cr, orc, ctx, group_pixels):
    """Depth and colour passes over groups of views (one view per group, a
    few views per group, all views in one group) share one fragment arena;
    every grouping gives the per-view images."""
    pos, rgba = blob_cloud(50000, 13)
    cloud = make_cloud(cr, orc, ctx, pos, rgba)
    try:
        ctx.set_tuning(viewGroupPixels=group_pixels)
        mv = cr.MultiViewRasteriser(ctx, SIZES)
        mv.addPointCloud(cloud)
        cams = cameras(cr, SIZES, 17)
        mv.render(cams)
        assert_views_match(cr, ctx, mv, [cloud], mv.configuration, cams, SIZES)
    finally:
        ctx.set_tuning(viewGroupPixels=4194304)


def test_batched_views_reject_bad_arguments(cr, orc, ctx):
    pos, rgba = blob_cloud(2000, 1)
    cloud = make_cloud(cr, orc, ctx, pos, rgba)
    mv = cr.MultiViewRasteriser(ctx, [(16, 16), (8, 8)])
    mv.addPointCloud(cloud)
    cams = cameras(cr, [(16, 16), (8, 8)], 1)
    with pytest.raises(cr.CRError):
        mv.render(cams[:1])
    mv.configuration = cr.ComputeRasteriserConfiguration(mode=cr.MODE_NEAREST)
    with pytest.raises(cr.CRError) as e:
        mv.render(cams)
    assert e.value.status == 4  # CR_ERR_UNSUPPORTED
    mv.configuration = cr.ComputeRasteriserConfiguration()
    mv.frames[1] = mv.frames[0]
    with pytest.raises(cr.CRError):
        mv.render(cams)


def test_batched_views_match_oracle_directly(cr, orc, ctx):
    """Every batched view against the CPU oracle itself (not only against the
    per-view GPU path): RGBA8, float depth, depth plane and R, G, B, count
    planes, bit for bit, with two clouds (one moved by a model matrix)."""
    from scenes import oracle_cloud_from_device, oracle_config
    pos, rgba = lattice_cloud(30, 21)
    a = make_cloud(cr, orc, ctx, pos, rgba)
    pos2, rgba2 = blob_cloud(40000, 22)
    b = make_cloud(cr, orc, ctx, pos2, rgba2, ppb=777)
    b.position = (0.3, -0.2, 0.1)
    sizes = [(96, 64), (160, 90), (64, 128)]
    mv = cr.MultiViewRasteriser(ctx, sizes)
    mv.addPointCloud(a)
    mv.addPointCloud(b)
    cams = cameras(cr, sizes, 9)
    mv.render(cams)
    cfg = oracle_config(orc, mv.configuration)
    for i, (cam, (w, h)) in enumerate(zip(cams, sizes)):
        clouds = []
        for c in (a, b):
            oc = oracle_cloud_from_device(orc, c)
            vp = cr.matrix_multiply(cam.projectionMatrix, cam.viewMatrix)
            oc.files = orc.update_files(orc.identity_file(), vp, c.worldMatrix)
            clouds.append(oc)
        ref = orc.render(clouds, cfg, cam.viewMatrix, cam.projectionMatrix, w, h)
        assert np.array_equal(mv.outputRGBA8(i), ref.rgba), f"view {i} rgba"
        assert np.array_equal(mv.depthTexture(i).view(np.uint32), ref.depthf.view(np.uint32))
        px = mv.pixels(i)
        assert np.array_equal(px["depth"], ref.depth), f"view {i} depth"
        acc = np.stack([px["red"], px["green"], px["blue"], px["count"]], -1)
        assert np.array_equal(acc, ref.accum), f"view {i} accum"
        assert ref.accum[..., 3].any()
