"""PLY file -> GPU pack -> render: PLYPointCloudLoader.load packs the parsed
vertices on the GPU; the image is bit-identical to the oracle's pack of the
oracle's parse, rendered by the oracle."""
import os

import numpy as np
import pytest

import oracle.ply as oply
from scenes import oracle_cloud_from_device, oracle_config

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("binary", [False, True])
def test_ply_load_pack_render_matches_oracle(cr, orc, tmp_path, binary):
    ctx = cr.Context(0)
    rng = np.random.default_rng(11 + binary)
    n = 30000
    pos = rng.normal(0, 0.4, (n, 3)).astype(np.float32)
    rgb = rng.integers(0, 65536, (n, 3)).astype(np.uint16)
    head = ("ply\nformat %s 1.0\nelement vertex %d\nproperty float x\nproperty float y\n"
            "property float z\nproperty ushort red\nproperty ushort green\nproperty ushort blue\n"
            "end_header\n" % ("binary_little_endian" if binary else "ascii", n)).encode()
    if binary:
        rec = np.zeros(n, np.dtype([("p", "<f4", 3), ("c", "<u2", 3)]))
        rec["p"], rec["c"] = pos, rgb
        data = head + rec.tobytes()
    else:
        data = head + "\n".join(f"{float(a)!r} {float(b)!r} {float(c)!r} {r} {g} {bl}"
                                for (a, b, c), (r, g, bl) in zip(pos, rgb)).encode()
    path = os.path.join(tmp_path, "cloud.ply")
    with open(path, "wb") as f:
        f.write(data)
    cloud = cr.PLYPointCloudLoader.load(ctx, path, pointsPerBatch=1024)
    assert cloud.pointCount == n

    opos, ocol = oply.parse(data)
    packed = orc.pack(opos[:, :3], colors=ocol, pointsPerBatch=1024)
    assert np.array_equal(cloud.batches()["numPoints"][:packed.batchCount],
                          packed.batches["numPoints"])
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cr.ComputeRasteriserConfiguration(holeFillIterations=1)
    ras.addPointCloud(cloud)
    ras.resize((160, 120))
    cam = cr.PerspectiveCamera(position=(0.9, 0.5, 1.7), near=0.01, far=100.0, fov=55.0,
                               aspect=160 / 120)
    cam.lookAt((0.0, 0.0, 0.0))
    ras.update(cam)
    ras.encode()
    ocl = oracle_cloud_from_device(orc, cloud)
    pts = cloud.points()
    # The device pool holds the oracle pack's points (same order, words, colours).
    for b, pb in zip(cloud.batches()[:packed.batchCount], packed.batches):
        f, k, g = int(b["firstPoint"]), int(b["numPoints"]), int(pb["firstPoint"])
        for name in ("xyzLow", "xyzMed", "xyzHigh", "colors", "levels"):
            assert np.array_equal(pts[name][f:f + k], getattr(packed, name)[g:g + k]), name
    ref = orc.render(ocl, oracle_config(orc, ras.configuration), cam.viewMatrix,
                     cam.projectionMatrix, 160, 120)
    assert np.array_equal(ras.outputRGBA8(), ref.rgba)
    assert ref.accum[..., 3].any()
