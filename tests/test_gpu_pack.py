"""GPU packer parity against the CPU oracle's pack (bit-exact).

Restates GPUPackerParityTests.swift:109-324 (single batch, multi batch,
slot-targeted chunks, two chunks in one call) with exact per-index equality
of every output, and adds duplicate-key clouds, 63-bit keys and the input
layouts.  The reference test only asserts AABBs to 1e-5 and positions to
4 quantisation steps; here batches, words, levels, colours and the source
permutation are compared bit for bit.
"""
import numpy as np
import pytest

from scenes import blob_cloud

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(cr):
    return cr.Context(0)


def lattice(n):
    """GPUPackerParityTests.swift:58-73."""
    g = np.arange(n, dtype=np.float32) / np.float32(n - 1)
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    fx, fy, fz = x.ravel(), y.ravel(), z.ravel()
    pos = np.stack([fx - np.float32(0.5), fy - np.float32(0.5), fz - np.float32(0.5)], 1)
    col = np.stack([fx, fy, fz, np.ones_like(fx)], 1)
    return pos.astype(np.float32), col.astype(np.float32)


def check_region(cloud, ref, first_slot, ppb, src=None, cmp_src=True):
    nb = ref.batchCount
    n = ref.pointCount
    gb = cloud.batches(first_slot, nb)
    exp = ref.batches.copy()
    exp["firstPoint"] = (first_slot + np.arange(nb)) * ppb
    assert gb.tobytes() == exp.tobytes()
    pts = cloud.points(first_slot * ppb, n)
    for k in ("xyzLow", "xyzMed", "xyzHigh", "colors", "levels"):
        assert np.array_equal(pts[k], getattr(ref, k)), k
    if src is not None and cmp_src:
        assert np.array_equal(src, ref.sourceIndices)


def gpu_pack(cr, ctx, pos, col=None, rgba=None, ppb=10240, bits=10, lod=4, divs=64, slots=1):
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(slots, ppb))
    packer = cr.GPUPacker(ctx, lodLevels=lod, coarseVoxelDivisions=divs, mortonBits=bits)
    src = packer.pack(pos, col if col is not None else rgba, into=cloud, sourceIndices=True)
    return cloud, src


@pytest.mark.parametrize("n", [16, 40])
def test_lattice_pack_bit_exact(cr, orc, ctx, n):
    pos, col = lattice(n)
    ref = orc.pack(pos, col)
    cloud, src = gpu_pack(cr, ctx, pos, col)
    assert cloud.residentBatchCount == ref.batchCount
    assert cloud.pointCount == len(pos)
    check_region(cloud, ref, 0, 10240, src)


@pytest.mark.parametrize("bits", [10, 21])
@pytest.mark.parametrize("ppb", [10240, 777, 64])
def test_duplicate_key_cloud_bit_exact(cr, orc, ctx, bits, ppb):
    """Clustered points share Morton keys; both sorts are stable, so the
    order (and everything after it) is identical."""
    pos, rgba = blob_cloud(50000, 5 + bits + ppb)
    ref = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=ppb, morton_bits=bits)
    cloud, src = gpu_pack(cr, ctx, pos, rgba=rgba, ppb=ppb, bits=bits)
    check_region(cloud, ref, 0, ppb, src)


@pytest.mark.parametrize("lod,divs", [(1, 64), (2, 3), (8, 2), (4, 8)])
def test_lod_parameters(cr, orc, ctx, lod, divs):
    pos, rgba = blob_cloud(30000, 99, scale=3.0)
    ref = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=2048, lodLevels=lod,
                   coarseVoxelDivisions=divs)
    cloud, src = gpu_pack(cr, ctx, pos, rgba=rgba, ppb=2048, lod=lod, divs=divs)
    check_region(cloud, ref, 0, 2048, src)


def test_input_layouts(cr, orc, ctx):
    pos, rgba = blob_cloud(20000, 4)
    ref = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=4096)
    # 16-byte records {x, y, z, rgba8}.
    rec = np.zeros((len(pos), 4), np.float32)
    rec[:, :3] = pos
    rec.view(np.uint32)[:, 3] = rgba
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(1, 4096))
    src = cr.GPUPacker(ctx).pack(records=rec, into=cloud, sourceIndices=True)
    check_region(cloud, ref, 0, 4096, src)
    # float3 in 16-byte slots + packed colours.
    p4 = np.zeros((len(pos), 4), np.float32)
    p4[:, :3] = pos
    cloud2, src2 = gpu_pack(cr, ctx, p4, rgba=rgba, ppb=4096)
    check_region(cloud2, ref, 0, 4096, src2)
    # float colours truncate as uint(clamp(c) * 255).
    colf = np.random.default_rng(1).uniform(-0.2, 1.2, (len(pos), 4)).astype(np.float32)
    ref3 = orc.pack(pos, colf, pointsPerBatch=4096)
    cloud3, src3 = gpu_pack(cr, ctx, pos, col=colf, ppb=4096)
    check_region(cloud3, ref3, 0, 4096, src3)


def test_device_resident_input(cr, orc, ctx):
    torch = pytest.importorskip("torch")
    pos, rgba = blob_cloud(12000, 8)
    ref = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=1000)
    dp = torch.from_numpy(pos).cuda()
    dc = torch.from_numpy(rgba.view(np.int32)).cuda()
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(1, 1000))
    torch.cuda.synchronize()
    src = cr.GPUPacker(ctx).pack(dp, dc, into=cloud, sourceIndices=True)
    check_region(cloud, ref, 0, 1000, src)


def test_pack_grows_pool_and_empties_other_slots(cr, orc, ctx):
    pos, rgba = blob_cloud(5000, 2)
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(2, 512))
    packer = cr.GPUPacker(ctx)
    packer.pack(pos, rgba, into=cloud)
    assert cloud.capacity.maxResidentBatches == 10
    assert cloud.residentBatchCount == 10
    small = pos[:700]
    packer.pack(small, rgba[:700], into=cloud)
    assert cloud.residentBatchCount == 2 and cloud.pointCount == 700
    b = cloud.batches()
    assert list(b["state"]) == [1, 1] + [0] * 8
    packer.pack(np.zeros((0, 3), np.float32), np.zeros(0, np.uint32), into=cloud)
    assert cloud.residentBatchCount == 0


def test_slot_targeted_chunks_non_destructive(cr, orc, ctx):
    """GPUPackerParityTests.swift:262-295."""
    ppb = 10240
    posA, colA = lattice(40)
    posB, colB = lattice(32)
    refA = orc.pack(posA, colA)
    refB = orc.pack(posB, colB)
    cloud = cr.ComputeRasteriserPointCloud(
        ctx, cr.ComputeRasteriserCapacity(refA.batchCount + refB.batchCount + 3, ppb))
    packer = cr.GPUPacker(ctx)
    assert cloud.addRawChunksGPU(packer, [(posA, colA)]) == [0]
    assert cloud.residentBatchCount == refA.batchCount
    assert cloud.pointCount == len(posA)
    check_region(cloud, refA, 0, ppb)
    assert cloud.addRawChunksGPU(packer, [(posB, colB)]) == [refA.batchCount]
    assert cloud.residentBatchCount == refA.batchCount + refB.batchCount
    check_region(cloud, refB, refA.batchCount, ppb)
    check_region(cloud, refA, 0, ppb)


def test_two_chunks_one_call(cr, orc, ctx):
    """GPUPackerParityTests.swift:297-323."""
    ppb = 10240
    posA, colA = lattice(36)
    posB, colB = lattice(28)
    refA, refB = orc.pack(posA, colA), orc.pack(posB, colB)
    cloud = cr.ComputeRasteriserPointCloud(
        ctx, cr.ComputeRasteriserCapacity(refA.batchCount + refB.batchCount + 1, ppb))
    slots = cloud.addRawChunksGPU(cr.GPUPacker(ctx), [(posA, colA), (posB, colB)])
    assert slots == [0, refA.batchCount]
    check_region(cloud, refA, 0, ppb)
    check_region(cloud, refB, refA.batchCount, ppb)


def test_chunk_without_room_is_skipped(cr, orc, ctx):
    pos, col = lattice(12)
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(2, 1024))
    packer = cr.GPUPacker(ctx)
    # 1728 points need 2 slots; the second chunk finds no free run.
    assert cloud.addRawChunksGPU(packer, [(pos, col), (pos, col)]) == [0]
    assert cloud.residentBatchCount == 2


def test_packed_cloud_renders_like_cpu_packed(cr, orc, ctx):
    """A GPU-packed cloud and a CPU-packed cloud produce the same frame."""
    from scenes import to_product_packed
    pos, rgba = blob_cloud(40000, 17)
    ref = orc.pack(pos, colors_rgba8=rgba)
    cpu_cloud = cr.ComputeRasteriserPointCloud(ctx, packed=to_product_packed(cr, ref))
    gpu_cloud, _ = gpu_pack(cr, ctx, pos, rgba=rgba)
    imgs = []
    for cloud in (cpu_cloud, gpu_cloud):
        ras = cr.ComputeRasteriser(ctx)
        ras.addPointCloud(cloud)
        ras.resize((200, 120))
        cam = cr.PerspectiveCamera(position=(0.3, 0.2, 1.4), near=0.01, far=100, fov=60,
                                   aspect=200 / 120)
        ras.update(cam)
        ras.encode()
        imgs.append(ras.outputRGBA8())
    assert np.array_equal(imgs[0], imgs[1])
    assert (imgs[0][..., 3] > 0).sum() > 500


def test_heightfield_63_bit_pack_bit_exact(cr, orc, ctx):
    """The 63-bit packer (21 bits per axis) on a 4M-point heightfield (GPU
    synthesised 16-byte records, the 400M-point configuration's generator at
    a size the CPU pack handles in seconds): every batch, word, level, colour
    and the source permutation equal the CPU pack's."""
    n, ppb = 4_000_000, 10240
    recs = cr.synth_terrain(ctx, cr.TerrainParams(seed=0xC0FFEE03), n)
    host = recs.download()
    pos = np.ascontiguousarray(host[:, :3])
    rgba = host[:, 3].view(np.uint32).copy()
    ref = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=ppb, morton_bits=21)
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(ref.batchCount, ppb))
    src = cr.GPUPacker(ctx, mortonBits=21).pack(records=recs, into=cloud, sourceIndices=True)
    recs.close()
    check_region(cloud, ref, 0, ppb, src)


def test_device_generators_match_host_restatement(cr, orc, ctx):
    """The device's seeded generators and the oracle's host restatement give
    bit-identical records (the benchmark's CPU side builds its clouds with the
    restatement, without the library)."""
    params = cr.TerrainParams(seed=0xC0FFEE02)
    n = 3_000_000
    dev = cr.synth_terrain(ctx, params, n)
    got = dev.download()
    dev.close()
    want = orc.synth_terrain(orc.Terrain(seed=0xC0FFEE02), n, threads=8)
    assert got.tobytes() == want.tobytes()
    for x, y in ((0.0, 0.0), (1234.5, 3210.25), (3999.0, 17.0)):
        assert np.float32(cr.terrain_height(params, x, y)) == np.float32(
            orc.terrain_height(orc.Terrain(seed=0xC0FFEE02), x, y))
    lat = cr.synth_lattice(ctx, 100)
    got = lat.download()
    lat.close()
    assert got.tobytes() == orc.synth_lattice(100, threads=8).tobytes()


def test_lattice_1m_pack_bit_exact(cr, orc, ctx):
    """The 1,000,000-point jittered 100^3 lattice (seed 0xC0FFEE01) packed into
    10,240-point batches on the GPU equals the CPU pack bit for bit."""
    recs = cr.synth_lattice(ctx, 100)
    host = recs.download()
    ref = orc.pack(np.ascontiguousarray(host[:, :3]), colors_rgba8=host[:, 3].view(np.uint32).copy(),
                   pointsPerBatch=10240, threads=8)
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(ref.batchCount, 10240))
    src = cr.GPUPacker(ctx).pack(records=recs, into=cloud, sourceIndices=True)
    recs.close()
    assert ref.batchCount == 98
    check_region(cloud, ref, 0, 10240, src)
    cloud.close()


@pytest.mark.parametrize("bits", [10, 21])
def test_constant_and_single_digit_keys(cr, orc, ctx, bits):
    """Edge cases of the radix sort's digit skipping: every point at the same
    position (every digit of every key the same: no pass runs, the input
    order stands) and points that differ along one axis only (most digits
    constant), at sizes around the 4096-key tile."""
    for n in (1, 4095, 4096, 4097, 9000):
        pos = np.tile(np.array([[0.25, -0.5, 1.0]], np.float32), (n, 1))
        rgba = np.arange(n, dtype=np.uint32) | np.uint32(0xff000000)
        ref = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=1000, morton_bits=bits)
        cloud, src = gpu_pack(cr, ctx, pos, rgba=rgba, ppb=1000, bits=bits)
        check_region(cloud, ref, 0, 1000, src)
        cloud.close()
    n = 20000
    pos = np.zeros((n, 3), np.float32)
    pos[:, 1] = np.random.default_rng(3).integers(0, 7, n).astype(np.float32)
    rgba = np.arange(n, dtype=np.uint32)
    ref = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=512, morton_bits=bits)
    cloud, src = gpu_pack(cr, ctx, pos, rgba=rgba, ppb=512, bits=bits)
    check_region(cloud, ref, 0, 512, src)
    cloud.close()
