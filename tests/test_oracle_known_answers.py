"""Pins the CPU oracle against the reference's own known-answer tests.

Each test restates one test of Tests/SatinComputeRasteriserTests/ (the Swift
test target of Satin-ComputeRasteriser) against the oracle, with the same
inputs and the same expected values.
"""
import numpy as np
import pytest


def jittered_cloud(count=3000, seed=0x5EED):
    """LODBucketingTests.swift:12-27: seeded LCG cloud."""
    state = seed
    mask = (1 << 64) - 1

    def nxt():
        nonlocal state
        state = (state * 6364136223846793005 + 1442695040888963407) & mask
        return np.float32(state >> 40) / np.float32(1 << 24)

    pos = np.zeros((count, 3), np.float32)
    col = np.zeros((count, 4), np.float32)
    for i in range(count):
        pos[i] = [nxt() * np.float32(10) - np.float32(5) for _ in range(3)]
        col[i] = [nxt(), nxt(), nxt(), np.float32(1)]
    return pos, col


def cum_counts(batch):
    words = [int(batch["lodCum01"]), int(batch["lodCum23"]), int(batch["lodCum45"]),
             int(batch["lodCum67"])]
    out = []
    for w in words:
        out += [w & 0xFFFF, w >> 16]
    return out


# --- NearestPointReferenceTests.swift:5-62 -------------------------------------

def test_nearest_reference_uses_reverse_z_depth(orc):
    packed = orc.pack([[0, 0, 0.25], [0, 0, 0.75]], [[1, 0, 0, 1], [0, 1, 0, 1]],
                      pointsPerBatch=2)
    d, ix = orc.nearest_cpu_reference(packed.cloud(), 4, 4)
    center = 1 * 4 + 2
    assert ix[center] == 1
    assert packed.colors[ix[center]] == 0xFF00FF00


def test_nearest_reference_keeps_lowest_index_on_depth_tie(orc):
    packed = orc.pack([[0, 0, 0.5], [0, 0, 0.5]], [[1, 0, 0, 1], [0, 1, 0, 1]],
                      pointsPerBatch=2)
    d, ix = orc.nearest_cpu_reference(packed.cloud(), 4, 4)
    center = 1 * 4 + 2
    assert ix[center] == 0
    assert packed.colors[ix[center]] == 0xFF0000FF


def test_nearest_reference_rejects_background_and_out_of_clip(orc):
    packed = orc.pack([[2, 0, 0.5], [0, 0, -0.5]], [[1, 0, 0, 1], [0, 1, 0, 1]],
                      pointsPerBatch=2)
    d, ix = orc.nearest_cpu_reference(packed.cloud(), 4, 4)
    assert np.all(ix == 0xFFFFFFFF)
    assert np.all(d == 0)


# --- LayoutTests.swift ---------------------------------------------------------

def test_layout_strides_and_offsets(orc):
    import ctypes as C
    assert C.sizeof(orc.orc_batch) == 64 == orc.BATCH_DTYPE.itemsize
    assert C.sizeof(orc.orc_file) == 256 == orc.FILE_DTYPE.itemsize
    assert C.sizeof(orc.orc_visible) == 16 == orc.VISIBLE_DTYPE.itemsize
    offs = {n: orc.BATCH_DTYPE.fields[n][1] for n in orc.BATCH_DTYPE.names}
    assert (offs["state"], offs["minX"], offs["maxZ"], offs["numPoints"], offs["firstPoint"],
            offs["fileIndex"]) == (0, 4, 24, 28, 32, 36)


def test_fixture_packing_produces_consistent_counts(orc):
    packed = orc.cube_grid(4)
    assert packed.pointCount == 64
    assert len(packed.xyzLow) == len(packed.xyzMed) == len(packed.xyzHigh) == 64
    assert packed.batchCount > 0
    assert len(packed.files) == 1


def test_pack_assigns_lod_levels_and_covers_all_points(orc):
    z, y, x = np.meshgrid(np.arange(8), np.arange(8), np.arange(8), indexing="ij")
    pos = np.stack([x.ravel(), y.ravel(), z.ravel()], 1).astype(np.float32)
    col = np.ones((len(pos), 4), np.float32)
    packed = orc.pack(pos, col, pointsPerBatch=128, lodLevels=4, coarseVoxelDivisions=2)
    counts = np.bincount(packed.levels, minlength=8)
    assert counts[:4].sum() == len(pos)
    assert 0 < counts[0] < len(pos)
    assert np.all(packed.colors >> 24 == 0xFF)


def test_pack_preserves_color_multiset_under_morton(orc):
    pos = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]]
    col = [[1, 0, 0, 1], [0, 1, 0, 1], [0, 0, 1, 1], [1, 1, 0, 1], [1, 1, 1, 1]]
    packed = orc.pack(pos, col, pointsPerBatch=2)
    assert packed.pointCount == 5 and packed.batchCount == 3
    assert sorted(packed.colors.tolist()) == sorted(
        [0xFF0000FF, 0xFF00FF00, 0xFFFF0000, 0xFF00FFFF, 0xFFFFFFFF])


# --- LODBucketingTests.swift:50-153 -------------------------------------------

@pytest.fixture(scope="module")
def lod_fixtures(orc):
    pos, col = jittered_cloud()
    return [orc.pack(pos, col, pointsPerBatch=512, lodLevels=4, coarseVoxelDivisions=8),
            orc.cube_grid(24)]


def test_pack_buckets_batches_with_matching_prefix_counts(lod_fixtures):
    for packed in lod_fixtures:
        assert packed.batchCount > 0
        for b in packed.batches:
            first, n = int(b["firstPoint"]), int(b["numPoints"])
            sl = packed.levels[first:first + n]
            assert np.all(np.diff(sl.astype(int)) >= 0)
            recount = np.cumsum(np.bincount(sl & 7, minlength=8)).tolist()
            assert cum_counts(b) == recount
            assert recount[7] == n
            assert b["lodCum67"] != 0


def test_pack_permutation_consistent_after_bucketing(orc):
    pos, col = jittered_cloud(2000, 0xB0CE7)
    packed = orc.pack(pos, col, pointsPerBatch=512, lodLevels=4, coarseVoxelDivisions=8)
    src = packed.sourceIndices
    assert len(set(src.tolist())) == len(pos)
    assert np.array_equal(packed.orderedPositions, pos[src])
    c = np.clip(col, 0, 1) * np.float32(255)
    q = c.astype(np.uint32)
    expect = q[:, 0] | (q[:, 1] << 8) | (q[:, 2] << 16) | (q[:, 3] << 24)
    assert np.array_equal(packed.colors, expect[src])


def test_survivor_prefix_is_exact_upper_bound(lod_fixtures):
    for packed in lod_fixtures:
        for thr in [0, 0.4, 0.5, 1.0, 1.7, 3.0, 99]:
            lmax = min(max(int(np.floor(np.float32(thr) + np.float32(0.5))), 0), 7)
            for b in packed.batches:
                active = cum_counts(b)[lmax]
                first, n = int(b["firstPoint"]), int(b["numPoints"])
                tail = packed.levels[first + active:first + n].astype(np.float32)
                assert np.sum(tail < np.float32(thr) + np.float32(0.5)) == 0


def test_clod_off_sentinel_activates_full_batch(lod_fixtures):
    assert min(max(int(np.floor(99 + 0.5)), 0), 7) == 7
    for packed in lod_fixtures:
        for b in packed.batches:
            assert cum_counts(b)[7] == b["numPoints"]


# --- Oracle-internal consistency ----------------------------------------------

def test_log2_contract_accuracy(orc):
    xs = np.concatenate([np.geomspace(1e-3, 1e6, 2000), [1.0, 2.0, 0.04, 25.0, 400.0]])
    for x in xs.astype(np.float32):
        got = orc.log2f(float(x))
        assert abs(got - np.log2(np.float64(x))) <= 4e-6 * max(1.0, abs(np.log2(x)))
    assert orc.log2f(1.0) == 0.0
    assert orc.log2f(8.0) == 3.0


def test_depth_to_uint_saturates(orc):
    assert orc.depth_to_uint(1.0) == 0xFFFFFFFF
    assert orc.depth_to_uint(0.0) == 0
    assert orc.depth_to_uint(0.5) == 0x80000000
    assert orc.depth_to_uint(-3.0) == 0


def test_general_nearest_pass_equals_cpu_reference(orc):
    """With CLOD, dither and frustum culling off and unit point size, the
    oracle's nearest pass (the shaders' semantics) must equal the reference's
    literal NearestPointCPUReference."""
    pos, col = jittered_cloud(1500, 0x1234)
    packed = orc.pack(pos * np.float32(0.15), col, pointsPerBatch=256)
    view = np.eye(4, dtype=np.float32)
    # A perspective-ish projection: w = -z + 2 so points stay in front.
    proj = np.array([[1.2, 0, 0, 0], [0, 1.2, 0, 0], [0, 0, -0.5, -1], [0, 0, 1.5, 2]],
                    np.float32).reshape(16)
    files = orc.update_files(orc.identity_file(), orc.mat4_mul(proj, view), np.eye(4))
    cloud = packed.cloud(files)
    cfg = orc.Config(mode=1, enableCLOD=False, enableLODDither=False,
                     enableFrustumCulling=False)
    fr = orc.render(cloud, cfg, view, proj, 64, 48)
    d, ix = orc.nearest_cpu_reference(cloud, 64, 48, view, proj)
    assert np.array_equal(fr.nearest_depth.ravel(), d)
    assert np.array_equal(fr.nearest_index.ravel(), ix)
    assert np.count_nonzero(ix != 0xFFFFFFFF) > 100


def test_multithreaded_render_matches_single(orc):
    pos, col = jittered_cloud(4000, 0x77)
    packed = orc.pack(pos * np.float32(0.2), col, pointsPerBatch=300)
    view = np.eye(4, dtype=np.float32)
    proj = np.array([[1.2, 0, 0, 0], [0, 1.2, 0, 0], [0, 0, -0.5, -1], [0, 0, 1.5, 2]],
                    np.float32).reshape(16)
    files = orc.update_files(orc.identity_file(), orc.mat4_mul(proj, view), np.eye(4))
    cloud = packed.cloud(files)
    for mode in (0, 1):
        cfg = orc.Config(mode=mode, minimumPointSize=1, maximumPointSize=5, pointSizeScale=4,
                         holeFillIterations=1)
        a = orc.render(cloud, cfg, view, proj, 80, 60, threads=1)
        b = orc.render(cloud, cfg, view, proj, 80, 60, threads=4)
        assert np.array_equal(a.rgba, b.rgba)
        assert np.array_equal(a.accum, b.accum)
        assert np.array_equal(a.nearest_index, b.nearest_index)


def test_project_exp_neg_accuracy(orc):
    """The coverage resolve's e^-x (written for this project, shared by the
    kernels and the oracle) against float64 exp: within 2 float ulps."""
    xs = np.concatenate([np.linspace(0, 1, 2001), np.linspace(1, 20, 4001),
                         np.array([1e-6, 1e-3, 0.5, 10.0, 40.0, 80.0, 87.0])]).astype(np.float32)
    got = np.array([orc.exp_neg(float(x)) for x in xs], np.float32)
    want = np.exp(-xs.astype(np.float64))
    ulp = np.spacing(want.astype(np.float32)).astype(np.float64)
    assert (np.abs(got - want) <= 2 * ulp + 1e-45).all()
    assert orc.exp_neg(0.0) == 1.0 and orc.exp_neg(200.0) == 0.0
