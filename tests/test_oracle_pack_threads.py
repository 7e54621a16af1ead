"""The oracle's multi-threaded pack and host generators (CPU only).

orc_pack_threads must give the single-threaded restatement of
PackedPointCloudFixtures.pack (PackedPointCloudFixtures.swift:30-344) bit for
bit: it builds the benchmark's CPU-side clouds and the large packer parity
check.  The host generators must be deterministic in the thread count (every
record is a function of seed and index alone).
"""
import math

import numpy as np
import pytest

from scenes import blob_cloud

FIELDS = ("batches", "xyzLow", "xyzMed", "xyzHigh", "colors", "levels", "sourceIndices",
          "orderedPositions", "boundsMin", "boundsMax")


def same(a, b):
    for k in FIELDS:
        assert getattr(a, k).tobytes() == getattr(b, k).tobytes(), k


@pytest.mark.parametrize("bits", [10, 21])
@pytest.mark.parametrize("ppb", [10240, 777, 16])
@pytest.mark.parametrize("threads", [2, 5, 8])
def test_threaded_pack_matches_single(orc, bits, ppb, threads):
    recs = orc.synth_terrain(orc.Terrain(seed=0xABC + ppb), 120_000)
    pos, rgba = np.ascontiguousarray(recs[:, :3]), recs[:, 3].view(np.uint32).copy()
    a = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=ppb, morton_bits=bits)
    b = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=ppb, morton_bits=bits, threads=threads)
    same(a, b)


@pytest.mark.parametrize("bits", [10, 21])
def test_threaded_pack_duplicate_keys_and_float_colours(orc, bits):
    """Integer lattice points share keys (the stable order decides) and the
    colours go through the truncating float path."""
    rng = np.random.default_rng(7)
    pos = rng.integers(0, 6, (60_000, 3)).astype(np.float32)
    col = rng.uniform(0, 1, (60_000, 4)).astype(np.float32)
    a = orc.pack(pos, col, pointsPerBatch=1000, morton_bits=bits)
    b = orc.pack(pos, col, pointsPerBatch=1000, morton_bits=bits, threads=7)
    same(a, b)
    pos, rgba = blob_cloud(40_000, 3)
    for lod, divs in ((1, 64), (8, 2), (3, 5)):
        a = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=500, lodLevels=lod,
                     coarseVoxelDivisions=divs, morton_bits=bits)
        b = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=500, lodLevels=lod,
                     coarseVoxelDivisions=divs, morton_bits=bits, threads=3)
        same(a, b)


def test_threaded_pack_degenerate_clouds(orc):
    one = np.zeros((1, 3), np.float32)
    same(orc.pack(one, colors_rgba8=np.array([7], np.uint32)),
         orc.pack(one, colors_rgba8=np.array([7], np.uint32), threads=4))
    flat = np.zeros((5000, 3), np.float32)
    flat[:, 0] = np.linspace(-1, 1, 5000)
    c = np.arange(5000, dtype=np.uint32)
    same(orc.pack(flat, colors_rgba8=c, pointsPerBatch=64),
         orc.pack(flat, colors_rgba8=c, pointsPerBatch=64, threads=6))


def test_generators_independent_of_threads(orc):
    t = orc.Terrain()
    a = orc.synth_terrain(t, 50_000, first=123_456)
    b = orc.synth_terrain(t, 50_000, first=123_456, threads=6)
    assert a.tobytes() == b.tobytes()
    # Records are a function of the index: a sub-range equals the same slice.
    c = orc.synth_terrain(t, 1000, first=123_456 + 777)
    assert c.tobytes() == a[777:1777].tobytes()
    la = orc.synth_lattice(20)
    lb = orc.synth_lattice(20, threads=5)
    assert la.tobytes() == lb.tobytes()


def test_generators_shape(orc):
    """The heightfield's x, y span [0, extent), the outliers are about 5 % of
    the points, the colours are opaque; the lattice is jittered by at most
    0.002 around its grid."""
    t = orc.Terrain()
    r = orc.synth_terrain(t, 200_000, threads=4)
    assert (r[:, 0] >= 0).all() and (r[:, 0] < t.extent).all()
    rgba = r[:, 3].view(np.uint32)
    assert ((rgba >> 24) == 255).all()
    h = np.array([orc.terrain_height(t, float(x), float(y)) for x, y in r[:2000, :2]])
    outl = np.abs(r[:2000, 2] - h) > 1e-3
    assert 0.03 < outl.mean() < 0.07
    lat = orc.synth_lattice(10)
    g = np.linspace(-1, 1, 10, dtype=np.float32)
    gx = np.tile(g, 100)
    assert np.abs(lat[:, 0] - gx).max() <= 0.0021


def test_project_ln_and_cos_accuracy(orc):
    """The colour noise's ln(u) and cos(2 pi u), written for this project and
    evaluated identically by the device generator: close to float64."""
    us = np.concatenate([np.linspace(1e-7, 1.0, 20001), np.array([1e-7, 0.5, 0.999999])])
    for u in us.astype(np.float32)[::7]:
        assert abs(orc._load().orc_ln_unit(float(u)) - math.log(float(u))) <= 2e-6 * max(
            1.0, abs(math.log(float(u))))
    for u in np.linspace(0, 1, 4001, endpoint=False).astype(np.float32):
        assert abs(orc._load().orc_cos_2pi(float(u)) - math.cos(2 * math.pi * float(u))) < 1e-6
